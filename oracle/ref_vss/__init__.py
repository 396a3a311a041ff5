"""The reference's own vss-gll gas-mixture collision kernels, rendered and
compiled for golden vectors (test infrastructure)."""
