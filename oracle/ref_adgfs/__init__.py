"""The reference's own BGK-family relaxation kernels (bgk-, esbgk- and
shakov-direct-gll with their common ARS/BDF update kernels), rendered and
driven in the order of its ARS stepper for golden vectors (test
infrastructure)."""
