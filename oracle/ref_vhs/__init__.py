"""The reference's own fast-spectral VHS collision kernels, rendered from
its Mako template and run as test infrastructure (the checker of the
oracle, never part of the product).

``render.py`` renders ``frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako``
(read from a reference checkout at build time; the rendered CUDA source is
written to ``oracle/_ref/`` only, which stays out of version control) with a
small renderer for the Mako subset the template uses.  ``harness.cu``
drives the rendered kernels and cuFFT in the order of the reference's
``DGFSVHSGLLScatteringModel.perform_precomputation`` / ``fs``
(frfs/solvers/dgfs/scattering.py:67-286) for a batch of distributions.
``build.py`` compiles one shared library per velocity grid into
``oracle/_ref/``; ``tests/golden/make_reference_q.py`` runs them on a GPU
and writes the golden Q vectors the tests compare with.
"""
