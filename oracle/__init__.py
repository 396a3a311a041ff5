"""CPU oracle for the DGFS hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package (``frfs_b200``)
imports, links or runs anything from this directory; only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` use it, and only as the checker or as the timed CPU
restatement of the reference algorithm.

Every function restates, in FP64 numpy, the reference algorithm of
jaisw7/frfs for one row of the hot path and cites the reference file:line
it follows.  The restatement keeps the reference's own operation order and
normalisations (cuFFT Z2Z conventions: forward exp(-2*pi*i*jk/n),
inverse exp(+2*pi*i*jk/n), both unnormalised).

Parity pins: FR operator matrices, quadrature rules and spherical designs
are pinned against fixtures produced by the reference's own Python modules
(``tests/golden/make_golden.py``); the VHS precompute tables are pinned
against the reference's own numpy formulation of them (the docstring block
in ``frfs/solvers/dgfs/scattering.py:94-126``, executed by the same
script).  The collision operator is pinned against the reference's own
CUDA kernels: ``oracle/ref_vhs`` renders its vhs-gll template and drives
the kernels with cuFFT in its host order (test infrastructure, built into
``oracle/_ref``); the oracle's Q matches the golden vectors they wrote to
1.8e-14 (16^3) and 5.5e-15 (24^3) relative L2.  The gas-mixture
operator likewise: ``oracle/ref_vss`` renders the vss-gll template; the
mixture oracle's Q_p matches its golden vectors to 5.4e-15 (two species,
16^3), with 1 + s.t in B rounded as the kernel evaluates it (three fused
multiply-adds).  The BGK, ES-BGK and Shakov relaxation steps likewise:
``oracle/ref_adgfs`` renders the reference's *-direct-gll templates and
runs its ARS and BDF steppers' kernel sequences; the oracle's ARS steps
and BDF updates match to 4.7e-14 of the step's change.  Known-answer tests add
Q(Maxwellian) ~ 0, conservation of mass/momentum/energy and the
Bobylev-Krook-Wu analytic solution for Maxwell molecules.
"""
