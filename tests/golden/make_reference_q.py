"""Golden collision-operator vectors from the reference's own CUDA kernels.

Runs the reference's vhs-gll kernels and cuFFT (built by
``python -m oracle.ref_vhs.build <reference-root>`` into ``oracle/_ref/``;
the host sequence of frfs/solvers/dgfs/scattering.py:227-286) on seeded
distributions and writes ``tests/golden/reference_q_<tag>.npz`` (f and the
reference's Q, FP64, no conservation projection); likewise the gas-mixture
vss-gll kernels (``python -m oracle.ref_vss.build``; the host sequence of
frfs/solvers/dgfsbi/scattering.py:256-330) into
``tests/golden/reference_qbi_<tag>.npz`` (f and Q as [dof][species][Nv^3]):

    python tests/golden/make_reference_q.py [outdir]

Needs a CUDA GPU and the built libraries; the tests then compare the oracle
and the product with the committed vectors.
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, 'oracle', '_ref')
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))


def inputs(tag, vm):
    """Seeded distributions: the 4x4-mesh FP64 family on 16^3 (two
    Maxwellians, n ~ U(0.5, 1.5), |u| < 0.5, T ~ U(0.7, 1.3)); the batched
    family on 24^3 (1-3 Maxwellians + 1 % noise)."""
    from helpers import maxwellian, mixed_maxwellians, random_ball
    cv = vm.cv
    if tag == 'nv16':
        rng = np.random.default_rng(161)
        F = []
        for _ in range(4):
            f = 0.0
            for _ in range(2):
                f = f + maxwellian(cv, rng.uniform(0.5, 1.5), random_ball(rng, 0.5), rng.uniform(0.7, 1.3))
            F.append(f)
        return np.stack(F)
    rng = np.random.default_rng(241)
    return np.stack([mixed_maxwellians(cv, rng) for _ in range(2)])


def main(outdir):
    from oracle.ref_vhs.build import GRIDS, grid_tables
    for tag in GRIDS:
        so = os.path.join(REF, f'libref_vhs_{tag}.so')
        with open(os.path.join(REF, f'ref_vhs_{tag}.json')) as fh:
            g = json.load(fh)
        vm, _, _ = grid_tables(g)
        F = np.ascontiguousarray(inputs(tag, vm), dtype=np.float64)
        Q = np.zeros_like(F)
        lib = C.CDLL(so)
        lib.ref_vhs_q.restype = C.c_int
        lib.ref_vhs_q.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        rc = lib.ref_vhs_q(g['Nv'], g['Nrho'], g['M'], F.shape[0], F.ctypes.data, Q.ctypes.data)
        if rc != 0:
            raise RuntimeError(f'{tag}: reference run failed ({rc})')
        path = os.path.join(outdir, f'reference_q_{tag}.npz')
        np.savez_compressed(path, f=F, Q=Q, **{k: v for k, v in g.items() if k != 'tag'})
        print(path, F.shape, float(np.abs(Q).max()))


def mixture_inputs(vm):
    """Seeded two-species distributions: per species a sum of two
    Maxwellians n (m/(pi T))^1.5 exp(-m |c-u|^2/T), n ~ U(0.3, 1.2),
    T ~ U(0.7, 1.3), u ~ U(-0.3, 0.3)^3."""
    from helpers import mixture
    rng = np.random.default_rng(1616)
    return np.stack([np.stack(mixture(vm.cv, vm.masses, rng)) for _ in range(3)])


def run_vss(so, g, vm, par, F):
    """Q of the reference's mixture kernels for F [dof][2][Nv^3] (FP64)."""
    F = np.ascontiguousarray(F, dtype=np.float64)
    Q = np.zeros_like(F)
    gam = np.ascontiguousarray([par[(p, q)]['gamma'] for p in range(2) for q in range(2)])
    sz = np.ascontiguousarray(vm.sz, dtype=np.float64)
    qz = np.ascontiguousarray(vm.qz, dtype=np.float64)
    qw = np.ascontiguousarray(vm.qw, dtype=np.float64)
    lib = C.CDLL(so)
    lib.ref_vss_q.restype = C.c_int
    lib.ref_vss_q.argtypes = [C.c_int] * 5 + [C.c_void_p] * 3 + [C.c_double] * 3 + [C.c_void_p] * 3
    rc = lib.ref_vss_q(g['Nv'], g['Nrho'], g['M'], 2, F.shape[0], sz.ctypes.data, qz.ctypes.data,
                       qw.ctypes.data, vm.L, vm.sw, 4 * np.pi / g['Mpre'], gam.ctypes.data,
                       F.ctypes.data, Q.ctypes.data)
    if rc != 0:
        raise RuntimeError(f'reference mixture run failed ({rc})')
    return Q


def main_bi(outdir):
    from oracle.ref_vss.build import GRIDS, grid_tables
    for tag in GRIDS:
        so = os.path.join(REF, f'libref_vss_{tag}.so')
        with open(os.path.join(REF, f'ref_vss_{tag}.json')) as fh:
            g = json.load(fh)
        vm, _, _, par = grid_tables(g)
        F = mixture_inputs(vm)
        Q = run_vss(so, g, vm, par, F)
        path = os.path.join(outdir, f'reference_qbi_{tag}.npz')
        np.savez_compressed(path, f=F, Q=Q, **{k: np.asarray(v) for k, v in g.items() if k != 'tag'})
        print(path, F.shape, float(np.abs(Q).max()))


if __name__ == '__main__':
    out = sys.argv[1] if len(sys.argv) > 1 else HERE
    main(out)
    main_bi(out)
