"""Render the reference's vhs-gll kernels for the test grids and compile
each with the harness into ``oracle/_ref/libref_vhs_<tag>.so`` (test
infrastructure; the outputs stay out of version control).

    python -m oracle.ref_vhs.build <reference-root>

Grids: 'nv16' (Nv = 16 on [-5, 5]^3, Nrho = 8, M = 6, hard spheres) and
'nv24' (Nv = 24 on [-6, 6]^3, Nrho = M = 12, VHS omega = 0.81), with the
oracle's velocity mesh, radial rule, half-sphere directions and VHS
prefactor (the reference's template arguments, scattering.py:154-160).
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(ROOT, 'oracle', '_ref')
NONDIM = dict(T0=273.0, H0=1e-3, rho0=0.00011140244750324529, molarMass0=39.96e-3)
GRIDS = {'nv16': dict(Nv=16, Nrho=8, M=6, dev=5.0, omega=0.5),
         'nv24': dict(Nv=24, Nrho=12, M=12, dev=6.0, omega=0.81)}


def grid_tables(g):
    """Oracle velocity mesh and prefactor of one grid."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from frfs_b200.sphericaldesign import half_sphere_design
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import vhs_prefactor
    vm = VelocityMesh(g['Nv'], g['Nrho'], half_sphere_design(g['M']), cmax=0.0, Tmax=NONDIM['T0'],
                      dev=g['dev'], **NONDIM)
    gam, pref, _ = vhs_prefactor(vm, g['omega'], 4.17e-10, NONDIM['T0'])
    return vm, gam, pref


def build(reference_root, nvcc='nvcc'):
    from oracle.ref_vhs.render import render_vhs_gll
    os.makedirs(OUT, exist_ok=True)
    built = []
    for tag, g in GRIDS.items():
        vm, gam, pref = grid_tables(g)
        src = render_vhs_gll(reference_root, vm.Nrho, vm.M, vm.vsize, vm.sw, pref, vm.qw, vm.sz,
                             gam, vm.L, vm.qz)
        cu = os.path.join(OUT, f'vhs_gll_{tag}.cu')
        with open(cu, 'w') as fh:
            fh.write(src)
        so = os.path.join(OUT, f'libref_vhs_{tag}.so')
        subprocess.check_call([nvcc, '-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a',
                               '-Xcompiler', '-fPIC', '-shared', f'-DREF_KERNELS="{cu}"',
                               os.path.join(HERE, 'harness.cu'), '-lcufft', '-o', so])
        with open(os.path.join(OUT, f'ref_vhs_{tag}.json'), 'w') as fh:
            json.dump(dict(g, tag=tag), fh)
        built.append(so)
    return built


if __name__ == '__main__':
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], 'frfs')):
        sys.exit('usage: python -m oracle.ref_vhs.build <reference-root>')
    print('\n'.join(build(os.path.abspath(sys.argv[1]))))
