"""Render the reference's vss-gll gas-mixture kernels for the test grid and
compile them with the harness into ``oracle/_ref/libref_vss_<tag>.so`` (test
infrastructure; the outputs stay out of version control).

    python -m oracle.ref_vss.build <reference-root>

Grid 'bi16': two species of molar masses 39.96e-3 and 83.798e-3 kg/mol
(argon, krypton), Nv = 16 on [-5, 5]^3, Nrho = 6, M = 12 full-sphere
directions, Mpre = 12 pre-computation directions, every ordered pair VSS
with alpha = 1.3, omega = 0.81, dRef = 4.17e-10 m, Tref = 273 K; the
oracle's velocity mesh and pair parameters, and the template arguments of
frfs/solvers/dgfsbi/scattering.py:145-153.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(ROOT, 'oracle', '_ref')
NONDIM = dict(T0=273.0, H0=1e-3, rho0=0.00011140244750324529, molarMass0=39.96e-3)
GRIDS = {'bi16': dict(Nv=16, Nrho=6, M=12, Mpre=12, dev=5.0, molar=[39.96e-3, 83.798e-3],
                      alpha=1.3, omega=0.81, dRef=4.17e-10, Tref=273.0)}


def grid_tables(g):
    """Oracle mixture velocity mesh, pre-computation directions and pair
    parameters of one grid."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from frfs_b200.sphericaldesign import full_sphere_design
    from oracle.vss import BiVelocityMesh, all_pairs, vss_parameters
    masses = [m / NONDIM['molarMass0'] for m in g['molar']]
    vm = BiVelocityMesh(g['Nv'], g['Nrho'], full_sphere_design(g['M']), masses, cmax=0.0,
                        Tmax=NONDIM['T0'], dev=g['dev'], **NONDIM)
    szpre = full_sphere_design(g['Mpre'])
    pairs = all_pairs(len(masses), alpha=g['alpha'], omega=g['omega'], dRef=g['dRef'],
                      Tref=g['Tref'])
    return vm, szpre, pairs, vss_parameters(vm, pairs)


def render_vss_gll(reference_root, vm, szpre, par, soasz=32):
    """The rendered CUDA source of the reference's mixture kernels with the
    template arguments of scattering.py:145-153 (prefac, gamma, eta keyed by
    the pair string 'pq')."""
    from oracle.ref_vhs.render import render
    path = os.path.join(reference_root, 'frfs', 'solvers', 'dgfsbi', 'kernels', 'scattering',
                        'vss-gll.mako')
    with open(path) as fh:
        src = fh.read()
    S = len(vm.masses)
    cases = [(p, q) for p in range(S) for q in range(S)]
    key = lambda p, q: f'{p}{q}'
    return render(src, Nrho=vm.Nrho, M=vm.M, vsize=vm.vsize, sw=vm.sw,
                  prefac={key(*c): par[c]['prefac'] for c in cases}, soasz=soasz, cases=cases,
                  masses=vm.masses, qw=vm.qw, qz=vm.qz, L=vm.L, sz=vm.sz,
                  gamma={key(*c): par[c]['gamma'] for c in cases},
                  eta={key(*c): par[c]['eta'] for c in cases},
                  Mpre=szpre.shape[0], szpre=szpre, swpre=4 * 3.141592653589793 / szpre.shape[0])


def build(reference_root, nvcc='nvcc'):
    os.makedirs(OUT, exist_ok=True)
    built = []
    for tag, g in GRIDS.items():
        vm, szpre, _, par = grid_tables(g)
        src = render_vss_gll(reference_root, vm, szpre, par)
        cu = os.path.join(OUT, f'vss_gll_{tag}.cu')
        with open(cu, 'w') as fh:
            fh.write(src)
        so = os.path.join(OUT, f'libref_vss_{tag}.so')
        subprocess.check_call([nvcc, '-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a',
                               '-Xcompiler', '-fPIC', '-shared', f'-DREF_KERNELS="{cu}"',
                               os.path.join(HERE, 'harness.cu'), '-lcufft', '-o', so])
        with open(os.path.join(OUT, f'ref_vss_{tag}.json'), 'w') as fh:
            json.dump(dict(g, tag=tag), fh)
        built.append(so)
    return built


if __name__ == '__main__':
    if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], 'frfs')):
        sys.exit('usage: python -m oracle.ref_vss.build <reference-root>')
    print('\n'.join(build(os.path.abspath(sys.argv[1]))))
