"""Generate golden fixtures from the reference's own Python modules.

Run in a container that has the reference checkout (read-only), giving
the checkout's root as the one argument:

    python tests/golden/make_golden.py <reference-root>

It imports the reference's pure-numpy modules unchanged, with four alias
shims for Python 3.12 / numpy 2 (``collections.Iterable``/``Sequence``,
``configparser.SafeConfigParser``, ``np.float``) and a stub for the absent
``pycuda`` package (only its names are touched at import time), and writes
``tests/golden/*.npz``:

* ``shapes_<kind>_p<order>.npz``  upts, fpts, M0, M1, M2, M3, M1-M3*M2,
  norm_fpts, M12 (the inverse mass matrix) from ``frfs/shapes.py``
  (QuadShape / HexShape, GLL points), and ``interp_from_p<q>`` for q =
  order -+ 1, the restart interpolation of ``solvers/dgfs/system.py:100-104``;
* ``metrics_<kind>_p<order>.npz``  smats, rcpdjac, pnorms, ploc for a small
  affine mesh via ``frfs/solvers/base/elements.py``;
* ``vmesh_<case>.npz``  cv, cw, L, qz, qw, sz, sw from
  ``DGFSVelocityMesh`` (``frfs/solvers/dgfs/velocitymesh.py``);
* ``vhs_precompute_nv8.npz``  aa, bb1, bb2 from the reference's own numpy
  formulation of the VHS tables (``frfs/solvers/dgfs/scattering.py:94-126``,
  executed as written);
* ``initcond.npz``  Maxwellian and BKW initial values
  (``frfs/solvers/dgfs/initcond.py:39-140``);
* ``sphdesign.npz``  the shipped symmetric designs used here (2M=12, 32).
"""
import collections
import collections.abc
import configparser
import os
import sys
import types

import numpy as np

if len(sys.argv) != 2 or not os.path.isdir(os.path.join(sys.argv[1], 'frfs')):
    sys.exit('usage: make_golden.py <reference-root>  (the directory holding frfs/)')
REF = os.path.abspath(sys.argv[1])
OUT = os.path.dirname(os.path.abspath(__file__))

# --- alias shims (no edits to the reference) -------------------------------
collections.Iterable = collections.abc.Iterable
collections.Sequence = collections.abc.Sequence
configparser.SafeConfigParser = configparser.ConfigParser
np.float = float
pycuda = types.ModuleType('pycuda')
pycuda.gpuarray = types.ModuleType('pycuda.gpuarray')
pycuda.compiler = types.ModuleType('pycuda.compiler')
pycuda.driver = types.ModuleType('pycuda.driver')
for m in (pycuda, pycuda.gpuarray, pycuda.compiler, pycuda.driver):
    sys.modules[m.__name__] = m
sys.path.insert(0, REF)


def _bare_pkg(name):
    """Register a package without running its __init__ (those pull in
    MPI/plugin machinery that is absent here); submodules still import."""
    mod = types.ModuleType(name)
    mod.__path__ = [os.path.join(REF, *name.split('.'))]
    sys.modules[name] = mod


for _p in ('frfs.solvers', 'frfs.solvers.base', 'frfs.solvers.dgfs'):
    _bare_pkg(_p)

from frfs.inifile import Inifile                       # noqa: E402
from frfs.shapes import QuadShape, HexShape            # noqa: E402
from frfs.sphericaldesign import get_sphquadrule      # noqa: E402
from frfs.quadratures import zwgj                      # noqa: E402


def _cfg(order, extra=''):
    return Inifile(f"""
[solver]
system = dgfs
order = {order}
[solver-interfaces-line]
flux-pts = gauss-legendre-lobatto
[solver-interfaces-quad]
flux-pts = gauss-legendre-lobatto
[solver-elements-quad]
soln-pts = gauss-legendre-lobatto
[solver-elements-hex]
soln-pts = gauss-legendre-lobatto
{extra}
""")


def shapes():
    out = {}
    for cls, order in ((QuadShape, 2), (QuadShape, 3), (HexShape, 2)):
        cfg = _cfg(order)
        nspts = 2**cls.ndims            # linear shape points
        s = cls(nspts, cfg)
        d = dict(upts=np.array(s.upts), fpts=np.array(s.fpts),
                 M0=s.opmat('M0'), M1=s.opmat('M1'), M2=s.opmat('M2'),
                 M3=s.opmat('M3'), M132=s.opmat('M1 - M3*M2'),
                 norm_fpts=np.array(s.norm_fpts),
                 nfacefpts=np.array(s.nfacefpts), M12=s.opmat('M12'))
        # restart interpolation onto this basis from a solution of order q
        # (solvers/dgfs/system.py:100-104: the stored basis' nodal_basis_at
        # of the current solution points)
        for q in (order - 1, order + 1):
            solnb = cls(None, _cfg(q))
            d[f'interp_from_p{q}'] = solnb.ubasis.nodal_basis_at(s.upts)
        name = f'shapes_{cls.name}_p{order}.npz'
        np.savez(os.path.join(OUT, name), **d)
        out[(cls.name, order)] = (cls, cfg)
    return out


def metrics(shp):
    from frfs.solvers.base.elements import BaseElements

    class _Eles(BaseElements):
        privarmap = {2: ['f'], 3: ['f']}
        convarmap = privarmap
        _scratch_bufs = set()

        def set_backend(self, *a, **k):
            pass

        @staticmethod
        def pri_to_con(pris, cfg):
            return pris

    rng = np.random.default_rng(1)
    for (kind, order), (cls, cfg) in shp.items():
        ndims = cls.ndims
        # affine elements: a 2x1 (quad) or 2x1x1 (hex) brick of sizes hx,hy,hz
        # with a small shear so that every metric term is exercised
        h = np.array([0.25, 0.125, 0.5])[:ndims]
        A = np.diag(h / 2) + 0.01 * rng.standard_normal((ndims, ndims))
        corners = np.array(cls.std_ele(1))            # (nspts, ndims) in [-1,1]
        eles = []
        for e in range(2):
            off = np.zeros(ndims)
            off[0] = e * h[0]
            eles.append((corners @ A.T) + off)
        eles = np.stack(eles, axis=1)                  # (nspts, neles, ndims)
        el = _Eles(cls, eles, cfg)
        smats = el.smat_at_np('upts')                  # (ndims, nupts, ndims, neles)
        rcpdjac = el.rcpdjac_at_np('upts')             # (nupts, neles)
        np.savez(os.path.join(OUT, f'metrics_{kind}_p{order}.npz'),
                 eles=eles, smats=smats, rcpdjac=rcpdjac,
                 smats_fpts=el.smat_at_np('fpts'),
                 norm_pnorm_fpts=el._norm_pnorm_fpts,
                 mag_pnorm_fpts=el._mag_pnorm_fpts,
                 ploc_upts=el.ploc_at_np('upts'),
                 plocfpts=el.plocfpts)


class _StubBackend:
    soasz = 32

    def const_matrix(self, a, **kw):
        return np.array(a)


def vmesh():
    from frfs.solvers.dgfs.velocitymesh import DGFSVelocityMesh
    cases = {
        'c1': dict(Nv=16, Nrho=8, M=6, dev=5, rule='womersley'),
        'nv8': dict(Nv=8, Nrho=4, M=6, dev=5, rule='womersley'),
        'm16': dict(Nv=24, Nrho=12, M=16, dev=6, rule='womersley'),
    }
    for name, c in cases.items():
        cfg = Inifile(f"""
[constants]
Nv = {c['Nv']}
NvBatchSize = {c['Nv']**2}
Nrho = {c['Nrho']}
[non-dim]
T0 = 273
H0 = 1e-3
rho0 = 0.00011140244750324529
molarMass0 = 39.96e-3
[velocity-mesh]
dev = {c['dev']}
cmax = 0
Tmax = 273
[spherical-design-rule]
ssrule = {c['rule']}
M = {c['M']}
""")
        vm = DGFSVelocityMesh(_StubBackend(), cfg)
        np.savez(os.path.join(OUT, f'vmesh_{name}.npz'), cv=vm.cv(),
                 cw=vm.cw(), L=vm.L(), qz=vm.qz(), qw=vm.qw(), sz=vm.sz(),
                 sw=vm.sw(), u0=vm.u0(), n0=vm.n0(), Nv=c['Nv'],
                 Nrho=c['Nrho'], M=c['M'])


def vhs_precompute():
    """Execute the reference's numpy formulation of aa/bb1/bb2 as written
    (the string block inside ``perform_precomputation``)."""
    # scattering.py imports Mako/cuFFT at module level, so the block is read
    # from the source text of DGFSVHSGLLScatteringModel.perform_precomputation
    path = os.path.join(REF, 'frfs', 'solvers', 'dgfs', 'scattering.py')
    text = open(path).read()
    cls = text.index('class DGFSVHSGLLScatteringModel')
    src = text[text.index('def perform_precomputation', cls):]
    start = src.index('"""') + 3
    block = src[start:src.index('"""', start)]
    body = block[:block.index('# load precomputed weights onto the memory')]
    body = '\n'.join(l[8:] if l.startswith(' ' * 8) else l.lstrip()
                     for l in body.splitlines())
    g = np.load(os.path.join(OUT, 'vmesh_nv8.npz'))
    Nv, Nrho, M = int(g['Nv']), int(g['Nrho']), int(g['M'])
    vsize = Nv**3
    l0 = np.concatenate((np.arange(0, Nv / 2), np.arange(-Nv / 2, 0)))
    l = np.zeros((3, vsize))
    for idv in range(vsize):
        I, J, K = idv // (Nv * Nv), (idv % (Nv * Nv)) // Nv, (idv % (Nv * Nv)) % Nv
        l[:, idv] = l0[I], l0[J], l0[K]
    gamma = 2.0 * (1 - 0.81)

    class _Self:
        _gamma = gamma
    ns = dict(np=np, Nrho=Nrho, M=M, vsize=vsize, L=float(g['L']),
              qz=g['qz'], qw=g['qw'], sz=g['sz'], l=l, self=_Self())
    exec(body, ns)
    np.savez(os.path.join(OUT, 'vhs_precompute_nv8.npz'),
             aa=ns['h_aa'], bb1=ns['h_bb1'], bb2=ns['h_bb2'], gamma=gamma)


def initcond():
    from frfs.solvers.dgfs.initcond import (DGFSMaxwellianInitCondition,
                                            DGFSBKWInitCondition)
    g = np.load(os.path.join(OUT, 'vmesh_c1.npz'))

    class _VM:
        def cv(self): return g['cv']
        def cw(self): return float(g['cw'])
        def vsize(self): return int(g['Nv'])**3
        def u0(self): return float(g['u0'])
        def T0(self): return 273.0
        def rho0(self): return 0.00011140244750324529
        def molarMass0(self): return 39.96e-3

    u0 = float(g['u0'])
    cfg = Inifile(f"""
[soln-ics]
rho = {0.00011140244750324529 * 1.1}
T = {273 * 0.9}
ux = {0.2 * u0}
uy = {-0.1 * u0}
uz = {0.05 * u0}
[bkw]
t0 = 5.5
""")
    mx = DGFSMaxwellianInitCondition(None, cfg, _VM(), 'soln-ics')
    bkw = DGFSBKWInitCondition(None, cfg, _VM(), 'bkw')
    np.savez(os.path.join(OUT, 'initcond.npz'), maxwellian=mx.get_init_vals(),
             rho=1.1, T=0.9, u=np.array([0.2, -0.1, 0.05]),
             bkw=bkw.get_init_vals(), bkw_t0=5.5)


def sphdesign():
    d = {}
    for npts in (12, 32):
        d[f'pts{npts}'] = get_sphquadrule('symmetric', rule='womersley',
                                          npts=npts).pts
    z, w = zwgj(8, 0.0, 0.0)
    d['gj8_z'], d['gj8_w'] = z, w
    z, w = zwgj(12, 0.0, 0.0)
    d['gj12_z'], d['gj12_w'] = z, w
    np.savez(os.path.join(OUT, 'sphdesign.npz'), **d)


if __name__ == '__main__':
    shp = shapes()
    metrics(shp)
    vmesh()
    vhs_precompute()
    initcond()
    sphdesign()
    print('fixtures written to', OUT)
