"""GPU parity of the boundary conditions other than the diffuse wall
(inlet, normal-shock inlet, outlet, vanish, specular, diffuse-cyl) against
the FP64 oracle, through every FR entry point."""
import numpy as np
import pytest
import torch

from frfs_b200 import _lib
from frfs_b200.backend import CUDABackend
from frfs_b200.integrators import get_integrator
from frfs_b200.mesh import StructuredMesh
from frfs_b200.system import DGFSSystem

from helpers import bc_cfg, oracle_for, rel_l2
from test_bcs_cpu import HEX, QUAD
from test_fr_gpu import _fr_oracle, _perturb

pytestmark = pytest.mark.gpu

QUAD2 = {'x-': 'dgfs-inlet', 'x+': 'dgfs-outlet', 'y-': 'dgfs-vanish', 'y+': 'dgfs-wall-diffuse'}


def _system(kind, order, prec, bcs, Nv=16, nreg=3, scheme='dgfs-tvd-rk2'):
    cfg = bc_cfg(Nv, order, bcs, precision=prec, scheme=scheme)
    be = CUDABackend(cfg)
    if kind == 'quad':
        mesh = StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5))
    else:
        mesh = StructuredMesh((2, 2, 2), (0.0, -0.5, 0.0), (1.0, 0.5, 1.0))
    return cfg, be, DGFSSystem(be, mesh, cfg, nreg=nreg)


CASES = [('quad', 2, 'double', QUAD, 1e-12), ('quad', 3, 'single', QUAD2, 2e-5),
         ('hex', 2, 'double', HEX, 1e-12), ('hex', 2, 'single', HEX, 2e-5),
         ('quad', 2, 'single', QUAD, 2e-5)]


@pytest.mark.parametrize('kind,order,prec,bcs,tol', CASES)
def test_bc_rhs_parity(cuda, kind, order, prec, bcs, tol):
    """L(u) with these boundaries: the system's path vs the oracle, and the
    dense / gather / factored entries against one another."""
    cfg, be, s = _system(kind, order, prec, bcs)
    _perturb(s, 21)
    orc = _fr_oracle(s, kind, order)
    u = s.eles_scal_upts_inb_full[0]
    un = u.double().cpu().numpy()
    s.updatebc(0.0, 0, 1)
    s.rhs(0.0, 0, 1)
    torch.cuda.synchronize()
    L_o = orc.rhs(un)
    assert rel_l2(s.eles_scal_upts_inb_full[1].double().cpu().numpy(), L_o) < 10 * tol
    # every entry point on the same state
    L, fsel = _lib.lib(), s.ele.fsel.data_ptr()
    x1, x2 = u * 1.5, u * 0.5
    args = (0.5, 2.0, x1.data_ptr(), 0.25, x2.data_ptr(), -0.5, _lib.stream_ptr())
    s._disu()
    if s.walls.has_diffuse:
        s._update_bc()
    outs = {}
    outs['dense'] = torch.empty_like(u)
    _lib.check(L.bdgfs_fr_rhs(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), u.data_ptr(),
                              s._uf_rows.data_ptr(), outs['dense'].data_ptr(), *args), 'rhs')
    outs['gather'] = torch.empty_like(u)
    _lib.check(L.bdgfs_fr_rhs_gather(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel,
                                     u.data_ptr(), outs['gather'].data_ptr(), *args), 'gather')
    outs['tensor'] = torch.empty_like(u)
    _lib.check(L.bdgfs_fr_rhs_tensor(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct),
                                     _lib.ref(s.ele.tensor), u.data_ptr(), None,
                                     outs['tensor'].data_ptr(), *args), 'tensor')
    if prec == 'single':
        s.ele.struct.engine = 1
        outs['tcgen05'] = torch.empty_like(u)
        _lib.check(L.bdgfs_fr_rhs(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), u.data_ptr(),
                                  s._uf_rows.data_ptr(), outs['tcgen05'].data_ptr(), *args), 'tc')
        s.ele.struct.engine = 0
    torch.cuda.synchronize()
    assert torch.equal(outs['dense'], outs['gather'])
    base = (0.5 * un + 0.25 * 1.5 * un - 0.5 * 0.5 * un)
    for k, o in outs.items():
        Lg = (o.double().cpu().numpy() - base) / 2.0
        assert rel_l2(Lg, L_o) < 10 * tol, k


@pytest.mark.parametrize('kind,bcs,nsteps', [('quad', QUAD, 3), ('quad', QUAD2, 3), ('hex', HEX, 1)])
def test_bc_steps_match_oracle(cuda, kind, bcs, nsteps):
    """Graph-replayed SSP-RK2 DG steps (FP64, with collisions, no
    conservation projection) against the oracle stepper on a mesh with these
    boundaries."""
    from oracle.fr import step_rk2
    cfg, be, s = _system(kind, 2, 'double', bcs, Nv=16)
    _perturb(s, 22)
    orc = _fr_oracle(s, kind, 2)
    vo = oracle_for(s.vm)
    Q = lambda x: np.stack([np.stack([vo.Q(x[e, j]) for j in range(x.shape[1])])
                            for e in range(x.shape[0])])
    s.sm._project = False
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    dt = 2e-4
    for _ in range(nsteps):
        u = step_rk2(u, dt, orc.rhs, Q)
        integ.step(integ.tcurr, dt)
        integ.tcurr += dt
    torch.cuda.synchronize()
    assert rel_l2(s.eles_scal_upts_inb_full[0].double().cpu().numpy(), u) < 1e-11


@pytest.mark.parametrize('prec,tol', [('double', 1e-13), ('single', 1e-6)])
def test_maxwellian_expr_initial_condition(cuda, prec, tol):
    """'maxwellianExpr': every solution point holds the Maxwellian of the
    expressions at its location."""
    from helpers import maxwellian
    cfg = bc_cfg(16, 2, QUAD, precision=prec)
    u0 = np.sqrt(2 * 8.3144598 / 39.96e-3 * 273.0)
    cfg.set('constants', 'rl', '0.00011140244750324529')
    for k, v in (('type', 'maxwellianExpr'), ('rho', 'rl*(1 + 0.1*sin(2*pi*x))'),
                 ('ux', f'{0.1 * u0}*y'), ('uy', f'{0.05 * u0}*x'), ('uz', '0'),
                 ('T', '273*(1 + 0.05*x)')):
        cfg.set('soln-ics', k, v)
    be = CUDABackend(cfg)
    s = DGFSSystem(be, StructuredMesh((3, 2), (0.0, -0.5), (1.0, 0.5)), cfg, nreg=2)
    torch.cuda.synchronize()
    cv = s.vm.cv()
    p = s.geo.plocupts
    want = np.stack([np.stack([maxwellian(cv, 1 + 0.1 * np.sin(2 * np.pi * x), [0.1 * y, 0.05 * x, 0],
                                          1 + 0.05 * x) for x, y in pe]) for pe in p])
    got = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    assert rel_l2(got, want) < tol
