"""GPU parity of the FR operators, the diffuse-wall update and full DGFS
steps against the FP64 oracle (frfs_b200 C ABI vs oracle.fr)."""
import numpy as np
import pytest
import torch

from frfs_b200.backend import CUDABackend
from frfs_b200.mesh import StructuredMesh
from frfs_b200.system import DGFSSystem
from frfs_b200.integrators import get_integrator

from helpers import couette_cfg, oracle_for, rel_l2

pytestmark = pytest.mark.gpu

GOLD = __import__('os').path.join(__import__('os').path.dirname(__file__), 'golden')


def _ops(kind, order):
    g = np.load(f'{GOLD}/shapes_{kind}_p{order}.npz')
    return {'M0': g['M0'], 'M132': g['M132'], 'M3': g['M3']}


def _system(kind, order, precision, Nv=16, Nrho=8, M=6, dev=5, shape=None, nreg=3, **kw):
    cfg = couette_cfg(Nv, Nrho, M, dev, order, precision=precision, **kw)
    be = CUDABackend(cfg)
    if kind == 'quad':
        mesh = StructuredMesh(shape or (3, 2), (0.0, -0.5), (1.0, 0.5), periodic='x')
    else:
        mesh = StructuredMesh(shape or (2, 2, 2), (0.0, -0.5, 0.0), (1.0, 0.5, 1.0),
                              periodic='xz')
    return cfg, be, mesh, DGFSSystem(be, mesh, cfg, nreg=nreg)


def _perturb(sys_, seed):
    rng = np.random.default_rng(seed)
    u = sys_.eles_scal_upts_inb_full[0]
    x = sys_.geo.plocupts                     # (E, nupts, ndims)
    amp = 0.2 * np.sin(2 * np.pi * x[..., 0]) + 0.1 * np.cos(np.pi * x[..., 1])
    vel = rng.uniform(-0.3, 0.3, size=u.shape[-1])
    pert = 1.0 + amp[..., None] * (1.0 + vel[None, None, :])
    u.mul_(torch.from_numpy(pert).to(u))


def _fr_oracle(sys_, kind, order):
    from oracle.fr import FROracle
    walls, rows = sys_.walls.oracle_walls()
    return FROracle(_ops(kind, order), sys_.geo, sys_.vm.c0(), sys_.vm.cw(), walls, bcid=rows)


@pytest.mark.parametrize('kind,order,prec,tol', [
    ('quad', 2, 'double', 1e-12), ('quad', 3, 'double', 1e-12), ('hex', 2, 'double', 1e-12),
    ('quad', 3, 'single', 2e-5), ('hex', 2, 'single', 2e-5)])
def test_fr_rhs_parity(cuda, kind, order, prec, tol):
    cfg, be, mesh, s = _system(kind, order, prec)
    _perturb(s, 1)
    orc = _fr_oracle(s, kind, order)
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    # disu + bc update
    s.updatebc(0.0, 0, 1)
    uf_o = orc.disu(u)
    assert rel_l2(s._uf.double().cpu().numpy(), uf_o) < tol
    bc_o = orc.update_bc(uf_o)
    bc_g = s.walls.bcv.double().cpu().numpy()[:len(bc_o)]
    assert np.allclose(bc_g, bc_o, rtol=10 * tol, atol=0)
    # full rhs: L(u) into bank 1
    s.rhs(0.0, 0, 1)
    L_g = s.eles_scal_upts_inb_full[1].double().cpu().numpy()
    L_o = orc.rhs(u, bc=bc_o)
    assert rel_l2(L_g, L_o) < 10 * tol


def test_fr_free_stream_periodic(cuda):
    """A uniform state on a fully periodic mesh is preserved: L(u) = 0."""
    cfg = couette_cfg(16, 8, 6, 5, 3, precision='double')
    be = CUDABackend(cfg)
    mesh = StructuredMesh((4, 3), (0.0, 0.0), (1.0, 1.0), periodic='xy')
    s = DGFSSystem(be, mesh, cfg)
    s.rhs(0.0, 0, 1)
    L = s.eles_scal_upts_inb_full[1]
    assert float(L.abs().max()) < 1e-12 * float(s.eles_scal_upts_inb_full[0].abs().max())


@pytest.mark.parametrize('scheme', ['dgfs-tvd-rk2', 'dgfs-euler'])
def test_steps_match_oracle(cuda, scheme):
    """Three steps of the graph-captured stepper vs the oracle stepper (FP64,
    exact-Nyquist collision operator)."""
    from oracle.fr import step_rk2, step_euler
    cfg, be, mesh, s = _system('quad', 2, 'double', scheme=scheme, dt=2e-3, uw=0.3)
    _perturb(s, 2)
    orc = _fr_oracle(s, 'quad', 2)
    vo = oracle_for(s.vm)
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    integ = get_integrator(be, s, cfg)
    nsteps, dt = 3, 2e-3
    L = lambda x: orc.rhs(x)
    Q = lambda x: np.stack([np.stack([vo.Q(x[e, j]) for j in range(x.shape[1])])
                            for e in range(x.shape[0])])
    # conservation projection is new (not in the reference): compare without it
    s.sm._project = False
    for _ in range(nsteps):
        u = (step_rk2 if scheme == 'dgfs-tvd-rk2' else step_euler)(u, dt, L, Q)
        integ.step(integ.tcurr, dt)
        integ.tcurr += dt
    got = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    assert rel_l2(got, u) < 1e-11


def test_graph_replay_equals_eager(cuda):
    cfg, be, mesh, s1 = _system('quad', 3, 'single', Nv=16, Nrho=8, M=6, dev=5)
    _, _, _, s2 = _system('quad', 3, 'single', Nv=16, Nrho=8, M=6, dev=5)
    i1 = get_integrator(be, s1, cfg)
    i2 = get_integrator(be, s2, cfg)
    i2.use_graph = False
    for _ in range(3):
        i1.step(0.0, 5e-4)
        i2.step(0.0, 5e-4)
    assert torch.equal(s1.eles_scal_upts_inb_full[0], s2.eles_scal_upts_inb_full[0])


def test_moments_and_residual(cuda):
    from oracle.fr import moments
    cfg, be, mesh, s = _system('quad', 2, 'double', Nv=16, Nrho=8, M=6, dev=5)
    _perturb(s, 3)
    rho, U, T, q, P = s.moments(0)
    f = s.eles_scal_upts_inb_full[0].reshape(-1, s.vm.vsize()).cpu().numpy()
    for i in (0, 5, 17):
        r, u, t, qq, pp = moments(f[i], s.vm.cv(), s.vm.cw())
        assert abs(float(rho[i]) - r) < 1e-12 * r
        assert np.allclose(U[i].cpu().numpy(), u, atol=1e-12)
        assert abs(float(T[i]) - t) < 1e-11 * t
        assert np.allclose(q[i].cpu().numpy(), qq, atol=1e-10)
        assert np.allclose(P[i].cpu().numpy(), pp, rtol=1e-10, atol=1e-12)
    s.eles_scal_upts_inb_full[1].copy_(s.eles_scal_upts_inb_full[0] * 1.01)
    r = s.residual(1, 0).cpu().numpy()
    assert abs(np.sqrt(r[0] / r[1]) - 0.01) < 1e-10


def test_partitioned_virtual_ranks_equal_single_domain(cuda):
    """Three parts of a slab-partitioned mesh, stepped stage by stage with the
    in-process halo exchange, reproduce the single-domain steps exactly."""
    from frfs_b200.partition import LocalTransport, slab_partition, step_rk2_virtual
    cfg, be, mesh, s = _system('quad', 3, 'single', Nv=16, Nrho=8, M=6, dev=5, shape=(6, 2))
    _perturb(s, 4)
    parts = slab_partition(mesh, 3)
    systems = [DGFSSystem(be, mesh, cfg, nreg=3, partition=(parts, r)) for r in range(3)]
    tr = LocalTransport(systems)
    for r, sy in enumerate(systems):
        sy.transport = tr
        idx = torch.as_tensor(parts[r], device=be.device)
        sy.eles_scal_upts_inb_full[0].copy_(s.eles_scal_upts_inb_full[0].index_select(0, idx))
    integ = get_integrator(be, s, cfg)
    integ.use_graph = False
    for _ in range(2):
        integ.step(0.0, 5e-4)
        step_rk2_virtual(systems, 5e-4)
    torch.cuda.synchronize()
    for r, sy in enumerate(systems):
        idx = torch.as_tensor(parts[r], device=be.device)
        assert torch.equal(sy.eles_scal_upts_inb_full[0],
                           s.eles_scal_upts_inb_full[0].index_select(0, idx)), r


@pytest.mark.parametrize('kind,order', [('quad', 3), ('hex', 2), ('quad', 2)])
def test_tensor_core_rhs_matches_cuda_core_rhs(cuda, kind, order):
    """The tcgen05 (3xTF32) FR residual against the CUDA-core kernel on the
    same FP32 state: agreement to FP32 rounding, with walls and with the
    RK combination operands."""
    cfg, be, mesh, s = _system(kind, order, 'single', shape=(3, 2) if kind == 'quad' else (2, 2, 2))
    _perturb(s, 7)
    x1 = s.eles_scal_upts_inb_full[0] * 1.5
    x2 = s.eles_scal_upts_inb_full[0] * 0.5
    s.updatebc(0.0, 0, 1)
    outs = []
    for eng in (1, 0):                  # tensor cores, CUDA cores
        s.ele.struct.engine = eng
        o = torch.empty_like(x1)
        s._active = (0, 1)
        s._fused_rhs(a=0.5, b=2.0, x1=x1, c1=0.25, x2=x2, c2=-0.5, out=o)
        outs.append(o)
    s.ele.struct.engine = 0
    torch.cuda.synchronize()
    # 3xTF32 keeps ~22 significant bits per product; the residual is a sum with
    # cancellation: within the FP32 tolerance of the FR parity tests
    assert rel_l2(outs[0].double().cpu().numpy(), outs[1].double().cpu().numpy()) < 2e-5


@pytest.mark.parametrize('kind,order,prec', [('quad', 3, 'single'), ('hex', 2, 'single'),
                                             ('hex', 2, 'double')])
def test_gather_rhs_equals_disu_rhs(cuda, kind, order, prec):
    """GLL flux points: bdgfs_fr_bc_update_gather / bdgfs_fr_rhs_gather read
    the face values from the state itself and give bitwise the results of
    bdgfs_fr_disu + bdgfs_fr_bc_update + bdgfs_fr_rhs; the aliasing guard
    refuses out == u."""
    from frfs_b200 import _lib
    cfg, be, mesh, s = _system(kind, order, prec)
    assert s.ele.fsel is not None
    _perturb(s, 11)
    u = s.eles_scal_upts_inb_full[0]
    x1, x2 = u * 1.5, u * 0.5
    s.updatebc(0.0, 0, 1)
    bc_ref = s.walls.bcv.clone()
    ref = torch.empty_like(u)
    L, fsel = _lib.lib(), s.ele.fsel.data_ptr()
    _lib.check(L.bdgfs_fr_rhs(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), u.data_ptr(),
                              s._uf_rows.data_ptr(), ref.data_ptr(), 0.5, 2.0, x1.data_ptr(), 0.25,
                              x2.data_ptr(), -0.5, _lib.stream_ptr()), 'rhs')
    s.walls.bcv.zero_()
    _lib.check(L.bdgfs_fr_bc_update_gather(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel,
                                           u.data_ptr(), _lib.stream_ptr()), 'bc_update_gather')
    out = torch.empty_like(u)
    _lib.check(L.bdgfs_fr_rhs_gather(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel,
                                     u.data_ptr(), out.data_ptr(), 0.5, 2.0, x1.data_ptr(), 0.25,
                                     x2.data_ptr(), -0.5, _lib.stream_ptr()), 'rhs_gather')
    torch.cuda.synchronize()
    assert torch.equal(s.walls.bcv, bc_ref)
    assert torch.equal(out, ref)
    assert L.bdgfs_fr_rhs_gather(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel,
                                 u.data_ptr(), u.data_ptr(), 0.5, 2.0, None, 0.0, None, 0.0,
                                 _lib.stream_ptr()) == -1


def test_stepper_gather_path_equals_disu_path(cuda):
    """Two SSP-RK2 steps through the gather path (the default for one part
    and GLL points) equal the same steps with the face-value array."""
    outs = []
    for gather in (True, False):
        cfg, be, mesh, s = _system('hex', 2, 'single')
        _perturb(s, 3)
        if not gather:
            s.ele.fsel = None
        integ = get_integrator(be, s, cfg)
        for _ in range(2):
            integ.step(integ.tcurr, 1e-4)
            integ.tcurr += 1e-4
        torch.cuda.synchronize()
        outs.append(s.eles_scal_upts_inb_full[0].clone())
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize('kind,order,prec,tol', [('quad', 3, 'single', 2e-6), ('hex', 2, 'single', 2e-6),
                                                 ('hex', 2, 'double', 1e-13), ('quad', 2, 'double', 1e-13),
                                                 ('hex', 1, 'single', 1e-5), ('hex', 1, 'double', 1e-13)])
def test_tensor_factored_rhs_matches_dense(cuda, kind, order, prec, tol):
    """The factored residual R = M1 F~ + M3 (F^n - M2 F~) of
    bdgfs_fr_rhs_tensor against bdgfs_fr_rhs_gather (dense M1 - M3 M2):
    equal to rounding, with walls and the RK combination operands."""
    from frfs_b200 import _lib
    cfg, be, mesh, s = _system(kind, order, prec)
    assert s.ele.tensor is not None
    _perturb(s, 13)
    u = s.eles_scal_upts_inb_full[0]
    x1, x2 = u * 1.5, u * 0.5
    s.updatebc(0.0, 0, 1)
    L, fsel = _lib.lib(), s.ele.fsel.data_ptr()
    outs = []
    for tensor in (False, True):
        o = torch.empty_like(u)
        args = (u.data_ptr(), o.data_ptr(), 0.5, 2.0, x1.data_ptr(), 0.25, x2.data_ptr(), -0.5,
                _lib.stream_ptr())
        if tensor:
            rc = L.bdgfs_fr_rhs_tensor(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct),
                                       _lib.ref(s.ele.tensor), args[0], None, *args[1:])
        else:
            rc = L.bdgfs_fr_rhs_gather(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel, *args)
        _lib.check(rc, 'rhs')
        outs.append(o)
    o = torch.empty_like(u)
    s._disu()
    _lib.check(L.bdgfs_fr_rhs_tensor(_lib.ref(s.ele.struct), _lib.ref(s.walls.struct),
                                     _lib.ref(s.ele.tensor), u.data_ptr(), s._uf_rows.data_ptr(),
                                     o.data_ptr(), 0.5, 2.0, x1.data_ptr(), 0.25, x2.data_ptr(), -0.5,
                                     _lib.stream_ptr()), 'rhs_tensor_face_array')
    torch.cuda.synchronize()
    assert torch.equal(o, outs[1])          # face array or gather: the same arithmetic
    # the residual part only: out - (a u + c1 x1 + c2 x2) = b L(u)
    base = 0.5 * u + 0.25 * x1 - 0.5 * x2
    la, lb = (outs[0] - base).double(), (outs[1] - base).double()
    assert float((la - lb).norm() / la.norm()) < tol


def test_nancheck_plugin_detects_injected_nan(cuda):
    """[soln-plugin-nancheck] nsteps: a clean run passes; a NaN written into
    the state on the host side is caught by the device status word at the
    next check (plugins/nancheck.py:17-22), with RuntimeError."""
    cfg, be, mesh, s = _system('quad', 2, 'single')
    cfg.set('soln-plugin-nancheck', 'nsteps', '1')
    integ = get_integrator(be, s, cfg)
    integ.advance_to(2 * 5e-4)
    assert integ.nacptsteps == 2
    integ.soln[1, 3, 17] = float('nan')
    with pytest.raises(RuntimeError, match='NaNs detected'):
        integ.advance_to(3 * 5e-4)


@pytest.mark.parametrize('kind,order,prec,tol', [('quad', 2, 'double', 1e-14), ('quad', 3, 'single', 1e-6),
                                                 ('hex', 2, 'single', 1e-6), ('hex', 2, 'double', 1e-14)])
def test_invmass_equals_reference_operator(cuda, kind, order, prec, tol):
    """system.invmass (solvers/dgfs/system.py:221-231): out = M12 u per
    element with the reference's own M12 (frfs/shapes.py:163-166, golden
    fixture); the banks must differ."""
    from frfs_b200._lib import BdgfsError
    cfg, be, mesh, s = _system(kind, order, prec)
    _perturb(s, 3)
    m12 = np.load(f'{GOLD}/shapes_{kind}_p{order}.npz')['M12']
    s.invmass(0, 1)
    torch.cuda.synchronize()
    u = s.eles_scal_upts_inb_full[0].double().cpu().numpy()
    want = np.einsum('ij,ejv->eiv', m12, u)
    got = s.eles_scal_upts_inb_full[1].double().cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < tol
    with pytest.raises(BdgfsError):
        s.invmass(0, 0)
