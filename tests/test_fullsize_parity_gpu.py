"""Parity of the CUDA path with the FP64 oracle at the full workload sizes.

* 4x4 periodic quads P2, Nv=16, hard spheres, Nrho=8, M=6, two seeded
  Maxwellians per DOF: 10 dgfs-tvd-rk2 steps in FP64 on the whole mesh
  against the oracle stepper (reference algorithm, no projection).
* Couette, 16x8 quads P3, Nv=24, M=Nrho=12, FP32, and the lid-driven cavity,
  8^3 hexes P2, same velocity settings: one dgfs-tvd-rk2 step.  Each stage's
  output is checked at 128 seeded DOFs against the oracle's stage built from
  the GPU's own stage input (FR operator on the whole mesh, Q of the sampled
  DOFs followed by the launch's FP64 conservation projection); the stage's Q
  is checked on its own at the same DOFs.
* The two-grid batched collision launch (24576 distributions on 24^3, 8192
  on 32^3, mass ratio 2, Nrho=16, M=12) against the oracle on 256 seeded
  distributions of each grid.

Reference path: frfs/integrators/std/steppers.py:122-225 and
frfs/solvers/dgfs/scattering.py:227-286.  The oracle runs on the host cores
in a spawned process pool.
"""
import numpy as np
import pytest
import torch

from frfs_b200.backend import CUDABackend
from frfs_b200.integrators import get_integrator
from frfs_b200.mesh import StructuredMesh
from frfs_b200.system import DGFSSystem

from helpers import NONDIM, couette_cfg, rel_l2
from oracle_pool import OraclePool, grid_entry, project

pytestmark = pytest.mark.gpu

GOLD = __import__('os').path.join(__import__('os').path.dirname(__file__), 'golden')

# FP32 tolerances (relative L2 against the FP64 oracle)
TOL_Q32 = 1e-3          # the collision operator at the sampled DOFs
TOL_STAGE32 = 2e-3      # the stage increment (u_stage - combination) / dt at those DOFs
TOL_U32 = 1e-6          # the stage output itself


def _fr_oracle(s, kind, order):
    from oracle.fr import FROracle
    g = np.load(f'{GOLD}/shapes_{kind}_p{order}.npz')
    walls, rows = s.walls.oracle_walls()
    return FROracle({'M0': g['M0'], 'M132': g['M132'], 'M3': g['M3']}, s.geo, s.vm.c0(),
                    s.vm.cw(), walls, bcid=rows)


def _u0():
    return np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])


# ---------------------------------------------------------------------------
# 4x4 periodic quads P2, Nv = 16, FP64, 10 steps on the whole mesh
# ---------------------------------------------------------------------------

def _two_maxwellians(cv, rng, shape):
    """Per DOF: sum of 2 Maxwellians, n ~ U(0.5, 1.5), |u| < 0.5 (uniform in
    the ball), T ~ U(0.7, 1.3)."""
    F = np.empty(shape + (cv.shape[1],))
    for idx in np.ndindex(*shape):
        f = 0.0
        for _ in range(2):
            d = rng.normal(size=3)
            d = d / np.linalg.norm(d) * 0.5 * rng.uniform()**(1 / 3)
            T = rng.uniform(0.7, 1.3)
            f = f + rng.uniform(0.5, 1.5) / (np.pi * T)**1.5 * np.exp(
                -np.sum((cv - d[:, None])**2, axis=0) / T)
        F[idx] = f
    return F


def test_periodic_quad_p2_nv16_fp64_ten_steps(cuda):
    from oracle.fr import step_rk2
    cfg = couette_cfg(16, 8, 6, 5, 2, precision='double', omega=0.5, dt=1e-3)
    be = CUDABackend(cfg)
    mesh = StructuredMesh((4, 4), (0.0, 0.0), (1.0, 1.0), periodic='xy')
    s = DGFSSystem(be, mesh, cfg, nreg=3)
    u = s.eles_scal_upts_inb_full[0]
    assert tuple(u.shape[:2]) == (16, 9)          # 144 DOFs
    F = _two_maxwellians(s.vm.cv(), np.random.default_rng(11), tuple(u.shape[:2]))
    u.copy_(torch.from_numpy(F))
    s.sm._project = False                         # the reference algorithm has none
    integ = get_integrator(be, s, cfg)
    orc = _fr_oracle(s, 'quad', 2)
    dt, nsteps = 1e-3, 10
    E, J, n = F.shape
    with OraclePool({'g': grid_entry(s.vm, 0.5)}) as pool:
        Q = lambda x: pool.Q('g', x.reshape(E * J, n)).reshape(E, J, n)
        uo = F.copy()
        for _ in range(nsteps):
            uo = step_rk2(uo, dt, orc.rhs, Q)
            integ.step(integ.tcurr, dt)
            integ.tcurr += dt
    got = s.eles_scal_upts_inb_full[0].cpu().numpy()
    assert np.isfinite(got).all()
    err = rel_l2(got, uo)
    print(f'10 FP64 steps, 144 DOFs: rel L2 {err:.2e}')
    assert err < 1e-11
    # the steps moved the state well above the tolerance
    assert rel_l2(F, uo) > 1e-4


# ---------------------------------------------------------------------------
# one SSP-RK2 step at full size, stage outputs at 128 seeded DOFs (FP32)
# ---------------------------------------------------------------------------

def _smooth_state(s, rng):
    """Two Maxwellians per DOF with smooth seeded spatial fields (non-
    equilibrium, so Q and the FR operator are both non-trivial)."""
    cv = s.vm.cv()
    x = s.geo.plocupts                                  # (E, nupts, ndims)
    ph = rng.uniform(0, 2 * np.pi, size=4)
    X = x[..., 0]
    Y = x[..., 1]
    Z = x[..., 2] if x.shape[-1] > 2 else 0.0 * X
    out = np.empty(x.shape[:2] + (cv.shape[1],), dtype=np.float32)
    for e in range(x.shape[0]):
        for j in range(x.shape[1]):
            xx, yy, zz = X[e, j], Y[e, j], Z[e, j]
            n1 = 1.0 + 0.2 * np.sin(2 * np.pi * xx + ph[0]) * np.cos(np.pi * yy)
            u1 = np.array([0.2 * np.sin(np.pi * yy + ph[1]), 0.1 * np.cos(2 * np.pi * xx), 0.05 * np.sin(2 * np.pi * zz)])
            T1 = 1.0 + 0.1 * np.sin(2 * np.pi * xx + ph[2])
            n2 = 0.3 * (1.0 + 0.5 * np.cos(2 * np.pi * xx + np.pi * yy + ph[3]))
            u2 = np.array([-0.3, 0.2 * np.sin(np.pi * yy), 0.1])
            T2 = 0.8
            f = (n1 / (np.pi * T1)**1.5 * np.exp(-np.sum((cv - u1[:, None])**2, axis=0) / T1)
                 + n2 / (np.pi * T2)**1.5 * np.exp(-np.sum((cv - u2[:, None])**2, axis=0) / T2))
            out[e, j] = f
    return out


def _stage_parity(s, kind, order, dt, vsel=None, ndof_check=128, seed=3):
    """One dgfs-tvd-rk2 step through the graph-captured stepper, each stage
    against the oracle stage built from the GPU's stage input."""
    bank = s.eles_scal_upts_inb_full
    E, J, n = bank[0].shape
    rng = np.random.default_rng(seed)
    bank[0].copy_(torch.from_numpy(_smooth_state(s, rng)))
    pick = np.sort(rng.choice(E * J, size=ndof_check, replace=False))
    pe, pj = pick // J, pick % J
    c0 = s.vm.c0().astype(np.float64)
    orc = _fr_oracle(s, kind, order)
    sub = orc if vsel is None else orc.restrict(vsel)
    cols = slice(None) if vsel is None else vsel

    def oracle_L(u):
        bc = orc.update_bc_from_state(u)
        return sub.rhs(u if vsel is None else u[:, :, vsel], bc=bc)

    u0 = bank[0].cpu().numpy()                         # FP32 host copies (exact in FP64)
    s.collide(0.0, 0, 2)                               # Q(u0), the launch stage 1 makes
    q1 = bank[2].double().cpu().numpy()[pe, pj]
    integ = get_integrator(s.backend, s, s.cfg)
    integ.step(0.0, dt)                                # r1 = u1, r2 = Q(u1), r0 = u_new
    torch.cuda.synchronize()
    u1 = bank[1].cpu().numpy()
    q2 = bank[2].double().cpu().numpy()[pe, pj]
    u2 = bank[0].cpu().numpy()
    res = {}
    with OraclePool({'g': grid_entry(s.vm, 0.81)}) as pool:
        Qo1 = project(pool.Q('g', u0[pe, pj].astype(np.float64)), c0)
        Qo2 = project(pool.Q('g', u1[pe, pj].astype(np.float64)), c0)
    res['q1'] = rel_l2(q1, Qo1)
    res['q2'] = rel_l2(q2, Qo2)
    L1 = oracle_L(u0)[pe, pj]
    L2 = oracle_L(u1)[pe, pj]
    # stage 1: u1 = u0 + dt (L + Q)(u0)
    u0, u1, u2 = (x[pe, pj].astype(np.float64) for x in (u0, u1, u2))
    inc1 = (u1[:, cols] - u0[:, cols]) / dt
    ref1 = L1 + Qo1[:, cols]
    res['stage1_inc'] = rel_l2(inc1, ref1)
    res['stage1_u'] = rel_l2(u1[:, cols], u0[:, cols] + dt * ref1)
    # stage 2: u_new = u0/2 + u1/2 + dt/2 (L + Q)(u1)
    base = 0.5 * u0[:, cols] + 0.5 * u1[:, cols]
    inc2 = (u2[:, cols] - base) / (0.5 * dt)
    ref2 = L2 + Qo2[:, cols]
    res['stage2_inc'] = rel_l2(inc2, ref2)
    res['stage2_u'] = rel_l2(u2[:, cols], base + 0.5 * dt * ref2)
    res['L_share'] = float(np.linalg.norm(L1) / np.linalg.norm(ref1))
    print(kind, {k: f'{v:.2e}' for k, v in res.items()})
    assert res['q1'] < TOL_Q32 and res['q2'] < TOL_Q32, res
    assert res['stage1_inc'] < TOL_STAGE32 and res['stage2_inc'] < TOL_STAGE32, res
    assert res['stage1_u'] < TOL_U32 and res['stage2_u'] < TOL_U32, res
    return res


def test_couette_16x8_p3_nv24_stage_parity(cuda):
    cfg = couette_cfg(24, 12, 12, 6, 3, precision='single', uw=0.3, dt=5e-4)
    be = CUDABackend(cfg)
    mesh = StructuredMesh((16, 8), (0.0, -0.5), (2.0, 0.5), periodic='x')
    s = DGFSSystem(be, mesh, cfg, nreg=3)
    assert s.eles_scal_upts_inb_full[0].shape[0] * s.eles_scal_upts_inb_full[0].shape[1] == 2048
    _stage_parity(s, 'quad', 3, 5e-4)


def test_lid_cavity_8cube_hex_p2_stage_parity(cuda):
    from helpers import vhs_cfg
    rho0, T0 = NONDIM['rho0'], NONDIM['T0']
    walls = ''.join(f"""
[soln-bcs-{name}]
type = dgfs-wall-diffuse
rho = {rho0}
T = {T0}
ux = {ux}
uy = 0
uz = 0
""" for name, ux in (('lid', 0.5 * _u0()), ('walls', 0.0)))
    cfg = vhs_cfg(24, 12, 12, 6, precision='single', extra=f"""
[solver]
system = dgfs
order = 2
[solver-time-integrator]
scheme = dgfs-tvd-rk2
controller = none
tstart = 0.0
tend = 1.0
dt = 2e-4
[soln-ics]
type = maxwellian
rho = {rho0}
T = {T0}
ux = 0
uy = 0
uz = 0
{walls}""")
    be = CUDABackend(cfg)
    names = {'x-': 'walls', 'x+': 'walls', 'y-': 'walls', 'y+': 'lid', 'z-': 'walls',
             'z+': 'walls'}
    mesh = StructuredMesh((8, 8, 8), (0, 0, 0), (1, 1, 1), periodic='', bcnames=names)
    s = DGFSSystem(be, mesh, cfg, nreg=3)
    assert s.eles_scal_upts_inb_full[0].shape[0] * s.eles_scal_upts_inb_full[0].shape[1] == 13824
    # the FR operator of the oracle on 512 seeded velocities (velocities are
    # independent there; the wall sums use all of them), Q on all
    vsel = np.sort(np.random.default_rng(5).choice(s.vm.vsize(), size=512, replace=False))
    _stage_parity(s, 'hex', 2, 2e-4, vsel=vsel)


# ---------------------------------------------------------------------------
# the two-grid batched launch, 256 seeded distributions per grid
# ---------------------------------------------------------------------------

def test_batched_two_grid_launch_256_per_grid(cuda):
    from frfs_b200.scattering import VHSCollider, VHSGrid, vhs_prefactor
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    from helpers import mixed_maxwellians, vhs_cfg
    sizes, masses = {24: 24576, 32: 8192}, {24: 1.0, 32: 2.0}
    rng = np.random.default_rng(8)
    grids, fs, qs, picks, entries, c0s = [], [], [], {}, {}, {}
    for Nv in (24, 32):
        cfg = vhs_cfg(Nv, 16, 12, 6, precision='single')
        be = CUDABackend(cfg)
        vm = DGFSVelocityMesh(be, cfg)
        gam, pref, _ = vhs_prefactor(vm, 0.81, 4.17e-10, NONDIM['T0'], mass=masses[Nv])
        grids.append(VHSGrid(Nv, vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(), gam, pref, vm.cw(),
                             vm.c0(), torch.float32, be.device))
        scale = pref / vhs_prefactor(vm, 0.81, 4.17e-10, NONDIM['T0'], mass=1.0)[1]
        entries[Nv] = grid_entry(vm, 0.81, scale)
        c0s[Nv] = vm.c0().astype(np.float64)
        # 64 seeded cubes tiled to the full count, then 256 seeded positions
        # overwritten by 256 further distinct cubes: the checked rows
        cv = vm.cv()
        base = np.stack([mixed_maxwellians(cv, rng) for _ in range(64)]).astype(np.float32)
        f = torch.from_numpy(base).to(cuda).repeat(sizes[Nv] // 64, 1).contiguous()
        picks[Nv] = np.sort(rng.choice(sizes[Nv], size=256, replace=False))
        chk = np.stack([mixed_maxwellians(cv, rng) for _ in range(256)]).astype(np.float32)
        f[torch.from_numpy(picks[Nv]).to(cuda)] = torch.from_numpy(chk).to(cuda)
        fs.append(f)
        qs.append(torch.full_like(f, float('nan')))
    col = VHSCollider(grids, cuda)
    col([(1, fs[1], qs[1], None), (0, fs[0], qs[0], None)], project=True)
    torch.cuda.synchronize()
    for q in qs:
        assert bool(torch.isfinite(q).all())
    errs = {}
    with OraclePool({f'{Nv}': entries[Nv] for Nv in (24, 32)}) as pool:
        for gi, Nv in enumerate((24, 32)):
            F = fs[gi][torch.from_numpy(picks[Nv]).to(cuda)].double().cpu().numpy()
            Qo = project(pool.Q(f'{Nv}', F), c0s[Nv])
            Qg = qs[gi][torch.from_numpy(picks[Nv]).to(cuda)].double().cpu().numpy()
            errs[Nv] = rel_l2(Qg, Qo)
    print('batched two-grid launch, 256 per grid:', errs)
    for Nv, e in errs.items():
        assert e < TOL_Q32, (Nv, e)
