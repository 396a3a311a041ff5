"""Benchmark: DG time steps/s of the DGFS Couette workload on B200.

Workload (the configuration the headline metric is quoted on): 2-D mesh of
16 x 8 quadrilaterals at P = 3 (2048 DOFs), Nv = 24^3 velocities on
[-6, 6]^3, VHS omega = 0.81, Nrho = 12, M = 12, diffuse walls at y = -+0.5
moving at -+0.3 with T = 1, initial Maxwellian n = 1, T = 1, SSP-RK2
(dgfs-tvd-rk2), dt = 5e-4, FP32 state, FP64 moments/projection.  A step is
one full DG time step (two collision-operator evaluations of every DOF plus
two FR advection stages), captured as one CUDA graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun with N ranks the channel is N times longer, each rank owns
one 16 x 8 slab (2048 DOFs, the single-GPU workload) and neighbouring slabs
exchange face values over NCCL every stage (weak scaling); value = N *
steps / the slowest rank's device time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NONDIM = dict(T0=273.0, H0=1e-3, rho0=0.00011140244750324529, molarMass0=39.96e-3)
WORK = dict(Nv=24, Nrho=12, M=12, dev=6, omega=0.81, order=3, nx=16, ny=8,
            uw=0.3, dt=5e-4)
METRIC = 'DG steps/s and Q evals/s: plain FP64 vs FP32 batched vs surrogate at stated L2 err'


def couette_ini(precision='single', w=WORK):
    import numpy as np
    u0 = np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])
    rho0, T0 = NONDIM['rho0'], NONDIM['T0']
    walls = ''.join(f"""
[soln-bcs-{name}]
type = dgfs-wall-diffuse
rho = {rho0}
T = {T0}
ux = {sgn * w['uw'] * u0}
uy = 0
uz = 0
""" for name, sgn in (('y-', -1), ('y+', 1)))
    return f"""
[backend]
precision = {precision}
[constants]
Nv = {w['Nv']}
Nrho = {w['Nrho']}
[non-dim]
T0 = {T0}
H0 = {NONDIM['H0']}
rho0 = {rho0}
molarMass0 = {NONDIM['molarMass0']}
[velocity-mesh]
dev = {w['dev']}
cmax = 0
Tmax = {T0}
[spherical-design-rule]
ssrule = womersley
M = {w['M']}
[scattering-model]
type = vhs-gll
omega = {w['omega']}
dRef = 4.17e-10
Tref = {T0}
[solver]
system = dgfs
order = {w['order']}
[solver-time-integrator]
scheme = dgfs-tvd-rk2
controller = none
tstart = 0.0
tend = 0.1
dt = {w['dt']}
[soln-ics]
type = maxwellian
rho = {rho0}
T = {T0}
ux = 0
uy = 0
uz = 0
{walls}"""


def q_flops_per_eval(Nv, Nrho, M):
    """Algorithmic FLOP of one collision-operator evaluation (packed
    algorithm): (M*Nrho + Nrho + 2) complex FFTs at 5 n log2 n plus the
    per-(p,q) multiplier/product work 8 n, n = Nv^3."""
    import math
    n = Nv**3
    return (M * Nrho + Nrho + 2) * 5.0 * n * math.log2(n) + 8.0 * M * Nrho * n


def q_flops_reference_equivalent(Nv, Nrho, M):
    """FLOP of the reference's own evaluation of one Q (scattering.py:
    239-281): 3 M Nrho + 3 complex FFTs at 5 n log2 n, n = Nv^3.  Reported
    beside the roofline only as context; the roofline uses the packed count."""
    import math
    n = Nv**3
    return (3 * M * Nrho + 3) * 5.0 * n * math.log2(n)


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()

    def start(self):
        q = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
             'clocks_event_reasons.sw_power_cap')
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '-i', str(self.index), f'--query-gpu={q}',
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def stop(self):
        if self.proc is None:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        import statistics
        sm = [float(r[0]) for r in self.rows if len(r) >= 7 and r[0].replace('.', '').isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 7 and r[1].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[k] for r in self.rows if len(r) >= 7
                          for k in range(4) if r[3 + k].lower() == 'active'})
        return {'sm_mhz': statistics.median(sm) if sm else None,
                'sm_max_mhz': max(mx) if mx else None, 'reasons': reasons,
                'samples': len(sm)}


def dist_init():
    import torch
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        backend = 'nccl' if torch.cuda.is_available() else 'gloo'
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return ws, rank, local


def reduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64,
                     device='cuda' if torch.cuda.is_available() else 'cpu')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- CPU legs
_ORC = None


def _oracle_init(Nv, Nrho, sz, dev, omega):
    """Pool initializer: build the reference-algorithm tables once per worker."""
    global _ORC
    sys.path.insert(0, ROOT)
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import VHSOracle
    vm = VelocityMesh(Nv, Nrho, sz, cmax=0.0, Tmax=NONDIM['T0'], dev=dev, **NONDIM)
    _ORC = VHSOracle(vm, omega, 4.17e-10, NONDIM['T0'])


def _oracle_q_worker(F):
    import numpy as np
    if len(F) == 0:
        return np.zeros((0, 0))
    return np.stack([_ORC.Q(f) for f in F])


def _oracle_init_multi(grids):
    """Pool initializer: one reference-algorithm oracle per (key, Nv, Nrho, sz,
    dev, omega, scale) entry; scale multiplies Q (species mass)."""
    global _ORCS
    sys.path.insert(0, ROOT)
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import VHSOracle
    _ORCS = {}
    for key, Nv, Nrho, sz, dev, omega, scale in grids:
        vm = VelocityMesh(Nv, Nrho, sz, cmax=0.0, Tmax=NONDIM['T0'], dev=dev, **NONDIM)
        _ORCS[key] = (VHSOracle(vm, omega, 4.17e-10, NONDIM['T0']), scale)


def _oracle_q_keyed(item):
    import numpy as np
    key, F = item
    orc, scale = _ORCS[key]
    if len(F) == 0:
        return key, np.zeros((0, orc.vm.vsize))
    return key, np.stack([scale * orc.Q(f) for f in F])


def batched_q_error(arrays, per_grid=64, seed=5, counts=None):
    """Relative L2 error of the batched launch's Q against the FP64 reference
    algorithm on a seeded sample of per_grid distributions of each grid
    (host cores, spawned pool), and the host cores' Q evaluations per second
    for the workload's mix of grids (counts: distributions per grid),
    timed per grid on that sample and extrapolated."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    import numpy as np
    from frfs_b200.scattering import vhs_prefactor
    from frfs_b200.sphericaldesign import half_sphere_design
    grids, fs, qs = arrays
    w = BATCHED
    rng = np.random.default_rng(seed)
    cfgs, items, picks = [], {}, {}
    for gi, (g, mass) in enumerate(zip(grids, (1.0, w['mass2']))):
        key = f'Nv{g.Nv}'
        from frfs_b200.inifile import Inifile
        from frfs_b200.velocitymesh import DGFSVelocityMesh
        from frfs_b200.backend import CUDABackend
        cfg = Inifile(couette_ini('single', dict(WORK, Nv=g.Nv, Nrho=w['Nrho'], M=w['M'])))
        vm = DGFSVelocityMesh(CUDABackend(cfg), cfg)
        scale = (vhs_prefactor(vm, w['omega'], 4.17e-10, NONDIM['T0'], mass=mass)[1]
                 / vhs_prefactor(vm, w['omega'], 4.17e-10, NONDIM['T0'], mass=1.0)[1])
        cfgs.append((key, g.Nv, w['Nrho'], half_sphere_design(w['M']), WORK['dev'], w['omega'], scale))
        idx = np.sort(rng.choice(fs[gi].shape[0], size=per_grid, replace=False))
        picks[key] = (gi, idx)
        F = fs[gi][idx].double().cpu().numpy()
        items[key] = [(key, c) for c in np.array_split(F, per_grid)]
    ncores = min(os.cpu_count() or 1, per_grid)
    err, secs = {}, {}
    with ProcessPoolExecutor(max_workers=ncores, mp_context=mp.get_context('spawn'),
                             initializer=_oracle_init_multi, initargs=(cfgs,)) as pool:
        list(pool.map(_oracle_q_keyed, [(cfgs[0][0], []) for _ in range(ncores)]))  # start
        for key, (gi, idx) in picks.items():
            t0 = time.perf_counter()
            outs = list(pool.map(_oracle_q_keyed, items[key]))
            secs[key] = (time.perf_counter() - t0) / per_grid       # wall s per Q, all cores
            Qo = np.concatenate([q for _, q in outs])
            # the same conservation projection as the kernel, applied in FP64
            c0 = grids[gi].c0.double().cpu().numpy()
            cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
            Phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
            lam = np.linalg.solve(Phi @ Phi.T, Phi @ Qo.T)
            Qo = Qo - (Phi.T @ lam).T
            Qg = qs[gi][idx].double().cpu().numpy()
            err[key] = float(np.linalg.norm(Qg - Qo) / np.linalg.norm(Qo))
    cpu = None
    if counts is not None:
        keys = list(picks)
        t = sum(counts[i] * secs[k] for i, k in enumerate(keys))
        cpu = {'value': sum(counts) / t, 'unit': 'Q evals/s', 'cores': ncores, 'kind': 'port',
               'sample': (f'{per_grid} seeded distributions of each grid (reference algorithm, '
                          '3+3*M*Nrho FP64 FFTs each, spread over the host cores), wall time '
                          'per distribution extrapolated to the workload mix '
                          f'{dict(zip(keys, counts))}')}
    return err, cpu


def make_pool(ncores, Nv, Nrho, sz, dev, omega):
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    pool = ProcessPoolExecutor(max_workers=ncores, mp_context=mp.get_context('spawn'),
                               initializer=_oracle_init, initargs=(Nv, Nrho, sz, dev, omega))
    list(pool.map(_oracle_q_worker, [[] for _ in range(ncores)]))   # start workers
    return pool


def cpu_reference_step_time(F_sample, fr_state, ndof_total, pool, ncores):
    """Time of one full DG step of the reference algorithm on the host cores,
    from a bounded sample: Q of the sample DOFs spread over the pool (wall
    time), and the FR operator on the full mesh."""
    import numpy as np
    chunks = [c for c in np.array_split(F_sample, ncores) if len(c)]
    t0 = time.perf_counter()
    outs = list(pool.map(_oracle_q_worker, chunks))
    tq = time.perf_counter() - t0
    Q = np.concatenate(outs)
    orc_fr, u = fr_state
    t1 = time.perf_counter()
    orc_fr.rhs(u)
    tfr = time.perf_counter() - t1
    # per step: 2 stages x (Q over all DOFs + one FR operator)
    t_step = 2.0 * (tq * ndof_total / len(F_sample) + tfr)
    return t_step, Q, tq, tfr


def make_fr_oracle(system):
    import numpy as np
    from oracle.fr import FROracle
    shp = system.geo.shape
    ops = {'M0': shp.opmat('M0'), 'M132': shp.opmat('M1 - M3*M2'), 'M3': shp.opmat('M3')}
    walls, rows = system.walls.oracle_walls()
    return FROracle(ops, system.geo, system.vm.c0(), system.vm.cw(), walls, bcid=rows)


def _oracle_gl_worker(F):
    """(Q, loss term) of the reference algorithm for each row of F."""
    import numpy as np
    if len(F) == 0:
        return np.zeros((0, 0)), np.zeros((0, 0))
    out = [_ORC.gain_loss(f) for f in F]
    return (np.stack([g - l for g, l in out]), np.stack([l for _, l in out]))


def upt_weights(geo):
    """Quadrature weight x |J| of every solution point, [E * nupts] (the
    tensor-product GLL rule of the element's solution points)."""
    import numpy as np
    shp = geo.shape
    pts, wts = np.asarray(shp.pts1), np.asarray(shp.wts1)
    w = np.prod([wts[np.argmin(np.abs(pts[None, :] - shp.upts[:, d:d + 1]), axis=1)]
                 for d in range(shp.upts.shape[1])], axis=0)
    return (geo.djac * w[None, :]).reshape(-1)


def state_totals(system, bank):
    """Mesh integrals, in FP64, of the mass, momentum and energy (sum of
    |c|^2 f cw) of a solution bank."""
    import torch
    from frfs_b200.system import raw_moments
    m = raw_moments(system.eles_scal_upts_inb_full[bank], system.vm)
    dens = torch.stack([m[:, 0], m[:, 1], m[:, 2], m[:, 3], m[:, 4] + m[:, 7] + m[:, 9]], 1)
    w = torch.as_tensor(upt_weights(system.geo), dtype=torch.float64, device=m.device)
    return (w[:, None] * dens).sum(0).cpu().numpy()


def drift(before, after, conserved=(0, 1, 2, 3, 4)):
    """Relative change of the conserved totals over one step: mass and
    energy relative to themselves, momentum relative to the mass (unit
    speed)."""
    out = {}
    names = ['mass', 'momentum_x', 'momentum_y', 'momentum_z', 'energy']
    for k in conserved:
        ref = abs(before[0]) if 1 <= k <= 3 else abs(before[k])
        out[names[k]] = float(abs(after[k] - before[k]) / ref)
    return out


def q_conservation(collide, f, q, c0, cw, chunk=2048):
    """Conservation of one collision launch over every distribution of f:
    the FP64 moments C.Q the launch reports before and after its projection
    (after: FP64, before the cast to the state's type) and the FP64 moments
    of the Q it wrote, each relative to C.|Q| (C = cw {1, c, |c|^2}); max
    over distributions and the five moments."""
    import torch
    n3 = c0.numel()**3
    f2, q2 = f.reshape(-1, n3), q.reshape(-1, n3)
    ndof = f2.shape[0]
    mom = torch.empty(ndof, 10, dtype=torch.float64, device=f.device)
    collide(f2, q2, mom)
    cx, cy, cz = torch.meshgrid(c0, c0, c0, indexing='ij')
    phi = torch.stack([torch.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
    worst = {'projected_fp64': 0.0, 'written': 0.0, 'unprojected': 0.0}
    for i0 in range(0, ndof, chunk):
        Q = q2[i0:i0 + chunk].double()
        scale = (Q.abs() @ phi.abs().T) * cw
        wr = (Q @ phi.T) * cw
        m = mom[i0:i0 + chunk]
        worst['projected_fp64'] = max(worst['projected_fp64'], float((m[:, 5:].abs() / scale).max()))
        worst['written'] = max(worst['written'], float((wr.abs() / scale).max()))
        worst['unprojected'] = max(worst['unprojected'], float((m[:, :5].abs() / scale).max()))
    return {'max_rel_' + k: v for k, v in worst.items()} | {
        'definition': 'max over distributions and moments of |cw sum phi Q| / (cw sum |phi| |Q|), '
                      'phi = {1, c, |c|^2}: FP64 sums of the launch before its projection '
                      '(unprojected), after it (projected_fp64, before the cast) and of the '
                      'FP32 Q it wrote'}


def run_reference(args):
    """--impl reference: the reference's algorithm (FP64 CPU restatement,
    oracle/) timed on all host cores; each step a bounded sample."""
    import numpy as np
    ws, rank, local = int(os.environ.get('WORLD_SIZE', '1')), int(os.environ.get('RANK', '0')), 0
    if rank != 0:
        return
    ncores = os.cpu_count() or 1
    from frfs_b200.inifile import Inifile
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    from frfs_b200.mesh import StructuredMesh, ElementGeometry
    from oracle.fr import FROracle
    cfg = Inifile(couette_ini('double'))
    vm = DGFSVelocityMesh(None, cfg)
    mesh = StructuredMesh((WORK['nx'], WORK['ny']), (0.0, -0.5), (2.0, 0.5), periodic='x')
    geo = ElementGeometry(mesh, WORK['order'])
    shp = geo.shape
    from frfs_b200.initcond import DGFSMaxwellianInitCondition
    walls = []
    for name in geo.wall_names:
        bc = DGFSMaxwellianInitCondition(None, cfg, vm, f'soln-bcs-{name}')
        walls.append((bc.unondim()[:, 0], bc.get_init_vals()))
    ic = DGFSMaxwellianInitCondition(None, cfg, vm, 'soln-ics').get_init_vals()
    u = np.broadcast_to(ic, (geo.neles, geo.nupts, vm.vsize())).copy()
    orc_fr = FROracle({'M0': shp.opmat('M0'), 'M132': shp.opmat('M1 - M3*M2'),
                       'M3': shp.opmat('M3')}, geo, vm.c0(), vm.cw(), walls)
    nsample = 8 * ncores
    rng = np.random.default_rng(0)
    F = u.reshape(-1, vm.vsize())[:nsample] * (1 + 0.01 * rng.uniform(-1, 1, (nsample, vm.vsize())))
    pool = make_pool(ncores, WORK['Nv'], WORK['Nrho'], vm.sz(), WORK['dev'], WORK['omega'])
    times = []
    for i in range(args.warmup + args.steps):
        t, _, tq, tfr = cpu_reference_step_time(F, (orc_fr, u), geo.neles * geo.nupts, pool,
                                                ncores)
        if i >= args.warmup:
            times.append(t)
    pool.shutdown()
    mean = sum(times) / len(times)
    v = 1.0 / mean
    sample = (f'{nsample} of {geo.neles * geo.nupts} DOFs for Q (3+3*M*Nrho FFTs each, '
              f'FP64 pocketfft) + FR operator on the full mesh, extrapolated per DOF to 1 step')
    line = {'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'DG steps/s',
            'n_gpus': args.gpus, 'steps': args.steps, 'warmup': args.warmup,
            'ms_per_step': mean * 1e3, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
            'config': config_block(args.gpus),
            'q_evals_per_s': geo.neles * geo.nupts * 2 / mean,
            'cpu_baseline': {'value': v, 'unit': 'DG steps/s', 'cores': ncores,
                             'kind': 'port', 'sample': sample},
            'e2e': {'value': v, 'unit': 'DG steps/s', 'h2d_bytes_per_step': 0,
                    'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def config_block(n):
    return {'workload': ('couette-2d: 16x8 quads P3 (2048 DOFs), Nv=24^3 on [-6,6]^3, '
                         'VHS omega=0.81, Nrho=12, M=12, diffuse walls +-0.3, SSP-RK2 dt=5e-4'),
            'ndof': 2048, 'Nv': 24, 'Nrho': 12, 'M': 12, 'order': 3, 'mesh': [16, 8],
            'parallelism': (f'{n} slabs of a {16 * n}x8 channel, NCCL face-value halo '
                            'exchange per stage (weak scaling)') if n > 1 else 'single GPU',
            'l2': 'flushed before every timed step (256 MiB write); step working set 452 MB > L2'}


# ---------------------------------------------------------------- other configs
BATCHED = dict(n24=24576, n32=8192, Nrho=16, M=12, dev=6, omega=0.81, mass2=2.0)
# DRAM bytes (read + write) of one collision launch on the 2048-DOF Couette
# state, from an ncu capture of the tuner's Nv=24 variant (the balanced
# packed variant with the z-pass spectra in tensor memory: 114.2 MB + 93.5 MB)
Q_LAUNCH_DRAM_BYTES = 114.22e6 + 93.46e6
SMALL64 = dict(Nv=16, Nrho=8, M=6, dev=5, omega=0.5, order=2, nx=4, ny=4, dt=1e-3)


def batched_q(flush, reps=3, sizes=None):
    """Two species on uneven grids (24^3 and 32^3, mass ratio 2) in one
    persistent launch captured in a CUDA graph; returns Q evals/s and the
    FP32 arrays for the error check.  sizes: (n24, n32) instead of the
    workload's (profiling case)."""
    import numpy as np
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.scattering import VHSGrid, VHSCollider, vhs_prefactor
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    from frfs_b200.autotune import tune_vhs
    w = dict(BATCHED)
    if sizes is not None:
        w['n24'], w['n32'] = sizes
    grids, fs = [], []
    gen = torch.Generator(device='cuda').manual_seed(7)
    for Nv, ndof, mass in ((24, w['n24'], 1.0), (32, w['n32'], w['mass2'])):
        cfg = Inifile(couette_ini('single', dict(WORK, Nv=Nv, Nrho=w['Nrho'], M=w['M'])))
        be = CUDABackend(cfg)
        vm = DGFSVelocityMesh(be, cfg)
        gam, pref, _ = vhs_prefactor(vm, w['omega'], 4.17e-10, NONDIM['T0'], mass=mass)
        g = VHSGrid(Nv, vm.L(), vm.qz(), vm.qw(), vm.sz(), vm.sw(), gam, pref, vm.cw(), vm.c0(),
                    torch.float32, be.device)
        grids.append(g)
        # seeded sums of 1-3 Maxwellians (n ~ U(0.2,2), |u| < 1, T ~ U(0.5,2)) + 1% noise,
        # generated on the device from per-distribution parameters
        c0 = torch.as_tensor(vm.c0(), dtype=torch.float32, device=be.device)
        cx, cy, cz = c0.view(-1, 1, 1), c0.view(1, -1, 1), c0.view(1, 1, -1)
        f = torch.zeros(ndof, Nv, Nv, Nv, device=be.device)
        k = torch.randint(1, 4, (ndof,), generator=gen, device=be.device)
        for j in range(3):
            n = 0.2 + 1.8 * torch.rand(ndof, generator=gen, device=be.device)
            d = torch.randn(ndof, 3, generator=gen, device=be.device)
            d = d / d.norm(dim=1, keepdim=True) * torch.rand(ndof, 1, generator=gen,
                                                            device=be.device).pow(1 / 3)
            T = 0.5 + 1.5 * torch.rand(ndof, generator=gen, device=be.device)
            on = (k > j).float() * n / (torch.pi * T)**1.5
            for i0 in range(0, ndof, 2048):
                sl = slice(i0, i0 + 2048)
                r2 = ((cx[None] - d[sl, 0, None, None, None])**2
                      + (cy[None] - d[sl, 1, None, None, None])**2
                      + (cz[None] - d[sl, 2, None, None, None])**2)
                f[sl] += on[sl, None, None, None] * torch.exp(-r2 / T[sl, None, None, None])
        f *= 1 + 0.01 * (2 * torch.rand(f.shape, generator=gen, device=be.device) - 1)
        fs.append(f.reshape(ndof, -1).contiguous())
    tune_vhs(grids, grids[0].phase.device)
    col = VHSCollider(grids, grids[0].phase.device)
    qs = [torch.empty_like(f) for f in fs]
    batches = [(1, fs[1], qs[1], None), (0, fs[0], qs[0], None)]   # expensive grid first
    col(batches)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        col(batches)
    torch.cuda.current_stream().wait_stream(s)
    with torch.cuda.graph(g):
        col(batches)
    st = torch.cuda.current_stream()
    ms = []
    for _ in range(reps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        g.replay()
        b.record(st)
        torch.cuda.synchronize()
        ms.append(a.elapsed_time(b))
    t = sum(ms) / len(ms)
    ndof = w['n24'] + w['n32']
    cons = {}
    for gi, g in enumerate(grids):
        cons[f'Nv{g.Nv}'] = q_conservation(lambda f2, q2, m, gi=gi: col([(gi, f2, q2, m)]),
                                           fs[gi], qs[gi], g.c0.double(), float(g.struct.cw))
    return {'workload': f"two species, {w['n24']} x 24^3 + {w['n32']} x 32^3, mass ratio 2, Nrho=16, M=12, "
                        'one persistent launch in a CUDA graph, FP32 + FP64 projection',
            'q_evals_per_s': ndof / (t * 1e-3), 'ms_per_launch': t,
            'tiles': [int(x.struct.tile) for x in grids], 'conservation': cons}, (grids, fs, qs)


def small_fp64(flush, steps=20, ncores=0):
    """Plain FP64 method: 4x4 periodic quads P2 (144 DOFs), Nv=16, hard
    spheres, Nrho=8, M=6, two seeded Maxwellians per DOF, SSP-RK2 dt=1e-3."""
    import numpy as np
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.integrators import get_integrator
    from frfs_b200.mesh import StructuredMesh
    from frfs_b200.system import DGFSSystem
    w = SMALL64
    ini = couette_ini('double', dict(WORK, Nv=w['Nv'], Nrho=w['Nrho'], M=w['M'], dev=w['dev'],
                                     omega=w['omega'], order=w['order'], dt=w['dt']))
    cfg = Inifile(ini)
    be = CUDABackend(cfg)
    mesh = StructuredMesh((w['nx'], w['ny']), (0.0, 0.0), (1.0, 1.0), periodic='xy')
    s = DGFSSystem(be, mesh, cfg, nreg=3)
    rng = np.random.default_rng(2)
    cv = s.vm.cv()
    u = s.eles_scal_upts_inb_full[0]
    F = np.empty(u.shape)
    for e in range(u.shape[0]):
        for j in range(u.shape[1]):
            f = 0.0
            for _ in range(2):
                d = rng.normal(size=3)
                d = d / np.linalg.norm(d) * 0.5 * rng.uniform()**(1 / 3)
                T = rng.uniform(0.7, 1.3)
                f = f + rng.uniform(0.5, 1.5) / (np.pi * T)**1.5 * np.exp(
                    -np.sum((cv - d[:, None])**2, axis=0) / T)
            F[e, j] = f
    u.copy_(torch.from_numpy(F))
    integ = get_integrator(be, s, cfg)
    # one step from the seeded state: conservation, and the same step of the
    # reference algorithm (FP64 oracle, whole mesh, its Q followed by the
    # launch's FP64 projection) on the host cores, timed and compared
    tot0 = state_totals(s, 0)
    integ.step(0.0, w['dt'])
    torch.cuda.synchronize()
    tot1 = state_totals(s, 0)
    got = s.eles_scal_upts_inb_full[0].cpu().numpy()
    cpu = err = None
    if ncores:
        from oracle.fr import step_rk2
        from frfs_b200.sphericaldesign import half_sphere_design
        pool = make_pool(ncores, w['Nv'], w['Nrho'], half_sphere_design(w['M']), w['dev'], w['omega'])
        orc = make_fr_oracle(s)
        c0 = s.vm.c0().astype(np.float64)
        cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
        Phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
        E, J, n = F.shape

        def Qo(x):
            rows = x.reshape(E * J, n)
            q = np.concatenate(list(pool.map(_oracle_q_worker, np.array_split(rows, ncores))))
            q -= (Phi.T @ np.linalg.solve(Phi @ Phi.T, Phi @ q.T)).T
            return q.reshape(E, J, n)
        t0 = time.perf_counter()
        uo = step_rk2(F, w['dt'], orc.rhs, Qo)
        t_cpu = time.perf_counter() - t0
        pool.shutdown()
        err = float(np.linalg.norm(got - uo) / np.linalg.norm(uo - F))
        cpu = {'value': 1.0 / t_cpu, 'unit': 'DG steps/s', 'cores': ncores, 'kind': 'port',
               'sample': ('one whole SSP-RK2 step of the same state (288 Q evaluations, '
                          '3+3*M*Nrho FP64 FFTs each, on the host cores + the FR operator '
                          'twice), no extrapolation')}
    for _ in range(3):
        integ.step(0.0, w['dt'])
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        integ.step(0.0, w['dt'])
        b.record(st)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    c0t = torch.as_tensor(s.vm.c0(), dtype=torch.float64, device=be.device)
    qc = q_conservation(lambda f, q, m: s.sm.collide(f, q, moments=m),
                        s.eles_scal_upts_inb_full[0], s.eles_scal_upts_inb_full[2], c0t, s.vm.cw())
    return {'workload': '4x4 periodic quads P2 (144 DOFs), Nv=16^3 on [-5,5]^3, hard sphere, '
                        'Nrho=8, M=6, SSP-RK2 dt=1e-3, FP64 (exact-Nyquist collision operator)',
            'dg_steps_per_s': steps / (tot * 1e-3), 'ms_per_step': tot / steps,
            'dtype': 'f64',
            'step_rel_l2_err_vs_fp64_oracle': err,
            'error_definition': ('|u_gpu - u_oracle| / |u_oracle - u_0| after one step from the '
                                 'seeded state (relative to the change the step makes)'),
            'conservation': {'collision': qc,
                             'state_drift_per_step': drift(tot0, tot1),
                             'state_totals': 'GLL-quadrature integrals over the periodic mesh'},
            'cpu_baseline': cpu}


MIXTURE = dict(Nv=24, Nrho=12, M=12, Mpre=12, ndof=1024, masses=(39.96e-3, 83.798e-3),
               alpha=1.3, omega=0.81, dev=6)


def mixture_ini(w=MIXTURE):
    """Binary argon-krypton mixture, 'vss-gll' with the same VSS parameters
    for every ordered species pair, FP32 state."""
    S = len(w['masses'])
    pairs = '\n'.join(f"alpha{p}{q} = {w['alpha']}\nomega{p}{q} = {w['omega']}\n"
                      f"dRef{p}{q} = 4.17e-10\nTref{p}{q} = {NONDIM['T0']}"
                      for p in range(S) for q in range(S))
    mm = '\n'.join(f'molarMass{p + 1} = {m}' for p, m in enumerate(w['masses']))
    return f"""
[backend]
precision = single
[constants]
Nv = {w['Nv']}
Nrho = {w['Nrho']}
[non-dim]
T0 = {NONDIM['T0']}
H0 = {NONDIM['H0']}
rho0 = {NONDIM['rho0']}
molarMass0 = {NONDIM['molarMass0']}
[velocity-mesh]
dev = {w['dev']}
cmax = 0
Tmax = {NONDIM['T0']}
{mm}
[spherical-design-rule]
ssrule = womersley
M = {w['M']}
[scattering-model]
type = vss-gll
Mpre = {w['Mpre']}
ssrulepre = womersley
{pairs}
"""


def vss_mixture(flush, peak=None, reps=3, ndof=None, check=True):
    """Gas-mixture collision operator ('vss-gll', Q_p = sum_q Q_pq for both
    species of ndof distribution pairs, one launch): Q_p evals/s, FLOP-model
    roofline and the error of the FP32 launch against the FP64 oracle on two
    seeded pairs.  FLOP per (distribution, species) item with S species,
    P = Nrho M slices and n = Nv^3: (S (3 P + 1) + 2) 5 n log2 n for the
    FFTs (F and the partners' transforms, three 3-D transforms per slice,
    two inverse transforms at the end) + 38 S P n for the phase, product and
    kernel-weight arithmetic."""
    import numpy as np
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.dgfsbi import DGFSBiVelocityMesh, DGFSBiVSSGLLScatteringModel
    from frfs_b200.inifile import Inifile
    w = dict(MIXTURE)
    if ndof is not None:
        w['ndof'] = ndof
    cfg = Inifile(mixture_ini(w))
    be = CUDABackend(cfg)
    S = len(w['masses'])
    vm = DGFSBiVelocityMesh(be, cfg, S)
    sm = DGFSBiVSSGLLScatteringModel(be, cfg, vm)
    n, nd = vm.vsize(), w['ndof']
    # seeded sums of two Maxwellians n (m/(pi T))^1.5 exp(-m |c-u|^2/T) per
    # species, n ~ U(0.3, 1.2), T ~ U(0.7, 1.3), |u_i| < 0.3, built on the device
    rng = np.random.default_rng(11)
    cv = torch.as_tensor(vm.cv(), dtype=torch.float64, device=be.device)
    fs = []
    for m in vm.masses():
        f = torch.zeros((nd, n), dtype=torch.float64, device=be.device)
        for _ in range(2):
            dn = torch.as_tensor(rng.uniform(0.3, 1.2, nd), device=be.device)[:, None]
            T = torch.as_tensor(rng.uniform(0.7, 1.3, nd), device=be.device)[:, None]
            u = torch.as_tensor(rng.uniform(-0.3, 0.3, (nd, 3, 1)), device=be.device)
            f += dn * (m / (np.pi * T))**1.5 * torch.exp(-m * ((cv[None] - u)**2).sum(1) / T)
        fs.append(f.float())
        del f
    Qs = [torch.empty_like(f) for f in fs]
    st = torch.cuda.current_stream()
    sm.collide(fs, Qs)
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(reps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        sm.collide(fs, Qs)
        b.record(st)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    ms = tot / reps
    P = vm.Nrho() * vm.M()
    flop_item = (S * (3 * P + 1) + 2) * 5 * n * math.log2(n) + 38 * S * P * n
    flop = flop_item * S * nd
    res = {'workload': (f"binary gas mixture (molar masses {w['masses'][0]}, {w['masses'][1]} kg/mol), "
                        f"'vss-gll' alpha={w['alpha']} omega={w['omega']}, Nv={w['Nv']}^3 on "
                        f"[-{w['dev']},{w['dev']}]^3, Nrho={w['Nrho']}, M={w['M']} full-sphere "
                        f"directions, Mpre={w['Mpre']}; {nd} distribution pairs, Q_p = sum_q Q_pq "
                        f"for both species in one launch, FP32, then the FP64 conservation "
                        f"projection (one more launch)"),
           'launch_ms': ms, 'q_p_evals_per_s': S * nd / (ms * 1e-3),
           'flop_per_launch': flop, 'achieved_tflops': flop / (ms * 1e-3) / 1e12}
    if peak:
        res['frac_of_fp32_fma_probe'] = res['achieved_tflops'] / peak
    if check:
        sys.path.insert(0, ROOT)
        from oracle.vss import BiVelocityMesh, VSSOracle, project_mixture
        ovm = BiVelocityMesh(vm.Nv(), vm.Nrho(), vm.sz(), vm.masses(), cmax=0.0, Tmax=NONDIM['T0'],
                             dev=vm.L(), **NONDIM)
        prm = dict(alpha=w['alpha'], omega=w['omega'], dRef=4.17e-10, Tref=NONDIM['T0'])
        orc = VSSOracle(ovm, sm._szpre, {(p, q): prm for p in range(S) for q in range(S)})
        err, t_or = 0.0, 0.0
        for d in (0, nd - 1):
            t0 = time.perf_counter()
            want = orc.Q([fs[p][d].double().cpu().numpy() for p in range(S)])
            t_or += time.perf_counter() - t0
            want = project_mixture(want, ovm.cv, vm.masses())
            for p in range(S):
                got = Qs[p][d].double().cpu().numpy()
                err = max(err, float(np.linalg.norm(got - want[p]) / np.linalg.norm(want[p])))
        res['q_rel_l2_err_vs_fp64_oracle'] = err
        res['error_sample'] = ('distribution pairs 0 and ndof-1, both species, FP64 oracle (1 host '
                               'core) followed by the same conservation projection as the launch')
        res['oracle_s_per_pair_1core'] = t_or / 2
    del fs, Qs
    torch.cuda.empty_cache()
    return res


def dgfsbi_couette(flush, steps=3):
    """'dgfsbi' system: the binary mixture of ``vss_mixture`` in the Couette
    geometry (16 x 8 quads P3, 2048 DOFs per species, x periodic, diffuse
    walls at y = -+0.5 moving at -+0.3 u0, T = 1), number densities 0.3 /
    0.7 n0, dgfsbi-tvd-rk2 at dt = 5e-4 as one CUDA graph per step; DG
    steps/s."""
    import numpy as np
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.dgfsbi import DGFSBiSystem
    from frfs_b200.inifile import Inifile
    from frfs_b200.integrators import get_integrator
    from frfs_b200.mesh import StructuredMesh
    w = MIXTURE
    u0 = np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])
    n0 = NONDIM['rho0'] / NONDIM['molarMass0'] * 6.0221409e+23
    walls = ''.join(f"""
[soln-bcs-{name}]
type = dgfsbi-wall-diffuse
T = {NONDIM['T0']}
ux = {sgn * WORK['uw'] * u0}
uy = 0
uz = 0
""" for name, sgn in (('y-', -1), ('y+', 1)))
    cfg = Inifile(mixture_ini(w) + f"""
[solver]
system = dgfsbi
order = {WORK['order']}
[solver-time-integrator]
scheme = dgfsbi-tvd-rk2
controller = none
tstart = 0.0
tend = 1.0
dt = {WORK['dt']}
[soln-ics]
type = maxwellian
nden1 = {0.3 * n0}
nden2 = {0.7 * n0}
T = {NONDIM['T0']}
ux = 0
uy = 0
uz = 0
""" + walls)
    be = CUDABackend(cfg)
    mesh = StructuredMesh((WORK['nx'], WORK['ny']), (0.0, -0.5), (2.0, 0.5), periodic='x')
    s = DGFSBiSystem(be, mesh, cfg, nreg=3)
    integ = get_integrator(be, s, cfg)
    dt = WORK['dt']
    for _ in range(3):                      # warm-up: eager run, capture, one replay
        integ.step(0.0, dt)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        integ.step(0.0, dt)
        b.record(st)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    ok = all(bool(torch.isfinite(u).all()) for u in integ.soln)
    res = {'workload': (f"'dgfsbi' binary mixture Couette: 16 x 8 quads P3 (2048 DOFs per species), "
                        f"the vss_mixture operator settings, diffuse walls -+0.3 u0 at T = 1, "
                        f"nden 0.3 / 0.7 n0, dgfsbi-tvd-rk2 dt = {dt}, FP32"),
           'dg_steps_per_s': steps / (tot * 1e-3), 'ms_per_step': tot / steps,
           'finite': ok}
    del s, integ
    torch.cuda.empty_cache()
    return res


def ars_bgk(flush, steps=20):
    """adgfs system: the Couette workload's mesh and velocity grid (16 x 8
    quads P3, Nv=24^3, FP32) with BGK relaxation (omega 0.81) and the
    ARS-222 IMEX stepper; DG steps/s and the HBM roofline of the fused
    ARS stage kernel (stage 2: reads f0, L0, L1, f1 and L1 once more for
    its moments, writes f2)."""
    import torch
    from frfs_b200.adgfs import ARS_DIST, ARS_MOML, ARS_MOMU, ADGFSSystem
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.integrators import get_integrator
    from frfs_b200.mesh import StructuredMesh
    cfg = Inifile(couette_ini('single'))
    for k, v in (('type', 'bgk-direct-gll'), ('muRef', '2.117e-5'), ('Tref', '273')):
        cfg.set('scattering-model', k, v)
    cfg.set('solver', 'system', 'adgfs')
    cfg.set('solver-time-integrator', 'scheme', 'adgfs-ars-222')
    be = CUDABackend(cfg)
    mesh = StructuredMesh((WORK['nx'], WORK['ny']), (0.0, -0.5), (2.0, 0.5), periodic='x')
    s = ADGFSSystem(be, mesh, cfg, nreg=4)
    integ = get_integrator(be, s, cfg)
    dt = WORK['dt']
    for _ in range(3):
        integ.step(0.0, dt)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        integ.step(0.0, dt)
        b.record(st)
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    # the stage-2 kernel alone (same banks as inside the step)
    Ae, Ai = integ._A_expl(2), integ._A_impl(2)
    kt = 0.0
    reps = 10
    for _ in range(reps):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.ars_stage(dt, 2, ARS_MOML | ARS_MOMU | ARS_DIST, Ae, Ai, integ._F[:2], integ._F[2],
                    integ._L[:2], integ._U[:3], integ._LU[:2])
        b.record(st)
        torch.cuda.synchronize()
        kt += a.elapsed_time(b)
    kt /= reps
    elems = s.ndof * s.vm.vsize()
    nbytes = elems * 4 * 6                       # 5 reads + 1 write of FP32 rows
    peak = hbm_peak_gbs()
    ach = nbytes / (kt * 1e-3) / 1e9
    return {'workload': ('adgfs: 16x8 quads P3 (2048 DOFs), Nv=24^3, BGK (bgk-direct-gll, '
                         'omega 0.81), ARS-222, dt=5e-4, FP32 state / FP64 moments'),
            'dg_steps_per_s': steps / (tot * 1e-3), 'ms_per_step': tot / steps,
            'stage_kernel': {'kernel': 'bdgfs::ars_kernel (stage 2)', 'ms': kt,
                             'bytes': nbytes, 'achieved_gbs': ach, 'peak_gbs': peak,
                             'frac': ach / peak, 'bound': 'hbm'}}


def cavity_ini():
    """Config 5's .ini (8^3 hex P2, lid 0.5 at T=1, diffuse walls) and the
    mesh boundary names."""
    import numpy as np
    u0 = np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])
    ini = couette_ini('single', dict(WORK, order=2)).split('[soln-bcs-y-]')[0]
    ini += f"""
[soln-bcs-lid]
type = dgfs-wall-diffuse
rho = {NONDIM['rho0']}
T = {NONDIM['T0']}
ux = {0.5 * u0}
uy = 0
uz = 0
[soln-bcs-walls]
type = dgfs-wall-diffuse
rho = {NONDIM['rho0']}
T = {NONDIM['T0']}
ux = 0
uy = 0
uz = 0
"""
    names = {'x-': 'walls', 'x+': 'walls', 'y-': 'walls', 'y+': 'lid', 'z-': 'walls',
             'z+': 'walls'}
    return ini, names


def run_hybrid_steps(nsteps, nwarm=3):
    """Profiling case: SSP-RK2 steps of the lid-driven cavity with the
    hybrid collision operator, the surrogate randomly initialised with its
    head scales at zero (Q = 0 on surrogate cells; the kernels, shapes and
    cell counts of the hybrid step; timing only)."""
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.integrators import get_integrator
    from frfs_b200.mesh import StructuredMesh
    from frfs_b200.surrogate import HybridCollider, QSurrogate
    from frfs_b200.system import DGFSSystem
    ini, names = cavity_ini()
    cfg = Inifile(ini)
    cfg.set('solver-time-integrator', 'dt', '2e-4')
    be = CUDABackend(cfg)
    mesh = StructuredMesh((8, 8, 8), (0, 0, 0), (1, 1, 1), periodic='', bcnames=names)
    s5 = DGFSSystem(be, mesh, cfg, nreg=3)
    q = QSurrogate(s5.sm.grid, nmodes=512, width=1024, center=False)   # the cavity hybrid's model
    dev = be.device
    g = torch.Generator(device=dev).manual_seed(0)
    n = q.n
    q.Bd = torch.linalg.qr(torch.randn(n, 512, device=dev, generator=g))[0].t().contiguous()
    q.Bq = torch.linalg.qr(torch.randn(n, 1536, device=dev, generator=g))[0].t().contiguous()
    q.mu = torch.zeros(512, device=dev)
    q.sigma = torch.full((512,), 0.05, device=dev)
    q.hscale = torch.zeros(3, device=dev)
    q._init_params(g)
    q._fold()
    hc = HybridCollider(q, threshold=0.05, recheck=0.02, recheck_every=2)
    n3 = s5.vm.vsize()
    s5.sm.collide = lambda fin, fout, **kw: hc(fin.reshape(-1, n3), fout.reshape(-1, n3))
    integ = get_integrator(be, s5, cfg)
    for _ in range(nwarm):
        integ.step(0.0, 2e-4)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(nsteps):
        integ.step(0.0, 2e-4)
    b.record(st)
    torch.cuda.synchronize()
    stt = hc.stats()
    print(json.dumps({'hybrid_steps': nsteps, 'ms_per_step': a.elapsed_time(b) / nsteps,
                      'spectral_cells_per_call': stt['spectral_cells'],
                      'surrogate_cells_per_call': stt['surrogate_cells']}))


def fp64_subcheck(pool, ncores, f, outs, c0):
    """Errors of device Q arrays (outs: name -> [m][n]) on the distributions
    f against the FP64 oracle (reference algorithm + the launch's FP64
    projection), relative to the oracle's Q and to its loss term
    prefac f (IFFT(bb2 F^)) (the collision frequency times f)."""
    import numpy as np
    F = f.double().cpu().numpy()
    t0 = time.perf_counter()
    res = list(pool.map(_oracle_gl_worker, [c for c in np.array_split(F, 4 * ncores) if len(c)]))
    t = time.perf_counter() - t0
    Qo = np.concatenate([r[0] for r in res])
    Lo = np.concatenate([r[1] for r in res])
    c0 = np.asarray(c0, np.float64)
    cx, cy, cz = np.meshgrid(c0, c0, c0, indexing='ij')
    Phi = np.stack([np.ones_like(cx), cx, cy, cz, cx * cx + cy * cy + cz * cz]).reshape(5, -1)
    Qo = Qo - (Phi.T @ np.linalg.solve(Phi @ Phi.T, Phi @ Qo.T)).T
    out = {'n': int(F.shape[0]), 'oracle_s': t}
    for name, q in outs.items():
        d = q.double().cpu().numpy() - Qo
        row = np.linalg.norm(d, axis=1) / np.linalg.norm(Qo, axis=1)
        out[name] = {'rel_l2_vs_q': float(np.linalg.norm(d) / np.linalg.norm(Qo)),
                     'rel_l2_vs_loss_term': float(np.linalg.norm(d) / np.linalg.norm(Lo)),
                     'per_row_median': float(np.median(row)),
                     'per_row_p90': float(np.percentile(row, 90))}
    return out


def cavity_cpu_step(s5, bank, pool, ncores, nq=128, nv=512):
    """Host cores: one SSP-RK2 step of the reference algorithm on the cavity
    state, from a bounded sample: Q of nq seeded DOFs (pool) and the FR
    operator on nv seeded velocities (velocities are independent there),
    each extrapolated to the whole state."""
    import numpy as np
    import torch
    u = s5.eles_scal_upts_inb_full[bank]
    E, J, n = u.shape
    rng = np.random.default_rng(6)
    pick = np.sort(rng.choice(E * J, nq, replace=False))
    F = u.reshape(-1, n)[torch.as_tensor(pick, device=u.device)].double().cpu().numpy()
    t0 = time.perf_counter()
    list(pool.map(_oracle_q_worker, [c for c in np.array_split(F, ncores) if len(c)]))
    tq = time.perf_counter() - t0
    orc = make_fr_oracle(s5)
    vsel = np.sort(rng.choice(n, nv, replace=False))
    uh = u[:, :, torch.as_tensor(vsel, device=u.device)].double().cpu().numpy()
    full = u.cpu().numpy()
    t1 = time.perf_counter()
    bc = orc.update_bc_from_state(full)
    orc.restrict(vsel).rhs(uh, bc=bc)
    tfr = time.perf_counter() - t1
    t_step = 2.0 * (tq * (E * J) / nq + tfr * n / nv)
    return {'value': 1.0 / t_step, 'unit': 'DG steps/s', 'cores': ncores, 'kind': 'port',
            'sample': (f'Q of {nq} seeded DOFs ({tq:.1f} s on {ncores} processes, reference '
                       f'algorithm) and the FR operator on {nv} of {n} velocities ({tfr:.2f} s, '
                       'wall sums over all), each extrapolated to the whole state, 2 stages')}


def surrogate_legs(flush, log=None, pool=None, ncores=0):
    """Config 4 (surrogate trained on the Couette family, evaluated on 50000
    held-out seeded distributions) and config 5 (8^3 hex P2 lid-driven
    cavity: plain FP32 spectral vs surrogate hybrid, DG steps/s)."""
    import time
    import numpy as np
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.integrators import get_integrator
    from frfs_b200.mesh import StructuredMesh
    from frfs_b200.scattering import DGFSVHSGLLScatteringModel
    from frfs_b200.surrogate import CAVITY, HybridCollider, QSurrogate, sample_family
    from frfs_b200.system import DGFSSystem
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    cfg = Inifile(couette_ini('single'))
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    t0 = time.time()
    q = QSurrogate(sm.grid, nmodes=512, width=1024)
    q.fit(nsamples=200000, ntest=50000, epochs=20, lr=3e-4, batch=1024, seed=0)
    t_fit = time.time() - t0
    # surrogate vs spectral throughput on near-equilibrium cells
    gen = torch.Generator(device=be.device).manual_seed(3)
    f = sample_family(vm.c0(), 8192, gen, be.device)
    out = torch.empty_like(f)
    h = HybridCollider(q, threshold=float('inf'), recheck=0.0)
    st = torch.cuda.current_stream()

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            fn()
            b.record(st)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps
    t_sur = timed(lambda: h(f, out))
    t_spec = timed(lambda: sm.collide(f, out, project=True, exact=False))
    # what the hidden layers add: the same model with only its linear skip path
    saved = q.W[3].clone()
    q.W[3][:, :q.w] = 0.0
    q._fold()
    lin = q.evaluate(10000, seed=1)
    q.W[3].copy_(saved)
    q._fold()
    c4 = {'workload': ('surrogate of Q on Nv=24^3 (M=Nrho=12): every cell re-centred at zero '
                       'velocity by a spectral shift (Q shifted back), 512-mode bases '
                       '(randomised SVD) of the Maxwellian-deviation direction and of Q/rho^2, '
                       'input = modes x, (T-1) x, (T-1)^2 x, products of the 24 leading modes, '
                       'T-1; 4-layer GELU MLP width 1024 with a linear skip and 3 output heads '
                       '(Q/rho^2 = y0 + s y1 + s^2 y2, s the deviation size), BF16 weights / '
                       'FP32 accumulation on tcgen05, least-squares skip path (kept fixed), '
                       'AdamW lr 3e-4, 20 epochs, 200000 training / 50000 held-out seeded '
                       'distributions of the Couette family, FP64 conservation projection'),
          'modes': q.k, 'train_steps': q.steps, 'train_s': q.train_seconds,
          'ridge_start_train_rel_residual': q.ridge_residual,
          'basis_truncation_heads': q.basis_err_heads,
          'heldout_rel_l2_linear_skip_only': lin,
          'data_s': q.data_seconds, 'fit_s_total': t_fit,
          'final_loss': q.history[-1], 'first_epoch_loss': q.history[0],
          'heldout_rel_l2_vs_spectral_q': q.test_err,
          'surrogate_q_evals_per_s': 8192 / (t_sur * 1e-3),
          'spectral_q_evals_per_s': 8192 / (t_spec * 1e-3)}
    if pool is not None:
        # 1000 further held-out distributions against the FP64 oracle
        fo = sample_family(vm.c0(), 1000, torch.Generator(device=be.device).manual_seed(987654),
                           be.device)
        qs, qh = torch.empty_like(fo), torch.empty_like(fo)
        sm.collide(fo, qs, project=True, exact=False)
        h.collide_surrogate_only(fo, qh)
        c4['fp64_oracle_subcheck'] = fp64_subcheck(pool, ncores, fo, {'surrogate': qh,
                                                                      'fp32_spectral': qs},
                                                   vm.c0())

    # ---- config 5: lid-driven cavity
    ini, names = cavity_ini()
    # surrogate for the cavity's near-equilibrium cells (CAVITY family)
    t0 = time.time()
    # raw rows (no re-centring): the hybrid's near-equilibrium cells have Q
    # of the size of the spectral operator's shift-equivariance error
    qc = QSurrogate(sm.grid, nmodes=512, width=1024, family=CAVITY, center=False)
    qc.fit(nsamples=200000, ntest=20000, epochs=20, lr=3e-4, batch=1024, seed=10)
    t_fit_c = time.time() - t0
    res, fields = {}, {}
    nsteps, nwarm = 40, 3
    for mode in ('plain', 'hybrid'):
        c5cfg = Inifile(ini)
        c5cfg.set('solver-time-integrator', 'dt', '2e-4')
        be5 = CUDABackend(c5cfg)
        mesh = StructuredMesh((8, 8, 8), (0, 0, 0), (1, 1, 1), periodic='', bcnames=names)
        s5 = DGFSSystem(be5, mesh, c5cfg, nreg=3)
        hc = None
        if mode == 'hybrid':
            # 2 % of the surrogate cells re-checked every time step: on the
            # first of the SSP-RK2 step's two collide calls
            hc = HybridCollider(qc, threshold=0.05, recheck=0.02, recheck_every=2)
            n3 = s5.vm.vsize()
            s5.sm.collide = lambda fin, fout, **kw: hc(fin.reshape(-1, n3), fout.reshape(-1, n3))
        integ = get_integrator(be5, s5, c5cfg)
        for _ in range(nwarm):
            integ.step(0.0, 2e-4)
        torch.cuda.synchronize()
        tot = 0.0
        sur = rec = spc = 0
        num = den = 0.0
        for _ in range(nsteps - nwarm):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            integ.step(0.0, 2e-4)
            b.record(st)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
            if hc is not None:
                # the step's second call (last) and its re-checking first call
                sst = hc.stats()
                sur += sst['surrogate_cells']
                rec += sst['rechecked_cells']
                spc += sst['spectral_cells'] + int(hc.rc_counts[1])
                e = hc.recheck_err.cpu().tolist()
                num += e[0]
                den += e[1]
        k = nsteps - nwarm
        res[mode] = {'dg_steps_per_s': k / (tot * 1e-3), 'ms_per_step': tot / k}
        if hc is not None:
            res[mode].update({'surrogate_cells_per_call': sur / k, 'rechecked_cells_per_step': rec / k,
                              'spectral_cells_per_step': spc / k,
                              'recheck_rel_l2': math.sqrt(num / den) if den > 0 else None})
        if mode == 'plain' and pool is not None:
            res[mode]['cpu_baseline'] = cavity_cpu_step(s5, integ._idxcurr, pool, ncores)
        if hc is not None and pool is not None:
            # the surrogate on 64 seeded cells it handles in the final state,
            # against the FP64 oracle: relative to Q and to the loss term
            fin = s5.eles_scal_upts_inb_full[integ._idxcurr].reshape(-1, s5.vm.vsize())
            hc.classify(fin, seed=1, recheck=0.0)
            nsur = int(hc.counts[0])
            pick = torch.as_tensor(np.sort(np.random.default_rng(4).choice(nsur, min(64, nsur),
                                                                           replace=False)),
                                   device=fin.device)
            fsel = fin.index_select(0, hc.sur_idx[:nsur].long()[pick]).contiguous()
            qs, qh = torch.empty_like(fsel), torch.empty_like(fsel)
            sm.collide(fsel, qs, project=True, exact=False)
            HybridCollider(qc, threshold=float('inf'), recheck=0.0).collide_surrogate_only(fsel, qh)
            res[mode]['surrogate_cells_fp64_oracle_check'] = fp64_subcheck(
                pool, ncores, fsel, {'surrogate': qh, 'fp32_spectral': qs}, s5.vm.c0())
        rho, U, T, _, _ = s5.moments(integ._idxcurr)
        fields[mode] = (rho.cpu(), U.cpu(), T.cpu())
        del s5, integ, hc
        torch.cuda.empty_cache()
    (rp, up, Tp), (rh, uh, Th) = fields['plain'], fields['hybrid']
    c5 = {'workload': ('3-D lid-driven cavity: 8^3 hex P2 (13824 DOFs), Nv=24^3, VHS 0.81, '
                       'Nrho=M=12, lid 0.5, diffuse walls T=1, uniform Maxwellian start, SSP-RK2 '
                       f'dt=2e-4, {nsteps} steps ({nwarm} untimed); hybrid threshold 0.05, 2% '
                       'of the surrogate cells re-checked by the spectral operator every time '
                       'step (first collide call of each step); surrogate (512 modes, raw rows) '
                       'trained on the cavity family'),
          'surrogate_fit_s': t_fit_c, 'surrogate_heldout_rel_l2': qc.test_err,
          'surrogate_basis_truncation_heads': qc.basis_err_heads,
          'surrogate_final_loss': qc.history[-1], 'surrogate_first_epoch_loss': qc.history[0],
          'plain_fp32_spectral': res['plain'], 'hybrid': res['hybrid'],
          'speedup': res['hybrid']['dg_steps_per_s'] / res['plain']['dg_steps_per_s'],
          'fields_after_steps': nsteps,
          'hybrid_vs_plain_max_abs_diff': {
              'rho_rel': float(((rh - rp).abs() / rp).max()),
              'U_over_lid_speed': float((uh - up).abs().max() / 0.5),
              'T_rel': float(((Th - Tp).abs() / Tp).max())}}
    return c4, c5


# ---------------------------------------------------------------- GPU leg
def run_gpu(args):
    import numpy as np
    import torch
    ws, rank, local = dist_init()
    # CPU baseline pool before any GPU work (spawned workers)
    pool = None
    ncores = os.cpu_count() or 1
    if rank == 0 and ws == 1 and not args.no_cpu:
        from frfs_b200.sphericaldesign import half_sphere_design
        pool = make_pool(ncores, WORK['Nv'], WORK['Nrho'], half_sphere_design(WORK['M']),
                         WORK['dev'], WORK['omega'])
    from frfs_b200 import _lib
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.integrators import get_integrator
    from frfs_b200.mesh import StructuredMesh
    from frfs_b200.system import DGFSSystem
    cfg = Inifile(couette_ini('single'))
    be = CUDABackend(cfg)
    dev = be.device
    if ws == 1:
        mesh = StructuredMesh((WORK['nx'], WORK['ny']), (0.0, -0.5), (2.0, 0.5), periodic='x')
        system = DGFSSystem(be, mesh, cfg, nreg=3)
    else:
        # weak scaling: a ws-times longer channel, one 16 x 8 slab per rank,
        # face values of neighbouring slabs exchanged over NCCL every stage
        from frfs_b200.partition import NCCLTransport, slab_partition
        mesh = StructuredMesh((WORK['nx'] * ws, WORK['ny']), (0.0, -0.5), (2.0 * ws, 0.5),
                              periodic='x')
        parts = slab_partition(mesh, ws)
        system = DGFSSystem(be, mesh, cfg, nreg=3, partition=(parts, rank),
                            transport=NCCLTransport())
    integ = get_integrator(be, system, cfg)
    if ws > 1:
        integ.use_graph = False       # NCCL exchange inside the step: eager launches
    ndof = system.ele.neles * system.ele.nupts
    dt = WORK['dt']
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # ---------------- device-timed steps (graph replay, inputs resident)
    for _ in range(max(args.warmup, 3)):
        integ.step(integ.tcurr, dt)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
    barrier(ws)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    evs = []
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        integ.step(integ.tcurr, dt)
        e1.record(st)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    barrier(ws)
    clocks = sampler.stop() if sampler else None
    t_dev = sum(a.elapsed_time(b) for a, b in evs) / 1e3          # seconds, this rank
    t_max = reduce_max(t_dev, ws)
    value = ws * args.steps / t_max
    ms_per_step = t_max / args.steps * 1e3
    # ---------------- conservation: one more step's state totals, one launch's moments
    fin = system.eles_scal_upts_inb_full[0]
    qout = system.eles_scal_upts_inb_full[2]
    conservation = None
    if ws == 1:
        tot0 = state_totals(system, 0)
        integ.step(integ.tcurr, dt)
        tot1 = state_totals(system, 0)
        c0t = torch.as_tensor(system.vm.c0(), dtype=torch.float64, device=dev)
        conservation = {
            'collision': q_conservation(lambda f, q, m: system.sm.collide(f, q, moments=m),
                                        fin, qout, c0t, system.vm.cw()),
            'state_drift_per_step': drift(tot0, tot1, conserved=(0,)),
            'state_totals': ('GLL-quadrature integrals over the mesh; the diffuse walls exchange '
                             'momentum and energy with the gas, so mass is the conserved total')}
    # ---------------- dominant kernel: Q alone, events on its stream
    for _ in range(2):
        system.sm.collide(fin, qout)
    torch.cuda.synchronize()
    qt = []
    for _ in range(5):
        flush.fill_(1)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        system.sm.collide(fin, qout)
        b.record(st)
        qt.append((a, b))
    torch.cuda.synchronize()
    q_ms = sum(x.elapsed_time(y) for x, y in qt) / len(qt)
    flop = q_flops_per_eval(WORK['Nv'], WORK['Nrho'], WORK['M']) * ndof
    achieved = flop / (q_ms * 1e-3) / 1e12
    # measured FP32 FMA peak on this GPU (probe kernel in libbdgfs)
    probe = torch.zeros(1, device=dev)
    nsm = torch.cuda.get_device_properties(dev).multi_processor_count
    iters = 4096
    _lib.check(_lib.lib().bdgfs_fma_probe(_lib.ptr(probe), nsm * 8, 64, _lib.stream_ptr()), 'probe')
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    _lib.check(_lib.lib().bdgfs_fma_probe(_lib.ptr(probe), nsm * 8, iters, _lib.stream_ptr()), 'probe')
    b.record(st)
    torch.cuda.synchronize()
    pk_ms = a.elapsed_time(b)
    peak = nsm * 8 * 256 * iters * 16 * 8 * 2 / (pk_ms * 1e-3) / 1e12
    # ---------------- e2e: host buffers, copies inside the timed region.  Every
    # step uploads its input from pinned host memory and reads its result back.
    # Uploads go to one of two device input buffers on their own copy stream,
    # so the next step's upload overlaps this step's compute (the first one
    # does not); the step starts from its buffer with a device copy.  The
    # result is first copied to a device staging bank, so its device->host
    # read (a second copy stream) overlaps the next step too.  One interval
    # covers all steps, the L2 flushes and the last read-back.
    nbytes = fin.numel() * fin.element_size()
    host_in = torch.empty(fin.shape, dtype=fin.dtype, pin_memory=True)
    host_out = torch.empty(fin.shape, dtype=fin.dtype, pin_memory=True)
    host_in.copy_(fin)
    stage = torch.empty_like(fin)
    dev_in = [torch.empty_like(fin), torch.empty_like(fin)]
    cs = torch.cuda.Stream(device=dev)
    cu = torch.cuda.Stream(device=dev)
    uploaded, consumed = [None, None], [None, None]

    def upload(k):
        with torch.cuda.stream(cu):
            if consumed[k % 2] is not None:
                cu.wait_event(consumed[k % 2])     # its previous input has been taken
            dev_in[k % 2].copy_(host_in, non_blocking=True)
            uploaded[k % 2] = torch.cuda.Event()
            uploaded[k % 2].record(cu)
    copied = None
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    cu.wait_event(a)
    upload(0)
    for k in range(args.steps):
        flush.fill_(1)
        if k + 1 < args.steps:
            upload(k + 1)
        st.wait_event(uploaded[k % 2])
        fin.copy_(dev_in[k % 2])
        consumed[k % 2] = torch.cuda.Event()
        consumed[k % 2].record(st)
        integ.step(integ.tcurr, dt)
        if copied is not None:
            st.wait_event(copied)                  # the previous read-back has left stage
        stage.copy_(fin)
        done = torch.cuda.Event()
        done.record(st)
        cs.wait_event(done)
        with torch.cuda.stream(cs):
            host_out.copy_(stage, non_blocking=True)
            copied = torch.cuda.Event()
            copied.record(cs)
    st.wait_event(copied)
    b.record(st)
    torch.cuda.synchronize()
    t_e2e = reduce_max(a.elapsed_time(b) / 1e3, ws)
    e2e = ws * args.steps / t_e2e
    # ---------------- CPU baseline (rank 0, N = 1): reference algorithm sample
    cpu = None
    qerr = None
    if pool is not None:
        f_host = fin.reshape(-1, system.vm.vsize()).double().cpu().numpy()
        rng = np.random.default_rng(1)
        idx = rng.choice(ndof, size=min(ndof, 32 * ncores), replace=False)
        F = f_host[idx]
        orc_fr = make_fr_oracle(system)
        u_host = fin.double().cpu().numpy()
        t_step, Qo, tq, tfr = cpu_reference_step_time(F, (orc_fr, u_host), ndof, pool, ncores)
        # L2 error of the FP32 GPU operator vs the FP64 reference algorithm on the sample
        system.sm.collide(fin, qout, project=False)
        qg = qout.reshape(-1, system.vm.vsize())[torch.as_tensor(idx, device=dev)].double().cpu().numpy()
        qerr = float(np.linalg.norm(qg - Qo) / np.linalg.norm(Qo))
        cpu = {'value': 1.0 / t_step, 'unit': 'DG steps/s', 'cores': ncores, 'kind': 'port',
               'sample': (f'Q of {len(idx)} random DOFs of the same state (reference algorithm, '
                          f'3+3*M*Nrho FP64 FFTs each, {tq:.1f} s on {ncores} processes) + FR '
                          f'operator on the full mesh ({tfr:.2f} s), extrapolated to one step')}
    # other measured configurations of the metric (rank 0, single GPU)
    extra = {}
    if ws == 1 and not args.no_extra:
        extra['plain_fp64_small'] = small_fp64(flush, ncores=0 if args.no_cpu else ncores)
        bq, arrays = batched_q(flush)
        bq['q_rel_l2_err_vs_fp64_reference'], bq['cpu_baseline'] = batched_q_error(
            arrays, counts=[BATCHED['n24'], BATCHED['n32']])
        bq['error_sample'] = ('64 seeded distributions per grid, FP64 reference algorithm on the '
                              'host cores followed by the same conservation projection as the '
                              'kernel (applied in FP64)')
        extra['batched_q'] = bq
        del arrays
        extra['ars_bgk'] = ars_bgk(flush)
        extra['vss_mixture'] = vss_mixture(flush, peak)
        extra['dgfsbi_couette'] = dgfsbi_couette(flush)
    if ws == 1 and not args.no_surrogate:
        c4, c5 = surrogate_legs(flush, pool=pool, ncores=ncores)
        extra['surrogate'] = c4
        extra['hybrid_lid_cavity'] = c5
    if pool is not None:
        pool.shutdown()
    # gpu launches per step: 2 stages x (collide [+ disu] [+ bc_update] + rhs); the
    # one-part GLL system reads face values from the state (no disu)
    gathers = system.ele.fsel is not None and system.domain is None
    per_stage = 2 + (0 if gathers else 1) + (1 if system.walls.has_diffuse else 0)
    launches = 2 * per_stage * args.steps
    line = {
        'metric': METRIC, 'value': value, 'unit': 'DG steps/s', 'n_gpus': ws,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms_per_step,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic', 'config': config_block(ws),
        'q_evals_per_s': ws * 2 * ndof * args.steps / t_max,
        'q_rel_l2_err_vs_fp64_reference': qerr,
        'roofline': {'bound': 'fp32', 'kernel': 'bdgfs::vhs_collide_kernel',
                     'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
                     'frac': achieved / peak,
                     'peak_source': 'measured FP32 FMA probe on this GPU (MEASURED_PEAKS.json has '
                                    'no FP32 CUDA-core figure)',
                     'flop_per_launch': flop, 'launch_ms': q_ms,
                     'reference_equivalent': {
                         'flop_per_launch': ndof * q_flops_reference_equivalent(24, 12, 12),
                         'tflops': ndof * q_flops_reference_equivalent(24, 12, 12) / (q_ms * 1e-3) / 1e12,
                         'note': ("the reference's 3 M Nrho + 3 FFTs per Q in the same launch time; "
                                  'context only (above the peak: the packed algorithm does fewer)')},
                     # algorithmic: f in + Q out = 2 x 113 MB
                     'traffic': Q_LAUNCH_DRAM_BYTES, 'traffic_alg': 2 * 4 * ndof * 24**3,
                     'traffic_source': ('not measured in this run: dram__bytes_read.sum + '
                                        'dram__bytes_write.sum of one ncu capture of this '
                                        'kernel variant on the same 2048 Couette cubes '
                                        '(profiles/vhs_collide_nv24.md)')},
        'e2e': {'value': e2e, 'unit': 'DG steps/s', 'h2d_bytes_per_step': nbytes,
                'd2h_bytes_per_step': nbytes},
        'gpu_launches': launches,
        'clocks': clocks,
        'cpu_baseline': cpu,
        'conservation': conservation,
        **extra,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_q_only(ndof):
    """Collision kernel alone on ndof seeded Couette-family cubes (profiling)."""
    import numpy as np
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.scattering import DGFSVHSGLLScatteringModel
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    cfg = Inifile(couette_ini('single'))
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    rng = np.random.default_rng(0)
    cv = vm.cv()
    base = np.exp(-np.sum(cv**2, axis=0)) / np.pi**1.5
    f = torch.from_numpy(base).float().to(be.device).repeat(ndof, 1)
    f *= 1 + 0.01 * torch.rand(f.shape, device=be.device, generator=torch.Generator(
        device=be.device).manual_seed(int(rng.integers(1 << 30))))
    q = torch.empty_like(f)
    for _ in range(3):
        sm.collide(f, q)
    torch.cuda.synchronize()
    print(json.dumps({'q_only_ndof': ndof, 'finite': bool(torch.isfinite(q).all())}))


def run_surrogate_curve(modes=(64, 128, 256, 384, 512)):
    """Analysis case: the Couette-family surrogate (drift-free rows, the
    config-4 model and training) at several basis sizes: held-out error
    against the FP32 spectral Q (50000 distributions), the bases'
    truncation of the heads, and the error of the fixed linear path alone
    (the hidden layers' output zeroed), one JSON line per size."""
    import time
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.scattering import DGFSVHSGLLScatteringModel
    from frfs_b200.surrogate import QSurrogate
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    cfg = Inifile(couette_ini('single'))
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    for k in modes:
        t0 = time.time()
        q = QSurrogate(sm.grid, nmodes=k, width=1024)
        q.fit(nsamples=200000, ntest=50000, epochs=20, lr=3e-4, batch=1024, seed=0)
        saved = q.W[3].clone()
        q.W[3][:, :q.w] = 0.0
        q._fold()
        lin = q.evaluate(10000, seed=1)
        q.W[3].copy_(saved)
        q._fold()
        print(json.dumps({'modes': k, 'heldout_rel_l2_vs_spectral_q': q.test_err,
                          'basis_truncation_heads': q.basis_err_heads,
                          'heldout_rel_l2_linear_skip_only': lin, 'fit_s': time.time() - t0}),
              flush=True)
        del q


def run_surrogate_call(ndof, reps=2):
    """Profiling case: all-surrogate hybrid calls on ndof Couette-family
    cells with a randomly initialised 256-mode / width-1024 network (the
    kernels and shapes of inference; timing only)."""
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.scattering import DGFSVHSGLLScatteringModel
    from frfs_b200.surrogate import HybridCollider, QSurrogate, sample_family
    from frfs_b200.velocitymesh import DGFSVelocityMesh
    cfg = Inifile(couette_ini('single'))
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    q = QSurrogate(sm.grid, nmodes=512, width=1024)
    dev = be.device
    g = torch.Generator(device=dev).manual_seed(0)
    n = q.n
    q.Bd = torch.linalg.qr(torch.randn(n, 512, device=dev, generator=g))[0].t().contiguous()
    q.Bq = torch.linalg.qr(torch.randn(n, 1536, device=dev, generator=g))[0].t().contiguous()
    q.mu = torch.zeros(512, device=dev)
    q.sigma = torch.full((512,), 0.05, device=dev)
    q.hscale = torch.full((3,), 1e-3, device=dev)
    q._init_params(g)
    q._fold()
    f = sample_family(vm.c0(), ndof, g, dev)
    out = torch.empty_like(f)
    h = HybridCollider(q, threshold=float('inf'), recheck=0.0)
    for _ in range(2):
        h(f, out)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        h(f, out)
    b.record(st)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    print(json.dumps({'surrogate_call_ndof': ndof, 'ms': ms, 'q_evals_per_s': ndof / ms * 1e3}))


def hbm_peak_gbs():
    """HBM copy bandwidth of MEASURED_PEAKS.json (measured on this pool's
    B200s), else the pool's earlier measurement, 6650 GB/s."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'MEASURED_PEAKS.json')
    if os.path.exists(path):
        return json.load(open(path))['hbm_gbs']
    return 6650.0


def run_fr_only(kind, reps=10):
    """Profiling case: the FR kernels of one SSP-RK2 stage (disu, wall
    update, fused rhs with two combination operands) on the Couette
    (16x8 quads P3) or lid-cavity (8^3 hex P2) mesh, Nv=24^3, FP32; device
    time per kernel and the fused rhs kernel's HBM roofline."""
    import torch
    from frfs_b200.backend import CUDABackend
    from frfs_b200.inifile import Inifile
    from frfs_b200.mesh import StructuredMesh
    from frfs_b200.system import DGFSSystem
    if kind == 'couette':
        cfg = Inifile(couette_ini('single'))
        mesh = StructuredMesh((WORK['nx'], WORK['ny']), (0.0, -0.5), (2.0, 0.5), periodic='x')
    else:
        ini = couette_ini('single', dict(WORK, order=2)).split('[soln-bcs-y-]')[0]
        ini += """
[soln-bcs-walls]
type = dgfs-wall-diffuse
rho = {rho}
T = {T}
ux = 0
uy = 0
uz = 0
""".format(rho=NONDIM['rho0'], T=NONDIM['T0'])
        cfg = Inifile(ini)
        mesh = StructuredMesh((8, 8, 8), (0, 0, 0), (1, 1, 1), periodic='',
                              bcnames={k: 'walls' for k in ('x-', 'x+', 'y-', 'y+', 'z-', 'z+')})
    be = CUDABackend(cfg)
    s = DGFSSystem(be, mesh, cfg, nreg=3)
    st = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=be.device)
    x1, x2 = s._bank(1), s._bank(2)
    x1.copy_(s._bank(0))
    x2.copy_(s._bank(0))

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            fn()
            b.record(st)
            torch.cuda.synchronize()
            tot += a.elapsed_time(b)
        return tot / reps
    s._active = (0, 1)
    t_disu = timed(s._disu)
    t_bc = timed(s._update_bc) if s.walls.has_diffuse else 0.0
    out = s._bank(1).clone()
    from frfs_b200 import _lib as _lb
    t_rhs = timed(lambda: _lb.lib().bdgfs_fr_rhs(
        _lb.ref(s.ele.struct), _lb.ref(s.walls.struct), s._bank(0).data_ptr(), s._uf_rows.data_ptr(),
        out.data_ptr(), 0.5, 2.5e-4, x1.data_ptr(), 2.5e-4, x2.data_ptr(), 0.5, _lb.stream_ptr()))
    E, U, F, nv = s.ele.neles, s.ele.nupts, s.ele.nfpts, s.vm.vsize()
    nbytes = 4 * nv * E * (4 * U + 2 * F)          # u, x1, x2 in + out; own and neighbour faces
    peak = hbm_peak_gbs()
    res = {'fr_only': kind, 'neles': E, 'nupts': U, 'nfpts': F, 'nv': nv,
           'disu_ms': t_disu, 'bc_update_ms': t_bc, 'rhs_ms': t_rhs,
           'rhs_bytes': nbytes, 'rhs_gbs': nbytes / (t_rhs * 1e-3) / 1e9,
           'rhs_frac_of_hbm': nbytes / (t_rhs * 1e-3) / 1e9 / peak,
           'disu_gbs': 4 * nv * E * (U + F) / (t_disu * 1e-3) / 1e9}
    if s.ele.fsel is not None:
        # face values read from the state (no disu): u, x1, x2 in + out, neighbour faces
        from frfs_b200 import _lib
        L, fsel = _lib.lib(), s.ele.fsel.data_ptr()
        u = s._bank(0)
        t_bcg = timed(lambda: L.bdgfs_fr_bc_update_gather(
            _lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel, u.data_ptr(),
            _lib.stream_ptr())) if s.walls.has_diffuse else 0.0
        t_rg = timed(lambda: L.bdgfs_fr_rhs_gather(
            _lib.ref(s.ele.struct), _lib.ref(s.walls.struct), fsel, u.data_ptr(), out.data_ptr(),
            0.5, 2.5e-4, x1.data_ptr(), 2.5e-4, x2.data_ptr(), 0.5, _lib.stream_ptr()))
        gbytes = 4 * nv * E * (4 * U + F)
        res.update({'gather_bc_update_ms': t_bcg, 'gather_rhs_ms': t_rg, 'gather_rhs_bytes': gbytes,
                    'gather_rhs_frac_of_hbm': gbytes / (t_rg * 1e-3) / 1e9 / peak,
                    'stage_ms_disu_path': t_disu + t_bc + t_rhs,
                    'stage_ms_gather_path': t_bcg + t_rg})
        if s.ele.tensor is not None:
            # factored residual R = M1 F~ + M3 (F^n - M2 F~) on the gather path
            t_rt = timed(lambda: L.bdgfs_fr_rhs_tensor(
                _lib.ref(s.ele.struct), _lib.ref(s.walls.struct), _lib.ref(s.ele.tensor),
                u.data_ptr(), None, out.data_ptr(), 0.5, 2.5e-4, x1.data_ptr(), 2.5e-4, x2.data_ptr(), 0.5,
                _lib.stream_ptr()))
            res.update({'tensor_rhs_ms': t_rt,
                        'tensor_rhs_frac_of_hbm': gbytes / (t_rt * 1e-3) / 1e9 / peak,
                        'stage_ms_tensor_path': t_bcg + t_rt})
    print(json.dumps(res))


def run_ars_only():
    """The adgfs ARS-222 leg alone (profiling case)."""
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    print(json.dumps(ars_bgk(flush)))


def run_dgfsbi_only():
    """The 'dgfsbi' mixture Couette leg alone (profiling case)."""
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    print(json.dumps(dgfsbi_couette(flush)))


def run_vss_only(ndof):
    """The gas-mixture collision launch alone on ndof distribution pairs
    (profiling case, no oracle check)."""
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    print(json.dumps(vss_mixture(flush, reps=2, ndof=ndof, check=False)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=20)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='frfs_b200', choices=['frfs_b200', 'reference'])
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline leg')
    ap.add_argument('--no-surrogate', action='store_true',
                    help='skip the surrogate training and hybrid lid-cavity legs')
    ap.add_argument('--no-extra', action='store_true',
                    help='skip the FP64 small and batched-collision measurements')
    ap.add_argument('--q-only', type=int, default=0, metavar='NDOF',
                    help='profiling case: 3 launches of the collision kernel on NDOF cubes')
    ap.add_argument('--surrogate-call', type=int, default=0, metavar='NDOF',
                    help='profiling case: all-surrogate hybrid calls on NDOF cells')
    ap.add_argument('--surrogate-curve', action='store_true',
                    help='analysis case: the Couette surrogate at 64..512 modes')
    ap.add_argument('--q-batched', type=int, default=0, metavar='NDOF24',
                    help='profiling case: the two-species collision launch on NDOF24 24^3 and '
                         'NDOF24/3 32^3 cubes')
    ap.add_argument('--hybrid-steps', type=int, default=0, metavar='N',
                    help='profiling case: N hybrid SSP-RK2 steps of the lid-driven cavity '
                         '(random surrogate with zero head scales)')
    ap.add_argument('--ars-only', action='store_true',
                    help='profiling case: the adgfs ARS-222 leg alone')
    ap.add_argument('--dgfsbi-only', action='store_true',
                    help='profiling case: the dgfsbi mixture Couette leg alone')
    ap.add_argument('--vss-only', type=int, default=0, metavar='NDOF',
                    help='profiling case: the gas-mixture collision launch on NDOF pairs')
    ap.add_argument('--fr-only', choices=['couette', 'cavity'],
                    help='profiling case: the FR kernels of one RK stage')
    args = ap.parse_args()
    if args.q_only:
        run_q_only(args.q_only)
    elif args.surrogate_call:
        run_surrogate_call(args.surrogate_call)
    elif args.surrogate_curve:
        run_surrogate_curve()
    elif args.hybrid_steps:
        run_hybrid_steps(args.hybrid_steps)
    elif args.q_batched:
        import torch
        flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
        res, _ = batched_q(flush, reps=2, sizes=(args.q_batched, args.q_batched // 3))
        print(json.dumps(res))
    elif args.ars_only:
        run_ars_only()
    elif args.vss_only:
        run_vss_only(args.vss_only)
    elif args.dgfsbi_only:
        run_dgfsbi_only()
    elif args.fr_only:
        run_fr_only(args.fr_only)
    elif args.impl == 'reference':
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
