"""Shared test set-up: configs, seeded distributions, oracle construction."""
import numpy as np

from frfs_b200.inifile import Inifile

NONDIM = dict(T0=273.0, H0=1e-3, rho0=0.00011140244750324529, molarMass0=39.96e-3)


def vhs_cfg(Nv, Nrho, M, dev, omega=0.81, precision='single', extra=''):
    return Inifile(f"""
[backend]
precision = {precision}
[constants]
Nv = {Nv}
Nrho = {Nrho}
[non-dim]
T0 = {NONDIM['T0']}
H0 = {NONDIM['H0']}
rho0 = {NONDIM['rho0']}
molarMass0 = {NONDIM['molarMass0']}
[velocity-mesh]
dev = {dev}
cmax = 0
Tmax = 273
[spherical-design-rule]
ssrule = womersley
M = {M}
[scattering-model]
type = vhs-gll
omega = {omega}
dRef = 4.17e-10
Tref = 273
{extra}
""")


def oracle_for(vm_prod, omega=0.81):
    """FP64 oracle on the same mesh parameters and directions."""
    from oracle.velocitymesh import VelocityMesh
    from oracle.vhs import VHSOracle
    dev = vm_prod.L()          # cmax = 0, Tmax = T0 -> L = dev
    vm = VelocityMesh(vm_prod.Nv(), vm_prod.Nrho(), vm_prod.sz(), cmax=0.0,
                      Tmax=NONDIM['T0'], dev=dev, **NONDIM)
    return VHSOracle(vm, omega, 4.17e-10, 273.0)


def maxwellian(cv, n, u, T):
    u = np.asarray(u, dtype=np.float64)[:, None]
    return n / (np.pi * T)**1.5 * np.exp(-np.sum((cv - u)**2, axis=0) / T)


def random_ball(rng, rmax):
    u = rng.normal(size=3)
    return u / np.linalg.norm(u) * rmax * rng.uniform()**(1 / 3)


def mixed_maxwellians(cv, rng, k=None, nrange=(0.2, 2.0), umax=1.0,
                      Trange=(0.5, 2.0), noise=0.01):
    """Sum of 1-3 seeded Maxwellians plus uniform relative noise (the batched
    collision workload's distribution family)."""
    k = rng.integers(1, 4) if k is None else k
    f = 0.0
    for _ in range(k):
        f = f + maxwellian(cv, rng.uniform(*nrange), random_ball(rng, umax),
                           rng.uniform(*Trange))
    if noise:
        f = f * (1.0 + noise * rng.uniform(-1.0, 1.0, size=f.shape))
    return f


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def couette_cfg(Nv, Nrho, M, dev, order, precision='single', uw=0.3, scheme='dgfs-tvd-rk2',
                dt=5e-4, omega=0.81, T=1.0, extra=''):
    """Couette-type config: walls at y = -+0.5 moving at -+uw (non-dim)."""
    import numpy as np
    u0 = np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])
    rho0 = NONDIM['rho0']
    return vhs_cfg(Nv, Nrho, M, dev, omega=omega, precision=precision, extra=f"""
[solver]
system = dgfs
order = {order}
[solver-time-integrator]
scheme = {scheme}
controller = none
tstart = 0.0
tend = 1.0
dt = {dt}
[soln-ics]
type = maxwellian
rho = {rho0}
T = {NONDIM['T0'] * T}
ux = 0
uy = 0
uz = 0
[soln-bcs-y-]
type = dgfs-wall-diffuse
rho = {rho0}
T = {NONDIM['T0']}
ux = {-uw * u0}
uy = 0
uz = 0
[soln-bcs-y+]
type = dgfs-wall-diffuse
rho = {rho0}
T = {NONDIM['T0']}
ux = {uw * u0}
uy = 0
uz = 0
{extra}
""")


def bc_cfg(Nv, order, bcs, precision='single', scheme='dgfs-tvd-rk2', dt=5e-4, Nrho=8, M=6,
           dev=5):
    """A config whose named boundaries ('x-', 'x+', ...) carry the boundary
    types of ``bcs``: inlets at 0.2 u0 into the domain along x with 1.2 T0,
    diffuse walls at rest, 'dgfs-wall-diffuse-cyl' with a wall temperature
    and tangential speed that vary along the wall."""
    u0 = np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])
    rho0, T0 = NONDIM['rho0'], NONDIM['T0']
    sects = []
    for name, t in bcs.items():
        if t == 'dgfs-wall-diffuse-cyl':
            body = (f"rho = {rho0}\nT = {T0} * (1.0 + 0.2 * (x < 0.5) * x)\n"
                    f"ux = {0.1 * u0} * (1 + y)\nuy = 0\nuz = {0.05 * u0} * abs(x - 0.5)")
        elif t in ('dgfs-inlet', 'dgfs-inlet-normalshock'):
            body = f"rho = {1.1 * rho0}\nT = {1.2 * T0}\nux = {0.2 * u0}\nuy = 0\nuz = 0"
        elif t == 'dgfs-wall-diffuse':
            body = f"rho = {rho0}\nT = {T0}\nux = 0\nuy = 0\nuz = 0"
        else:
            body = ''
        sects.append(f"[soln-bcs-{name}]\ntype = {t}\n{body}\n")
    return vhs_cfg(Nv, Nrho, M, dev, precision=precision, extra=f"""
[solver]
system = dgfs
order = {order}
[solver-time-integrator]
scheme = {scheme}
controller = none
tstart = 0.0
tend = 1.0
dt = {dt}
[soln-ics]
type = maxwellian
rho = {rho0}
T = {T0}
ux = 0
uy = 0
uz = 0
""" + '\n'.join(sects))


def vss_cfg(Nv, Nrho, M, Mpre, masses=(39.96e-3, 83.798e-3), alpha=1.3, omega=0.81, dev=5,
            precision='double', project=False):
    """Gas-mixture config of the 'vss-gll' model: every ordered species pair
    with the same VSS parameters."""
    S = len(masses)
    pairs = '\n'.join(f'alpha{p}{q} = {alpha}\nomega{p}{q} = {omega}\ndRef{p}{q} = 4.17e-10\n'
                      f'Tref{p}{q} = 273' for p in range(S) for q in range(S))
    mm = '\n'.join(f'molarMass{p + 1} = {m}' for p, m in enumerate(masses))
    return Inifile(f"""
[backend]
precision = {precision}
[constants]
Nv = {Nv}
Nrho = {Nrho}
[non-dim]
T0 = {NONDIM['T0']}
H0 = {NONDIM['H0']}
rho0 = {NONDIM['rho0']}
molarMass0 = {NONDIM['molarMass0']}
[velocity-mesh]
dev = {dev}
cmax = 0
Tmax = 273
{mm}
[spherical-design-rule]
ssrule = womersley
M = {M}
[scattering-model]
type = vss-gll
Mpre = {Mpre}
ssrulepre = womersley
conservation-projection = {'true' if project else 'false'}
{pairs}
""")


def dgfsbi_cfg(Nv=16, Nrho=4, M=6, Mpre=6, order=2, precision='double', dev=4, uw=0.3,
               scheme='dgfsbi-tvd-rk2', dt=2e-4, masses=(39.96e-3, 83.798e-3)):
    """Gas mixture between diffuse walls at y = -+0.5 moving at -+uw
    (non-dim), x periodic: the 'dgfsbi' system with 'vss-gll'."""
    u0 = np.sqrt(2 * 8.3144598 / NONDIM['molarMass0'] * NONDIM['T0'])
    n0 = NONDIM['rho0'] / NONDIM['molarMass0'] * 6.0221409e+23
    cfg = vss_cfg(Nv, Nrho, M, Mpre, masses=masses, dev=dev, precision=precision)
    extra = f"""
[solver]
system = dgfsbi
order = {order}
[solver-time-integrator]
scheme = {scheme}
controller = none
tstart = 0.0
tend = 1.0
dt = {dt}
[soln-ics]
type = maxwellian
{chr(10).join(f'nden{p + 1} = {n0 * (0.7 if p else 0.3)}' for p in range(len(masses)))}
T = {NONDIM['T0']}
ux = 0
uy = 0
uz = 0
[soln-bcs-y-]
type = dgfsbi-wall-diffuse
T = {NONDIM['T0']}
ux = {-uw * u0}
uy = 0
uz = 0
[soln-bcs-y+]
type = dgfsbi-wall-diffuse
T = {NONDIM['T0'] * 1.1}
ux = {uw * u0}
uy = 0
uz = 0
"""
    return Inifile(cfg.tostr() + extra)


def vss_oracle_for(sm):
    """The oracle on the model's mesh, directions and pair parameters."""
    from oracle.vss import BiVelocityMesh, VSSOracle
    vm = sm.vm
    ovm = BiVelocityMesh(vm.Nv(), vm.Nrho(), vm.sz(), vm.masses(), cmax=0.0, Tmax=NONDIM['T0'],
                         dev=vm.L(), **NONDIM)
    pairs = {}
    for p in range(vm.nspcs()):
        for q in range(vm.nspcs()):
            pq = f'{p}{q}'
            c = sm.cfg
            pairs[(p, q)] = dict(alpha=c.getfloat('scattering-model', 'alpha' + pq),
                                 omega=c.getfloat('scattering-model', 'omega' + pq),
                                 dRef=c.getfloat('scattering-model', 'dRef' + pq),
                                 Tref=c.getfloat('scattering-model', 'Tref' + pq))
    return VSSOracle(ovm, sm._szpre, pairs)


def mixture(cv, masses, rng, k=2):
    """Seeded non-equilibrium distributions of each species: sums of
    Maxwellians n (m/(pi T))^1.5 exp(-m |c-u|^2/T)."""
    out = []
    for m in masses:
        f = 0.0
        for _ in range(k):
            n, T = rng.uniform(0.3, 1.2), rng.uniform(0.7, 1.3)
            u = rng.uniform(-0.3, 0.3, size=3)[:, None]
            f = f + n * (m / (np.pi * T))**1.5 * np.exp(-m * np.sum((cv - u)**2, axis=0) / T)
        out.append(f)
    return out
