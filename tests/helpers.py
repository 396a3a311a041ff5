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
