"""Oracle: BGK relaxation ('bgk-direct-gll') and the ARS IMEX steppers (FP64).

Restates, in numpy, for test use only:
  prefactor     t0 p0 / visc, t0 = H0/u0, visc = muRef (T0/Tref)^omega,
                p0 = n0 R0/NA T0           (frfs/solvers/adgfs/scattering.py,
                                            ADGFSBGKDirectGLLScatteringModel.load_parameters)
  moments       U = (sum f, sum c f, sum |c|^2 f) cw  (mat of perform_precomputation)
  Maxwellian    T = (U4 - |U1:3|^2/U0)/(1.5 U0), M = U0/(pi T)^1.5 exp(-|c-u|^2/T)
                                           (kernels/scattering/bgk-direct-gll.mako:4-50)
  nu            prefac U0 T^(1-omega)      (linear-common-direct-gll.mako:121-130)
  ARS stage ar  U_ar = U_0 + dt sum_{j<ar} _A[ar][j] LU_j        (updateMom{ar}_ARS)
                f_ar = (f_0 + sum_{j<ar} _A[ar][j] dt L_j
                        + sum_{j=1}^{ar-1} A[ar][j] dt nu_j (M_j - f_j)
                        + A[ar][ar] dt nu_ar M_ar) / (1 + A[ar][ar] dt nu_ar)
                                           (updateDistribution{ar}_ARS,
                                            linear-common-direct-gll.mako:90-145)
  stepper       ARSabcAstdStepper.step     (frfs/integrators/std/steppers.py:531-585)
                with the tables of ARS-111/222/443 (steppers.py:589-670).
Distributions are arrays [..., nv]; moments [..., 5].
"""
import numpy as np

R0 = 8.3144598
NA = 6.0221409e+23

_g = 1.0 - 2.0**0.5 / 2.0
_d = 1.0 - 1.0 / (2.0 * _g)
ARS = {
    'adgfs-ars-111': ([[0., 0.], [1., 0.]],
                      [[0., 0.], [0., 1.]]),
    'adgfs-ars-222': ([[0., 0., 0.], [_g, 0., 0.], [_d, 1 - _d, 0.]],
                      [[0., 0., 0.], [0., _g, 0.], [0., 1 - _g, _g]]),
    'adgfs-ars-443': ([[0., 0., 0., 0., 0.], [1 / 2, 0., 0., 0., 0.],
                       [11 / 18, 1 / 18, 0., 0., 0.], [5 / 6, -5 / 6, 1 / 2, 0., 0.],
                       [1 / 4, 7 / 4, 3 / 4, -7 / 4, 0.]],
                      [[0., 0., 0., 0., 0.], [0., 1 / 2, 0., 0., 0.],
                       [0., 1 / 6, 1 / 2, 0., 0.], [0., -1 / 2, 1 / 2, 1 / 2, 0.],
                       [0., 3 / 2, -3 / 2, 1 / 2, 1 / 2]]),
}


def bgk_prefactor(H0, u0, T0, n0, omega, muRef, Tref):
    t0 = H0 / u0
    visc = muRef * (T0 / Tref)**omega
    p0 = n0 * R0 / NA * T0
    return t0 * p0 / visc


def moments5(f, cv, cw):
    c2 = np.sum(cv * cv, axis=0)
    return np.stack([f.sum(-1), f @ cv[0], f @ cv[1], f @ cv[2], f @ c2], axis=-1) * cw


def _state(U):
    rho = U[..., 0]
    u = U[..., 1:4] / rho[..., None]
    T = (U[..., 4] - np.sum(U[..., 1:4]**2, axis=-1) / rho) / (1.5 * rho)
    return rho, u, T


def maxwellian(U, cv):
    rho, u, T = _state(U)
    d2 = sum((cv[k][None] - u.reshape(-1, 3)[:, k:k + 1])**2 for k in range(3))
    d2 = d2.reshape(U.shape[:-1] + (cv.shape[1],))
    return (rho / (np.pi * T)**1.5)[..., None] * np.exp(-d2 / T[..., None])


def nu(U, prefac, omega):
    rho, _, T = _state(U)
    return prefac * rho * T**(1.0 - omega)


def step_ars(f0, dt, L, scheme, prefac, omega, cv, cw):
    """One ARS step of df/dt = L(f) + nu (M[f] - f); L(f) is the explicit
    (advection) part, a callable on arrays shaped like f0."""
    _A, A = ARS[scheme]
    s = len(_A) - 1
    F, Ls, LU = [f0], [], []
    U = [moments5(f0, cv, cw)]
    for i in range(s):
        ar = i + 1
        Ls.append(L(F[i]))
        LU.append(moments5(Ls[i], cv, cw))
        U.append(U[0] + dt * sum(_A[ar][j] * LU[j] for j in range(ar)))
        num = F[0] + sum(_A[ar][j] * dt * Ls[j] for j in range(ar))
        for j in range(1, ar):
            num = num + A[ar][j] * dt * nu(U[j], prefac, omega)[..., None] * (
                maxwellian(U[j], cv) - F[j])
        nar = nu(U[ar], prefac, omega)[..., None]
        num = num + A[ar][ar] * dt * nar * maxwellian(U[ar], cv)
        F.append(num / (1.0 + A[ar][ar] * dt * nar))
    return F[s]


# ---------------------------------------------------------------------------
# ES-BGK ('esbgk-direct-gll', frfs/solvers/adgfs/scattering.py,
# ADGFSESBGKDirectGLLScatteringModel; kernels/scattering/esbgk-direct-gll.mako)
#   moments     11: (sum f, sum c f, sum |c|^2 f, sum cx^2 f, sum cy^2 f,
#               sum cz^2 f, sum cx cy f, sum cy cz f, sum cz cx f) cw
#   prefactor   t0 Pr p0 / visc (nu = prefac rho T^(1-omega) as for BGK)
#   Gaussian    (momentNorm, cmaxwellian) T_ii = T/Pr + 2 (1 - 1/Pr)
#               (P_ii/rho - u_i^2), T_ij = 2 (1 - 1/Pr)(P_ij/rho - u_i u_j),
#               G = rho / (pi^1.5 sqrt(det T)) exp(-(c-u)^T T^-1 (c-u))
#   ARS moments (updateMom{ar}_ARS): the conserved five as for BGK; the six
#               second moments relax implicitly at rate nu/Pr to the
#               Maxwellian's (rho T/2 + rho u_i^2, rho u_i u_j).

def esbgk_prefactor(H0, u0, T0, n0, omega, muRef, Tref, Pr):
    return Pr * bgk_prefactor(H0, u0, T0, n0, omega, muRef, Tref)


def moments11(f, cv, cw):
    c2 = np.sum(cv * cv, axis=0)
    cx, cy, cz = cv
    rows = [np.ones_like(cx), cx, cy, cz, c2, cx * cx, cy * cy, cz * cz, cx * cy, cy * cz, cz * cx]
    return np.stack([f @ r for r in rows], axis=-1) * cw


def es_tensor(U, Pr):
    """(rho, u[3], T, Tij[3x3]) of 11-moment rows."""
    rho, u, T = _state(U)
    k = 2.0 * (1.0 - 1.0 / Pr)
    P = np.empty(U.shape[:-1] + (3, 3))
    P[..., 0, 0], P[..., 1, 1], P[..., 2, 2] = U[..., 5], U[..., 6], U[..., 7]
    P[..., 0, 1] = P[..., 1, 0] = U[..., 8]
    P[..., 1, 2] = P[..., 2, 1] = U[..., 9]
    P[..., 2, 0] = P[..., 0, 2] = U[..., 10]
    Tij = k * (P / rho[..., None, None] - u[..., :, None] * u[..., None, :])
    Tij = Tij + (T / Pr)[..., None, None] * np.eye(3)
    return rho, u, T, Tij


def es_gaussian(U, Pr, cv):
    rho, u, T, Tij = es_tensor(U, Pr)
    lead = U.shape[:-1]
    flat = lambda a, s: a.reshape((-1,) + s)
    rho_, u_, Tij_ = flat(rho, ()), flat(u, (3,)), flat(Tij, (3, 3))
    out = np.empty((rho_.shape[0], cv.shape[1]))
    for i in range(rho_.shape[0]):
        d = cv - u_[i][:, None]
        Ti = np.linalg.inv(Tij_[i])
        q = np.einsum('av,ab,bv->v', d, Ti, d)
        out[i] = rho_[i] / (np.pi**1.5 * np.sqrt(np.linalg.det(Tij_[i]))) * np.exp(-q)
    return out.reshape(lead + (cv.shape[1],))


def _es_targets(U):
    """Second moments of the Maxwellian of U: rho T/2 + rho u_i^2, rho u_i u_j."""
    rho, u, T = _state(U)
    t = np.empty(U.shape[:-1] + (6,))
    for k in range(3):
        t[..., k] = 0.5 * rho * T + rho * u[..., k]**2
    t[..., 3] = rho * u[..., 0] * u[..., 1]
    t[..., 4] = rho * u[..., 1] * u[..., 2]
    t[..., 5] = rho * u[..., 2] * u[..., 0]
    return t


def step_ars_es(f0, dt, L, scheme, prefac, omega, Pr, cv, cw):
    """One ARS step of df/dt = L(f) + nu (G[f] - f) (ES-BGK)."""
    _A, A = ARS[scheme]
    s = len(_A) - 1
    F, Ls, LU = [f0], [], []
    U = [moments11(f0, cv, cw)]
    for i in range(s):
        ar = i + 1
        Ls.append(L(F[i]))
        LU.append(moments11(Ls[i], cv, cw))
        Ua = U[0] + dt * sum(_A[ar][j] * LU[j] for j in range(ar))
        # second moments: implicit relaxation at nu/Pr towards the Maxwellian's
        rate = lambda Uj: nu(Uj, prefac, omega) / Pr
        num = Ua[..., 5:].copy()
        for j in range(1, ar):
            num += A[ar][j] * dt * rate(U[j])[..., None] * (_es_targets(U[j]) - U[j][..., 5:])
        ra = rate(Ua)[..., None]
        num += A[ar][ar] * dt * ra * _es_targets(Ua)
        Ua[..., 5:] = num / (1.0 + A[ar][ar] * dt * ra)
        U.append(Ua)
        num = F[0] + sum(_A[ar][j] * dt * Ls[j] for j in range(ar))
        for j in range(1, ar):
            num = num + A[ar][j] * dt * nu(U[j], prefac, omega)[..., None] * (
                es_gaussian(U[j], Pr, cv) - F[j])
        nar = nu(U[ar], prefac, omega)[..., None]
        num = num + A[ar][ar] * dt * nar * es_gaussian(U[ar], Pr, cv)
        F.append(num / (1.0 + A[ar][ar] * dt * nar))
    return F[s]


# ---------------------------------------------------------------------------
# Shakov ('shakov-direct-gll', frfs/solvers/adgfs/scattering.py,
# ADGFSShakovDirectGLLScatteringModel; kernels/scattering/shakov-direct-gll.mako)
#   moments     14: the 11 ES-BGK rows and |c|^2 c (x, y, z), times cw
#   prefactor   t0 p0 / visc (as BGK), Pr from the .ini (default 2/3)
#   heat flux   (momentNorm) q_i = Q_i - 2 P_ij u_j + rho u_i |u|^2 - 1.5 rho T u_i
#   target      (cmaxwellian) S = M (1 + 2 (1 - Pr)/5 (q.d)/(rho T^2) (2|d|^2/T - 5)),
#               d = c - u
#   ARS moments (updateMom{ar}_ARS): the conserved five explicit; the six
#               second moments relax implicitly at nu to the Maxwellian's;
#               Q relaxes as dQ/dt = nu (Q(M) + (1 - Pr)(q - Q) - Pr Q), only
#               the -Pr Q part implicit, with this stage's second moments.

def shakov_prefactor(H0, u0, T0, n0, omega, muRef, Tref):
    return bgk_prefactor(H0, u0, T0, n0, omega, muRef, Tref)


def moments14(f, cv, cw):
    c2 = np.sum(cv * cv, axis=0)
    rows = [c2 * cv[0], c2 * cv[1], c2 * cv[2]]
    return np.concatenate([moments11(f, cv, cw), np.stack([f @ r for r in rows], axis=-1) * cw],
                          axis=-1)


def _stress(U):
    """Raw second moments of 14-moment rows as [..., 3, 3]."""
    P = np.empty(U.shape[:-1] + (3, 3))
    P[..., 0, 0], P[..., 1, 1], P[..., 2, 2] = U[..., 5], U[..., 6], U[..., 7]
    P[..., 0, 1] = P[..., 1, 0] = U[..., 8]
    P[..., 1, 2] = P[..., 2, 1] = U[..., 9]
    P[..., 2, 0] = P[..., 0, 2] = U[..., 10]
    return P


def heat_flux(U):
    rho, u, T = _state(U)
    Pu = np.einsum('...ij,...j->...i', _stress(U), u)
    u2 = np.sum(u * u, axis=-1)
    return (U[..., 11:14] - 2.0 * Pu + (rho * u2)[..., None] * u
            - 1.5 * (rho * T)[..., None] * u)


def shakov_target(U, Pr, cv):
    rho, u, T = _state(U)
    q = heat_flux(U)
    M = maxwellian(U[..., :5], cv)
    lead = U.shape[:-1]
    u_, q_ = u.reshape(-1, 3), q.reshape(-1, 3)
    d = cv[None] - u_[:, :, None]                       # [n, 3, nv]
    qd = np.einsum('ni,niv->nv', q_, d).reshape(lead + (cv.shape[1],))
    d2 = np.sum(d * d, axis=1).reshape(lead + (cv.shape[1],))
    k = 2.0 * (1.0 - Pr) / 5.0 / (rho * T * T)
    return M * (1.0 + k[..., None] * qd * (2.0 * d2 / T[..., None] - 5.0))


def _heat_targets(U, Pr):
    """Q(M) + (1 - Pr)(q - Q): the explicit part of the heat-flux relaxation
    (q - Q written out, as the reference does, so that Q cancels exactly)."""
    rho, u, T = _state(U)
    u2 = np.sum(u * u, axis=-1)
    QM = (rho * u2)[..., None] * u + 2.5 * (rho * T)[..., None] * u
    qmQ = (-2.0 * np.einsum('...ij,...j->...i', _stress(U), u) + (rho * u2)[..., None] * u
           - 1.5 * (rho * T)[..., None] * u)
    return QM + (1.0 - Pr) * qmQ


def step_ars_sk(f0, dt, L, scheme, prefac, omega, Pr, cv, cw):
    """One ARS step of df/dt = L(f) + nu (S[f] - f) (Shakov)."""
    _A, A = ARS[scheme]
    s = len(_A) - 1
    F, Ls, LU = [f0], [], []
    U = [moments14(f0, cv, cw)]
    for i in range(s):
        ar = i + 1
        Ls.append(L(F[i]))
        LU.append(moments14(Ls[i], cv, cw))
        Ua = U[0] + dt * sum(_A[ar][j] * LU[j] for j in range(ar))
        rate = lambda Uj: nu(Uj, prefac, omega)
        ra = rate(Ua)[..., None]
        num = Ua[..., 5:11].copy()
        for j in range(1, ar):
            num += A[ar][j] * dt * rate(U[j])[..., None] * (_es_targets(U[j]) - U[j][..., 5:11])
        num += A[ar][ar] * dt * ra * _es_targets(Ua)
        Ua[..., 5:11] = num / (1.0 + A[ar][ar] * dt * ra)
        num = Ua[..., 11:14].copy()
        for j in range(1, ar):
            num += A[ar][j] * dt * rate(U[j])[..., None] * (
                _heat_targets(U[j], Pr) - Pr * U[j][..., 11:14])
        # this stage's heat-flux target uses the explicit Q_ar only through
        # (1 - Pr)(q - Q), which does not depend on Q
        num += A[ar][ar] * dt * ra * _heat_targets(Ua, Pr)
        Ua[..., 11:14] = num / (1.0 + Pr * A[ar][ar] * dt * ra)
        U.append(Ua)
        num = F[0] + sum(_A[ar][j] * dt * Ls[j] for j in range(ar))
        for j in range(1, ar):
            num = num + A[ar][j] * dt * nu(U[j], prefac, omega)[..., None] * (
                shakov_target(U[j], Pr, cv) - F[j])
        nar = nu(U[ar], prefac, omega)[..., None]
        num = num + A[ar][ar] * dt * nar * shakov_target(U[ar], Pr, cv)
        F.append(num / (1.0 + A[ar][ar] * dt * nar))
    return F[s]


# ---------------------------------------------------------------------------
# IMEX-BDF steppers ('adgfs-bdf-1/2/3', frfs/integrators/std/steppers.py:675-860)
#   moments  N = -sum_i (a_i U_i + g_i dt LU_i); U = N / a_q (conserved five);
#            second moments (ES-BGK: rate b nu/Pr, Shakov: b nu) and the Shakov
#            heat flux (denominator a_q + Pr b dt nu) relax implicitly
#            (updateMom{q}_BDF of the three scattering .mako files)
#   dist     f = (-sum_i (a_i f_i + g_i dt L_i) + b dt nu M[U]) / (a_q + b dt nu)
#            (updateDistribution{q}_BDF, linear-common-direct-gll.mako:40-88)
#   start    the first q - 1 steps: nstepsInit ARS-222 sub-steps each
BDF = {2: ([1. / 3., -4. / 3., 1.], [-2. / 3., 4. / 3.], 2. / 3., 10),
       3: ([-2. / 11., 9. / 11., -18. / 11., 1.], [6. / 11., -18. / 11., 18. / 11.], 6. / 11., 100)}

MODELS = {
    'bgk': (moments5, lambda U, Pr, cv: maxwellian(U, cv)),
    'esbgk': (moments11, es_gaussian),
    'shakov': (moments14, shakov_target),
}


def bdf_update(fs, Ls, Us, LUs, a, g, b, dt, prefac, omega, Pr, cv, model):
    """One BDF update from histories (oldest first); returns (U_new, f_new).
    g are the coefficients as passed to the reference kernels (-G)."""
    q = len(fs)
    N = -sum(a[i] * Us[i] + g[i] * dt * LUs[i] for i in range(q))
    U = N / a[q]
    rate = nu(U, prefac, omega)[..., None]
    if model == 'esbgk':
        w = b * dt * rate / Pr
        U[..., 5:11] = (N[..., 5:11] + w * _es_targets(U)) / (a[q] + w)
    if model == 'shakov':
        w = b * dt * rate
        U[..., 5:11] = (N[..., 5:11] + w * _es_targets(U)) / (a[q] + w)
        U[..., 11:14] = (N[..., 11:14] + w * _heat_targets(U, Pr)) / (a[q] + Pr * w)
    M = MODELS[model][1](U, Pr, cv)
    Nf = -sum(a[i] * fs[i] + g[i] * dt * Ls[i] for i in range(q))
    return U, (Nf + b * dt * rate * M) / (a[q] + b * dt * rate)


def run_bdf(f0, dt, L, nsteps, q, prefac, omega, Pr, cv, cw, model='bgk'):
    """nsteps calls of the BDF-q stepper from f0: the first q - 1 calls take
    nstepsInit ARS-222 sub-steps of dt / nstepsInit, then BDF steps."""
    A, G, b, ninit = BDF[q]
    g = [-x for x in G]
    mom = MODELS[model][0]

    def ars(f, h):
        if model == 'bgk':
            return step_ars(f, h, L, 'adgfs-ars-222', prefac, omega, cv, cw)
        if model == 'esbgk':
            return step_ars_es(f, h, L, 'adgfs-ars-222', prefac, omega, Pr, cv, cw)
        return step_ars_sk(f, h, L, 'adgfs-ars-222', prefac, omega, Pr, cv, cw)
    hist = [f0]
    f = f0
    for k in range(nsteps):
        if k < q - 1:
            for _ in range(ninit):
                f = ars(f, dt / ninit)
            hist.append(f)
            continue
        fs = hist[-q:]
        Ls = [L(x) for x in fs]
        Us = [mom(x, cv, cw) for x in fs]
        LUs = [mom(x, cv, cw) for x in Ls]
        _, f = bdf_update(fs, Ls, Us, LUs, A, g, b, dt, prefac, omega, Pr, cv, model)
        hist.append(f)
    return f
