"""Oracle: fast-spectral VSS collision operator of a gas mixture, FP64.

Restates ``DGFSBiVSSGLLScatteringModel`` (frfs/solvers/dgfsbi/scattering.py:
45-330), its velocity mesh (frfs/solvers/dgfsbi/velocitymesh.py:25-180) and
its kernels (frfs/solvers/dgfsbi/kernels/scattering/vss-gll.mako:31-300)
step by step, with the reference's operation order:

  per species pair (p, q) and distribution
    F = FFT(f_p)/n, G = FFT(f_q)/n                       (r2z, FFT, cosSinMul)
    for every radius r and full-sphere direction s, a = pi/L qz_r (s . l):
      t1 = e^{+i a m_q/(m_p+m_q)} F,  t2 = e^{-i a m_p/(m_p+m_q)} G
      T  = IFFT(t1) * IFFT(t2)      (complex product, unnormalised IFFTs)
      G^ += qw_r sw/n  b_pq[r, s] * FFT(T)               (computeQG)
    Q_pq = prefac_pq (Re IFFT(G^) - f_p Re IFFT(c_pq G)) (ax2, output)
  Q_p = sum_q Q_pq

  b_pq[r, s, l] = sum_t B swpre qz_r^(gamma_pq+2) e^{-i m_q/(m_p+m_q) pi/L qz_r (t . l)}
  c_pq[l]       = sum_{r, s, t} B qw_r sw swpre qz_r^(gamma_pq+2) e^{-i pi/L qz_r (t . l)}
  B = (1 + s . t)^(alpha_pq - 1), t over the Mpre pre-computation directions
                                                          (precompute_bc_pq)
Test infrastructure only.
"""
from fractions import Fraction
from itertools import product
from math import gamma as _gamma

import numpy as np

from oracle.velocitymesh import NA, R0, gauss_jacobi
from oracle.vhs import _fftn, _ifftn_unnorm, lgrid


class BiVelocityMesh:
    """velocitymesh.py:25-180 of dgfsbi (FP64): the box [-L, L]^3 with the
    mass-ratio-dependent radius R = 2 S and full-sphere directions sz (M
    points, sw = 4 pi / M)."""

    def __init__(self, Nv, Nrho, sz, masses, *, H0, T0, rho0, molarMass0, cmax, Tmax, dev,
                 quad_alpha=0.0, quad_beta=0.0):
        self.Nv, self.Nrho = int(Nv), int(Nrho)
        self.vsize = self.Nv**3
        self.H0, self.T0, self.rho0, self.molarMass0 = H0, T0, rho0, molarMass0
        self.n0 = rho0 / molarMass0 * NA
        self.u0 = np.sqrt(2 * R0 / molarMass0 * T0)
        self.masses = [float(m) for m in masses]              # molar masses / molarMass0
        mr = max(self.masses)
        self.L = cmax / self.u0 + dev * np.sqrt(Tmax / T0)
        self.S = min(self.L * 2.0 / (max(4. * mr / (1. + mr), 2.) + np.sqrt(1. + mr) + 1.),
                     self.L * 2.0 / (max(4. / (1. + mr), 2.) + np.sqrt(1. + 1. / mr) + 1.))
        self.R = 2 * self.S
        self.cw = (2.0 * self.L / self.Nv)**3
        N, L = self.Nv, self.L
        self.c0 = np.linspace(-L + L / N, L - L / N, N)
        I, J, K = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing='ij')
        self.cv = np.stack([self.c0[I].ravel(), self.c0[J].ravel(), self.c0[K].ravel()])
        qz, qw = gauss_jacobi(self.Nrho, quad_alpha, quad_beta)
        self.qz = (self.R / 2.0) * (1.0 + qz)
        self.qw = (self.R / 2.0) * qw
        self.sz = np.asarray(sz, dtype=np.float64)
        self.M = self.sz.shape[0]
        self.sw = 4 * np.pi / self.M


def vss_parameters(vm, pairs):
    """scattering.py:51-92: gamma_pq = 2 (1 - omega_pq), eta_pq = alpha_pq - 1
    and the prefactor of each ordered pair; pairs[(p, q)] = dict(alpha,
    omega, dRef, Tref)."""
    out = {}
    m = vm.masses
    for (p, q), c in pairs.items():
        alpha, omega, dRef, Tref = c['alpha'], c['omega'], c['dRef'], c['Tref']
        invKn = (np.sqrt(1. + m[p] / m[q]) * np.pi * vm.n0 * dRef * dRef
                 * (Tref / vm.T0)**(omega - 0.5) * vm.H0)
        mu = m[p] * m[q] / (m[p] + m[q])
        pref = invKn * alpha / (np.sqrt(1. + m[p] / m[q]) * mu**(omega - 0.5)
                                * 2.**(1 + alpha) * _gamma(2.5 - omega) * np.pi)
        out[(p, q)] = dict(gamma=2.0 * (1. - omega), eta=alpha - 1., prefac=pref)
    return out


def one_plus_cos(sz, szpre):
    """The base of B in precompute_bc_pq (vss-gll.mako:80-82),
    1 + szx[y] t_x + szy[y] t_y + szz[y] t_z, as the GPU evaluates the
    expression: three fused multiply-adds (the compiler's default
    contraction), each rounded once (emulated exactly with rationals).  At
    t = -s the exact value is 0 and this rounding decides B there."""
    def fma(a, b, c):
        return float(Fraction(a) * Fraction(b) + Fraction(c))
    out = np.empty((sz.shape[0], szpre.shape[0]))
    for y, s in enumerate(np.asarray(sz, dtype=np.float64).tolist()):
        for t, u in enumerate(np.asarray(szpre, dtype=np.float64).tolist()):
            out[y, t] = fma(s[2], u[2], fma(s[1], u[1], fma(s[0], u[0], 1.0)))
    return out


def precompute_bc(vm, szpre, gamma_pq, eta_pq, mq_frac):
    """precompute_bc_pq (vss-gll.mako:53-95): b[r*M+s, l] and c[l], complex."""
    l = lgrid(vm.Nv)
    Mpre = szpre.shape[0]
    swpre = 4 * np.pi / Mpre
    P = vm.Nrho * vm.M
    b = np.zeros((P, vm.vsize), complex)
    c = np.zeros(vm.vsize, complex)
    Bst = one_plus_cos(vm.sz, szpre)**eta_pq                  # [M, Mpre]
    tl = szpre @ l                                            # [Mpre, n]
    for r in range(vm.Nrho):
        fac = np.pi / vm.L * vm.qz[r]
        fac_b = swpre * vm.qz[r]**(gamma_pq + 2)
        fac_c = vm.qw[r] * vm.sw * fac_b
        eb = np.exp(-1j * mq_frac * fac * tl)                 # [Mpre, n]
        ec = np.exp(-1j * fac * tl)
        for s in range(vm.M):
            b[r * vm.M + s] = fac_b * (Bst[s] @ eb)
            c += fac_c * (Bst[s] @ ec)
    return b, c


class VSSOracle:
    """Q_p = sum_q Q_pq for every species p of one velocity point."""

    def __init__(self, vm, szpre, pairs, workers=1):
        self.vm = vm
        self.nspcs = len(vm.masses)
        self.par = vss_parameters(vm, pairs)
        self.l = lgrid(vm.Nv)
        self.workers = workers
        m = vm.masses
        self.b, self.c = {}, {}
        for (p, q), pr in self.par.items():
            mq = m[q] / (m[p] + m[q])
            self.b[(p, q)], self.c[(p, q)] = precompute_bc(vm, szpre, pr['gamma'], pr['eta'], mq)
        # a[r*M+s, l] = pi/L qz_r (s . l)                      (precompute_a)
        self.a = np.concatenate([np.pi / vm.L * vm.qz[r] * (vm.sz @ self.l)
                                 for r in range(vm.Nrho)])

    def Qpq(self, p, q, fp, fq):
        vm, N, n = self.vm, self.vm.Nv, self.vm.vsize
        m = vm.masses
        shp = (N, N, N)
        F = _fftn(fp.reshape(shp).astype(complex), self.workers).ravel() / n
        G = _fftn(fq.reshape(shp).astype(complex), self.workers).ravel() / n
        mq, mp = m[q] / (m[p] + m[q]), m[p] / (m[p] + m[q])
        t1 = np.exp(1j * mq * self.a) * F[None]
        t2 = np.exp(-1j * mp * self.a) * G[None]
        P = t1.shape[0]
        T = (_ifftn_unnorm(t1.reshape((P,) + shp), self.workers)
             * _ifftn_unnorm(t2.reshape((P,) + shp), self.workers))
        S = _fftn(T, self.workers).reshape(P, n)
        w = np.repeat(vm.qw * vm.sw / n, vm.M)                # r-major, as a
        QGh = np.sum(w[:, None] * self.b[(p, q)] * S, axis=0)
        QG = _ifftn_unnorm(QGh.reshape(shp), self.workers).ravel()
        QL = _ifftn_unnorm((self.c[(p, q)] * G).reshape(shp), self.workers).ravel()
        return self.par[(p, q)]['prefac'] * (QG.real - fp * QL.real)

    def Q(self, fs):
        """fs: list of species distributions [n]; returns [Q_p]."""
        return [sum(self.Qpq(p, q, fs[p], fs[q]) for q in range(self.nspcs))
                for p in range(self.nspcs)]


def full_sphere(half):
    """A full antipodal design from one point of each pair."""
    half = np.asarray(half, dtype=np.float64)
    return np.concatenate([half, -half])


def all_pairs(nspcs, alpha=1.0, omega=0.81, dRef=4.17e-10, Tref=273.0):
    return {(p, q): dict(alpha=alpha, omega=omega, dRef=dRef, Tref=Tref)
            for p, q in product(range(nspcs), repeat=2)}


def mixture_moments(fs, cv, cw, masses):
    """Per-species fields of one mixture distribution set, non-dimensional,
    as plugins/dgfsmomwriterbi.py:258-385 forms them before its dimensional
    scaling: rho_p = m_p sum f cw, U_p, T_p = (2/3) m_p sum f |c-U_p|^2 cw /
    (sum f cw); heat flux m_p^2 sum f |c-U|^2 (c-U) cw and pressure tensor
    2 m_p^2 sum f (c-U)_i (c-U)_j cw about the mixture velocity
    U = sum rho_p U_p / sum rho_p."""
    out = []
    for f, m in zip(fs, masses):
        mcw = m * cw
        rho = np.sum(f) * mcw
        U = cv @ f * mcw / rho
        c = cv - U[:, None]
        T = np.sum(f * np.sum(c * c, axis=0)) * (2.0 / 3.0 * mcw * m) / rho
        out.append({'rho': rho, 'U': U, 'T': T, 'nden': rho / m})
    rho = sum(o['rho'] for o in out)
    W = sum(o['rho'] * o['U'] for o in out) / rho
    c = cv - W[:, None]
    c2 = np.sum(c * c, axis=0)
    for f, m, o in zip(fs, masses, out):
        mcw = m * cw
        o['q'] = np.array([m * np.sum(f * c2 * c[a]) * mcw for a in range(3)])
        o['P'] = np.array([2 * m * np.sum(f * c[a] * c[b]) * mcw
                           for a, b in ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))])
    return out, {'rho': rho, 'U': W}


def project_mixture(Qs, cv, masses):
    """Minimal-norm change of the concatenated (Q_0 .. Q_{S-1}) that zeroes
    each species' mass and the total (mass-weighted) momentum and energy,
    solved directly from the stacked constraint vectors (the checker of the
    device projection; the reference has none)."""
    S, n = len(Qs), cv.shape[1]
    c2 = np.sum(cv * cv, axis=0)
    rows = []
    for p in range(S):
        r = np.zeros(S * n)
        r[p * n:(p + 1) * n] = 1.0
        rows.append(r)
    for phi in (cv[0], cv[1], cv[2], c2):
        rows.append(np.concatenate([m * phi for m in masses]))
    A = np.stack(rows)
    q = np.concatenate(Qs)
    lam = np.linalg.solve(A @ A.T, A @ q)
    q = q - A.T @ lam
    return [q[p * n:(p + 1) * n] for p in range(S)]
