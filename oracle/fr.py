"""Oracle: FR advection operator, diffuse-wall BC and DGFS steppers (FP64).

Restates, interface by interface as the reference does:
  disu        u_f = M0 u                        (frfs/solvers/dgfs/elements.py:56-59)
  tdisf       F~_i = sum_k smats[i][k] c_k u     (kernels/tflux.mako:6-25, flux.mako:4-20)
  tdivtpcorf  R = (M1 - M3 M2) F~                (elements.py:79-82)
  comm_flux   upwind: fn = 1/2 (n.c)(uL+uR) + 1/2 |n.c| (uL-uR);
              uL <- |n| fn, uR <- -|n| fn        (kernels/intcflux.mako:7-24,
                                                  rsolvers/rusanov.mako:5-52)
  bc flux     ghost uR = f_w (-bc0/bc1) if (c-Uw).n < 0 else uL, then the
              same upwind flux, uL <- |n| fn     (kernels/bccflux.mako:8-38,
                                                  bcs/dgfs-wall-diffuse.mako:4-20)
  update_bc   bc0 = sum_{(c-Uw).n >= 0} (c-Uw).n uL cw,
              bc1 = sum_{(c-Uw).n < 0} (c-Uw).n f_w cw
                                                 (bccupdate.mako:8-23,
                                                  bcs/dgfs-wall-diffuse-update.mako:4-38)
  other BCs   ghost uR by the boundary's type (kernels/bcs/<type>.mako):
              dgfs-inlet: f_in if (c-U).n < 0 else uL; dgfs-inlet-normalshock:
              f_in if c.n < 0 else uL; dgfs-vanish: 0 if c.n < 0 else uL;
              dgfs-outlet: uL; dgfs-wall-specular: uL at the grid velocity
              nearest to c - 2 (c.n) n (inters.py:232-311); dgfs-wall-diffuse-cyl
              is the diffuse wall with a per-point f_w (its own U, T)
  tdivtconf   R += M3 Fhat                       (elements.py:85-88)
  negdivconf  R = -rcpdjac R                     (kernels/negdivconf.mako:5-13)
  invmass     M12 u, M12 the inverse mass matrix (elements.py:161-164,
                                                  shapes.py:163-166)
and the steppers dgfs-euler / dgfs-tvd-rk2 (frfs/integrators/std/steppers.py:20-225).
Arrays are element-major: u[e][upt][v].  Test infrastructure only.
"""
import numpy as np


def velocities(c0):
    N = len(c0)
    idx = np.arange(N**3)
    return np.stack([c0[idx // (N * N)], c0[(idx // N) % N], c0[idx % N]])


class FROracle:
    """ops: dict with M0, M132, M3 (reference operator matrices);
    geo: object with smats[e][u][i][k], rcpdjac[e][u], norm_pnorm[e][f][d],
    mag_pnorm[e][f], nbr[e][f] (>= 0: e'*nfpts + f'; < 0: -1 - wall index),
    wall_fpts[w] = (e, f), wall_bcid[w]; walls: list of (Uw[3], f_w[nv]) or
    (Uw[3], f_w[nv], type) rows (type: the .ini boundary type, default
    'dgfs-wall-diffuse'); bcid[w]: the row of wall point w (default
    geo.wall_bcid)."""

    def __init__(self, ops, geo, c0, cw, walls=(), bcid=None):
        self.M0, self.M132, self.M3 = ops['M0'], ops['M132'], ops['M3']
        self.geo = geo
        self.c0 = np.asarray(c0, np.float64)
        self.cv = velocities(self.c0)
        self.cw = cw
        self.walls = [w if len(w) == 3 else (w[0], w[1], 'dgfs-wall-diffuse') for w in walls]
        self.bcid = np.asarray(geo.wall_bcid if bcid is None else bcid)
        self.ndims = geo.smats.shape[2]

    def mirror(self, n):
        """Index map of the specular reflection c -> c - 2 (c.n) n onto the
        nearest grid velocity (inters.py:232-311: argmin of the squared
        distance, which on the tensor-product grid is the nearest c0 per
        component)."""
        n3 = np.zeros(3)
        n3[:len(n)] = n
        cr = self.cv - 2.0 * (n3 @ self.cv)[None, :] * n3[:, None]
        idx = [np.argmin(np.abs(cr[d][:, None] - self.c0[None, :]), axis=1) for d in range(3)]
        N = len(self.c0)
        return (idx[0] * N + idx[1]) * N + idx[2]

    def disu(self, u):
        return np.einsum('fu,euv->efv', self.M0, u)

    def update_bc(self, uf):
        g = self.geo
        d = self.ndims
        nw = len(g.wall_fpts)
        bc = np.zeros((nw, 2))
        for w, (e, f) in enumerate(g.wall_fpts):
            Uw, fw, kind = self.walls[self.bcid[w]]
            if kind != 'dgfs-wall-diffuse':
                bc[w] = (0.0, -1.0)
                continue
            n = g.norm_pnorm[e, f]
            fac = sum((self.cv[j] - Uw[j]) * n[j] for j in range(d))
            ul = uf[e, f]
            bc[w, 0] = np.sum(np.where(fac >= 0, fac * ul * self.cw, 0.0))
            bc[w, 1] = np.sum(np.where(fac < 0, fac * fw * self.cw, 0.0))
        return bc

    def update_bc_from_state(self, u):
        """update_bc from the solution itself, with the face values formed
        only at the wall points (the same sums as ``update_bc(disu(u))``;
        keeps the full velocity set without a mesh-wide face array)."""
        g = self.geo
        uf = {}
        for e, f in g.wall_fpts:
            if (e, f) not in uf:
                uf[e, f] = self.M0[f] @ u[e]

        class _Faces:
            def __getitem__(_, ef):
                return uf[ef]
        return self.update_bc(_Faces())

    def restrict(self, vsel):
        """The same operator on the velocity subset vsel.  The FR operator
        acts on every velocity separately; only the diffuse-wall sums couple
        them, so pass ``bc`` from the full set (``update_bc_from_state``) to
        ``rhs`` of the restricted oracle."""
        import copy
        if any(kind == 'dgfs-wall-specular' for _, _, kind in self.walls):
            raise ValueError('the specular wall couples velocities: no restriction')
        sub = copy.copy(self)
        sub.cv = self.cv[:, vsel]
        sub.walls = [(Uw, np.asarray(fw)[vsel], kind) for Uw, fw, kind in self.walls]
        return sub

    def _rusanov(self, ul, ur, n):
        nc = sum(n[j] * self.cv[j] for j in range(self.ndims))
        return 0.5 * nc * (ul + ur) + 0.5 * np.abs(nc) * (ul - ur)

    def rhs(self, u, bc=None, ghost=None):
        """L(u).  ghost: face values of neighbours owned by other parts of a
        partitioned mesh (rows E*nfpts + i of the local neighbour table);
        their faces get the one-sided flux the reference's MPI interfaces
        compute (frfs/solvers/dgfs/inters.py:61-112)."""
        g = self.geo
        d = self.ndims
        E, nupts, nv = u.shape
        uf = self.disu(u)
        if bc is None and len(g.wall_fpts):
            bc = self.update_bc(uf)
        # tdisf: F~[e][i][u][v] = sum_k smats[e][u][i][k] c_k u
        Ft = np.einsum('euik,kv,euv->eiuv', g.smats, self.cv[:d], u)
        R = np.einsum('um,emv->euv', self.M132, Ft.reshape(E, d * nupts, nv))
        # common fluxes, interface by interface (lhs = lower global fpt index)
        nf = uf.shape[1]
        Fh = np.zeros_like(uf)
        done = np.zeros((E, nf), bool)
        for e in range(E):
            for f in range(nf):
                if done[e, f]:
                    continue
                nb = g.nbr[e, f]
                n = g.norm_pnorm[e, f]
                mag = g.mag_pnorm[e, f]
                ul = uf[e, f]
                if nb >= E * nf:
                    fn = self._rusanov(ul, ghost[int(nb) - E * nf], n)
                    Fh[e, f] = mag * fn
                elif nb >= 0:
                    e2, f2 = divmod(int(nb), nf)
                    fn = self._rusanov(ul, uf[e2, f2], n)
                    Fh[e, f] = mag * fn
                    Fh[e2, f2] = -mag * fn
                    done[e2, f2] = True
                else:
                    w = -1 - int(nb)
                    Uw, fw, kind = self.walls[self.bcid[w]]
                    fac = sum((self.cv[j] - Uw[j]) * n[j] for j in range(d))
                    cn = sum(self.cv[j] * n[j] for j in range(d))
                    if kind == 'dgfs-wall-diffuse':
                        ur = np.where(fac < 0, fw * (-bc[w, 0] / bc[w, 1]), ul)
                    elif kind == 'dgfs-inlet':
                        ur = np.where(fac < 0, fw, ul)
                    elif kind == 'dgfs-inlet-normalshock':
                        ur = np.where(cn < 0, fw, ul)
                    elif kind == 'dgfs-vanish':
                        ur = np.where(cn < 0, 0.0, ul)
                    elif kind == 'dgfs-outlet':
                        ur = ul
                    elif kind == 'dgfs-wall-specular':
                        ur = ul[self.mirror(n)]
                    else:
                        raise ValueError(kind)
                    Fh[e, f] = mag * self._rusanov(ul, ur, n)
                done[e, f] = True
        R = R + np.einsum('uf,efv->euv', self.M3, Fh)
        return -g.rcpdjac[:, :, None] * R


def inverse_mass(ndims, order):
    """M12 of frfs/shapes.py:163-166 (V^T V, V the orthonormal basis at the
    solution points) restated as the inverse of the nodal mass matrix
    M_ij = int l_i l_j over [-1, 1]^ndims (l the Lagrange basis at the GLL
    solution points, x index fastest), integrated exactly by a Gauss-Legendre
    product rule: for an orthonormal basis V^T V = M^-1."""
    from numpy.polynomial import legendre as L
    n = order + 1
    c = np.zeros(n)
    c[-1] = 1.0
    x = np.concatenate([[-1.0], np.sort(L.legroots(L.legder(c))), [1.0]])
    xq, wq = L.leggauss(n + 1)                     # exact for degree 2n + 1
    lag = np.ones((len(xq), n))
    for i in range(n):
        for j in range(n):
            if j != i:
                lag[:, i] *= (xq - x[j]) / (x[i] - x[j])
    m1 = lag.T @ (wq[:, None] * lag)
    M = m1
    for _ in range(ndims - 1):
        M = np.kron(m1, M)                         # slower index on the left
    return np.linalg.inv(M)


def invmass(minv, u):
    """system.invmass (solvers/dgfs/system.py:221-231): minv u per element."""
    return np.einsum('ij,ejv->eiv', minv, u)


def step_rk2(u, dt, L, Q):
    """dgfs-tvd-rk2 (steppers.py:122-225): u1 = u + dt (L+Q)(u);
    u_new = 1/2 u + 1/2 u1 + 1/2 dt (L+Q)(u1)."""
    u1 = u + dt * L(u) + dt * Q(u)
    return 0.5 * u + 0.5 * u1 + 0.5 * dt * (L(u1) + Q(u1))


def step_euler(u, dt, L, Q):
    """dgfs-euler (steppers.py:20-99)."""
    return u + dt * L(u) + dt * Q(u)


def moments(f, cv, cw):
    """Non-dimensional macroscopic fields of one distribution, as
    frfs/plugins/dgfsmomwriterstd.py:151-213 (_compute_moments_3D, mr = 1)
    computes them before dimensionalisation: rho, U[3], T, q[3], P[6]
    (xx, xy, xz, yy, yz, zz)."""
    rho = np.sum(f) * cw
    U = cv @ f * cw / rho
    c = cv - U[:, None]
    c2 = np.sum(c * c, axis=0)
    T = np.sum(f * c2) * (2.0 / 3.0 * cw) / rho
    q = (c @ (f * c2)) * cw
    P = 2.0 * np.array([np.sum(f * c[a] * c[b]) for a, b in
                        ((0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2))]) * cw
    return rho, U, T, q, P
