"""FR operator matrices of tensor-product elements with GLL points.

Restates, for quadrilaterals and hexahedra with Gauss-Legendre-Lobatto
solution and flux points, the operators of frfs/shapes.py:
  M0 = interpolation upts -> fpts                    (shapes.py:94-96)
  M1[u][d*nupts+u'] = d/dr_d l_u'(x_u)               (shapes.py:98-101)
  M2[f][d*nupts+u]  = n_ref[f][d] * M0[f][u]         (shapes.py:103-106)
  M3 = correction lifting gbasis_at(upts)            (shapes.py:108-120, 213-247)
The lifting of a face value at flux point x_f is the L2 projection of the
face-quadrature delta onto Q_P: M3[u][f] = w_f * K(x_u, x_f), with K the
reproducing kernel of Q_P on [-1, 1]^d (sum over an orthonormal basis, here
the product of normalised Legendre polynomials) and w_f the GLL face weight
at x_f (the face rule of shapes.py:223-226 has its nodes at the flux points).
Point orders follow the reference's tabulated rules (x fastest) and face
order/projections (shapes.py:368-402).
"""
import itertools as it

import numpy as np
from numpy.polynomial import legendre as npleg

from .quadratures import gll_points, gll_weights

QUAD_FACES = [  # (projection, reference normal)
    (lambda s: (s, -1.0), (0, -1)),
    (lambda s: (1.0, s), (1, 0)),
    (lambda s: (s, 1.0), (0, 1)),
    (lambda s: (-1.0, s), (-1, 0)),
]
HEX_FACES = [
    (lambda s, t: (s, t, -1.0), (0, 0, -1)),
    (lambda s, t: (s, -1.0, t), (0, -1, 0)),
    (lambda s, t: (1.0, s, t), (1, 0, 0)),
    (lambda s, t: (s, 1.0, t), (0, 1, 0)),
    (lambda s, t: (-1.0, s, t), (-1, 0, 0)),
    (lambda s, t: (s, t, 1.0), (0, 0, 1)),
]


def _lagrange_1d(nodes, x):
    """L[i][k] = l_k(x_i) and dL[i][k] = l_k'(x_i)."""
    x = np.atleast_1d(x)
    n = len(nodes)
    L = np.ones((len(x), n))
    dL = np.zeros((len(x), n))
    for k in range(n):
        others = [nodes[j] for j in range(n) if j != k]
        den = np.prod([nodes[k] - o for o in others])
        for i, xi in enumerate(x):
            L[i, k] = np.prod([xi - o for o in others]) / den
            s = 0.0
            for m in range(n - 1):
                s += np.prod([xi - o for j, o in enumerate(others) if j != m])
            dL[i, k] = s / den
    return L, dL


def _kernel_1d(n, s, t):
    """sum_{i<n} (i + 1/2) P_i(s) P_i(t)."""
    out = 0.0
    for i in range(n):
        c = [0] * i + [1]
        out = out + (i + 0.5) * npleg.legval(s, c) * npleg.legval(t, c)
    return out


class TensorShape:
    def __init__(self, name, order):
        if name not in ('quad', 'hex'):
            raise ValueError(f'unsupported element type {name}')
        self.name = name
        self.order = order
        self.ndims = 2 if name == 'quad' else 3
        self.n1 = n = order + 1
        self.pts1 = gll_points(n)
        self.wts1 = gll_weights(n)
        d = self.ndims
        # upts: x fastest
        self.upts = np.array([p[::-1] for p in it.product(self.pts1, repeat=d)])
        self.nupts = n**d
        faces = QUAD_FACES if d == 2 else HEX_FACES
        fp, fw, fn, nff = [], [], [], []
        if d == 2:
            for proj, nrm in faces:
                for s, w in zip(self.pts1, self.wts1):
                    fp.append(proj(s))
                    fw.append(w)
                    fn.append(nrm)
                nff.append(n)
        else:
            face_pts = [(p[1], p[0]) for p in it.product(self.pts1, repeat=2)]
            face_wts = [self.wts1[i] * self.wts1[j]
                        for j in range(n) for i in range(n)]
            for proj, nrm in faces:
                for (s, t), w in zip(face_pts, face_wts):
                    fp.append(proj(s, t))
                    fw.append(w)
                    fn.append(nrm)
                nff.append(n * n)
        self.fpts = np.array(fp, dtype=np.float64)
        self.fpts_wts = np.array(fw)
        self.norm_fpts = np.array(fn, dtype=np.float64)
        self.nfacefpts = nff
        self.nfpts = len(fp)
        self.facefpts = np.split(np.arange(self.nfpts), np.cumsum(nff)[:-1])

    def nodal_at(self, pts):
        """Tensor Lagrange basis at pts: (npts, nupts) and its gradient
        (ndims, npts, nupts)."""
        pts = np.atleast_2d(pts)
        d, n = self.ndims, self.n1
        Ls, dLs = zip(*[_lagrange_1d(self.pts1, pts[:, a]) for a in range(d)])
        # node index: x fastest -> node = ((k*n) + j)*n + i for (i, j, k)
        B = np.ones((len(pts), self.nupts))
        G = np.ones((d, len(pts), self.nupts))
        for node, idx in enumerate(it.product(range(n), repeat=d)):
            idx = idx[::-1]            # (ix, iy[, iz])
            for a in range(d):
                B[:, node] *= Ls[a][:, idx[a]]
                for g in range(d):
                    G[g, :, node] *= (dLs[a] if a == g else Ls[a])[:, idx[a]]
        return B, G

    @property
    def m0(self):
        return self.nodal_at(self.fpts)[0]

    @property
    def m1(self):
        _, G = self.nodal_at(self.upts)            # (d, nupts, nupts)
        return np.concatenate([G[a] for a in range(self.ndims)], axis=1)

    @property
    def m2(self):
        m0 = self.m0
        return np.concatenate([self.norm_fpts[:, a:a + 1] * m0
                               for a in range(self.ndims)], axis=1)

    @property
    def m3(self):
        n = self.n1
        K = np.ones((self.nupts, self.nfpts))
        for a in range(self.ndims):
            K *= _kernel_1d(n, self.upts[:, a][:, None], self.fpts[:, a][None, :])
        return K * self.fpts_wts[None, :]

    @property
    def m12(self):
        """Inverse of the nodal mass matrix, V^T V with V[k][u] the
        orthonormal basis (products of sqrt(k + 1/2) P_k) at the solution
        points (shapes.py:163-166); a product of 1-D factors per axis."""
        n = self.n1
        V1 = np.array([np.sqrt(k + 0.5) * npleg.legval(self.pts1, [0] * k + [1])
                       for k in range(n)])
        m1 = V1.T @ V1
        idx = np.array([p[::-1] for p in it.product(range(n), repeat=self.ndims)])
        M = np.ones((self.nupts, self.nupts))
        for a in range(self.ndims):
            M *= m1[np.ix_(idx[:, a], idx[:, a])]
        return M

    def interp_from(self, order):
        """(nupts, nupts of order) values at these solution points of the
        nodal basis of order ``order``: the restart interpolation of
        solvers/dgfs/system.py:100-104."""
        return TensorShape(self.name, order).nodal_at(self.upts)[0]

    def opmat(self, expr):
        mats = {'M0': self.m0, 'M1': self.m1, 'M2': self.m2, 'M3': self.m3,
                'M12': self.m12}
        if expr == 'M1 - M3*M2':
            return mats['M1'] - mats['M3'] @ mats['M2']
        return mats[expr]
