"""Learned surrogate of the collision operator and the hybrid collision step.

The reference has no learned component; this module adds one on top of the
spectral operator (``scattering.py``), which stays the fallback.

Model (per distribution f on an Nv^3 grid, n = Nv^3):
  rho   = sum(f) cw                                   (FP64 moments kernel)
  a     = Bf (f / rho)                                 Bf: nmodes x n basis
  y     = MLP((a - mu) / sigma)                        4 layers, GELU, width W
  Q     = rho^2 * s * Bq^T y                           Bq: nmodes x n basis
  Q    <- Q - phi^T G^{-1} (phi Q)                     FP64 conservation
Q(lambda f) = lambda^2 Q(f) is used exactly (density normalisation).  The
bases are fitted by a randomised SVD (Halko, Martinsson, Tropp 2011) whose
GEMMs are the project's FP32 kernels; every training GEMM (forward and
backward) runs on the tcgen05 tensor cores with BF16 operands and FP32
accumulation; AdamW and the loss are project kernels too.

Training family (the Couette workload's distributions): Maxwellians with
rho ~ U(0.8, 1.2), u_x ~ U(-0.35, 0.35), u_y, u_z ~ U(-0.05, 0.05),
T ~ U(0.85, 1.2), multiplied by 1 + A P(xi), xi = (c - u)/sqrt(T), with P a
random unit combination of the Grad-type shear-stress and heat-flux
polynomials (xi_i xi_j, xi_i^2 - xi_j^2, xi_i (|xi|^2 - 5/2)), which leave
rho, u and T unchanged, and A ~ U(0, 0.3); negative values are clipped.
Labels are the FP32 spectral Q with the conservation projection.

Hybrid step (``HybridCollider``): the Maxwellian-deviation indicator routes
cells with eps < threshold to the surrogate and the rest to the spectral
kernel; a seeded fraction of the surrogate cells is also evaluated
spectrally every step, keeps the spectral result and measures the
surrogate's error there.  Lists and counts live on the device, so a whole
hybrid step is captured in one CUDA graph.
"""
import ctypes as C
import math
import time

import numpy as np
import torch

from . import _lib
from .gemm import ACT_GELU, ACT_GELU_GRAD, adamw, colsum, gemm


# ------------------------------------------------------------------ data
GRAD_POLYS = ('xy', 'xz', 'yz', 'xx-yy', 'yy-zz', 'qx', 'qy', 'qz')


def sample_family(vm_c0, n, gen, device, dtype=torch.float32, amp=(0.0, 0.3)):
    """n distributions of the Couette-type family on the grid with cell
    centres vm_c0 (FP32 on the device)."""
    c0 = torch.as_tensor(vm_c0, dtype=torch.float32, device=device)
    N = c0.numel()
    cx, cy, cz = c0.view(1, -1, 1, 1), c0.view(1, 1, -1, 1), c0.view(1, 1, 1, -1)
    U = lambda lo, hi, *s: lo + (hi - lo) * torch.rand(*s, generator=gen, device=device)
    rho = U(0.8, 1.2, n).view(-1, 1, 1, 1)
    ux = U(-0.35, 0.35, n).view(-1, 1, 1, 1)
    uy = U(-0.05, 0.05, n).view(-1, 1, 1, 1)
    uz = U(-0.05, 0.05, n).view(-1, 1, 1, 1)
    T = U(0.85, 1.2, n).view(-1, 1, 1, 1)
    s = T.sqrt()
    xx, xy, xz = (cx - ux) / s, (cy - uy) / s, (cz - uz) / s
    x2 = xx * xx + xy * xy + xz * xz
    polys = [xx * xy, xx * xz, xy * xz, (xx * xx - xy * xy) / math.sqrt(2),
             (xy * xy - xz * xz) / math.sqrt(2),
             xx * (x2 - 2.5) / math.sqrt(2.5), xy * (x2 - 2.5) / math.sqrt(2.5),
             xz * (x2 - 2.5) / math.sqrt(2.5)]
    coef = torch.randn(n, len(polys), generator=gen, device=device)
    coef = coef / coef.norm(dim=1, keepdim=True)
    A = U(amp[0], amp[1], n).view(-1, 1, 1, 1)
    P = sum(coef[:, i].view(-1, 1, 1, 1) * p for i, p in enumerate(polys))
    f = rho / (math.pi * T)**1.5 * torch.exp(-((cx - ux)**2 + (cy - uy)**2 + (cz - uz)**2) / T)
    f = f * torch.clamp(1.0 + A * P, min=0.0)
    return f.reshape(n, N**3).to(dtype).contiguous()


# ------------------------------------------------------------------ basis
def _orth(Z):
    """Orthonormal columns spanning Z (n x r, device): Householder QR of the
    tall-skinny block in FP64 on the host (r is a few hundred)."""
    q, _ = np.linalg.qr(Z.double().cpu().numpy())
    return torch.from_numpy(q).float().to(Z.device).contiguous()


def fit_basis(X, k, oversample=64, power=2, gen=None):
    """Leading right singular vectors (at most k, orthonormal rows) of the
    sample matrix X (ns x n, FP32, device) by a randomised SVD."""
    ns, n = X.shape
    r = min(k + oversample, ns, n)
    Om = torch.randn(n, r, device=X.device, generator=gen)
    Y = torch.empty(ns, r, device=X.device)
    gemm(X, Om, tb=True, out=Y, engine=1)                        # X Omega
    for it in range(power):
        V = torch.empty(n, Y.shape[1], device=X.device)
        gemm(X, Y, ta=True, tb=True, out=V, engine=1)            # X^T Y
        V = _orth(V)
        if it < power - 1:
            Y = torch.empty(ns, V.shape[1], device=X.device)
            gemm(X, V, tb=True, out=Y, engine=1)                 # X V
    r = V.shape[1]
    B = torch.empty(ns, r, device=X.device)
    gemm(X, V, tb=True, out=B, engine=1)
    Cm = torch.empty(r, r, device=X.device)
    gemm(B, B, ta=True, tb=True, out=Cm, engine=1)               # B^T B
    w, U = np.linalg.eigh(Cm.double().cpu().numpy())
    order = np.argsort(w)[::-1]
    order = order[w[order] > 1e-12 * w[order[0]]][:k]
    Uk = torch.from_numpy(U[:, order].copy()).float().to(X.device)
    Vk = torch.empty(n, Uk.shape[1], device=X.device)
    gemm(V, Uk, tb=True, out=Vk, engine=1)                       # V U_k
    Vk = _orth(Vk)
    sv = np.sqrt(np.maximum(w[order], 0.0))
    return Vk.t().contiguous(), sv


# ------------------------------------------------------------------ model
class QSurrogate:
    """Basis projection + MLP (BF16 weights, FP32 accumulation) for Q."""

    def __init__(self, grid, nmodes=512, width=1024, device=None):
        self.grid = grid                    # scattering.VHSGrid (tables, c0, ginv)
        self.Nv = grid.Nv
        self.n = grid.Nv**3
        self.k = nmodes
        self.w = width
        self.device = device or grid.phase.device
        self.trained = False
        self.history = []

    # parameters ------------------------------------------------------
    def _init_params(self, gen):
        dims = [(self.w, self.k), (self.w, self.w), (self.w, self.w), (self.k, self.w)]
        self.W, self.b = [], []
        for (o, i) in dims:
            W = torch.randn(o, i, device=self.device, generator=gen) * math.sqrt(2.0 / i)
            self.W.append(W.contiguous())
            self.b.append(torch.zeros(o, device=self.device))
        self.W[-1] *= 0.1
        self.Wb = [W.bfloat16() for W in self.W]
        self.mW = [torch.zeros_like(W) for W in self.W]
        self.vW = [torch.zeros_like(W) for W in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.gW = [torch.zeros_like(W) for W in self.W]
        self.gb = [torch.zeros_like(b) for b in self.b]

    # training forward / backward (project kernels) ---------------------
    def forward_train(self, x_bf16):
        """x (B x k, bf16, standardised) -> y (B x k FP32); keeps activations."""
        B = x_bf16.shape[0]
        dev = self.device
        self._acts = [x_bf16]
        self._z = []
        h = x_bf16
        for l in range(3):
            z = torch.empty(B, self.w, device=dev)
            hn = torch.empty(B, self.w, device=dev, dtype=torch.bfloat16)
            gemm(h, self.Wb[l], bias=self.b[l], act=ACT_GELU, zout=z, out_bf16=hn)
            self._z.append(z)
            self._acts.append(hn)
            h = hn
        y = torch.empty(B, self.k, device=dev)
        gemm(h, self.Wb[3], bias=self.b[3], out=y)
        return y

    def backward_train(self, dy):
        """Gradients of all parameters from dL/dy (B x k FP32)."""
        g = dy
        for l in (3, 2, 1, 0):
            h = self._acts[l]
            gemm(g, h, ta=True, tb=True, out=self.gW[l])          # dW = g^T h
            colsum(g, self.gb[l])
            if l > 0:
                gn = torch.empty(g.shape[0], self.w, device=self.device)
                gemm(g, self.Wb[l], tb=True, act=ACT_GELU_GRAD, zin=self._z[l - 1], out=gn)
                g = gn

    def step(self, t, lr, wd=0.01):
        for l in range(4):
            adamw(self.W[l], self.gW[l], self.mW[l], self.vW[l], self.Wb[l], t, lr=lr, wd=wd)
            adamw(self.b[l], self.gb[l], self.mb[l], self.vb[l], None, t, lr=lr, wd=0.0)

    # data -> coefficients ------------------------------------------------
    def _labels(self, f, collider):
        Q = torch.empty_like(f)
        collider([(0, f, Q, None)], project=True, exact=False)
        return Q

    def _coeffs(self, f, Q):
        """FP32 coefficients a = Bf f/rho, c = Bq Q/rho^2 of a chunk."""
        from .system import raw_moments
        rho = (f.double().sum(1) * self.grid.cw).float()
        a = torch.empty(f.shape[0], self.k, device=self.device)
        c = torch.empty(f.shape[0], self.k, device=self.device)
        gemm(f, self.Bf, out=a, engine=1)
        gemm(Q, self.Bq, out=c, engine=1)
        a /= rho[:, None]
        c /= (rho * rho)[:, None]
        return a, c

    def fit(self, nsamples=200000, ntest=50000, epochs=20, lr=3e-4, batch=1024, seed=0,
            nbasis=16384, chunk=8192, log=None):
        """Generate data, fit the bases, train the MLP (all on the device)."""
        from .scattering import VHSCollider
        dev = self.device
        gen = torch.Generator(device=dev).manual_seed(seed)
        col = VHSCollider([self.grid], dev)
        c0 = self.grid.c0.double().cpu().numpy()
        t0 = time.time()
        # 1. bases from a sample
        fb = sample_family(c0, nbasis, gen, dev)
        Qb = self._labels(fb, col)
        rho = fb.double().sum(1) * self.grid.cw
        Xf = (fb / rho[:, None].float()).contiguous()
        Xq = (Qb / (rho * rho)[:, None].float()).contiguous()
        self.Bf, self.svf = fit_basis(Xf, self.k, gen=gen)
        self.Bq, self.svq = fit_basis(Xq, self.k, gen=gen)
        # the data may support fewer modes than requested
        self.k = min(self.Bf.shape[0], self.Bq.shape[0])
        self.Bf, self.Bq = self.Bf[:self.k].contiguous(), self.Bq[:self.k].contiguous()
        # basis truncation error on the fit sample (relative L2 of Q)
        cq = torch.empty(nbasis, self.k, device=dev)
        gemm(Xq, self.Bq, out=cq, engine=1)
        Xr = torch.empty_like(Xq)
        gemm(cq, self.Bq, tb=True, out=Xr, engine=1)
        self.basis_err_q = float((Xr - Xq).norm() / Xq.norm())
        del fb, Qb, Xf, Xq, Xr
        # 2. training coefficients
        A = torch.empty(nsamples, self.k, device=dev)
        Cc = torch.empty(nsamples, self.k, device=dev)
        for i0 in range(0, nsamples, chunk):
            m = min(chunk, nsamples - i0)
            f = sample_family(c0, m, gen, dev)
            a, c = self._coeffs(f, self._labels(f, col))
            A[i0:i0 + m] = a
            Cc[i0:i0 + m] = c
        self.mu = A.mean(0)
        self.sigma = A.std(0).clamp_min(1e-6 * float(A.std(0).max()))
        self.cscale = float(Cc.pow(2).mean().sqrt())
        X = ((A - self.mu) / self.sigma).bfloat16().contiguous()
        Tt = (Cc / self.cscale).contiguous()
        # loss floor: 1% of the mean target energy
        self.loss_delta = 0.01 * float(Tt.pow(2).sum(1).mean())
        del A, Cc
        t_data = time.time() - t0
        # 3. training (AdamW, relative MSE per sample)
        self._init_params(gen)
        loss = torch.zeros(1, dtype=torch.float64, device=dev)
        dy = torch.empty(batch, self.k, device=dev)
        step = 0
        t1 = time.time()
        for ep in range(epochs):
            perm = torch.randperm(nsamples, generator=gen, device=dev)
            nb = 0
            for i0 in range(0, nsamples - batch + 1, batch):
                idx = perm[i0:i0 + batch]
                xb, tb = X[idx].contiguous(), Tt[idx].contiguous()
                y = self.forward_train(xb)
                _lib.check(_lib.lib().bdgfs_relmse(y.data_ptr(), tb.data_ptr(), batch, self.k,
                                                   self.loss_delta, dy.data_ptr(), loss.data_ptr(),
                                                   _lib.stream_ptr()), 'bdgfs_relmse')
                self.backward_train(dy)
                step += 1
                self.step(step, lr)
                nb += 1
            self.history.append(float(loss.item()))
            if log:
                log(f'epoch {ep}: loss {self.history[-1]:.4e}')
        torch.cuda.synchronize(dev)
        self.train_seconds = time.time() - t1
        self.data_seconds = t_data
        self.steps = step
        self._fold()
        self.trained = True
        # 4. held-out evaluation against the spectral operator
        self.test_err = self.evaluate(ntest, seed=seed + 1, chunk=chunk)
        return self

    def _fold(self):
        """Fold input standardisation into layer 1 and the output scale into
        the reconstruction basis (exact rewrites of the trained model)."""
        W1 = self.W[0] / self.sigma[None, :]
        b1 = self.b[0] - W1 @ self.mu
        self.inf_W = [W1.bfloat16().contiguous()] + [w.bfloat16().contiguous() for w in self.W[1:]]
        self.inf_b = [b1.contiguous()] + [b.contiguous() for b in self.b[1:]]
        self.BfT_bf16 = self.Bf.bfloat16().contiguous()                 # k x n
        self.BqT_bf16 = (self.Bq.t() * self.cscale).bfloat16().contiguous()   # n x k

    # inference ------------------------------------------------------------
    def infer(self, f, rows, inv_rho, rho2, out, count=None, M=None):
        """Compact surrogate Q: out[m] = Q of f[rows[m]] (m < count) on the
        tensor cores; no conservation projection here."""
        M = M if M is not None else rows.numel()
        dev = self.device
        bufs = self._bufs(M)
        gemm(f, self.BfT_bf16, arow=rows, row_scale=inv_rho, mcount=count, M=M,
             out_bf16=bufs[0])
        h = bufs[0]
        for l in range(3):
            gemm(h, self.inf_W[l], bias=self.inf_b[l], act=ACT_GELU, mcount=count,
                 out_bf16=bufs[1 + (l % 2)])
            h = bufs[1 + (l % 2)]
        gemm(h, self.inf_W[3], bias=self.inf_b[3], mcount=count, out_bf16=bufs[3])
        gemm(bufs[3], self.BqT_bf16, row_scale=rho2, mcount=count, out=out)
        return out

    def _bufs(self, M):
        if getattr(self, '_buf_M', 0) < M:
            dev = self.device
            self._buf = [torch.empty(M, self.k, device=dev, dtype=torch.bfloat16),
                         torch.empty(M, self.w, device=dev, dtype=torch.bfloat16),
                         torch.empty(M, self.w, device=dev, dtype=torch.bfloat16),
                         torch.empty(M, self.k, device=dev, dtype=torch.bfloat16)]
            self._buf_M = M
        return [b[:M] for b in self._buf]

    def evaluate(self, nsamples, seed=1, chunk=8192):
        """Relative L2 error of the surrogate (with conservation projection)
        against the FP32 spectral Q on seeded held-out distributions:
        returns dict(mean, median, p90, aggregate)."""
        from .scattering import VHSCollider
        dev = self.device
        gen = torch.Generator(device=dev).manual_seed(seed)
        col = VHSCollider([self.grid], dev)
        c0 = self.grid.c0.double().cpu().numpy()
        errs = []
        num = den = 0.0
        h = HybridCollider(self, threshold=float('inf'), recheck=0.0)
        for i0 in range(0, nsamples, chunk):
            m = min(chunk, nsamples - i0)
            f = sample_family(c0, m, gen, dev)
            Qs = self._labels(f, col)
            Qh = torch.empty_like(f)
            h.collide_surrogate_only(f, Qh)
            d = (Qh.double() - Qs.double()).norm(dim=1)
            q = Qs.double().norm(dim=1)
            errs.append((d / q).cpu())
            num += float((d * d).sum())
            den += float((q * q).sum())
        e = torch.cat(errs).numpy()
        return {'mean': float(e.mean()), 'median': float(np.median(e)),
                'p90': float(np.percentile(e, 90)), 'aggregate': math.sqrt(num / den),
                'n': int(nsamples), 'basis_truncation_q': getattr(self, 'basis_err_q', None)}

    def state_dict(self):
        keys = ('Bf', 'Bq', 'mu', 'sigma')
        d = {k: getattr(self, k).cpu() for k in keys}
        d.update(W=[w.cpu() for w in self.W], b=[b.cpu() for b in self.b], cscale=self.cscale,
                 k=self.k, w=self.w, Nv=self.Nv)
        return d

    def load_state_dict(self, d):
        dev = self.device
        for k in ('Bf', 'Bq', 'mu', 'sigma'):
            setattr(self, k, d[k].to(dev))
        self.W = [w.to(dev) for w in d['W']]
        self.b = [b.to(dev) for b in d['b']]
        self.cscale = float(d['cscale'])
        self._fold()
        self.trained = True
        return self


# ------------------------------------------------------------------ hybrid
class HybridCollider:
    """Surrogate where the Maxwellian deviation is below ``threshold``,
    spectral elsewhere, spectral re-check of a seeded ``recheck`` fraction of
    the surrogate cells (their spectral result is kept)."""

    def __init__(self, model, threshold=0.05, recheck=0.02, project=True):
        from .scattering import VHSCollider
        self.model = model
        self.grid = model.grid
        self.threshold, self.recheck, self.project = float(threshold), float(recheck), project
        self.spectral = VHSCollider([self.grid], model.device)
        self._n = 0

    def _alloc(self, ndof):
        if self._n >= ndof:
            return
        dev = self.model.device
        self.counts = torch.zeros(3, dtype=torch.int64, device=dev)
        self.sur_idx = torch.zeros(ndof, dtype=torch.int32, device=dev)
        self.spec_idx = torch.zeros(ndof, dtype=torch.int32, device=dev)
        self.inv_rho = torch.zeros(ndof, device=dev)
        self.rho2 = torch.zeros(ndof, device=dev)
        self.flag = torch.zeros(ndof, dtype=torch.uint8, device=dev)
        self.eps = torch.zeros(ndof, device=dev)
        self.recheck_err = torch.zeros(2, dtype=torch.float64, device=dev)
        self.seed_dev = torch.zeros(1, dtype=torch.int64, device=dev)
        self.Qc = torch.empty(ndof, self.model.n, device=dev, dtype=self.grid.dtype)
        self._n = ndof

    def _args(self, ndof, seed):
        """seed None: the re-check sample follows a device step counter
        (advanced every call, also under CUDA-graph replay)."""
        g = self.grid
        return _lib.HybridArgs(
            ndof=ndof, Nv=g.Nv, fp64=int(g.dtype == torch.float64), c0=g.c0.data_ptr(),
            ginv=g.ginv.data_ptr(), cw=g.cw, threshold=self.threshold, recheck=self.recheck,
            seed=int(seed or 0), counts=self.counts.data_ptr(), sur_idx=self.sur_idx.data_ptr(),
            sur_inv_rho=self.inv_rho.data_ptr(), sur_rho2=self.rho2.data_ptr(),
            spec_idx=self.spec_idx.data_ptr(), flag=self.flag.data_ptr(),
            eps=self.eps.data_ptr(), recheck_err=self.recheck_err.data_ptr(),
            seed_dev=self.seed_dev.data_ptr() if seed is None else 0)

    def __call__(self, fin, fout, seed=None):
        """Q for every distribution of fin [ndof][n] into fout."""
        n = self.model.n
        f2, q2 = fin.reshape(-1, n), fout.reshape(-1, n)
        ndof = f2.shape[0]
        self._alloc(ndof)
        L = _lib.lib()
        args = self._args(ndof, seed)
        _lib.check(L.bdgfs_hybrid_classify(C.byref(args), f2.data_ptr(), _lib.stream_ptr()),
                   'bdgfs_hybrid_classify')
        # spectral cells (incl. re-checks): index list + device count
        self.spectral([(0, f2, q2, None)], project=self.project, exact=False,
                      index=self.spec_idx, count=self.counts[1:2])
        # surrogate cells: compact rows, projection, scatter
        self.model.infer(f2, self.sur_idx, self.inv_rho, self.rho2, self.Qc[:ndof],
                         count=self.counts[0:1], M=ndof)
        if self.project:
            _lib.check(L.bdgfs_hybrid_project(C.byref(args), self.Qc.data_ptr(), _lib.stream_ptr()),
                       'bdgfs_hybrid_project')
        _lib.check(L.bdgfs_hybrid_scatter(C.byref(args), self.Qc.data_ptr(), q2.data_ptr(),
                                          _lib.stream_ptr()), 'bdgfs_hybrid_scatter')

    def collide_surrogate_only(self, fin, fout):
        """Every cell through the surrogate (evaluation helper)."""
        saved = (self.threshold, self.recheck)
        self.threshold, self.recheck = float('inf'), 0.0
        try:
            self(fin, fout)
        finally:
            self.threshold, self.recheck = saved

    def stats(self):
        c = self.counts.cpu().tolist()
        e = self.recheck_err.cpu().tolist()
        return {'surrogate_cells': c[0], 'spectral_cells': c[1], 'rechecked_cells': c[2],
                'recheck_rel_l2': math.sqrt(e[0] / e[1]) if e[1] > 0 else None}
