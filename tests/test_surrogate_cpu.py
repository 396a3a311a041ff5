"""CPU checks of the surrogate's oracle and data family."""
import numpy as np
import torch

from oracle.surrogate import loss_and_grads
from frfs_b200.surrogate import sample_family


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    k, kin, w, B = 4, 6, 8, 5
    W = [rng.normal(size=(w, kin)) * 0.5, rng.normal(size=(w, w)) * 0.4,
         rng.normal(size=(w, w)) * 0.4, rng.normal(size=(3 * k, w + kin)) * 0.4]
    b = [rng.normal(size=w) * 0.1, rng.normal(size=w) * 0.1, rng.normal(size=w) * 0.1,
         rng.normal(size=3 * k) * 0.1]
    x, t = rng.normal(size=(B, kin)), rng.normal(size=(B, 3 * k))
    L, gW, gb = loss_and_grads(x, t, W, b)
    h = 1e-6
    for l in range(4):
        for (i, j) in ((0, 0), (1, 2), (W[l].shape[0] - 1, W[l].shape[1] - 1)):
            Wp = [m.copy() for m in W]
            Wp[l][i, j] += h
            Wm = [m.copy() for m in W]
            Wm[l][i, j] -= h
            fd = (loss_and_grads(x, t, Wp, b)[0] - loss_and_grads(x, t, Wm, b)[0]) / (2 * h)
            assert abs(fd - gW[l][i, j]) < 1e-6 * max(1.0, abs(fd))
        for i in (1, b[l].shape[0] - 1):
            bp = [v.copy() for v in b]
            bp[l][i] += h
            bm = [v.copy() for v in b]
            bm[l][i] -= h
            fd = (loss_and_grads(x, t, W, bp)[0] - loss_and_grads(x, t, W, bm)[0]) / (2 * h)
            assert abs(fd - gb[l][i]) < 1e-6 * max(1.0, abs(fd))


def test_cavity_family_ranges():
    from frfs_b200.surrogate import CAVITY
    c0 = np.linspace(-6 + 0.25, 6 - 0.25, 24)
    gen = torch.Generator().manual_seed(2)
    f = sample_family(c0, 16, gen, 'cpu', dtype=torch.float64, family=CAVITY).numpy()
    assert np.all(f >= 0) and np.all(np.isfinite(f))
    cw = (12.0 / 24)**3
    rho = f.sum(1) * cw
    assert np.all((rho > 0.88) & (rho < 1.12))


def test_family_moments_match_maxwellian_parameters():
    """The Grad-type perturbations leave rho, u, T unchanged (up to the
    clipping of negative values, rare at these amplitudes)."""
    c0 = np.linspace(-6 + 0.25, 6 - 0.25, 24)
    gen = torch.Generator().manual_seed(1)
    f = sample_family(c0, 32, gen, 'cpu', dtype=torch.float64, amp=(0.0, 0.1)).numpy()
    cw = (12.0 / 24)**3
    idx = np.arange(24**3)
    cv = np.stack([c0[idx // 576], c0[(idx // 24) % 24], c0[idx % 24]])
    rho = f.sum(1) * cw
    assert np.all((rho > 0.78) & (rho < 1.22))
    u = (f @ cv.T) * cw / rho[:, None]
    assert np.all(np.abs(u[:, 0]) < 0.36) and np.all(np.abs(u[:, 1:]) < 0.06)
    assert np.all(f >= 0)
