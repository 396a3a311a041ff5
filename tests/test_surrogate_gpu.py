"""Surrogate kernels: training gradients against the FP64 oracle, the
hybrid routing (all-spectral / all-surrogate limits, re-checks), and a small
end-to-end fit that must beat the method without the network."""
import math

import numpy as np
import pytest
import torch

from frfs_b200.backend import CUDABackend
from frfs_b200.scattering import DGFSVHSGLLScatteringModel
from frfs_b200.surrogate import HybridCollider, QSurrogate, sample_family
from frfs_b200.velocitymesh import DGFSVelocityMesh

from helpers import vhs_cfg

pytestmark = pytest.mark.gpu


def _model(Nv=16, Nrho=8, M=6, dev=5, k=64, w=128):
    cfg = vhs_cfg(Nv, Nrho, M, dev, precision='single')
    be = CUDABackend(cfg)
    vm = DGFSVelocityMesh(be, cfg)
    sm = DGFSVHSGLLScatteringModel(be, cfg, vm)
    return be, vm, sm, QSurrogate(sm.grid, nmodes=k, width=w)


def test_training_gradients_match_fp64_oracle(cuda):
    from oracle.surrogate import loss_and_grads
    be, vm, sm, q = _model(k=64, w=128)
    gen = torch.Generator(device=be.device).manual_seed(3)
    q._init_params(gen)
    for l in range(4):                              # non-trivial biases
        q.b[l].normal_(0, 0.1, generator=gen)
    B = 32
    x = torch.randn(B, 64, device=be.device, generator=gen).bfloat16()
    t = torch.randn(B, 64, device=be.device, generator=gen)
    y = q.forward_train(x)
    dy = torch.empty_like(y)
    loss = torch.zeros(1, dtype=torch.float64, device=be.device)
    from frfs_b200 import _lib
    _lib.check(_lib.lib().bdgfs_relmse(y.data_ptr(), t.data_ptr(), B, 64, 1e-12, dy.data_ptr(),
                                       loss.data_ptr(), _lib.stream_ptr()), 'relmse')
    q.backward_train(dy)
    torch.cuda.synchronize()
    W = [w.bfloat16().double().cpu().numpy() for w in q.W]
    b = [bb.double().cpu().numpy() for bb in q.b]
    L, gW, gb = loss_and_grads(x.double().cpu().numpy(), t.double().cpu().numpy(), W, b)
    assert abs(float(loss) - L) < 2e-2 * L
    for l in range(4):
        e = np.linalg.norm(q.gW[l].double().cpu().numpy() - gW[l]) / np.linalg.norm(gW[l])
        eb = np.linalg.norm(q.gb[l].double().cpu().numpy() - gb[l]) / np.linalg.norm(gb[l])
        assert e < 3e-2 and eb < 3e-2, (l, e, eb)   # bf16 operands, FP32 accumulation


@pytest.fixture(scope='module')
def small_fit(cuda):
    be, vm, sm, q = _model(k=64, w=256)
    q.fit(nsamples=16384, ntest=2048, epochs=6, lr=1e-3, batch=512, nbasis=4096, chunk=4096)
    return be, vm, sm, q


def test_small_fit_learns_and_gains(small_fit):
    """Training lowers the loss, the trained network is far more accurate
    than the same network untrained, and on the cells it serves it is much
    faster than the spectral method it replaces."""
    import time
    be, vm, sm, q = small_fit
    assert q.history[-1] < 0.5 * q.history[0]
    trained = q.test_err['aggregate']
    saved = [w.clone() for w in q.W], [b.clone() for b in q.b]
    gen = torch.Generator(device=be.device).manual_seed(77)
    q._init_params(gen)
    q._fold()
    untrained = q.evaluate(1024, seed=5)['aggregate']
    q.W, q.b = saved
    q._fold()
    assert trained < 0.5 * untrained, (trained, untrained)
    f = sample_family(vm.c0(), 2048, torch.Generator(device=be.device).manual_seed(8), be.device)
    out = torch.empty_like(f)
    h = HybridCollider(q, threshold=float('inf'), recheck=0.0)
    for _ in range(2):
        h(f, out)
        sm.collide(f, out, project=True, exact=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(3):
        h(f, out)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(3):
        sm.collide(f, out, project=True, exact=False)
    torch.cuda.synchronize()
    t_spec = time.perf_counter() - t0
    assert t_sur < t_spec / 3, (t_sur, t_spec)


def test_hybrid_limits(small_fit):
    be, vm, sm, q = small_fit
    gen = torch.Generator(device=be.device).manual_seed(9)
    f = sample_family(vm.c0(), 300, gen, be.device)
    plain = torch.empty_like(f)
    sm.collide(f, plain, project=True, exact=False)
    # threshold 0: everything spectral -> identical to the plain operator
    h0 = HybridCollider(q, threshold=0.0, recheck=0.02)
    q0 = torch.empty_like(f)
    h0(f, q0)
    torch.cuda.synchronize()
    assert torch.equal(q0, plain)
    assert h0.stats()['surrogate_cells'] == 0
    # everything surrogate, everything re-checked -> spectral kept everywhere,
    # the surrogate's error measured on all cells
    h1 = HybridCollider(q, threshold=float('inf'), recheck=1.0)
    q1 = torch.empty_like(f)
    h1(f, q1)
    torch.cuda.synchronize()
    st = h1.stats()
    assert st['surrogate_cells'] == 300 and st['rechecked_cells'] == 300
    assert torch.equal(q1, plain)
    assert st['recheck_rel_l2'] is not None and st['recheck_rel_l2'] < 2.0
    # re-check fraction is honoured approximately
    h2 = HybridCollider(q, threshold=float('inf'), recheck=0.2)
    h2(f, torch.empty_like(f))
    torch.cuda.synchronize()
    assert 30 <= h2.stats()['rechecked_cells'] <= 90


def test_surrogate_output_conserves(small_fit):
    be, vm, sm, q = small_fit
    gen = torch.Generator(device=be.device).manual_seed(10)
    f = sample_family(vm.c0(), 64, gen, be.device)
    h = HybridCollider(q, threshold=float('inf'), recheck=0.0)
    out = torch.empty_like(f)
    h(f, out)
    torch.cuda.synchronize()
    cv = torch.as_tensor(vm.cv(), device=be.device)
    phi = torch.stack([torch.ones_like(cv[0]), cv[0], cv[1], cv[2], (cv * cv).sum(0)])
    m = out.double() @ phi.T * vm.cw()
    scale = out.double().abs().sum(1, keepdim=True) * vm.cw() * 36.0
    assert bool((m.abs() < 1e-5 * scale).all())     # FP32 storage of FP64-projected rows
