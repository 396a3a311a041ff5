"""tcgen05 tensor-core GEMM and FP32 GEMM against a torch FP32 reference of
the same operation (operands rounded to bf16 for the tensor-core engine)."""
import math

import pytest
import torch

from frfs_b200.gemm import ACT_GELU, ACT_GELU_GRAD, gemm

pytestmark = pytest.mark.gpu


def _ref(A, B, alpha=1.0, bias=None):
    r = alpha * (A.double() @ B.double().T)
    if bias is not None:
        r = r + bias.double()
    return r


def _rel(x, y):
    return float((x.double() - y.double()).norm() / y.double().norm())


@pytest.mark.parametrize('M,N,K', [(128, 128, 64), (64, 40, 16), (300, 200, 130),
                                   (1024, 1024, 512), (257, 513, 1000)])
def test_tc_gemm_matches_fp32_reference(cuda, M, N, K):
    g = torch.Generator(device=cuda).manual_seed(M + N + K)
    A = torch.randn(M, K, device=cuda, generator=g).bfloat16()
    B = torch.randn(N, K, device=cuda, generator=g).bfloat16()
    C = torch.empty(M, N, device=cuda)
    gemm(A, B, out=C)
    torch.cuda.synchronize()
    assert _rel(C, _ref(A, B)) < 1e-5


def test_tc_gemm_strided_float_operands_bias_gelu(cuda):
    g = torch.Generator(device=cuda).manual_seed(5)
    At = torch.randn(96, 200, device=cuda, generator=g)       # A = At^T  (200 x 96)
    Bt = torch.randn(96, 150, device=cuda, generator=g)       # B = Bt^T  (150 x 96)
    bias = torch.randn(150, device=cuda, generator=g)
    C = torch.empty(200, 150, device=cuda)
    Z = torch.empty(200, 150, device=cuda)
    Cb = torch.empty(200, 150, device=cuda, dtype=torch.bfloat16)
    gemm(At, Bt, ta=True, tb=True, alpha=0.5, bias=bias, act=ACT_GELU, out=C, out_bf16=Cb, zout=Z)
    torch.cuda.synchronize()
    Ar, Br = At.bfloat16().float().T, Bt.bfloat16().float().T
    z = _ref(Ar, Br, 0.5, bias)
    assert _rel(Z, z) < 1e-5
    h = 0.5 * z * (1 + torch.erf(z / math.sqrt(2)))
    assert _rel(C, h) < 1e-5
    assert _rel(Cb.float(), h) < 1e-2
    # GELU-derivative epilogue
    D = torch.empty(200, 150, device=cuda)
    gemm(At, Bt, ta=True, tb=True, act=ACT_GELU_GRAD, zin=Z, out=D)
    torch.cuda.synchronize()
    phi = torch.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)
    cdf = 0.5 * (1 + torch.erf(z / math.sqrt(2)))
    assert _rel(D, _ref(Ar, Br) * (cdf + z * phi)) < 1e-5


def test_f32_gemm_engine(cuda):
    g = torch.Generator(device=cuda).manual_seed(9)
    A = torch.randn(333, 777, device=cuda, generator=g)
    B = torch.randn(129, 777, device=cuda, generator=g)
    C = torch.ones(333, 129, device=cuda)
    gemm(A, B, alpha=2.0, beta=1.0, out=C, engine=1)
    torch.cuda.synchronize()
    assert _rel(C, 2.0 * _ref(A, B) + 1.0) < 1e-6


@pytest.mark.parametrize('M,N,K', [(2048, 2560, 256),      # 160 tiles: >1 tile per CTA
                                   (300, 528, 13824),       # long K, ragged N
                                   (1, 8, 8), (129, 257, 72)])
def test_tma_engine_matches_general_engine(cuda, M, N, K):
    """The persistent TMA-fed engine (engine 0 on contiguous bf16 operands)
    against the general loader (engine 2) and an FP64 reference, with every
    epilogue option: bias, GELU, pre-activation, bf16 copy, row scale,
    scattered output rows and a device row count."""
    g = torch.Generator(device=cuda).manual_seed(M * 7 + N + K)
    Abig = torch.randn(M, K + 24, device=cuda, generator=g).bfloat16()
    A = Abig[:, 8:8 + K]                                   # row stride K+24, 16-byte aligned start
    B = torch.randn(N, K, device=cuda, generator=g).bfloat16()
    bias = torch.randn(N, device=cuda, generator=g)
    scale = torch.rand(M, device=cuda, generator=g) + 0.5
    crow = torch.randperm(M, device=cuda, generator=g).to(torch.int32)
    cnt = torch.tensor([max(1, M - 37)], dtype=torch.int64, device=cuda)
    outs = []
    for eng in (0, 2):
        C = torch.zeros(M, N, device=cuda)
        Cb = torch.zeros(M, N, device=cuda, dtype=torch.bfloat16)
        Z = torch.zeros(M, N, device=cuda)
        gemm(A, B, alpha=0.75, bias=bias, act=ACT_GELU, out=C, out_bf16=Cb, zout=Z,
             row_scale=scale, crow=crow, mcount=cnt, engine=eng)
        outs.append((C, Cb, Z))
    torch.cuda.synchronize()
    c = int(cnt.item())
    z = 0.75 * scale[:c, None].double() * (A[:c].double() @ B.double().T) + bias.double()
    h = 0.5 * z * (1 + torch.erf(z / math.sqrt(2)))
    rows = crow[:c].long()
    tol = 1e-5 * max(1.0, math.sqrt(K / 1024))     # FP32 accumulation over K
    for C, Cb, Z in outs:
        assert _rel(Z[rows], z) < tol
        assert _rel(C[rows], h) < tol
        assert _rel(Cb[rows].float(), h) < 1e-2
        # rows past the device count are untouched
        rest = torch.ones(M, dtype=torch.bool, device=cuda)
        rest[rows] = False
        assert float(C[rest].abs().sum()) == 0.0
    assert _rel(outs[0][0][rows], outs[1][0][rows]) < tol


def test_tma_engine_gelu_grad_and_plain(cuda):
    g = torch.Generator(device=cuda).manual_seed(3)
    A = torch.randn(640, 1024, device=cuda, generator=g).bfloat16()
    B = torch.randn(768, 1024, device=cuda, generator=g).bfloat16()
    Z = torch.randn(640, 768, device=cuda, generator=g)
    D = torch.empty(640, 768, device=cuda)
    gemm(A, B, act=ACT_GELU_GRAD, zin=Z, out=D)
    P = torch.empty(640, 768, device=cuda)
    gemm(A, B, out=P)
    torch.cuda.synchronize()
    z = Z.double()
    phi = torch.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)
    cdf = 0.5 * (1 + torch.erf(z / math.sqrt(2)))
    assert _rel(D, _ref(A, B) * (cdf + z * phi)) < 1e-5
    assert _rel(P, _ref(A, B)) < 1e-5


def test_bounded_wait_times_out_then_next_calls_are_correct(cuda):
    """The mbarrier polling loop of the tensor-core kernels, given a small
    limit on a barrier that nothing completes, gives up and reports
    BDGFS_ETIMEOUT (-4) instead of hanging; the context stays usable: the
    same wait on a completed barrier reports success and a GEMM that follows
    is correct."""
    from frfs_b200 import _lib
    L = _lib.lib()
    status = torch.full((1,), 99, dtype=torch.int32, device=cuda)
    assert L.bdgfs_wait_probe(1000, 0, status.data_ptr(), _lib.stream_ptr()) == 0
    torch.cuda.synchronize()
    assert int(status.item()) == -4
    assert L.bdgfs_wait_probe(1000, 1, status.data_ptr(), _lib.stream_ptr()) == 0
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert L.bdgfs_wait_probe(0, 0, status.data_ptr(), _lib.stream_ptr()) == -1
    g = torch.Generator(device=cuda).manual_seed(9)
    A = torch.randn(300, 130, device=cuda, generator=g).bfloat16()
    B = torch.randn(200, 130, device=cuda, generator=g).bfloat16()
    C = torch.empty(300, 200, device=cuda)
    gemm(A, B, out=C)
    torch.cuda.synchronize()
    assert _rel(C, _ref(A, B)) < 1e-5
