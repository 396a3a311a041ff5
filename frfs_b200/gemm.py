"""Host wrappers of the surrogate's GEMMs (``bdgfs_gemm``): tensor-core
(tcgen05, bf16 operands, FP32 accumulation) and FP32 CUDA-core engines."""
import ctypes as C

import torch

from . import _lib

ACT_NONE, ACT_GELU, ACT_GELU_GRAD = 0, 1, 2


def _operand(t, trans):
    """(pointer, row stride, k stride, is_bf16) of a 2-D operand viewed as
    [rows][K] (trans=False) or as the transpose of a [K][rows] tensor."""
    if t.dim() != 2:
        raise ValueError('GEMM operands are 2-D')
    if t.dtype not in (torch.float32, torch.bfloat16):
        raise TypeError('GEMM operands are float32 or bfloat16')
    s0, s1 = t.stride()
    return (t.data_ptr(), s1, s0, t.dtype == torch.bfloat16) if trans else \
        (t.data_ptr(), s0, s1, t.dtype == torch.bfloat16)


def gemm(a, b, *, ta=False, tb=False, alpha=1.0, beta=0.0, bias=None, act=ACT_NONE,
         out=None, out_bf16=None, zout=None, zin=None, engine=0, status=None, stream=None,
         arow=None, crow=None, row_scale=None, mcount=None, M=None, ldc=None):
    """out[m][n] = alpha * row_scale[m] * sum_k A(m,k) B(n,k) (+ beta*out)
    (+ bias) -> act.  A = a (M x K) or a^T if ta; B = b (N x K) or b^T if tb.
    arow gathers rows of A, crow scatters rows of the outputs, mcount is a
    device row count (rows beyond it are skipped)."""
    pa, sam, sak, abf = _operand(a, ta)
    pb, sbn, sbk, bbf = _operand(b, tb)
    K = a.shape[0] if ta else a.shape[1]
    if M is None:
        M = a.shape[1] if ta else a.shape[0]
    N = b.shape[1] if tb else b.shape[0]
    if (b.shape[0] if tb else b.shape[1]) != K:
        raise ValueError('inner dimensions differ')
    if bias is not None and (not bias.is_cuda or not bias.is_contiguous()):
        raise ValueError('bias must be a contiguous CUDA tensor')
    # outputs: 2-D row-major views (unit column stride); one leading
    # dimension for out/out_bf16 and one for zout/zin
    lds = {}
    for name, t in (('c', out), ('c', out_bf16), ('z', zout), ('z', zin)):
        if t is None:
            continue
        if not t.is_cuda or t.dim() != 2 or t.stride(1) != 1 or t.shape[1] != N:
            raise ValueError('outputs are 2-D CUDA views with N columns and unit column stride')
        if crow is None and t.shape[0] != M:
            raise ValueError('output rows differ from M')
        if lds.setdefault(name, t.stride(0)) != t.stride(0):
            raise ValueError('out and out_bf16 (zout and zin) must share a leading dimension')
    ldc = lds.get('c', N) if ldc is None else int(ldc)
    ldz = lds.get('z', N)
    for t, dt in ((arow, torch.int32), (crow, torch.int32), (row_scale, torch.float32),
                  (mcount, torch.int64)):
        if t is not None and (t.dtype != dt or not t.is_cuda):
            raise TypeError('index/scale/count tensors: int32 rows, float32 scale, int64 count')
    args = _lib.GemmArgs(M=M, N=N, K=K, A=pa, sam=sam, sak=sak, B=pb, sbn=sbn, sbk=sbk,
                         a_bf16=int(abf), b_bf16=int(bbf), alpha=float(alpha), beta=float(beta),
                         bias=bias.data_ptr() if bias is not None else 0, act=int(act),
                         engine=int(engine),
                         cf32=out.data_ptr() if out is not None else 0,
                         cbf16=out_bf16.data_ptr() if out_bf16 is not None else 0, ldc=ldc,
                         zout=zout.data_ptr() if zout is not None else 0,
                         zin=zin.data_ptr() if zin is not None else 0, ldz=ldz,
                         status=status.data_ptr() if status is not None else 0,
                         arow=arow.data_ptr() if arow is not None else 0,
                         crow=crow.data_ptr() if crow is not None else 0,
                         row_scale=row_scale.data_ptr() if row_scale is not None else 0,
                         mcount=mcount.data_ptr() if mcount is not None else 0)
    _lib.check(_lib.lib().bdgfs_gemm(C.byref(args), _lib.stream_ptr(stream)), 'bdgfs_gemm')
    return out if out is not None else out_bf16


def colsum(x, out):
    _lib.check(_lib.lib().bdgfs_colsum(x.data_ptr(), x.shape[0], x.shape[1], out.data_ptr(),
                                       _lib.stream_ptr()), 'bdgfs_colsum')
    return out


def adamw(p, g, m1, m2, p_bf16, step, lr=3e-4, betas=(0.9, 0.999), eps=1e-8, wd=0.01):
    _lib.check(_lib.lib().bdgfs_adamw(p.data_ptr(), g.data_ptr(), m1.data_ptr(), m2.data_ptr(),
                                      p_bf16.data_ptr() if p_bf16 is not None else None,
                                      p.numel(), lr, betas[0], betas[1], eps, wd, int(step),
                                      _lib.stream_ptr()), 'bdgfs_adamw')
