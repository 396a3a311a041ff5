// Tensor-core GEMM on the 5th-generation tensor cores (tcgen05.mma, BF16
// operands, FP32 accumulators in tensor memory), used by the learned
// collision-operator surrogate (projection onto the mode basis, the MLP and
// its backward pass, reconstruction).
//
//   C[m][n] = alpha * sum_k A(m,k) B(n,k)  (+ bias[n])  -> epilogue
//   A(m,k) = A[m*sam + k*sak],  B(n,k) = B[n*sbn + k*sbk]   (any strides)
//
// One CTA computes a 128 x 128 tile with four warps.  Operands are staged in
// shared memory by all threads (float or bf16 sources, converted to bf16) in
// the canonical K-major, no-swizzle layout of the MMA: 8-row x 16-byte core
// matrices, the two halves of each 16-wide K step LBO = 128 B apart and
// consecutive 8-row groups SBO = 1024 B apart.  One elected thread issues
// four kind::f16 MMAs (M=128, N=128, K=16) per 64-wide K stage into a
// 128-column TMEM accumulator and commits them to an mbarrier; the stage is
// double-buffered, so loading stage s+1 overlaps the MMAs of stage s.  The
// epilogue reads the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31 = tile rows) and applies bias / GELU / GELU-derivative.
// Every mbarrier wait is bounded; on expiry the kernel records
// BDGFS_ETIMEOUT in the status word and leaves.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "tcgen05.cuh"

namespace bdgfs {

namespace tc {

constexpr int BM = 128, BN = 128, BK = 64;
constexpr int THREADS = 128;
constexpr int TILE_BYTES = BM * BK * 2;          // 16 KB per operand per stage
constexpr uint32_t kWaitLimit = 1u << 26;        // bounded mbarrier polls
constexpr uint32_t kIdesc = idesc_bf16(BM, BN);

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase)
{
    return mbar_wait_bounded(bar, phase, kWaitLimit);
}

// Bounded-wait probe: one thread waits on an mbarrier of one expected
// arrival; with arrive = 0 nothing arrives, so the wait runs out after
// `limit` polls and the status word gets BDGFS_ETIMEOUT (no copy or MMA is
// in flight, no TMEM is held); with arrive = 1 the thread arrives first and
// the wait succeeds (BDGFS_OK).
__global__ void wait_probe_kernel(uint32_t limit, int arrive, int32_t* status)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    if (arrive) mbar_arrive(&bar);
    *status = mbar_wait_bounded(&bar, 0, limit) ? BDGFS_OK : BDGFS_ETIMEOUT;
}

__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return smem_desc(saddr, lbo, sbo, 0);
}

template <typename S>
__device__ __forceinline__ float to_f(S x);
template <>
__device__ __forceinline__ float to_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }

// Stage one 128 x 64 operand tile into the canonical layout:
// element (r, k) at ((r/8)*8 + k/8)*128 + (r%8)*16 + (k%8)*2 bytes.
template <typename S>
__device__ __forceinline__ void load_tile(unsigned char* dst, const S* src, int64_t rows,
                                          int64_t K, int64_t srow, int64_t sk, int64_t r0,
                                          int64_t k0, const int32_t* rowmap)
{
    // 128 rows x 8 k-groups = 1024 (row, kgroup) pairs, 8 per thread
    for (int p = threadIdx.x; p < BM * (BK / 8); p += THREADS) {
        const int r = p / (BK / 8), kg = p % (BK / 8);
        const int64_t gr = r0 + r;
        const int64_t sr = (gr < rows && rowmap) ? int64_t(rowmap[gr]) : gr;
        __align__(16) __nv_bfloat16 h[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int64_t gk = k0 + kg * 8 + j;
            float x = 0.f;
            if (gr < rows && gk < K) x = to_f<S>(src[sr * srow + gk * sk]);
            h[j] = __float2bfloat16_rn(x);
        }
        unsigned char* d = dst + ((r / 8) * (BK / 8) + kg) * 128 + (r % 8) * 16;
        *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(h);
    }
}

}  // namespace tc

template <typename SA, typename SB>
__global__ void __launch_bounds__(tc::THREADS, 1)
    tc_gemm_kernel(const bdgfs_gemm_args g, const SA* __restrict__ A, const SB* __restrict__ B)
{
    using namespace tc;
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char* sA[2] = {sm, sm + TILE_BYTES};
    unsigned char* sB[2] = {sm + 2 * TILE_BYTES, sm + 3 * TILE_BYTES};
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t m0 = int64_t(blockIdx.y) * BM, n0 = int64_t(blockIdx.x) * BN;
    // rows beyond a device-side count: nothing to do (uniform per CTA)
    int64_t Mrows = g.M;
    if (g.mcount) {
        const int64_t c = *g.mcount;
        Mrows = c < g.M ? (c < 0 ? 0 : c) : g.M;
    }
    if (m0 >= Mrows) return;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_s)),
                     "r"(uint32_t(BN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;

    const int64_t nk = (g.K + BK - 1) / BK;
    uint32_t phase[2] = {0, 0};
    bool ok = true;
    for (int64_t kt = 0; kt < nk; ++kt) {
        const int s = int(kt & 1);
        if (kt >= 2) {   // the MMAs that read this buffer two stages ago are done
            if (!mbar_wait(&bar[s], phase[s])) ok = false;
            phase[s] ^= 1;
        }
        if (!__syncthreads_and(ok)) break;
        load_tile<SA>(sA[s], A, Mrows, g.K, g.sam, g.sak, m0, kt * BK, g.arow);
        load_tile<SB>(sB[s], B, g.N, g.K, g.sbn, g.sbk, n0, kt * BK, nullptr);
        fence_async_smem();
        __syncthreads();
        if (warp == 0) {
            tc_fence_after();
            if (lane == 0) {
                const uint32_t a0 = smem_u32(sA[s]), b0 = smem_u32(sB[s]);
#pragma unroll
                for (int ks = 0; ks < BK / 16; ++ks) {
                    const uint64_t ad = make_desc(a0 + ks * 256, 128, 1024);
                    const uint64_t bd = make_desc(b0 + ks * 256, 128, 1024);
                    mma_bf16(tmem, ad, bd, kIdesc, (kt > 0 || ks > 0) ? 1u : 0u);
                }
                mma_commit(&bar[s]);
            }
            __syncwarp();
        }
    }
    // wait for the last one or two stages
    if (ok) {
        for (int64_t kt = nk > 2 ? nk - 2 : 0; kt < nk; ++kt) {
            const int s = int(kt & 1);
            if (!mbar_wait(&bar[s], phase[s])) ok = false;
            phase[s] ^= 1;
        }
    }
    tc_fence_after();
    if (!ok) abort_s = 1;
    __syncthreads();
    if (!abort_s) {
        // epilogue: warp w holds rows 32w + lane, 16 columns per load
        const int64_t row = m0 + warp * 32 + lane;
        const int64_t orow = (row < Mrows && g.crow) ? int64_t(g.crow[row]) : row;
        const float alpha = g.alpha * ((row < Mrows && g.row_scale) ? g.row_scale[row] : 1.f);
        const float* bias = static_cast<const float*>(g.bias);
        for (int c = 0; c < BN; c += 16) {
            float v[16];
            tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c), v);
            if (row >= Mrows) continue;
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int64_t col = n0 + c + j;
                if (col >= g.N) break;
                float x = alpha * v[j];
                if (bias) x += bias[col];
                if (g.zout) static_cast<float*>(g.zout)[orow * g.ldz + col] = x;
                if (g.act == 1) {
                    x = gelu(x);
                } else if (g.act == 2) {
                    const float z = static_cast<const float*>(g.zin)[orow * g.ldz + col];
                    x *= gelu_grad(z);
                }
                if (g.cf32) static_cast<float*>(g.cf32)[orow * g.ldc + col] = x;
                if (g.cbf16)
                    static_cast<__nv_bfloat16*>(g.cbf16)[orow * g.ldc + col] = __float2bfloat16_rn(x);
            }
        }
    } else if (threadIdx.x == 0 && g.status) {
        atomicExch(g.status, BDGFS_ETIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(BN)));
}

// ---------------------------------------------------------------------------
// FP32 SIMT GEMM (basis fitting needs FP32 accuracy): 64x64 tiles, 4x4 per
// thread, C[m][n] = alpha * sum_k A(m,k) B(n,k) + beta * C[m][n].
__global__ void __launch_bounds__(256) f32_gemm_kernel(const bdgfs_gemm_args g, const float* A,
                                                       const float* B)
{
    __shared__ float As[16][64 + 4], Bs[16][64 + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int64_t m0 = int64_t(blockIdx.y) * 64, n0 = int64_t(blockIdx.x) * 64;
    float acc[4][4] = {};
    for (int64_t k0 = 0; k0 < g.K; k0 += 16) {
        for (int p = threadIdx.x; p < 16 * 64; p += 256) {
            const int kk = p / 64, r = p % 64;
            const int64_t gm = m0 + r, gn = n0 + r, gk = k0 + kk;
            As[kk][r] = (gm < g.M && gk < g.K) ? A[gm * g.sam + gk * g.sak] : 0.f;
            Bs[kk][r] = (gn < g.N && gk < g.K) ? B[gn * g.sbn + gk * g.sbk] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) { a[i] = As[kk][ty * 4 + i]; b[i] = Bs[kk][tx * 4 + i]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
        }
        __syncthreads();
    }
    float* C = static_cast<float*>(g.cf32);
    for (int i = 0; i < 4; ++i) {
        const int64_t r = m0 + ty * 4 + i;
        if (r >= g.M) continue;
        for (int j = 0; j < 4; ++j) {
            const int64_t c = n0 + tx * 4 + j;
            if (c >= g.N) continue;
            float x = g.alpha * acc[i][j];
            if (g.beta != 0.f) x += g.beta * C[r * g.ldc + c];
            C[r * g.ldc + c] = x;
        }
    }
}

// column sums (bias gradients): out[n] = sum_m X[m][n]
__global__ void colsum_kernel(const float* X, int64_t M, int64_t N, float* out)
{
    const int64_t n = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int64_t m = 0; m < M; ++m) s += X[m * N + n];
    out[n] = s;
}

// AdamW on FP32 master weights; writes the bf16 working copy.
__global__ void adamw_kernel(float* p, const float* gr, float* m1, float* m2, __nv_bfloat16* pb,
                             int64_t n, float lr, float b1, float b2, float eps, float wd,
                             float bc1, float bc2)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = gr[i];
    const float a = b1 * m1[i] + (1.f - b1) * g;
    const float b = b2 * m2[i] + (1.f - b2) * g * g;
    m1[i] = a;
    m2[i] = b;
    const float mh = a / bc1, vh = b / bc2;
    float w = p[i];
    w -= lr * (mh / (sqrtf(vh) + eps) + wd * w);
    p[i] = w;
    if (pb) pb[i] = __float2bfloat16_rn(w);
}

// Per-row relative squared error and its gradient:
//   L = (1/M) sum_m |y_m - t_m|^2 / (|t_m|^2 + delta),  dy = dL/dy.
// delta floors the denominator (rows with tiny targets are weighted by
// their absolute error).
__global__ void __launch_bounds__(256) relmse_kernel(const float* y, const float* t, int64_t M,
                                                     int64_t N, float delta, float* dy,
                                                     double* loss)
{
    __shared__ double red[2 * 8];
    const int64_t m = blockIdx.x;
    const float* ym = y + m * N;
    const float* tm = t + m * N;
    double e[2] = {0, 0};
    for (int64_t j = threadIdx.x; j < N; j += blockDim.x) {
        const double d = double(ym[j]) - double(tm[j]);
        e[0] += d * d;
        e[1] += double(tm[j]) * double(tm[j]);
    }
    block_sum<2>(e, red);
    const double den = e[1] + double(delta);
    const float sc = float(2.0 / (den * double(M)));
    for (int64_t j = threadIdx.x; j < N; j += blockDim.x) dy[m * N + j] = sc * (ym[j] - tm[j]);
    if (threadIdx.x == 0 && loss) atomicAdd(loss, e[0] / den / double(M));
}

}  // namespace bdgfs

using namespace bdgfs;

extern "C" int32_t bdgfs_gemm(const bdgfs_gemm_args* g, void* stream)
{
    if (!g || !g->A || !g->B || g->M < 0 || g->N < 0 || g->K < 1) return BDGFS_EINVAL;
    if (!g->cf32 && !g->cbf16 && !g->zout) return BDGFS_EINVAL;
    if (g->act == 2 && !g->zin) return BDGFS_EINVAL;
    if (g->M == 0 || g->N == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (g->engine == 1) {           // FP32 SIMT
        if (g->a_bf16 || g->b_bf16 || !g->cf32 || g->act || g->bias || g->arow || g->crow ||
            g->row_scale || g->mcount)
            return BDGFS_EUNSUPPORTED;
        dim3 grid(unsigned((g->N + 63) / 64), unsigned((g->M + 63) / 64));
        f32_gemm_kernel<<<grid, 256, 0, st>>>(*g, static_cast<const float*>(g->A),
                                              static_cast<const float*>(g->B));
        return cuda_status(cudaGetLastError());
    }
    if (g->engine == 0) {           // TMA-fed persistent engine when the operands qualify
        const int rc = tma_gemm(*g, st);
        if (rc != BDGFS_EUNSUPPORTED) return rc;
    }
    if (g->beta != 0.f) return BDGFS_EUNSUPPORTED;
    const int64_t gy = (g->M + tc::BM - 1) / tc::BM, gx = (g->N + tc::BN - 1) / tc::BN;
    if (gy > 65535 || gx > 2147483647LL) return BDGFS_EINVAL;
    const dim3 grid{static_cast<unsigned>(gx), static_cast<unsigned>(gy), 1u};
    const size_t smem = 4 * tc::TILE_BYTES;
    auto launch = [&](auto kern, auto a, auto b) -> int32_t {
        if (const int rc = smem_optin(reinterpret_cast<const void*>(kern), smem)) return rc;
        kern<<<grid, tc::THREADS, smem, st>>>(*g, a, b);
        return cuda_status(cudaGetLastError());
    };
    const bool ab = g->a_bf16, bb = g->b_bf16;
    if (ab && bb)
        return launch(tc_gemm_kernel<__nv_bfloat16, __nv_bfloat16>,
                      static_cast<const __nv_bfloat16*>(g->A), static_cast<const __nv_bfloat16*>(g->B));
    if (ab && !bb)
        return launch(tc_gemm_kernel<__nv_bfloat16, float>, static_cast<const __nv_bfloat16*>(g->A),
                      static_cast<const float*>(g->B));
    if (!ab && bb)
        return launch(tc_gemm_kernel<float, __nv_bfloat16>, static_cast<const float*>(g->A),
                      static_cast<const __nv_bfloat16*>(g->B));
    return launch(tc_gemm_kernel<float, float>, static_cast<const float*>(g->A),
                  static_cast<const float*>(g->B));
}

extern "C" int32_t bdgfs_wait_probe(uint32_t limit, int32_t arrive, int32_t* status, void* stream)
{
    if (!status || limit < 1) return BDGFS_EINVAL;
    tc::wait_probe_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limit, arrive ? 1 : 0, status);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_colsum(const float* X, int64_t M, int64_t N, float* out, void* stream)
{
    if (!X || !out || M < 0 || N < 0) return BDGFS_EINVAL;
    if (N == 0) return BDGFS_OK;
    colsum_kernel<<<unsigned((N + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(X, M, N, out);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_adamw(float* p, const float* grad, float* m1, float* m2, void* p_bf16,
                               int64_t n, float lr, float beta1, float beta2, float eps,
                               float weight_decay, int64_t step, void* stream)
{
    if (!p || !grad || !m1 || !m2 || n < 0 || step < 1) return BDGFS_EINVAL;
    if (n == 0) return BDGFS_OK;
    const float bc1 = 1.f - powf(beta1, float(step)), bc2 = 1.f - powf(beta2, float(step));
    adamw_kernel<<<unsigned((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        p, grad, m1, m2, static_cast<__nv_bfloat16*>(p_bf16), n, lr, beta1, beta2, eps,
        weight_decay, bc1, bc2);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_relmse(const float* y, const float* t, int64_t M, int64_t N, float delta,
                                float* dy, double* loss, void* stream)
{
    if (!y || !t || !dy || M < 0 || N < 1 || M > 2147483647LL) return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (loss && cudaMemsetAsync(loss, 0, sizeof(double), st) != cudaSuccess) return BDGFS_ECUDA;
    if (M == 0) return BDGFS_OK;
    relmse_kernel<<<unsigned(M), 256, 0, st>>>(y, t, M, N, delta, dy, loss);
    return cuda_status(cudaGetLastError());
}
