// Persistent, warp-specialised tensor-core GEMM fed by TMA (sm_100a).
//
//   C[m][n] = alpha * row_scale[m] * sum_k A[m][k] B[n][k] (+ bias[n]) -> act
//
// for bf16 A and B whose K index is contiguous (the surrogate's inference
// chain: projection of the Maxwellian-deviation rows onto the input basis,
// the MLP layers, reconstruction from the output basis).
//
// Tile 128 x 256 x 64 (128 x 128 x 64 for GEMMs whose 256-wide tiles
// would occupy fewer than half the SMs).  One CTA per SM walks the output tiles
// (n-fastest, so CTAs that share an A row-block run together and the
// second read of it hits L2).  Warp roles:
//   warp 0      one thread issues the TMA loads of A (128 x 64) and
//               B (256 x 64) into a 4-stage ring (128-byte swizzle, one
//               swizzle atom per row), completion via mbarrier tx-count;
//   warp 1      owns 512 TMEM columns = two 128 x 256 f32 accumulators;
//               one thread issues tcgen05.mma (M=128, N=256, K=16) four
//               per stage, frees each stage with tcgen05.commit, and
//               signals a finished accumulator the same way;
//   warps 2-5   epilogue: tcgen05.ld the accumulator (warp w reads TMEM
//               lanes 32*(w%4)..+31 = tile rows), scale / bias / GELU /
//               GELU-derivative, vector stores, then release the
//               accumulator, so the epilogue of tile i overlaps the MMAs of
//               tile i+1.
// Every mbarrier wait is bounded.  A wait that runs out sets a CTA-wide
// abort flag (all other waits then give up), the status word gets
// BDGFS_ETIMEOUT, the TMA thread waits (bounded) for its loads in flight,
// the MMA thread waits (bounded) for its MMAs, and TMEM is freed.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <mutex>

#include "common.cuh"
#include "tc_gemm.cuh"
#include "tcgen05.cuh"

namespace bdgfs {
namespace tma {

using namespace tc;

constexpr int BM = 128, BK = 64;
constexpr int THREADS = 192;
constexpr uint32_t A_BYTES = BM * BK * 2;
constexpr uint32_t kPollLimit = 1u << 26;

// Tile shape by BN (output columns per tile): 256 (48 KB stages, 4 deep)
// or 128 (32 KB stages, 6 deep) for GEMMs with too few 256-wide tiles to
// fill the SMs.
template <int BN>
struct Cfg {
    static constexpr int STAGES = BN == 256 ? 4 : 6;
    static constexpr uint32_t B_BYTES = BN * BK * 2;
    static constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr uint32_t TMEM_COLS = 2 * BN;                 // two accumulators
    static constexpr size_t SMEM_BYTES = size_t(STAGES) * STAGE_BYTES + 1024;
    static constexpr uint32_t IDESC = idesc_bf16(BM, BN);
};

template <int STAGES>
struct Ctl {
    uint64_t full[STAGES], empty[STAGES], accf[2], acce[2], drain;
    uint32_t tmem;
    int abort;
};

// Bounded wait; gives up early once another role has aborted.
__device__ __forceinline__ bool wait(uint64_t* bar, uint32_t parity, volatile int* abort)
{
    for (uint32_t it = 0; it < kPollLimit; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 255u && *abort) return false;
    }
    *abort = 1;
    return false;
}

// Bounded wait that ignores the abort flag (draining work in flight).
__device__ __forceinline__ void drain_wait(uint64_t* bar, uint32_t parity)
{
    for (uint32_t it = 0; it < kPollLimit; ++it)
        if (mbar_try(bar, parity)) return;
}

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Epilogue for 32 consecutive columns col0.. of output row orow.
__device__ __forceinline__ void store_row32(const bdgfs_gemm_args& g, int64_t orow, int64_t col0,
                                            float alpha, const uint32_t (&r0)[16], const uint32_t (&r1)[16])
{
    float x[32];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        x[j] = alpha * __uint_as_float(r0[j]);
        x[16 + j] = alpha * __uint_as_float(r1[j]);
    }
    const bool full = col0 + 32 <= g.N;
    const int nv = full ? 32 : int(g.N - col0);
    const float* bias = static_cast<const float*>(g.bias);
    if (bias) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (j < nv) x[j] += __ldg(bias + col0 + j);
    }
    if (g.zout) {
        float* z = static_cast<float*>(g.zout) + orow * g.ldz + col0;
        if (full && aligned16(z) && (g.ldz & 3) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(z + j) = make_float4(x[j], x[j + 1], x[j + 2], x[j + 3]);
        } else {
            for (int j = 0; j < nv; ++j) z[j] = x[j];
        }
    }
    if (g.act == 1) {
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = gelu(x[j]);
    } else if (g.act == 2) {
        const float* zi = static_cast<const float*>(g.zin) + orow * g.ldz + col0;
        for (int j = 0; j < nv; ++j) x[j] *= gelu_grad(zi[j]);
    }
    if (g.cf32) {
        float* c = static_cast<float*>(g.cf32) + orow * g.ldc + col0;
        if (full && aligned16(c) && (g.ldc & 3) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(c + j) = make_float4(x[j], x[j + 1], x[j + 2], x[j + 3]);
        } else {
            for (int j = 0; j < nv; ++j) c[j] = x[j];
        }
    }
    if (g.cbf16) {
        __nv_bfloat16* c = static_cast<__nv_bfloat16*>(g.cbf16) + orow * g.ldc + col0;
        if (full && aligned16(c) && (g.ldc & 7) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 8) {
                __align__(16) __nv_bfloat162 h[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(x[j + 2 * i], x[j + 2 * i + 1]);
                *reinterpret_cast<uint4*>(c + j) = *reinterpret_cast<const uint4*>(h);
            }
        } else {
            for (int j = 0; j < nv; ++j) c[j] = __float2bfloat16_rn(x[j]);
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(THREADS, 1)
    tma_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                    const bdgfs_gemm_args g)
{
    using C = Cfg<BN>;
    constexpr int STAGES = C::STAGES;
    constexpr uint32_t STAGE_BYTES = C::STAGE_BYTES, TMEM_COLS = C::TMEM_COLS, kIdesc = C::IDESC;
    extern __shared__ unsigned char smraw[];
    __shared__ Ctl<STAGES> ctl;
    // stage buffers on a 1024-byte boundary (the 128-byte swizzle pattern)
    const uint32_t raw = smem_u32(smraw);
    unsigned char* sm = smraw + ((1024u - (raw & 1023u)) & 1023u);
    volatile int* abort = &ctl.abort;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int64_t Mrows = g.M;
    if (g.mcount) {
        const int64_t c = *g.mcount;
        Mrows = c < g.M ? (c < 0 ? 0 : c) : g.M;
    }
    const int64_t tilesM = (Mrows + BM - 1) / BM, tilesN = (g.N + BN - 1) / BN;
    const int64_t ntiles = tilesM * tilesN;
    const int64_t nk = (g.K + BK - 1) / BK;
    if (int64_t(blockIdx.x) >= ntiles) return;          // uniform per CTA, before any allocation

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&ctl.tmem)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&ctl.full[s], 1);
            mbar_init(&ctl.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&ctl.accf[a], 1);
            mbar_init(&ctl.acce[a], 128);
        }
        mbar_init(&ctl.drain, 1);
        ctl.abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = ctl.tmem;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer
            uint32_t stage = 0, ph = 0, used = 0, lastph = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; ok && t < ntiles; t += gridDim.x) {
                const int32_t ya = int32_t((t / tilesN) * BM), yb = int32_t((t % tilesN) * BN);
                for (int64_t kt = 0; kt < nk; ++kt) {
                    if (!wait(&ctl.empty[stage], ph ^ 1u, abort)) { ok = false; break; }
                    unsigned char* sa = sm + stage * STAGE_BYTES;
                    mbar_expect_tx(&ctl.full[stage], STAGE_BYTES);
                    tma_load_2d(sa, &tmA, int32_t(kt * BK), ya, &ctl.full[stage]);
                    tma_load_2d(sa + A_BYTES, &tmB, int32_t(kt * BK), yb, &ctl.full[stage]);
                    used |= 1u << stage;
                    lastph = (lastph & ~(1u << stage)) | (ph << stage);
                    if (++stage == STAGES) { stage = 0; ph ^= 1u; }
                }
            }
            // loads in flight complete before the CTA may exit
            for (int s = 0; s < STAGES; ++s)
                if (used & (1u << s)) drain_wait(&ctl.full[s], (lastph >> s) & 1u);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            uint32_t stage = 0, ph = 0, acc = 0, aph = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; ok && t < ntiles; t += gridDim.x) {
                if (!wait(&ctl.acce[acc], aph ^ 1u, abort)) break;
                tc_fence_after();
                const uint32_t d = tmem + acc * BN;
                for (int64_t kt = 0; kt < nk; ++kt) {
                    if (!wait(&ctl.full[stage], ph, abort)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(sm + stage * STAGE_BYTES), b0 = a0 + A_BYTES;
#pragma unroll
                    for (int ks = 0; ks < BK / 16; ++ks)
                        mma_bf16(d, smem_desc(a0 + ks * 32, 16, 1024, 2), smem_desc(b0 + ks * 32, 16, 1024, 2),
                                 kIdesc, (kt > 0 || ks > 0) ? 1u : 0u);
                    mma_commit(&ctl.empty[stage]);
                    if (++stage == STAGES) { stage = 0; ph ^= 1u; }
                }
                if (!ok) break;
                mma_commit(&ctl.accf[acc]);
                if (++acc == 2) { acc = 0; aph ^= 1u; }
            }
            // every MMA issued here is finished before TMEM is freed
            mma_commit(&ctl.drain);
            drain_wait(&ctl.drain, 0);
        }
    } else {
        // ---------------- epilogue (warps 2..5)
        const int q = warp & 3;                         // TMEM lane quadrant of this warp
        uint32_t acc = 0, aph = 0;
        for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
            if (!wait(&ctl.accf[acc], aph, abort)) break;
            tc_fence_after();
            const int64_t m0 = (t / tilesN) * BM, n0 = (t % tilesN) * BN;
            const int64_t row = m0 + q * 32 + lane;
            const bool live = row < Mrows;
            const int64_t orow = (live && g.crow) ? int64_t(g.crow[row]) : row;
            const float alpha = g.alpha * ((live && g.row_scale) ? g.row_scale[row] : 1.f);
            const uint32_t taddr = tmem + acc * BN + (uint32_t(q * 32) << 16);
            for (int c = 0; c < BN; c += 32) {
                if (n0 + c >= g.N) break;               // warp-uniform
                uint32_t r0[16], r1[16];
                tmem_ld16_issue(taddr + uint32_t(c), r0);
                tmem_ld16_issue(taddr + uint32_t(c + 16), r1);
                tmem_wait();
                if (live) store_row32(g, orow, n0 + c, alpha, r0, r1);
            }
            tc_fence_before();
            mbar_arrive(&ctl.acce[acc]);
            if (++acc == 2) { acc = 0; aph ^= 1u; }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
    if (threadIdx.x == 0 && ctl.abort && g.status) atomicExch(g.status, BDGFS_ETIMEOUT);
}

// ------------------------------------------------------------------ host
PFN_cuTensorMapEncodeTiled_v12000 encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// [rows][K] bf16, row stride ld elements; box 64 (K) x box_rows
bool make_map(CUtensorMap* m, const void* base, int64_t rows, int64_t K, int64_t ld, uint32_t box_rows)
{
    auto enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {cuuint64_t(K), cuuint64_t(rows)};
    const cuuint64_t strides[1] = {cuuint64_t(ld) * 2};
    const cuuint32_t box[2] = {uint32_t(BK), box_rows};
    const cuuint32_t es[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int sm_count()
{
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

}  // namespace tma

namespace {

template <int BN>
int launch_bn(const bdgfs_gemm_args& g, cudaStream_t st, const CUtensorMap& ma, int nsm)
{
    using namespace tma;
    using C = Cfg<BN>;
    CUtensorMap mb;
    if (!make_map(&mb, g.B, g.N, g.K, g.sbn, BN)) return BDGFS_EUNSUPPORTED;
    const int64_t tiles = ((g.M + BM - 1) / BM) * ((g.N + BN - 1) / BN);
    const unsigned grid = unsigned(tiles < nsm ? tiles : nsm);
    // dynamic shared-memory opt-in, once per device
    static std::mutex mu;
    static bool attr_set[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return BDGFS_ECUDA;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!attr_set[dev]) {
            if (cudaFuncSetAttribute(tma_gemm_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     int(C::SMEM_BYTES)) != cudaSuccess)
                return BDGFS_ECUDA;
            attr_set[dev] = true;
        }
    }
    tma_gemm_kernel<BN><<<grid, THREADS, C::SMEM_BYTES, st>>>(ma, mb, g);
    return cuda_status(cudaGetLastError());
}

}  // namespace

int tma_gemm(const bdgfs_gemm_args& g, cudaStream_t st)
{
    using namespace tma;
    const auto a16 = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    if (g.engine != 0 || !g.a_bf16 || !g.b_bf16 || g.sak != 1 || g.sbk != 1 || g.arow || g.beta != 0.f)
        return BDGFS_EUNSUPPORTED;
    if (g.K % 8 || g.sam % 8 || g.sbn % 8 || g.sam < g.K || g.sbn < g.K || !a16(g.A) || !a16(g.B))
        return BDGFS_EUNSUPPORTED;
    if (g.M > (int64_t(1) << 31) - BM || g.N > (int64_t(1) << 31) - 256 || g.K > (int64_t(1) << 31))
        return BDGFS_EUNSUPPORTED;
    if (g.act == 2 && !g.zin) return BDGFS_EINVAL;
    CUtensorMap ma;
    if (!make_map(&ma, g.A, g.M, g.K, g.sam, BM)) return BDGFS_EUNSUPPORTED;
    const int nsm = sm_count();
    if (nsm <= 0) return BDGFS_ECUDA;
    // 256-wide tiles unless they would occupy fewer than half the SMs (128-wide
    // tiles double the A traffic and run the MMA at half width: measured
    // slower whenever the 256-wide grid covers most SMs)
    const int64_t tiles256 = ((g.M + BM - 1) / BM) * ((g.N + 255) / 256);
    if (2 * tiles256 < int64_t(nsm)) return launch_bn<128>(g, st, ma, nsm);
    return launch_bn<256>(g, st, ma, nsm);
}

}  // namespace bdgfs
