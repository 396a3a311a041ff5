// Fused FR right-hand side on the 5th-generation tensor cores (FP32 state).
//
// For one element and 128 velocities the FR residual is a small GEMM,
//   R[v][i] = sum_k X[v][k] Op[i][k],   k < ND*NU:  X = F~[d][j] (flux at the
//   solution points, d = k / NU, j = k % NU),  Op = M1 - M3 M2;
//   ND*NU <= k < ND*NU + NF:  X = Fhat[f] (common normal flux at the face
//   points), Op = M3,
// followed by out = a u + b (-rcpdjac R) + c1 x1 + c2 x2 (the same quantity
// the CUDA-core rhs_kernel in fr.cu forms; reference operators as listed
// there).  Thread t of the CTA owns velocity v0 + t: it computes its row of
// X (in K-chunks of 32, tf32 hi/lo split), writes it into a K-major
// 128-byte-swizzled shared-memory tile, and after the MMAs reads its own
// row of the accumulator from TMEM lane t.  One thread issues
// tcgen05.mma.kind::tf32 with M = 128 (velocities), N = 16 or 32 (solution
// points, padded), K = 8, three products per step (hi*hi + hi*lo + lo*hi:
// the 3xTF32 split keeps FP32 accuracy).  X chunks are double-buffered, so
// building chunk c+1 overlaps the MMAs of chunk c.  Every mbarrier wait is
// bounded; a wait that runs out stops the CTA and sets *err.
//
// Measured on B200 this engine is slower than the CUDA-core kernel (lid
// cavity, hex P2: 11.2 ms vs 2.8 ms per launch): with 128 threads per CTA and
// every tile serialised as build -> barrier -> MMA -> wait, it is latency
// bound.  It is selected only on request (bdgfs_fr_eles.engine = 1).
#include "common.cuh"
#include "fr_tc.cuh"
#include "tcgen05.cuh"

namespace bdgfs {
namespace frtc {

using namespace tc;

constexpr int THREADS = 128;
constexpr uint32_t kPoll = 1u << 24;

template <int ND, int NU, int NF>
struct Shape {
    static constexpr int KV = ND * NU, K = KV + NF, KP = (K + 31) / 32 * 32, NCH = KP / 32;
    static constexpr int NP = NU <= 16 ? 16 : 32;              // MMA N (>= NU)
    static constexpr uint32_t B_CH = NP * 128;                 // bytes of one operator chunk (one copy)
    static constexpr uint32_t A_CH = 128 * 128;                // bytes of one X chunk (one copy)
    static constexpr uint32_t OFF_BLO = NCH * B_CH;
    static constexpr uint32_t OFF_A = 2 * NCH * B_CH;          // X buffers: [buf][hi|lo]
    static constexpr uint32_t BYTES = OFF_A + 4 * A_CH;
};

// byte offset of element (row r, column kk < 32) in a K-major tile of
// 128-byte rows with the 128-byte swizzle (8-row atoms, 1024 B apart)
__device__ __forceinline__ uint32_t sw128(int r, int kk)
{
    return uint32_t((r >> 3) * 1024 + (r & 7) * 128 + (((kk >> 2) ^ (r & 7)) << 4) + (kk & 3) * 4);
}

__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity)
{
    for (uint32_t it = 0; it < kPoll; ++it)
        if (mbar_try(bar, parity)) return true;
    return false;
}

template <int ND, int NU, int NF>
__global__ void __launch_bounds__(THREADS) rhs_tc_kernel(const bdgfs_fr_eles el, const bdgfs_fr_walls wl,
                                                         const float* __restrict__ u,
                                                         const float* __restrict__ uf, float* out, float a,
                                                         float b, const float* x1, float c1,
                                                         const float* x2, float c2, int64_t chunk,
                                                         int32_t* err)
{
    using S = Shape<ND, NU, NF>;
    extern __shared__ unsigned char smraw[];
    __shared__ float sm[NU * ND * ND], rj[NU], pn[NF * ND], mg[NF];
    __shared__ int nb[NF];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ uint32_t tmem_s;
    unsigned char* base = smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u);
    const int t = threadIdx.x, warp = t >> 5;
    const int64_t e = blockIdx.y, nv = el.nv;

    // ---- operator chunks (tf32 hi / lo), element data
    {
        const float* gd = static_cast<const float*>(el.dcorr);   // [NU][KV]
        const float* gm = static_cast<const float*>(el.m3);      // [NU][NF]
        for (int idx = t; idx < S::NP * S::KP; idx += THREADS) {
            const int n = idx / S::KP, k = idx - n * S::KP;
            float x = 0.f;
            if (n < NU) x = k < S::KV ? gd[n * S::KV + k] : (k < S::K ? gm[n * NF + (k - S::KV)] : 0.f);
            const uint32_t hi = to_tf32(x);
            const uint32_t lo = to_tf32(x - __uint_as_float(hi));
            const uint32_t off = (k >> 5) * S::B_CH + sw128(n, k & 31);
            *reinterpret_cast<uint32_t*>(base + off) = hi;
            *reinterpret_cast<uint32_t*>(base + S::OFF_BLO + off) = lo;
        }
        const float* gs = static_cast<const float*>(el.smats) + e * NU * ND * ND;
        for (int i = t; i < NU * ND * ND; i += THREADS) sm[i] = gs[i];
        const float* gr = static_cast<const float*>(el.rcpdjac) + e * NU;
        for (int i = t; i < NU; i += THREADS) rj[i] = gr[i];
        const float* gp = static_cast<const float*>(el.pnorm) + e * NF * ND;
        for (int i = t; i < NF * ND; i += THREADS) pn[i] = gp[i];
        const float* gg = static_cast<const float*>(el.magn) + e * NF;
        for (int i = t; i < NF; i += THREADS) {
            mg[i] = gg[i];
            nb[i] = el.nbr[e * NF + i];
        }
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_s)),
                     "r"(32u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_s;
    constexpr uint32_t idesc = idesc_tf32(128, S::NP);
    const uint32_t sbase = smem_u32(base);

    const float* c0 = static_cast<const float*>(el.c0);
    const float* uw = static_cast<const float*>(wl.uwall);
    const float* fw = static_cast<const float*>(wl.fw);
    const float* bcv = static_cast<const float*>(wl.bcv);
    const int64_t v1 = (int64_t(blockIdx.x) + 1) * chunk < nv ? (int64_t(blockIdx.x) + 1) * chunk : nv;
    uint32_t g = 0;          // chunks issued by this CTA (buffer = g & 1, use = g >> 1)
    bool failed = false;
    for (int64_t vt = int64_t(blockIdx.x) * chunk; vt < v1 && !failed; vt += THREADS) {
        const int64_t v = vt + t;
        const bool live = v < v1;
        float c[3] = {0.f, 0.f, 0.f};
        if (live) {
            const uint32_t vv = uint32_t(v), N = uint32_t(el.Nv);
            const uint32_t q = vv / N, iz = vv - q * N, ix = q / N, iy = q - ix * N;
            c[0] = c0[ix];
            c[1] = c0[iy];
            c[2] = c0[iz];
        }
        float uu[NU];
#pragma unroll
        for (int j = 0; j < NU; ++j) uu[j] = live ? u[(e * NU + j) * nv + v] : 0.f;
#pragma unroll
        for (int ch = 0; ch < S::NCH; ++ch) {
            const uint32_t buf = g & 1u, use = g >> 1;
            if (g >= 2) {
                const bool ok = wait_bar(&bar[buf], (use - 1) & 1u);
                if (__syncthreads_or(!ok)) { failed = true; break; }
            }
            // this thread's 32 values of the chunk
            float xv[32];
#pragma unroll
            for (int kk = 0; kk < 32; ++kk) {
                const int k = ch * 32 + kk;
                float x = 0.f;
                if (k < S::KV) {
                    const int d = k / NU, j = k - d * NU;
                    float al = 0.f;
#pragma unroll
                    for (int m = 0; m < ND; ++m) al += sm[(j * ND + d) * ND + m] * c[m];
                    x = al * uu[j];
                } else if (k < S::K && live) {
                    const int f = k - S::KV;
                    const float ul = uf[(e * NF + f) * nv + v];
                    float nc = 0.f;
#pragma unroll
                    for (int m = 0; m < ND; ++m) nc += pn[f * ND + m] * c[m];
                    const int n = nb[f];
                    float ur;
                    if (n >= 0) {
                        ur = uf[int64_t(n) * nv + v];
                    } else {
                        const int w = -1 - n;
                        const int bid = wl.bcid[w];
                        const int kd = wl.kind ? wl.kind[bid] : BDGFS_BC_DIFFUSE;
                        if (kd == BDGFS_BC_OUTLET) {
                            ur = ul;
                        } else if (kd >= BDGFS_BC_SPECULAR_X) {  // own face row at the mirrored velocity
                            const int64_t N = el.Nv;
                            const int64_t ix = v / (N * N), iy = (v / N) % N, iz = v % N;
                            const int64_t vm =
                                kd == BDGFS_BC_SPECULAR_X ? v + (N - 1 - 2 * ix) * N * N
                                : kd == BDGFS_BC_SPECULAR_Y ? v + (N - 1 - 2 * iy) * N
                                                            : v + (N - 1 - 2 * iz);
                            ur = uf[(e * NF + f) * nv + vm];
                        } else {
                            float fac = 0.f;
#pragma unroll
                            for (int m = 0; m < ND; ++m) fac += (c[m] - uw[bid * 3 + m]) * pn[f * ND + m];
                            const float sc = kd == BDGFS_BC_DIFFUSE ? -bcv[2 * w] / bcv[2 * w + 1] : 1.f;
                            ur = fac < 0.f ? fw[int64_t(bid) * nv + v] * sc : ul;
                        }
                    }
                    x = mg[f] * (0.5f * nc * (ul + ur) + 0.5f * fabsf(nc) * (ul - ur));
                }
                xv[kk] = x;
            }
            unsigned char* ahi = base + S::OFF_A + buf * 2 * S::A_CH;
            unsigned char* alo = ahi + S::A_CH;
#pragma unroll
            for (int s4 = 0; s4 < 8; ++s4) {
                uint4 h, l;
                uint32_t* hp = reinterpret_cast<uint32_t*>(&h);
                uint32_t* lp = reinterpret_cast<uint32_t*>(&l);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float x = xv[s4 * 4 + q];
                    hp[q] = to_tf32(x);
                    lp[q] = to_tf32(x - __uint_as_float(hp[q]));
                }
                const uint32_t off = sw128(t, s4 * 4);
                *reinterpret_cast<uint4*>(ahi + off) = h;
                *reinterpret_cast<uint4*>(alo + off) = l;
            }
            fence_async_smem();
            __syncthreads();
            if (t == 0) {
                tc_fence_after();
                const uint32_t a0 = sbase + S::OFF_A + buf * 2 * S::A_CH, a1 = a0 + S::A_CH;
                const uint32_t b0 = sbase + ch * S::B_CH, b1 = b0 + S::OFF_BLO;
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {
                    const uint64_t ah = smem_desc(a0 + ks * 32, 16, 1024, 2);
                    const uint64_t al = smem_desc(a1 + ks * 32, 16, 1024, 2);
                    const uint64_t bh = smem_desc(b0 + ks * 32, 16, 1024, 2);
                    const uint64_t bl = smem_desc(b1 + ks * 32, 16, 1024, 2);
                    mma_tf32(tmem, ah, bh, idesc, (ch > 0 || ks > 0) ? 1u : 0u);
                    mma_tf32(tmem, ah, bl, idesc, 1u);
                    mma_tf32(tmem, al, bh, idesc, 1u);
                }
                mma_commit(&bar[buf]);
            }
            ++g;
        }
        if (failed) break;
        // accumulator of this tile
        {
            const uint32_t lb = (g - 1) & 1u, lu = (g - 1) >> 1;
            const bool ok = wait_bar(&bar[lb], lu & 1u);
            if (__syncthreads_or(!ok)) { failed = true; break; }
        }
        tc_fence_after();
        float R[S::NP];
#pragma unroll
        for (int c16 = 0; c16 < S::NP; c16 += 16) {
            uint32_t r[16];
            tmem_ld16_issue(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c16), r);
            tmem_wait();
#pragma unroll
            for (int q = 0; q < 16; ++q) R[c16 + q] = __uint_as_float(r[q]);
        }
        tc_fence_before();
        if (live) {
#pragma unroll
            for (int i = 0; i < NU; ++i) {
                const int64_t idx = (e * NU + i) * nv + v;
                float o = a * uu[i] + b * (-rj[i] * R[i]);
                if (x1) o += c1 * x1[idx];
                if (x2) o += c2 * x2[idx];
                out[idx] = o;
            }
        }
        __syncthreads();          // TMEM read before the next tile overwrites it
    }
    if (failed && t == 0 && err) atomicExch(err, BDGFS_ETIMEOUT);
    // MMAs issued and not yet waited for (only after a failed wait): bounded drain
    if (failed && t == 0 && g > 0) wait_bar(&bar[(g - 1) & 1u], ((g - 1) >> 1) & 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(32u));
    }
}

template <int ND, int NU, int NF>
int launch(const bdgfs_fr_eles& el, const bdgfs_fr_walls& wl, const float* u, const float* uf, float* out,
           float a, float b, const float* x1, float c1, const float* x2, float c2, cudaStream_t st)
{
    using S = Shape<ND, NU, NF>;
    const int64_t chunk = 4 * THREADS;
    const int64_t bx = (el.nv + chunk - 1) / chunk;
    if (bx > 65535 || el.neles > 65535) return BDGFS_EUNSUPPORTED;
    const size_t smem = S::BYTES + 1024;
    // dynamic shared-memory opt-in, once per device
    if (const int rc = smem_optin(reinterpret_cast<const void*>(rhs_tc_kernel<ND, NU, NF>), smem))
        return rc;
    rhs_tc_kernel<ND, NU, NF><<<dim3(unsigned(bx), unsigned(el.neles)), THREADS, smem, st>>>(
        el, wl, u, uf, out, a, b, x1, c1, x2, c2, chunk, nullptr);
    return cuda_status(cudaGetLastError());
}

}  // namespace frtc

int fr_rhs_tc(const bdgfs_fr_eles& el, const bdgfs_fr_walls& wl, const void* u, const void* uf, void* out,
              double a, double b, const void* x1, double c1, const void* x2, double c2, cudaStream_t st)
{
    if (el.fp64 || el.engine != 1) return BDGFS_EUNSUPPORTED;
    const auto U = static_cast<const float*>(u), F = static_cast<const float*>(uf);
    const auto X1 = static_cast<const float*>(x1), X2 = static_cast<const float*>(x2);
    auto O = static_cast<float*>(out);
#define GO(D, NUv, NFv)                                                                                \
    if (el.ndims == D && el.nupts == NUv && el.nfpts == NFv)                                           \
        return frtc::launch<D, NUv, NFv>(el, wl, U, F, O, float(a), float(b), X1, float(c1), X2,        \
                                         float(c2), st);
    GO(2, 4, 8) GO(2, 9, 12) GO(2, 16, 16) GO(2, 25, 20) GO(3, 8, 24) GO(3, 27, 54)
#undef GO
    return BDGFS_EUNSUPPORTED;
}

}  // namespace bdgfs
