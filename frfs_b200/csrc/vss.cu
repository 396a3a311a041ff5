// Fast-spectral VSS collision operator of a gas mixture on one velocity grid:
// Q_p = sum_q Q_pq(f_p, f_q) for every species p of every distribution.
//
// Reference: DGFSBiVSSGLLScatteringModel.Qij / fs (frfs/solvers/dgfsbi/
// scattering.py:229-330) and its kernels r2z, cosSinMul_pq, prod,
// computeQG, ax2, output_pq (frfs/solvers/dgfsbi/kernels/scattering/
// vss-gll.mako:100-300).  Per pair (p, q), with F = FFT(f_p)/n,
// G = FFT(f_q)/n and a = pi/L qz_r (s . l):
//   t1 = e^{+i a m_q/(m_p+m_q)} F,  t2 = e^{-i a m_p/(m_p+m_q)} G
//   G^ += w_r b_pq[r, s] FFT(IFFT(t1) IFFT(t2))          (all r, s)
//   Q_pq = prefac_pq (Re IFFT(G^) - f_p Re IFFT(c_pq G))
//
// The reference runs 9 launches and 6 cuFFT executions per pair and
// distribution, each over the full P = Nrho M slab of scratch.  Here one
// persistent CTA owns a (distribution, species p) item and walks the P
// slices one at a time through five pencil passes over CTA-private scratch
// (L2 resident), with the DFTs in registers (generated codelets):
//   A  x: phase (separable: e^{i a} = Ex[lx] Ey[ly] Ez[lz], tables in shared
//         memory) and inverse DFT of t1 and t2
//   B  y: inverse DFT of both
//   C  z: inverse DFT of both, the product T, forward DFT of T
//   D  y: forward DFT of T
//   E  x: forward DFT of T and G^ += w_r prefac_pq b_pq T^
// The gain and loss terms of all partners q are linear, so they are summed
// in the spectral domain and transformed back once per item.
//
// FP32 at Nv <= 24 keeps the two working transforms Z1, Z2 of a slice in
// shared memory (rows of N + 1 complex values, so that the z pencils of a
// warp fall on distinct bank pairs; 231.5 KB at 24^3): passes B-D then touch
// no global memory, and per slice only F, G, b_pq and G^ travel through L2.
// Other grids keep Z1, Z2 in the CTA's global scratch (rows of N).
// In FP32 at Nv = 16, 24 and 32 the spectral gain accumulator G^ also
// stays on chip, in tensor memory: each thread owns the PPT x-pencils it
// transforms in pass E (1, 2, 4), so it keeps their complex sums in its
// TMEM lane (2 N PPT columns; warp w uses lanes 32 (w mod 4).. and the
// columns after those of warps w - 4, w - 8), read and written with
// tcgen05.ld / st, and G^ reaches global scratch once per item for the
// back-transform.
#include "common.cuh"
#include "fft_codelets.cuh"
#include "tcgen05.cuh"

namespace bdgfs {

namespace {

template <typename T, int N>
struct VssCfg {
    static constexpr int n = N * N * N;
    // one pencil per thread up to 256 pencils; 2 (24^3) or 4 (32^3) per
    // thread above, so a pencil pass keeps its N complex values in registers
    static constexpr int threads = sizeof(T) == 4 ? (N * N <= 256 ? N * N : N == 24 ? 288 : 256)
                                                  : N * N / ((N * N + 255) / 256);
    // Z1, Z2 in shared memory (row pitch N + 1) or in global scratch (pitch N)
    static constexpr bool smem = sizeof(T) == 4 && N <= 24;
    static constexpr int RP = smem ? N + 1 : N;
    static constexpr size_t smem_bytes = smem ? size_t(2) * N * N * RP * sizeof(cpx<T>) : 0;
    // G^ in tensor memory: every thread owns PPT whole x-pencils (FP32,
    // Nv = 16: 64 columns per CTA; 24: 288 of 512; 32: 512)
    static constexpr bool tmem = sizeof(T) == 4 && N % 8 == 0 && N >= 16;
    static constexpr int PPT = (N * N) / threads;
    static constexpr uint32_t tmem_cols = N == 16 ? 64 : 512;
    static_assert(!tmem || (PPT * threads == N * N && threads % 32 == 0 && N % 8 == 0 &&
                            ((threads / 32 + 3) / 4) * PPT * 2 * N <= int(tmem_cols)),
                  "TMEM accumulator layout");
};

// pencil pc of axis AX: first element and stride ([x][y][z], z fastest,
// rows of RP >= N elements)
template <int N, int AX, int RP = N>
__device__ __forceinline__ void pencil(int pc, int& base, int& stride)
{
    if constexpr (AX == 0) { base = (pc / N) * RP + (pc % N); stride = N * RP; }     // (y, z)
    else if constexpr (AX == 1) { base = (pc / N) * N * RP + (pc % N); stride = RP; } // (x, z)
    else { base = pc * RP; stride = 1; }                                              // (x, y)
}

// DFT (SIGN < 0 forward, > 0 inverse, unnormalised) of every pencil of
// axis AX of A, in place, times scale
template <typename T, int N, int SIGN, int AX, int RP = N>
__device__ __forceinline__ void pass(cpx<T>* __restrict__ A, T scale = T(1))
{
    for (int pc = threadIdx.x; pc < N * N; pc += blockDim.x) {
        int b, s;
        pencil<N, AX, RP>(pc, b, s);
        cpx<T> x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = A[b + k * s];
        dft<N, SIGN>(x);
#pragma unroll
        for (int k = 0; k < N; ++k) A[b + k * s] = cpx<T>{x[k].x * scale, x[k].y * scale};
    }
}

// 3-D forward DFT of a real row into A, scaled by 1/n
template <typename T, int N>
__device__ __forceinline__ void fft_real(const T* __restrict__ f, cpx<T>* __restrict__ A)
{
    for (int pc = threadIdx.x; pc < N * N; pc += blockDim.x) {
        cpx<T> x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = cpx<T>{f[pc * N + k], T(0)};
        dft<N, -1>(x);
#pragma unroll
        for (int k = 0; k < N; ++k) A[pc * N + k] = x[k];
    }
    __syncthreads();
    pass<T, N, -1, 1>(A);
    __syncthreads();
    pass<T, N, -1, 0>(A, T(1.0 / double(N * N * N)));
    __syncthreads();
}

__device__ __forceinline__ int lfreq(int k, int N) { return k < N / 2 ? k : k - N; }

template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b)
{
    return cpx<T>{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}

template <typename T, int N>
__global__ void __launch_bounds__(VssCfg<T, N>::threads) vss_kernel(const bdgfs_vss_args g,
                                                                     cpx<T>* __restrict__ scratch)
{
    constexpr int n = VssCfg<T, N>::n;
    constexpr int RP = VssCfg<T, N>::RP;       // row pitch of Z1, Z2
    __shared__ cpx<T> E1[3][N], E2[3][N];
    extern __shared__ __align__(16) unsigned char vss_smem[];
    cpx<T>* F = scratch + size_t(blockIdx.x) * 6 * n;
    cpx<T>* Gq = F + n;
    cpx<T>* Z1 = F + 2 * n;
    cpx<T>* Z2 = F + 3 * n;
    if constexpr (VssCfg<T, N>::smem) {
        Z1 = reinterpret_cast<cpx<T>*>(vss_smem);
        Z2 = Z1 + N * N * RP;
    }
    cpx<T>* Ga = F + 4 * n;
    cpx<T>* La = F + 5 * n;
    constexpr bool kTm = VssCfg<T, N>::tmem;
    constexpr int PPT = VssCfg<T, N>::PPT;
    __shared__ uint32_t s_tmem;
    uint32_t tsv = 0;                             // this thread's TMEM lane, first column
    if constexpr (kTm) {
        if (threadIdx.x < 32) tc::tmem_alloc(&s_tmem, VssCfg<T, N>::tmem_cols);
        tc::tc_fence_before();
        __syncthreads();
        tc::tc_fence_after();
        const uint32_t warp = threadIdx.x >> 5;
        tsv = s_tmem + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(PPT * 2 * N * (warp >> 2));
    }
    const int S = g.nspcs, P = g.Nrho * g.M;
    const int64_t nitems = g.ndof * S;
    for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int p = int(item / g.ndof);
        const int64_t dof = item - int64_t(p) * g.ndof;
        const T* fp = static_cast<const T*>(g.f[p]) + dof * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            if constexpr (!kTm) Ga[i] = cpx<T>{T(0), T(0)};
            La[i] = cpx<T>{T(0), T(0)};
        }
        fft_real<T, N>(fp, F);
        for (int q = 0; q < S; ++q) {
            const int pq = p * S + q;
            const cpx<T>* G = F;
            if (q != p) {
                fft_real<T, N>(static_cast<const T*>(g.f[q]) + dof * n, Gq);
                G = Gq;
            }
            const T pref = T(g.prefac[pq]);
            const cpx<T>* cq = static_cast<const cpx<T>*>(g.c) + size_t(pq) * n;
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const cpx<T> t = cmul(cq[i], G[i]);
                La[i].x += pref * t.x;
                La[i].y += pref * t.y;
            }
            const double mq = g.mfrac[pq], mp = 1.0 - mq;
            const cpx<T>* bq = static_cast<const cpx<T>*>(g.b) + size_t(pq) * P * n;
            for (int rs = 0; rs < P; ++rs) {
                const int r = rs / g.M, s = rs - r * g.M;
                __syncthreads();
                // separable phase tables e^{+i mq a_d l}, e^{-i mp a_d l} per axis
                for (int i = threadIdx.x; i < 6 * N; i += blockDim.x) {
                    const int w = i / (3 * N), d = (i / N) % 3, k = i % N;
                    const double ang = g.rfac[r] * g.sz[3 * s + d] * lfreq(k, N) * (w ? -mp : mq);
                    double sn, cs;
                    sincos(ang, &sn, &cs);
                    (w ? E2 : E1)[d][k] = cpx<T>{T(cs), T(sn)};
                }
                __syncthreads();
                // A: phases and inverse DFT along x
                for (int pc = threadIdx.x; pc < N * N; pc += blockDim.x) {
                    const int y = pc / N, z = pc % N;
                    const int zb = y * RP + z;           // (0, y, z) in Z1, Z2
                    const cpx<T> e1 = cmul(E1[1][y], E1[2][z]), e2 = cmul(E2[1][y], E2[2][z]);
                    cpx<T> x[N];
#pragma unroll
                    for (int k = 0; k < N; ++k) x[k] = cmul(cmul(E1[0][k], e1), F[pc + k * N * N]);
                    dft<N, +1>(x);
#pragma unroll
                    for (int k = 0; k < N; ++k) Z1[zb + k * N * RP] = x[k];
#pragma unroll
                    for (int k = 0; k < N; ++k) x[k] = cmul(cmul(E2[0][k], e2), G[pc + k * N * N]);
                    dft<N, +1>(x);
#pragma unroll
                    for (int k = 0; k < N; ++k) Z2[zb + k * N * RP] = x[k];
                }
                __syncthreads();
                // B: inverse DFT along y
                pass<T, N, +1, 1, RP>(Z1);
                pass<T, N, +1, 1, RP>(Z2);
                __syncthreads();
                // C: inverse DFT along z, product, forward DFT along z
                for (int pc = threadIdx.x; pc < N * N; pc += blockDim.x) {
                    cpx<T> x[N];
#pragma unroll
                    for (int k = 0; k < N; ++k) x[k] = Z1[pc * RP + k];
                    dft<N, +1>(x);
#pragma unroll
                    for (int k = 0; k < N; ++k) Z1[pc * RP + k] = x[k];
#pragma unroll
                    for (int k = 0; k < N; ++k) x[k] = Z2[pc * RP + k];
                    dft<N, +1>(x);
#pragma unroll
                    for (int k = 0; k < N; ++k) x[k] = cmul(Z1[pc * RP + k], x[k]);
                    dft<N, -1>(x);
#pragma unroll
                    for (int k = 0; k < N; ++k) Z1[pc * RP + k] = x[k];
                }
                __syncthreads();
                // D: forward DFT along y
                pass<T, N, -1, 1, RP>(Z1);
                __syncthreads();
                // E: forward DFT along x, weighted kernel product into G^
                const T w = T(g.rw[r]) * pref;
                const cpx<T>* brs = bq + size_t(rs) * n;
                if constexpr (kTm) {
                    const bool first = q == 0 && rs == 0;   // CTA-uniform
                    tc::tmem_wait_st();
#pragma unroll 1
                    for (int j = 0; j < PPT; ++j) {         // every thread: PPT pencils
                        const int pc = threadIdx.x + j * VssCfg<T, N>::threads;
                        const int zb = (pc / N) * RP + pc % N;
                        cpx<T> x[N];
#pragma unroll
                        for (int k = 0; k < N; ++k) x[k] = Z1[zb + k * N * RP];
                        dft<N, -1>(x);
#pragma unroll
                        for (int c = 0; c < N / 8; ++c) {
                            uint32_t acc[16];
                            const uint32_t col = tsv + uint32_t(j * 2 * N + 16 * c);
                            if (!first) {
                                tc::tmem_ld16_issue(col, acc);
                                tc::tmem_wait();
                            } else {
#pragma unroll
                                for (int e = 0; e < 16; ++e) acc[e] = 0u;
                            }
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const int k = 8 * c + e;
                                const cpx<T> t = cmul(brs[pc + k * N * N], x[k]);
                                acc[2 * e] = __float_as_uint(__uint_as_float(acc[2 * e]) + w * t.x);
                                acc[2 * e + 1] = __float_as_uint(__uint_as_float(acc[2 * e + 1]) + w * t.y);
                            }
                            tc::tmem_st16(col, acc);
                        }
                    }
                } else {
                    for (int pc = threadIdx.x; pc < N * N; pc += blockDim.x) {
                        const int zb = (pc / N) * RP + pc % N;
                        cpx<T> x[N];
#pragma unroll
                        for (int k = 0; k < N; ++k) x[k] = Z1[zb + k * N * RP];
                        dft<N, -1>(x);
#pragma unroll
                        for (int k = 0; k < N; ++k) {
                            const int i = pc + k * N * N;
                            const cpx<T> t = cmul(brs[i], x[k]);
                            Ga[i].x += w * t.x;
                            Ga[i].y += w * t.y;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if constexpr (kTm) {                      // G^: TMEM -> global scratch
            tc::tmem_wait_st();
#pragma unroll 1
            for (int j = 0; j < PPT; ++j) {
                const int pc = threadIdx.x + j * VssCfg<T, N>::threads;
#pragma unroll
                for (int c = 0; c < N / 8; ++c) {
                    uint32_t acc[16];
                    tc::tmem_ld16_issue(tsv + uint32_t(j * 2 * N + 16 * c), acc);
                    tc::tmem_wait();
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        Ga[pc + (8 * c + e) * N * N] =
                            cpx<T>{__uint_as_float(acc[2 * e]), __uint_as_float(acc[2 * e + 1])};
                }
            }
            __syncthreads();
        }
        // back to velocity space: Q_p = Re IFFT(G^) - f_p Re IFFT(L^)
        pass<T, N, +1, 2>(Ga);
        pass<T, N, +1, 2>(La);
        __syncthreads();
        pass<T, N, +1, 1>(Ga);
        pass<T, N, +1, 1>(La);
        __syncthreads();
        pass<T, N, +1, 0>(Ga);
        pass<T, N, +1, 0>(La);
        __syncthreads();
        T* Qp = static_cast<T*>(g.Q[p]) + dof * n;
        for (int i = threadIdx.x; i < n; i += blockDim.x) Qp[i] = Ga[i].x - fp[i] * La[i].x;
        __syncthreads();
    }
    if constexpr (kTm) {
        tc::tmem_wait_st();
        tc::tc_fence_before();
        __syncthreads();
        if (threadIdx.x < 32) {
            tc::tc_fence_after();
            tc::tmem_dealloc(s_tmem, VssCfg<T, N>::tmem_cols);
        }
    }
}

template <typename T, int N>
int vss_launch(const bdgfs_vss_args* a, void* scratch, size_t bytes, cudaStream_t st)
{
    constexpr int n = VssCfg<T, N>::n;
    const size_t per = size_t(6) * n * sizeof(cpx<T>);
    const int64_t nitems = a->ndof * a->nspcs;
    const int64_t ctas = int64_t(bytes / per) < nitems ? int64_t(bytes / per) : nitems;
    if (ctas < 1) return BDGFS_ESCRATCH;
    constexpr size_t sm = VssCfg<T, N>::smem_bytes;
    if constexpr (sm > 0) {
        if (const int rc = smem_optin(reinterpret_cast<const void*>(vss_kernel<T, N>), sm))
            return rc;
    }
    vss_kernel<T, N><<<unsigned(ctas > 65535 ? 65535 : ctas), VssCfg<T, N>::threads, sm, st>>>(
        *a, static_cast<cpx<T>*>(scratch));
    return cuda_status(cudaGetLastError());
}

// FP64 conservation projection of a mixture's Q: per distribution, the
// minimal-norm change of (Q_0 .. Q_{S-1}) that zeroes each species' mass
// sum f cw, the total momentum sum_p m_p c Q_p cw and the total energy
// sum_p m_p |c|^2 Q_p cw: Q_p -= lam_p + m_p (lam_S c + lam_{S+3} |c|^2),
// lam = G^-1 r with r the current constraint sums.
constexpr int VSS_PROJ_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(VSS_PROJ_THREADS) vss_project_kernel(const bdgfs_vss_proj_args a)
{
    __shared__ double red[5 * 4 * (VSS_PROJ_THREADS / 32)];
    const int N = a.Nv, S = a.nspcs, K = S + 4;
    const int64_t n = int64_t(N) * N * N;
    for (int64_t dof = blockIdx.x; dof < a.ndof; dof += gridDim.x) {
        double m[20];
#pragma unroll
        for (int j = 0; j < 20; ++j) m[j] = 0.0;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (p >= S) break;
            const T* Q = static_cast<const T*>(a.Q[p]) + dof * n;
            for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
                const double cx = a.c0[i / (N * N)], cy = a.c0[(i / N) % N], cz = a.c0[i % N];
                const double q = double(Q[i]);
                m[5 * p + 0] += q;
                m[5 * p + 1] += cx * q;
                m[5 * p + 2] += cy * q;
                m[5 * p + 3] += cz * q;
                m[5 * p + 4] += (cx * cx + cy * cy + cz * cz) * q;
            }
        }
        block_sum<20>(m, red);
        // constraint sums r and multipliers lam = G^-1 r (K <= 8)
        double r[8], lam[8];
        for (int k = 0; k < 8; ++k) r[k] = 0.0;
        for (int p = 0; p < S; ++p) {
            r[p] = m[5 * p];
            for (int d = 0; d < 4; ++d) r[S + d] += a.mass[p] * m[5 * p + 1 + d];
        }
        for (int k = 0; k < K; ++k) {
            double v = 0.0;
            for (int l = 0; l < K; ++l) v += a.ginv[k * K + l] * r[l];
            lam[k] = v;
        }
        for (int p = 0; p < S; ++p) {
            T* Q = static_cast<T*>(a.Q[p]) + dof * n;
            const double mp = a.mass[p];
            for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
                const double cx = a.c0[i / (N * N)], cy = a.c0[(i / N) % N], cz = a.c0[i % N];
                const double d = lam[p] + mp * (lam[S] * cx + lam[S + 1] * cy + lam[S + 2] * cz
                                                + lam[S + 3] * (cx * cx + cy * cy + cz * cz));
                Q[i] = T(double(Q[i]) - d);
            }
        }
        __syncthreads();
    }
}

}  // namespace

}  // namespace bdgfs

using namespace bdgfs;

extern "C" int32_t bdgfs_vss_project(const bdgfs_vss_proj_args* a, void* stream)
{
    if (!a || a->nspcs < 1 || a->nspcs > 4 || a->ndof < 0 || a->Nv < 1 || a->Nv > 64 || !a->c0 ||
        !a->mass || !a->ginv)
        return BDGFS_EINVAL;
    for (int p = 0; p < a->nspcs; ++p)
        if (!a->Q[p]) return BDGFS_EINVAL;
    if (a->ndof == 0) return BDGFS_OK;
    const int64_t grid = a->ndof < 148 * 8 ? a->ndof : 148 * 8;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (a->fp64)
        vss_project_kernel<double><<<unsigned(grid), VSS_PROJ_THREADS, 0, st>>>(*a);
    else
        vss_project_kernel<float><<<unsigned(grid), VSS_PROJ_THREADS, 0, st>>>(*a);
    return cuda_status(cudaGetLastError());
}

extern "C" size_t bdgfs_vss_scratch_bytes(int32_t Nv, int32_t fp64, int32_t nctas)
{
    if (Nv < 1 || Nv > 32 || nctas < 1) return 0;
    const size_t n = size_t(Nv) * Nv * Nv;
    return size_t(nctas) * 6 * n * (fp64 ? 16 : 8);
}

extern "C" int32_t bdgfs_vss_collide(const bdgfs_vss_args* a, void* scratch, size_t bytes, void* stream)
{
    if (!a || !scratch || a->nspcs < 1 || a->nspcs > 4 || a->ndof < 0 || a->Nrho < 1 || a->M < 1 ||
        !a->mfrac || !a->prefac || !a->rfac || !a->rw || !a->sz || !a->b || !a->c)
        return BDGFS_EINVAL;
    for (int p = 0; p < a->nspcs; ++p)
        if (!a->f[p] || !a->Q[p]) return BDGFS_EINVAL;
    if (a->ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define VSS_GO(NN)                                                                          \
    if (a->Nv == NN)                                                                        \
        return a->fp64 ? vss_launch<double, NN>(a, scratch, bytes, st)                      \
                       : vss_launch<float, NN>(a, scratch, bytes, st);
    VSS_GO(8)
    VSS_GO(12)
    VSS_GO(16)
    VSS_GO(24)
    VSS_GO(32)
#undef VSS_GO
    return BDGFS_EUNSUPPORTED;
}
