// Device-side pieces of the surrogate/spectral hybrid collision step.
//
// indicator: per distribution, FP64 moments (rho, u, T), the Maxwellian
//   M[f] = rho/(pi T)^{3/2} exp(-|c-u|^2/T) (the non-dimensional form of
//   frfs/solvers/dgfs/initcond.py:55-58) and eps = |f - M[f]|_2 / |f|_2;
//   eps < threshold -> surrogate list, else spectral list; a seeded fraction
//   of the surrogate cells is also put on the spectral list (re-check).
//   Lists are filled with atomics (order arbitrary, results per cell are
//   independent of it); counts stay on the device, so the whole step can be
//   captured in a CUDA graph.
// project: FP64 minimal-norm conservation projection of compact rows,
//   Q <- Q - phi^T G^{-1} (phi Q), phi = {1, c, |c|^2}.
// scatter: compact surrogate rows -> state-indexed Q, except on re-checked
//   cells, which keep the spectral result; there the surrogate's error is
//   accumulated (FP64 sums of |Qs - Qspec|^2 and |Qspec|^2).
#include <cuda_bf16.h>

#include "common.cuh"
#include "rows.cuh"

namespace bdgfs {

__device__ __forceinline__ uint32_t mix32(uint64_t x)
{
    // splitmix64 finaliser (Steele, Lea, Flood 2014)
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    x ^= x >> 31;
    return uint32_t(x >> 32);
}

// NVC > 0: the grid size at compile time (h.Nv == NVC)
template <typename T, int VEC, int NVC = 0>
__global__ void __launch_bounds__(256, NVC > 0 ? 5 : 0) indicator_kernel(const bdgfs_hybrid_args h,
                                                                         const T* __restrict__ f)
{
    __shared__ double red[8 * 8];
    __shared__ double cs[kMaxNv], ex[3][kMaxNv];
    __shared__ int64_t s_pos;
    const int64_t dof = blockIdx.x;
    const int Nv = NVC > 0 ? NVC : h.Nv;
    const int n = Nv * Nv * Nv;
    const T* fd = f + dof * int64_t(n);
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = h.c0[i];
    __syncthreads();
    double m[5] = {0, 0, 0, 0, 0};
    row_moments<T, VEC, NVC>(fd, n, Nv, cs, m);
    block_sum<5>(m, red);
    const double rho = m[0] * h.cw;
    const double ux = m[1] / m[0], uy = m[2] / m[0], uz = m[3] / m[0];
    const double Tt = (m[4] / m[0] - (ux * ux + uy * uy + uz * uz)) * (2.0 / 3.0);
    const bool ok = rho > 0.0 && Tt > 0.0;
    // separable Maxwellian: M = a * ex[0][ix] * ex[1][iy] * ex[2][iz]
    const double a = ok ? rho / pow(3.141592653589793 * Tt, 1.5) : 0.0;
    if (ok) {
        const double it = 1.0 / Tt;
        for (int i = threadIdx.x; i < 3 * Nv; i += blockDim.x) {
            const int d = i / Nv, j = i - d * Nv;
            const double c = cs[j] - (d == 0 ? ux : d == 1 ? uy : uz);
            ex[d][j] = exp(-c * c * it);
        }
    }
    __syncthreads();
    double e[2] = {0, 0};
    if (ok) {
#pragma unroll 2
        for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
            Chunk<T, VEC> c;
            c.load(fd + v);
            uint32_t ix, iy, iz;
            vsplit<NVC>(uint32_t(v), uint32_t(Nv), ix, iy, iz);
            const double axy = a * ex[0][ix] * ex[1][iy];
#pragma unroll
            for (int j = 0; j < VEC; ++j) {
                const double x = double(c.v[j]);
                const double d = x - axy * ex[2][iz + j];
                e[0] += d * d;
                e[1] += x * x;
            }
        }
    }
    block_sum<2>(e, red);
    if (threadIdx.x == 0) {
        const double eps = (ok && e[1] > 0.0) ? sqrt(e[0] / e[1]) : 1e30;
        s_pos = -1;
        if (h.eps) h.eps[dof] = float(eps);
        const bool sur = eps < double(h.threshold);
        const uint64_t seed = h.seed_dev ? *h.seed_dev : h.seed;
        const bool re = sur && (double(mix32(seed * 0x100000001B3ull + uint64_t(dof))) <
                                double(h.recheck) * 4294967296.0);
        if (h.flag) h.flag[dof] = uint8_t(sur ? (re ? 2 : 1) : 0);
        if (sur) {
            const int64_t p = int64_t(atomicAdd(reinterpret_cast<unsigned long long*>(h.counts), 1ull));
            h.sur_idx[p] = int32_t(dof);
            h.sur_inv_rho[p] = float(1.0 / rho);
            h.sur_rho2[p] = float(rho * rho);
            s_pos = p;
            if (h.sur_s) h.sur_s[p] = float(sqrt(e[0]) / rho);
            if (h.sur_uT) {
                h.sur_uT[4 * p + 0] = float(ux);
                h.sur_uT[4 * p + 1] = float(uy);
                h.sur_uT[4 * p + 2] = float(uz);
                h.sur_uT[4 * p + 3] = float(Tt);
            }
            if (h.feat) {
                __nv_bfloat16* fr = static_cast<__nv_bfloat16*>(h.feat) + p * h.feat_ld;
                fr[0] = __float2bfloat16_rn(h.center ? 0.f : float(ux));
                fr[1] = __float2bfloat16_rn(h.center ? 0.f : float(uy));
                fr[2] = __float2bfloat16_rn(h.center ? 0.f : float(uz));
                fr[3] = __float2bfloat16_rn(float(Tt - 1.0));
            }
        }
        if (!sur || re) {
            const int64_t p = int64_t(atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 1), 1ull));
            h.spec_idx[p] = int32_t(dof);
        }
        if (re) atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 2), 1ull);
    }
    __syncthreads();
    const int64_t p = s_pos;
    if (p >= 0 && h.dev_rows) {
        // (f - M[f]) / |f - M[f]|_2: direction of the deviation from the
        // local Maxwellian (its size, at unit density, is sur_s)
        __nv_bfloat16* out = static_cast<__nv_bfloat16*>(h.dev_rows) + p * int64_t(n);
        const double inv = (ok && e[0] > 0.0) ? 1.0 / sqrt(e[0]) : 0.0;
#pragma unroll 2
        for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
            Chunk<T, VEC> c;
            c.load(fd + v);
            uint32_t ix, iy, iz;
            vsplit<NVC>(uint32_t(v), uint32_t(Nv), ix, iy, iz);
            const double axy = a * ex[0][ix] * ex[1][iy];
            float d[VEC];
#pragma unroll
            for (int j = 0; j < VEC; ++j)
                d[j] = ok ? float((double(c.v[j]) - axy * ex[2][iz + j]) * inv) : 0.f;
            if constexpr (VEC == 4) {
                __align__(8) __nv_bfloat162 hv[2] = {__floats2bfloat162_rn(d[0], d[1]),
                                                     __floats2bfloat162_rn(d[2], d[3])};
                *reinterpret_cast<uint2*>(out + v) = *reinterpret_cast<const uint2*>(hv);
            } else {
                out[v] = __float2bfloat16_rn(d[0]);
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) project_kernel(const bdgfs_hybrid_args h, T* Qc)
{
    __shared__ double red[8 * 8];
    const int64_t row = blockIdx.x;
    const int64_t cnt = h.counts ? *h.counts : h.ndof;
    if (row >= cnt) return;
    const int Nv = h.Nv;
    const int64_t n = int64_t(Nv) * Nv * Nv;
    T* q = Qc + row * n;
    const double* c0 = h.c0;
    double m[5] = {0, 0, 0, 0, 0};
    for (int v = threadIdx.x; v < int(n); v += blockDim.x) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        const double cx = c0[ix], cy = c0[iy], cz = c0[iz];
        const double x = double(q[v]);
        m[0] += x;
        m[1] += cx * x;
        m[2] += cy * x;
        m[3] += cz * x;
        m[4] += (cx * cx + cy * cy + cz * cz) * x;
    }
    block_sum<5>(m, red);
    double lam[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j) s += h.ginv[i * 5 + j] * m[j];
        lam[i] = s;
    }
    for (int v = threadIdx.x; v < int(n); v += blockDim.x) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        const double cx = c0[ix], cy = c0[iy], cz = c0[iz];
        const double c2 = cx * cx + cy * cy + cz * cz;
        q[v] = T(double(q[v]) - (lam[0] + lam[1] * cx + lam[2] * cy + lam[3] * cz + lam[4] * c2));
    }
}

template <typename T>
__global__ void __launch_bounds__(256) scatter_kernel(const bdgfs_hybrid_args h, const T* __restrict__ Qc,
                                                      T* __restrict__ Q)
{
    __shared__ double red[2 * 8];
    const int64_t row = blockIdx.x;
    if (row == 0 && threadIdx.x == 0 && h.seed_dev) *h.seed_dev += 1;   // next step's sample
    const int64_t cnt = *h.counts;
    if (row >= cnt) return;
    const int64_t n = int64_t(h.Nv) * h.Nv * h.Nv;
    const int64_t dof = h.sur_idx[row];
    const T* src = Qc + row * n;
    T* dst = Q + dof * n;
    if (h.flag[dof] != 2) {
        int bad = 0;
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
            const T x = src[v];
            bad |= !isfinite(x);
            dst[v] = x;
        }
        // a non-finite row goes to the fallback list (the spectral launch
        // that follows overwrites it)
        if (__syncthreads_or(bad) && h.fb_idx && threadIdx.x == 0)
            h.fb_idx[atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 3), 1ull)] = int32_t(dof);
        return;
    }
    double e[2] = {0, 0};
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
        const double d = double(src[v]) - double(dst[v]);
        e[0] += d * d;
        e[1] += double(dst[v]) * double(dst[v]);
    }
    block_sum<2>(e, red);
    if (!isfinite(e[0])) return;                       // the cell keeps its spectral Q
    if (threadIdx.x == 0 && h.recheck_err) {
        atomicAdd(h.recheck_err, e[0]);
        atomicAdd(h.recheck_err + 1, e[1]);
    }
}

// Conservation projection of compact row `row` fused with its scatter:
// the corrected values go straight to Q[sur_idx[row]] (or, on a re-checked
// cell, are compared with the spectral values already there).
template <typename T, int VEC>
__global__ void __launch_bounds__(256) project_scatter_kernel(const bdgfs_hybrid_args h,
                                                              const T* __restrict__ Qc, T* __restrict__ Q)
{
    __shared__ double red[5 * 8];
    __shared__ double cs[kMaxNv];
    const int64_t row = blockIdx.x;
    if (row == 0 && threadIdx.x == 0 && h.seed_dev) *h.seed_dev += 1;   // next step's sample
    const int64_t cnt = *h.counts;
    if (row >= cnt) return;
    const int Nv = h.Nv;
    const int n = Nv * Nv * Nv;
    const T* src = Qc + row * int64_t(n);
    const int64_t dof = h.sur_idx[row];
    T* dst = Q + dof * int64_t(n);
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = h.c0[i];
    __syncthreads();
    double m[5] = {0, 0, 0, 0, 0};
    row_moments<T, VEC>(src, n, Nv, cs, m);
    block_sum<5>(m, red);
    const bool re = h.flag[dof] == 2;
    // a non-finite row (NaN / Inf anywhere makes its moments non-finite;
    // uniform per block): nothing is written; a surrogate cell goes to the
    // fallback list, a re-checked cell keeps its spectral Q
    if (!isfinite(m[0] + m[1] + m[2] + m[3] + m[4])) {
        if (!re && h.fb_idx && threadIdx.x == 0)
            h.fb_idx[atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 3), 1ull)] = int32_t(dof);
        return;
    }
    double lam[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j) t += h.ginv[i * 5 + j] * m[j];
        lam[i] = t;
    }
    double e[2] = {0, 0};
#pragma unroll 2
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        Chunk<T, VEC> c;
        c.load(src + v);
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        const double cx = cs[ix], cy = cs[iy];
        const double lxy = lam[0] + lam[1] * cx + lam[2] * cy + lam[4] * (cx * cx + cy * cy);
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            const double cz = cs[iz + j];
            c.v[j] = T(double(c.v[j]) - (lxy + lam[3] * cz + lam[4] * cz * cz));
        }
        if (!re) {
            c.store(dst + v);
        } else {
            Chunk<T, VEC> sp;
            sp.load(dst + v);
#pragma unroll
            for (int j = 0; j < VEC; ++j) {
                const double d = double(c.v[j]) - double(sp.v[j]);
                e[0] += d * d;
                e[1] += double(sp.v[j]) * double(sp.v[j]);
            }
        }
    }
    if (!re) return;                                   // uniform per block
    block_sum<2>(e, red);
    if (threadIdx.x == 0 && h.recheck_err) {
        atomicAdd(h.recheck_err, e[0]);
        atomicAdd(h.recheck_err + 1, e[1]);
    }
}

template <typename T>
__device__ __forceinline__ float to_f32(T x) { return float(x); }
template <>
__device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 x) { return __bfloat162float(x); }
template <typename T>
__device__ __forceinline__ T from_f32(float x) { return T(x); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_f32<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }

// Spectral shift (bdgfs_hybrid_shift).  Along one axis the shift by a is
// the circulant g_i = sum_j w[(i - j) mod N] f_j with
//   w[k] = (1/N) sum_{m=-N/2}^{N/2-1} cos(2 pi m (k + a/h) / N)
// (the real part of the trigonometric interpolant on the periodic grid);
// the three axes are applied in turn on a row staged in shared memory as a
// padded cube, element (x, y, z) at (x*N + y)*(N + 1) + z (the three pencil
// directions are then free of bank conflicts).  u: the shift per axis,
// sign * u[d] / h in grid units; wt: 3N floats.  Ends with a barrier.
template <int N>
__device__ __forceinline__ int cube_at(int v)
{
    const int xy = v / N;
    return xy * (N + 1) + (v - xy * N);
}

template <int N>
__device__ void cube_shift(float* cube, float* wt, const float* u, double sign, double hg)
{
    constexpr int S = N + 1;
    for (int i = threadIdx.x; i < 3 * N; i += blockDim.x) {
        const int d = i / N, k = i - d * N;
        const double a = sign * double(u[d]) / hg;
        double w = 0.0;
        for (int m = -N / 2; m < N / 2; ++m) w += cospi(2.0 * double(m) * (double(k) + a) / double(N));
        wt[i] = float(w / double(N));
    }
    __syncthreads();
#pragma unroll 1
    for (int d = 2; d >= 0; --d) {                  // z, y, x
        float w[N];
#pragma unroll
        for (int k = 0; k < N; ++k) w[k] = wt[d * N + k];
        for (int p = threadIdx.x; p < N * N; p += blockDim.x) {
            const int p0 = p / N, p1 = p - p0 * N;
            int base, stride;
            if (d == 2) { base = p * S; stride = 1; }                    // (x, y)
            else if (d == 1) { base = p0 * N * S + p1; stride = S; }     // (x, z)
            else { base = p0 * S + p1; stride = N * S; }                 // (y, z)
            float v[N];
#pragma unroll
            for (int j = 0; j < N; ++j) v[j] = cube[base + j * stride];
#pragma unroll
            for (int i = 0; i < N; ++i) {
                float acc = 0.f;
#pragma unroll
                for (int j = 0; j < N; ++j) acc = fmaf(w[(i - j + N) % N], v[j], acc);
                cube[base + i * stride] = acc;
            }
        }
        __syncthreads();
    }
}

template <int N>
constexpr size_t cube_smem_bytes()
{
    return sizeof(float) * (size_t(N) * N * (N + 1) + 3 * N);
}

// Grid-stride over the rows below the device count.
template <int N, typename TI, typename TO>
__global__ void __launch_bounds__(256) shift_kernel(const bdgfs_hybrid_args h, const TI* in, TO* out,
                                                    float sign)
{
    extern __shared__ float sh[];
    constexpr int n = N * N * N;
    float* cube = sh;
    float* wt = sh + N * N * (N + 1);
    const int64_t cnt = *h.counts;
    const double hg = h.c0[1] - h.c0[0];
    for (int64_t row = blockIdx.x; row < cnt; row += gridDim.x) {
        const TI* src = in + row * int64_t(n);
        TO* dst = out + row * int64_t(n);
        for (int v = threadIdx.x; v < n; v += blockDim.x) cube[cube_at<N>(v)] = to_f32(src[v]);
        cube_shift<N>(cube, wt, h.sur_uT + 4 * row, double(sign), hg);
        for (int v = threadIdx.x; v < n; v += blockDim.x) dst[v] = from_f32<TO>(cube[cube_at<N>(v)]);
        __syncthreads();                             // cube and wt reused by the next row
    }
}

// Indicator with the row staged once in shared memory (FP32 state): the
// moments, the Maxwellian deviation and the deviation row are computed
// from shared memory, so f is read from HBM once; with h.center the
// deviation row is also re-centred at zero velocity (cube_shift by +u)
// before its bf16 copy is written.  Same lists, counts and per-row outputs
// as indicator_kernel.
template <int N, bool CENTER>
__global__ void __launch_bounds__(256) indicator_smem_kernel(const bdgfs_hybrid_args h,
                                                             const float* __restrict__ f)
{
    extern __shared__ float sh[];
    constexpr int n = N * N * N;
    float* cube = sh;
    float* wt = sh + N * N * (N + 1);
    __shared__ double red[8 * 8];
    __shared__ double cs[N], ex[3][N];
    __shared__ int64_t s_pos;
    __shared__ float s_u[3];
    const int64_t dof = blockIdx.x;
    const float* fd = f + dof * int64_t(n);
    for (int i = threadIdx.x; i < N; i += blockDim.x) cs[i] = h.c0[i];
    for (int v = 4 * threadIdx.x; v < n; v += 4 * blockDim.x) {       // 16-byte loads
        const float4 x = *reinterpret_cast<const float4*>(fd + v);
        float* c = cube + cube_at<N>(v);                               // N % 4 == 0: one row
        c[0] = x.x; c[1] = x.y; c[2] = x.z; c[3] = x.w;
    }
    __syncthreads();
    // every pass walks chunks of 4 consecutive z (one index split per chunk)
    constexpr int NC = n / 4, NZ = N / 4;
    double m[5] = {0, 0, 0, 0, 0};
    for (int c = threadIdx.x; c < NC; c += blockDim.x) {
        const int xy = c / NZ, z0 = 4 * (c - xy * NZ), ix = xy / N, iy = xy - ix * N;
        const float* q = cube + xy * (N + 1) + z0;
        const double cx = cs[ix], cy = cs[iy], b = cx * cx + cy * cy;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double x = double(q[j]), cz = cs[z0 + j];
            m[0] += x;
            m[1] += cx * x;
            m[2] += cy * x;
            m[3] += cz * x;
            m[4] += (b + cz * cz) * x;
        }
    }
    block_sum<5>(m, red);
    const double rho = m[0] * h.cw;
    const double ux = m[1] / m[0], uy = m[2] / m[0], uz = m[3] / m[0];
    const double Tt = (m[4] / m[0] - (ux * ux + uy * uy + uz * uz)) * (2.0 / 3.0);
    const bool ok = rho > 0.0 && Tt > 0.0;
    const double a = ok ? rho / pow(3.141592653589793 * Tt, 1.5) : 0.0;
    if (ok) {
        const double it = 1.0 / Tt;
        for (int i = threadIdx.x; i < 3 * N; i += blockDim.x) {
            const int d = i / N, j = i - d * N;
            const double c = cs[j] - (d == 0 ? ux : d == 1 ? uy : uz);
            ex[d][j] = exp(-c * c * it);
        }
    }
    __syncthreads();
    double e[2] = {0, 0};
    if (ok) {
        for (int c = threadIdx.x; c < NC; c += blockDim.x) {
            const int xy = c / NZ, z0 = 4 * (c - xy * NZ), ix = xy / N, iy = xy - ix * N;
            const float* q = cube + xy * (N + 1) + z0;
            const double axy = a * ex[0][ix] * ex[1][iy];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double x = double(q[j]);
                const double d = x - axy * ex[2][z0 + j];
                e[0] += d * d;
                e[1] += x * x;
            }
        }
    }
    block_sum<2>(e, red);
    if (threadIdx.x == 0) {
        const double eps = (ok && e[1] > 0.0) ? sqrt(e[0] / e[1]) : 1e30;
        s_pos = -1;
        if (h.eps) h.eps[dof] = float(eps);
        const bool sur = eps < double(h.threshold);
        const uint64_t seed = h.seed_dev ? *h.seed_dev : h.seed;
        const bool re = sur && (double(mix32(seed * 0x100000001B3ull + uint64_t(dof))) <
                                double(h.recheck) * 4294967296.0);
        if (h.flag) h.flag[dof] = uint8_t(sur ? (re ? 2 : 1) : 0);
        if (sur) {
            const int64_t p = int64_t(atomicAdd(reinterpret_cast<unsigned long long*>(h.counts), 1ull));
            h.sur_idx[p] = int32_t(dof);
            h.sur_inv_rho[p] = float(1.0 / rho);
            h.sur_rho2[p] = float(rho * rho);
            s_pos = p;
            if (h.sur_s) h.sur_s[p] = float(sqrt(e[0]) / rho);
            if (h.sur_uT) {
                h.sur_uT[4 * p + 0] = float(ux);
                h.sur_uT[4 * p + 1] = float(uy);
                h.sur_uT[4 * p + 2] = float(uz);
                h.sur_uT[4 * p + 3] = float(Tt);
            }
            if (h.feat) {
                __nv_bfloat16* fr = static_cast<__nv_bfloat16*>(h.feat) + p * h.feat_ld;
                fr[0] = __float2bfloat16_rn(h.center ? 0.f : float(ux));
                fr[1] = __float2bfloat16_rn(h.center ? 0.f : float(uy));
                fr[2] = __float2bfloat16_rn(h.center ? 0.f : float(uz));
                fr[3] = __float2bfloat16_rn(float(Tt - 1.0));
            }
            s_u[0] = float(ux);
            s_u[1] = float(uy);
            s_u[2] = float(uz);
        }
        if (!sur || re) {
            const int64_t p = int64_t(atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 1), 1ull));
            h.spec_idx[p] = int32_t(dof);
        }
        if (re) atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 2), 1ull);
    }
    __syncthreads();
    const int64_t p = s_pos;
    if (p < 0 || !h.dev_rows) return;                  // uniform per block
    const double inv = (ok && e[0] > 0.0) ? 1.0 / sqrt(e[0]) : 0.0;
    for (int c = threadIdx.x; c < NC; c += blockDim.x) {
        const int xy = c / NZ, z0 = 4 * (c - xy * NZ), ix = xy / N, iy = xy - ix * N;
        float* q = cube + xy * (N + 1) + z0;
        const double axy = a * ex[0][ix] * ex[1][iy];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            q[j] = ok ? float((double(q[j]) - axy * ex[2][z0 + j]) * inv) : 0.f;
    }
    __syncthreads();
    if constexpr (CENTER) cube_shift<N>(cube, wt, s_u, 1.0, cs[1] - cs[0]);
    __nv_bfloat16* out = static_cast<__nv_bfloat16*>(h.dev_rows) + p * int64_t(n);
    for (int v = 4 * threadIdx.x; v < n; v += 4 * blockDim.x) {
        const float* c = cube + cube_at<N>(v);
        __align__(8) __nv_bfloat162 hv[2] = {__floats2bfloat162_rn(c[0], c[1]),
                                             __floats2bfloat162_rn(c[2], c[3])};
        *reinterpret_cast<uint2*>(out + v) = *reinterpret_cast<const uint2*>(hv);
    }
}

// project_scatter with each compact row staged once in shared memory
// (FP32; Qc read from HBM once); SHIFT (centred surrogate): the row is first
// moved back to its cell's drift (cube_shift by -u).  Then projected in
// FP64 and scattered exactly as project_scatter_kernel does.  Qc is left
// unchanged.
template <int N, bool SHIFT>
__global__ void __launch_bounds__(256) shift_project_scatter_kernel(const bdgfs_hybrid_args h,
                                                                    const float* __restrict__ Qc,
                                                                    float* __restrict__ Q)
{
    extern __shared__ float sh[];
    constexpr int n = N * N * N;
    float* cube = sh;
    float* wt = sh + N * N * (N + 1);
    __shared__ double red[5 * 8];
    __shared__ double cs[N];
    const int64_t row = blockIdx.x;
    if (row == 0 && threadIdx.x == 0 && h.seed_dev) *h.seed_dev += 1;   // next step's sample
    const int64_t cnt = *h.counts;
    if (row >= cnt) return;
    const float* src = Qc + row * int64_t(n);
    const int64_t dof = h.sur_idx[row];
    float* dst = Q + dof * int64_t(n);
    for (int i = threadIdx.x; i < N; i += blockDim.x) cs[i] = h.c0[i];
    for (int v = 4 * threadIdx.x; v < n; v += 4 * blockDim.x) {
        const float4 x = *reinterpret_cast<const float4*>(src + v);
        float* c = cube + cube_at<N>(v);
        c[0] = x.x; c[1] = x.y; c[2] = x.z; c[3] = x.w;
    }
    __syncthreads();
    if constexpr (SHIFT) cube_shift<N>(cube, wt, h.sur_uT + 4 * row, -1.0, cs[1] - cs[0]);
    constexpr int NC = n / 4, NZ = N / 4;
    double m[5] = {0, 0, 0, 0, 0};
    for (int c = threadIdx.x; c < NC; c += blockDim.x) {
        const int xy = c / NZ, z0 = 4 * (c - xy * NZ), ix = xy / N, iy = xy - ix * N;
        const float* q = cube + xy * (N + 1) + z0;
        const double cx = cs[ix], cy = cs[iy], b = cx * cx + cy * cy;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double x = double(q[j]), cz = cs[z0 + j];
            m[0] += x;
            m[1] += cx * x;
            m[2] += cy * x;
            m[3] += cz * x;
            m[4] += (b + cz * cz) * x;
        }
    }
    block_sum<5>(m, red);
    const bool re = h.flag[dof] == 2;
    if (!isfinite(m[0] + m[1] + m[2] + m[3] + m[4])) {
        if (!re && h.fb_idx && threadIdx.x == 0)
            h.fb_idx[atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 3), 1ull)] = int32_t(dof);
        return;
    }
    double lam[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j) t += h.ginv[i * 5 + j] * m[j];
        lam[i] = t;
    }
    double e[2] = {0, 0};
    for (int v = 4 * threadIdx.x; v < n; v += 4 * blockDim.x) {
        const int xy = v / N, iz = v - xy * N, ix = xy / N, iy = xy - ix * N;
        const double cx = cs[ix], cy = cs[iy];
        const double lxy = lam[0] + lam[1] * cx + lam[2] * cy + lam[4] * (cx * cx + cy * cy);
        const float* c = cube + xy * (N + 1) + iz;
        float o[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double cz = cs[iz + j];
            o[j] = float(double(c[j]) - (lxy + lam[3] * cz + lam[4] * cz * cz));
        }
        if (!re) {
            *reinterpret_cast<float4*>(dst + v) = make_float4(o[0], o[1], o[2], o[3]);
        } else {
            const float4 sp = *reinterpret_cast<const float4*>(dst + v);
            const float spv[4] = {sp.x, sp.y, sp.z, sp.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const double d = double(o[j]) - double(spv[j]);
                e[0] += d * d;
                e[1] += double(spv[j]) * double(spv[j]);
            }
        }
    }
    if (!re) return;                                   // uniform per block
    block_sum<2>(e, red);
    if (threadIdx.x == 0 && h.recheck_err) {
        atomicAdd(h.recheck_err, e[0]);
        atomicAdd(h.recheck_err + 1, e[1]);
    }
}

__global__ void __launch_bounds__(256) tfeat_kernel(const bdgfs_hybrid_args h, __nv_bfloat16* xc, int64_t ld,
                                                    int64_t x0, int64_t x1, int64_t k, int k2, int64_t xq)
{
    __shared__ float xs[64];
    const int64_t cnt = *h.counts;
    const int nq = k2 * (k2 + 1) / 2;
    for (int64_t row = blockIdx.x; row < cnt; row += gridDim.x) {
        const float t = h.sur_uT[4 * row + 3] - 1.f;
        __nv_bfloat16* r = xc + row * ld;
        for (int64_t j = threadIdx.x; j < k; j += blockDim.x) {
            const float x = __bfloat162float(r[x0 + j]);
            r[x1 + j] = __float2bfloat16_rn(t * x);
            r[x1 + k + j] = __float2bfloat16_rn(t * t * x);
            if (j < k2) xs[j] = x;
        }
        __syncthreads();
        // products x_i x_j, i <= j < k2, row-major over the upper triangle
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            int i = 0, rem = q;
            while (rem >= k2 - i) { rem -= k2 - i; ++i; }
            r[xq + q] = __float2bfloat16_rn(xs[i] * xs[i + rem]);
        }
        __syncthreads();
    }
}

// out[m][i*k + j] = s_m^i Y[m][i*k + j]
__global__ void __launch_bounds__(128) heads_kernel(const bdgfs_hybrid_args h, const float* __restrict__ Y,
                                                    int64_t ldy, int64_t k, int nheads,
                                                    __nv_bfloat16* __restrict__ out, int64_t ldo)
{
    const int64_t row = blockIdx.x;
    if (row >= *h.counts) return;
    const float s = h.sur_s[row];
    const float* y = Y + row * ldy;
    float p = 1.f;
    for (int i = 0; i < nheads; ++i) {
        for (int64_t j = threadIdx.x; j < k; j += blockDim.x)
            out[row * ldo + i * k + j] = __float2bfloat16_rn(p * y[i * k + j]);
        p *= s;
    }
}

// Split-bf16 heads: v = s_m^i Y[m][i*k + j] as hi = bf16(v), lo = bf16(v - hi),
// written at columns c, K + c and 2K + c (K = nheads * k, c = i*k + j) as
// [hi | hi | lo], to meet an output basis stored as [B_hi | B_lo | B_hi]:
// one GEMM then sums hi*B_hi + hi*B_lo + lo*B_hi (the bf16 x bf16 terms of
// an FP32-accurate product; lo*B_lo is below FP32 rounding).
__global__ void __launch_bounds__(128) heads_split_kernel(const bdgfs_hybrid_args h,
                                                          const float* __restrict__ Y, int64_t ldy,
                                                          int64_t k, int nheads,
                                                          __nv_bfloat16* __restrict__ out, int64_t ldo)
{
    const int64_t row = blockIdx.x;
    if (row >= *h.counts) return;
    const float s = h.sur_s[row];
    const float* y = Y + row * ldy;
    const int64_t K = int64_t(nheads) * k;
    __nv_bfloat16* o = out + row * ldo;
    float p = 1.f;
    for (int i = 0; i < nheads; ++i) {
        for (int64_t j = threadIdx.x; j < k; j += blockDim.x) {
            const float v = p * y[i * k + j];
            const __nv_bfloat16 hi = __float2bfloat16_rn(v);
            const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
            o[i * k + j] = hi;
            o[K + i * k + j] = hi;
            o[2 * K + i * k + j] = lo;
        }
        p *= s;
    }
}

}  // namespace bdgfs

using namespace bdgfs;

static int check_h(const bdgfs_hybrid_args* h)
{
    if (!h || h->ndof < 0 || h->Nv < 1 || h->Nv > kMaxNv || !h->c0) return BDGFS_EINVAL;
    if (h->ndof > 2147483647LL) return BDGFS_EINVAL;
    return BDGFS_OK;
}

static int shift_any(const bdgfs_hybrid_args* h, const void* in, int in_bf16, void* out, int out_bf16,
                     float sign, cudaStream_t st);

static bool cube_grid(int Nv)
{
    return Nv == 8 || Nv == 12 || Nv == 16 || Nv == 24 || Nv == 32;
}

template <int N, bool CENTER>
static int indicator_smem_launch(const bdgfs_hybrid_args* h, const float* f, cudaStream_t st)
{
    constexpr size_t smem = cube_smem_bytes<N>();
    if (const int rc = smem_optin(reinterpret_cast<const void*>(indicator_smem_kernel<N, CENTER>), smem))
        return rc;
    indicator_smem_kernel<N, CENTER><<<unsigned(h->ndof), 256, smem, st>>>(*h, f);
    return cuda_status(cudaGetLastError());
}

template <bool CENTER>
static int indicator_smem_dispatch(const bdgfs_hybrid_args* h, const float* f, cudaStream_t st)
{
    switch (h->Nv) {
    case 8: return indicator_smem_launch<8, CENTER>(h, f, st);
    case 12: return indicator_smem_launch<12, CENTER>(h, f, st);
    case 16: return indicator_smem_launch<16, CENTER>(h, f, st);
    case 24: return indicator_smem_launch<24, CENTER>(h, f, st);
    case 32: return indicator_smem_launch<32, CENTER>(h, f, st);
    default: return BDGFS_EUNSUPPORTED;
    }
}

template <int N, bool SHIFT>
static int shift_project_scatter_launch(const bdgfs_hybrid_args* h, const float* Qc, float* Q, cudaStream_t st)
{
    constexpr size_t smem = cube_smem_bytes<N>();
    if (const int rc = smem_optin(reinterpret_cast<const void*>(shift_project_scatter_kernel<N, SHIFT>), smem))
        return rc;
    shift_project_scatter_kernel<N, SHIFT><<<unsigned(h->ndof), 256, smem, st>>>(*h, Qc, Q);
    return cuda_status(cudaGetLastError());
}

template <bool SHIFT>
static int staged_project_scatter(const bdgfs_hybrid_args* h, const float* q, float* o, cudaStream_t st)
{
    switch (h->Nv) {
    case 8: return shift_project_scatter_launch<8, SHIFT>(h, q, o, st);
    case 12: return shift_project_scatter_launch<12, SHIFT>(h, q, o, st);
    case 16: return shift_project_scatter_launch<16, SHIFT>(h, q, o, st);
    case 24: return shift_project_scatter_launch<24, SHIFT>(h, q, o, st);
    default: return shift_project_scatter_launch<32, SHIFT>(h, q, o, st);
    }
}

extern "C" int32_t bdgfs_hybrid_classify(const bdgfs_hybrid_args* h, const void* f, void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!f || !h->counts || !h->sur_idx || !h->spec_idx || !h->sur_inv_rho || !h->sur_rho2 ||
        !h->flag)
        return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(h->counts, 0, (h->fb_idx ? 4 : 3) * sizeof(int64_t), st) != cudaSuccess)
        return BDGFS_ECUDA;
    if (h->recheck_err && cudaMemsetAsync(h->recheck_err, 0, 2 * sizeof(double), st) != cudaSuccess)
        return BDGFS_ECUDA;
    if (h->ndof == 0) return BDGFS_OK;
    const bool v4 = h->Nv % 4 == 0 && (reinterpret_cast<uintptr_t>(f) & 15u) == 0 &&
                    (!h->dev_rows || (reinterpret_cast<uintptr_t>(h->dev_rows) & 7u) == 0);
    if (h->center && (!h->sur_uT || !h->dev_rows)) return BDGFS_EINVAL;
    if (h->center && !h->fp64 && v4 && cube_grid(h->Nv)) {
        // the row staged once in shared memory and the deviation row
        // re-centred in the same launch (without centring the streaming
        // kernel below is faster: more CTAs per SM keep more loads in flight)
        return indicator_smem_dispatch<true>(h, static_cast<const float*>(f), st);
    }
    if (h->fp64) {
        if (v4)
            indicator_kernel<double, 4><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const double*>(f));
        else
            indicator_kernel<double, 1><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const double*>(f));
    } else {
        if (v4 && h->Nv == 24)
            indicator_kernel<float, 4, 24><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(f));
        else if (v4)
            indicator_kernel<float, 4><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(f));
        else
            indicator_kernel<float, 1><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(f));
    }
    if (cudaGetLastError() != cudaSuccess) return BDGFS_ECUDA;
    if (h->center) return shift_any(h, h->dev_rows, 1, h->dev_rows, 1, 1.f, st);
    return BDGFS_OK;
}

extern "C" int32_t bdgfs_hybrid_project(const bdgfs_hybrid_args* h, void* Qc, void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!Qc || !h->ginv) return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (h->fp64)
        project_kernel<double><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<double*>(Qc));
    else
        project_kernel<float><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<float*>(Qc));
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_hybrid_scatter(const bdgfs_hybrid_args* h, const void* Qc, void* Q,
                                        void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!Qc || !Q || !h->counts || !h->sur_idx || !h->flag) return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (h->center) {                   // back to each cell's drift, in place
        if (!h->sur_uT) return BDGFS_EINVAL;
        if (const int r = shift_any(h, Qc, 0, const_cast<void*>(Qc), 0, -1.f, st)) return r;
    }
    if (h->fp64)
        scatter_kernel<double><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const double*>(Qc),
                                                                  static_cast<double*>(Q));
    else
        scatter_kernel<float><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(Qc),
                                                                 static_cast<float*>(Q));
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_hybrid_project_scatter(const bdgfs_hybrid_args* h, const void* Qc, void* Q,
                                                void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!Qc || !Q || !h->counts || !h->sur_idx || !h->flag || !h->ginv) return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = h->Nv % 4 == 0 && (reinterpret_cast<uintptr_t>(Qc) & 15u) == 0 &&
                    (reinterpret_cast<uintptr_t>(Q) & 15u) == 0;
    if (h->center) {
        if (!h->sur_uT) return BDGFS_EINVAL;
        if (!h->fp64 && v4 && cube_grid(h->Nv))       // shift back, project, scatter: one pass
            return staged_project_scatter<true>(h, static_cast<const float*>(Qc), static_cast<float*>(Q), st);
        if (const int r = shift_any(h, Qc, 0, const_cast<void*>(Qc), 0, -1.f, st)) return r;
    }
    if (h->fp64) {
        if (v4)
            project_scatter_kernel<double, 4><<<unsigned(h->ndof), 256, 0, st>>>(
                *h, static_cast<const double*>(Qc), static_cast<double*>(Q));
        else
            project_scatter_kernel<double, 1><<<unsigned(h->ndof), 256, 0, st>>>(
                *h, static_cast<const double*>(Qc), static_cast<double*>(Q));
    } else {
        if (v4)
            project_scatter_kernel<float, 4><<<unsigned(h->ndof), 256, 0, st>>>(
                *h, static_cast<const float*>(Qc), static_cast<float*>(Q));
        else
            project_scatter_kernel<float, 1><<<unsigned(h->ndof), 256, 0, st>>>(
                *h, static_cast<const float*>(Qc), static_cast<float*>(Q));
    }
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_hybrid_heads(const bdgfs_hybrid_args* h, const float* Y, int64_t ldy, int64_t k,
                                      int32_t nheads, void* out, int64_t ldo, void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!Y || !out || !h->counts || !h->sur_s || k < 1 || nheads < 1 || ldy < nheads * k ||
        ldo < nheads * k)
        return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    heads_kernel<<<unsigned(h->ndof), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        *h, Y, ldy, k, nheads, static_cast<__nv_bfloat16*>(out), ldo);
    return cuda_status(cudaGetLastError());
}

template <int N, typename TI, typename TO>
static int shift_launch(const bdgfs_hybrid_args* h, const void* in, void* out, float sign, cudaStream_t st)
{
    constexpr size_t smem = cube_smem_bytes<N>();
    if (const int rc = smem_optin(reinterpret_cast<const void*>(shift_kernel<N, TI, TO>), smem)) return rc;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BDGFS_ECUDA;
    int64_t grid = int64_t(nsm) * 4;
    if (grid > h->ndof) grid = h->ndof;
    shift_kernel<N, TI, TO><<<unsigned(grid), 256, smem, st>>>(*h, static_cast<const TI*>(in),
                                                               static_cast<TO*>(out), sign);
    return cuda_status(cudaGetLastError());
}

template <int N>
static int shift_types(const bdgfs_hybrid_args* h, const void* in, int in_bf16, void* out, int out_bf16,
                       float sign, cudaStream_t st)
{
    using B = __nv_bfloat16;
    if (h->fp64) {
        if (in_bf16 && out_bf16) return shift_launch<N, B, B>(h, in, out, sign, st);
        if (in_bf16) return shift_launch<N, B, double>(h, in, out, sign, st);
        if (out_bf16) return shift_launch<N, double, B>(h, in, out, sign, st);
        return shift_launch<N, double, double>(h, in, out, sign, st);
    }
    if (in_bf16 && out_bf16) return shift_launch<N, B, B>(h, in, out, sign, st);
    if (in_bf16) return shift_launch<N, B, float>(h, in, out, sign, st);
    if (out_bf16) return shift_launch<N, float, B>(h, in, out, sign, st);
    return shift_launch<N, float, float>(h, in, out, sign, st);
}

extern "C" int32_t bdgfs_hybrid_shift(const bdgfs_hybrid_args* h, const void* in, int32_t in_bf16,
                                      void* out, int32_t out_bf16, float sign, void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!in || !out || !h->counts || !h->sur_uT || h->Nv < 2) return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    return shift_any(h, in, in_bf16, out, out_bf16, sign, static_cast<cudaStream_t>(stream));
}

static int shift_any(const bdgfs_hybrid_args* h, const void* in, int in_bf16, void* out, int out_bf16,
                     float sign, cudaStream_t st)
{
    switch (h->Nv) {
    case 8: return shift_types<8>(h, in, in_bf16, out, out_bf16, sign, st);
    case 12: return shift_types<12>(h, in, in_bf16, out, out_bf16, sign, st);
    case 16: return shift_types<16>(h, in, in_bf16, out, out_bf16, sign, st);
    case 24: return shift_types<24>(h, in, in_bf16, out, out_bf16, sign, st);
    case 32: return shift_types<32>(h, in, in_bf16, out, out_bf16, sign, st);
    default: return BDGFS_EUNSUPPORTED;
    }
}

extern "C" int32_t bdgfs_hybrid_tfeatures(const bdgfs_hybrid_args* h, void* xc, int64_t ld, int64_t x0,
                                          int64_t x1, int64_t k, int32_t k2, int64_t xq, void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    const int64_t nq = int64_t(k2) * (k2 + 1) / 2;
    if (!xc || !h->counts || !h->sur_uT || k < 1 || x0 < 0 || x1 < 0 || x0 + k > ld || x1 + 2 * k > ld ||
        (x1 < x0 + k && x0 < x1 + 2 * k) || k2 < 0 || k2 > 64 || k2 > k ||
        (k2 > 0 && (xq < 0 || xq + nq > ld || (xq < x0 + k && x0 < xq + nq) ||
                    (xq < x1 + 2 * k && x1 < xq + nq))))
        return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BDGFS_ECUDA;
    int64_t grid = int64_t(nsm) * 8;
    if (grid > h->ndof) grid = h->ndof;
    tfeat_kernel<<<unsigned(grid), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        *h, static_cast<__nv_bfloat16*>(xc), ld, x0, x1, k, k2, xq);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_hybrid_heads_split(const bdgfs_hybrid_args* h, const float* Y, int64_t ldy,
                                            int64_t k, int32_t nheads, void* out, int64_t ldo,
                                            void* stream)
{
    int rc = check_h(h);
    if (rc) return rc;
    if (!Y || !out || !h->counts || !h->sur_s || k < 1 || nheads < 1 || ldy < nheads * k ||
        ldo < 3 * nheads * k)
        return BDGFS_EINVAL;
    if (h->ndof == 0) return BDGFS_OK;
    heads_split_kernel<<<unsigned(h->ndof), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        *h, Y, ldy, k, nheads, static_cast<__nv_bfloat16*>(out), ldo);
    return cuda_status(cudaGetLastError());
}

