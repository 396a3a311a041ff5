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

template <typename T, int VEC>
__global__ void __launch_bounds__(256) indicator_kernel(const bdgfs_hybrid_args h, const T* __restrict__ f)
{
    __shared__ double red[8 * 8];
    __shared__ double cs[kMaxNv], ex[3][kMaxNv];
    __shared__ int64_t s_pos;
    const int64_t dof = blockIdx.x;
    const int Nv = h.Nv;
    const int n = Nv * Nv * Nv;
    const T* fd = f + dof * int64_t(n);
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = h.c0[i];
    __syncthreads();
    double m[5] = {0, 0, 0, 0, 0};
    row_moments<T, VEC>(fd, n, Nv, cs, m);
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
            vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
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
            if (h.feat) {
                __nv_bfloat16* fr = static_cast<__nv_bfloat16*>(h.feat) + p * h.feat_ld;
                fr[0] = __float2bfloat16_rn(float(ux));
                fr[1] = __float2bfloat16_rn(float(uy));
                fr[2] = __float2bfloat16_rn(float(uz));
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
            vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
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

}  // namespace bdgfs

using namespace bdgfs;

static int check_h(const bdgfs_hybrid_args* h)
{
    if (!h || h->ndof < 0 || h->Nv < 1 || h->Nv > kMaxNv || !h->c0) return BDGFS_EINVAL;
    if (h->ndof > 2147483647LL) return BDGFS_EINVAL;
    return BDGFS_OK;
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
    if (h->fp64) {
        if (v4)
            indicator_kernel<double, 4><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const double*>(f));
        else
            indicator_kernel<double, 1><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const double*>(f));
    } else {
        if (v4)
            indicator_kernel<float, 4><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(f));
        else
            indicator_kernel<float, 1><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(f));
    }
    return cuda_status(cudaGetLastError());
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
