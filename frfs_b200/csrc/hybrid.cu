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
#include "common.cuh"

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

template <typename T>
__global__ void __launch_bounds__(256) indicator_kernel(const bdgfs_hybrid_args h, const T* __restrict__ f)
{
    __shared__ double red[8 * 8];
    const int64_t dof = blockIdx.x;
    const int Nv = h.Nv;
    const int64_t n = int64_t(Nv) * Nv * Nv;
    const T* fd = f + dof * n;
    const double* c0 = h.c0;
    double m[5] = {0, 0, 0, 0, 0};
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
        const double cx = c0[v / (int64_t(Nv) * Nv)], cy = c0[(v / Nv) % Nv], cz = c0[v % Nv];
        const double x = double(fd[v]);
        m[0] += x;
        m[1] += cx * x;
        m[2] += cy * x;
        m[3] += cz * x;
        m[4] += (cx * cx + cy * cy + cz * cz) * x;
    }
    block_sum<5>(m, red);
    const double rho = m[0] * h.cw;
    const double ux = m[1] / m[0], uy = m[2] / m[0], uz = m[3] / m[0];
    const double Tt = (m[4] / m[0] - (ux * ux + uy * uy + uz * uz)) * (2.0 / 3.0);
    double e[2] = {0, 0};
    const bool ok = rho > 0.0 && Tt > 0.0;
    if (ok) {
        const double a = rho / pow(3.141592653589793 * Tt, 1.5), it = 1.0 / Tt;
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
            const double cx = c0[v / (int64_t(Nv) * Nv)] - ux, cy = c0[(v / Nv) % Nv] - uy,
                         cz = c0[v % Nv] - uz;
            const double x = double(fd[v]);
            const double d = x - a * exp(-(cx * cx + cy * cy + cz * cz) * it);
            e[0] += d * d;
            e[1] += x * x;
        }
    }
    block_sum<2>(e, red);
    if (threadIdx.x == 0) {
        const double eps = (ok && e[1] > 0.0) ? sqrt(e[0] / e[1]) : 1e30;
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
        }
        if (!sur || re) {
            const int64_t p = int64_t(atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 1), 1ull));
            h.spec_idx[p] = int32_t(dof);
        }
        if (re) atomicAdd(reinterpret_cast<unsigned long long*>(h.counts + 2), 1ull);
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
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
        const double cx = c0[v / (int64_t(Nv) * Nv)], cy = c0[(v / Nv) % Nv], cz = c0[v % Nv];
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
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
        const double cx = c0[v / (int64_t(Nv) * Nv)], cy = c0[(v / Nv) % Nv], cz = c0[v % Nv];
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
        for (int64_t v = threadIdx.x; v < n; v += blockDim.x) dst[v] = src[v];
        return;
    }
    double e[2] = {0, 0};
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
        const double d = double(src[v]) - double(dst[v]);
        e[0] += d * d;
        e[1] += double(dst[v]) * double(dst[v]);
    }
    block_sum<2>(e, red);
    if (threadIdx.x == 0 && h.recheck_err) {
        atomicAdd(h.recheck_err, e[0]);
        atomicAdd(h.recheck_err + 1, e[1]);
    }
}

}  // namespace bdgfs

using namespace bdgfs;

static int check_h(const bdgfs_hybrid_args* h)
{
    if (!h || h->ndof < 0 || h->Nv < 1 || !h->c0) return BDGFS_EINVAL;
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
    if (cudaMemsetAsync(h->counts, 0, 3 * sizeof(int64_t), st) != cudaSuccess) return BDGFS_ECUDA;
    if (h->recheck_err && cudaMemsetAsync(h->recheck_err, 0, 2 * sizeof(double), st) != cudaSuccess)
        return BDGFS_ECUDA;
    if (h->ndof == 0) return BDGFS_OK;
    if (h->fp64)
        indicator_kernel<double><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const double*>(f));
    else
        indicator_kernel<float><<<unsigned(h->ndof), 256, 0, st>>>(*h, static_cast<const float*>(f));
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
