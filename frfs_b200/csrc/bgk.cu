// BGK relaxation and the ARS IMEX stage update of the 'adgfs' system.
//
// Reference: ADGFSBGKDirectGLLScatteringModel (frfs/solvers/adgfs/
// scattering.py), kernels cmaxwellian / updateMom{q}_ARS
// (kernels/scattering/bgk-direct-gll.mako:4-113) and
// updateDistribution{q}_ARS (linear-common-direct-gll.mako:90-145), driven
// by ARSabcAstdStepper.step (frfs/integrators/std/steppers.py:531-585).
//
// One CTA per distribution.  The reference computes the moments with a
// cuBLAS product against [1, c, |c|^2] cw, stores every stage Maxwellian in
// a full-size bank and updates f in separate launches; here one launch per
// stage reduces the moments (FP64), forms the stage moments and updates f,
// with each Maxwellian built on the fly from separable exponential tables
// (3 Nv exponentials per Maxwellian instead of Nv^3).
#include "common.cuh"
#include "rows.cuh"

namespace bdgfs {

constexpr double kPi = 3.141592653589793;

// temperature and density of a moment row
__device__ __forceinline__ void row_state(const double (&U)[5], double& rho, double& ux, double& uy, double& uz,
                                          double& T)
{
    rho = U[0];
    ux = U[1] / U[0];
    uy = U[2] / U[0];
    uz = U[3] / U[0];
    T = (U[4] - (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0]) / (1.5 * U[0]);
}

template <typename T, int VEC>
__global__ void __launch_bounds__(256) bgk_moments_kernel(const T* __restrict__ f, int Nv, const double* c0,
                                                          double cw, double* __restrict__ U)
{
    __shared__ double red[5 * 8];
    __shared__ double cs[kMaxNv];
    const int64_t dof = blockIdx.x;
    const int n = Nv * Nv * Nv;
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = c0[i];
    __syncthreads();
    double m[5] = {0, 0, 0, 0, 0};
    row_moments<T, VEC>(f + dof * int64_t(n), n, Nv, cs, m);
    block_sum<5>(m, red);
    if (threadIdx.x < 5) U[dof * 5 + threadIdx.x] = m[threadIdx.x] * cw;
}

template <typename T, int VEC>
__global__ void __launch_bounds__(256) bgk_maxwellian_kernel(const double* __restrict__ U, int Nv,
                                                             const double* c0, T* __restrict__ M)
{
    __shared__ double ex[3][kMaxNv];
    const int64_t dof = blockIdx.x;
    const int n = Nv * Nv * Nv;
    double u[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) u[i] = U[dof * 5 + i];
    double rho, ux, uy, uz, Tt;
    row_state(u, rho, ux, uy, uz, Tt);
    const double a = rho / pow(kPi * Tt, 1.5), it = 1.0 / Tt;
    for (int i = threadIdx.x; i < 3 * Nv; i += blockDim.x) {
        const int d = i / Nv, j = i - d * Nv;
        const double c = c0[j] - (d == 0 ? ux : d == 1 ? uy : uz);
        ex[d][j] = exp(-c * c * it);
    }
    __syncthreads();
    T* row = M + dof * int64_t(n);
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        const double axy = a * ex[0][ix] * ex[1][iy];
        Chunk<T, VEC> c;
#pragma unroll
        for (int j = 0; j < VEC; ++j) c.v[j] = T(axy * ex[2][iz + j]);
        c.store(row + v);
    }
}

template <typename T, int VEC>
__global__ void __launch_bounds__(256) ars_kernel(const bdgfs_ars_args g)
{
    __shared__ double red[5 * 8];
    __shared__ double cs[kMaxNv];
    __shared__ double ex[4][3][kMaxNv];
    __shared__ double am[4], nu[4];
    const int64_t dof = blockIdx.x;
    const int Nv = g.Nv, ar = g.stage, flags = g.flags;
    const int n = Nv * Nv * Nv;
    const int64_t off = dof * int64_t(n);
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = g.c0[i];
    __syncthreads();

    double U0[5], LUl[5], Uar[5];
    // ---- moments of f_0 (updateMom / moment)
    if (flags & BDGFS_ARS_MOM0) {
        double m[5] = {0, 0, 0, 0, 0};
        row_moments<T, VEC>(static_cast<const T*>(g.f[0]) + off, n, Nv, cs, m);
        block_sum<5>(m, red);
#pragma unroll
        for (int i = 0; i < 5; ++i) U0[i] = m[i] * g.cw;
        if (threadIdx.x == 0)
            for (int i = 0; i < 5; ++i) g.U[0][dof * 5 + i] = U0[i];
    } else if (flags & BDGFS_ARS_MOMU) {
#pragma unroll
        for (int i = 0; i < 5; ++i) U0[i] = g.U[0][dof * 5 + i];
    }
    // ---- moments of the newest explicit part L_{ar-1}
    if (flags & BDGFS_ARS_MOML) {
        double m[5] = {0, 0, 0, 0, 0};
        row_moments<T, VEC>(static_cast<const T*>(g.L[ar - 1]) + off, n, Nv, cs, m);
        block_sum<5>(m, red);
#pragma unroll
        for (int i = 0; i < 5; ++i) LUl[i] = m[i] * g.cw;
        if (threadIdx.x == 0)
            for (int i = 0; i < 5; ++i) g.LU[ar - 1][dof * 5 + i] = LUl[i];
    }
    // ---- stage moments U_ar = U_0 + dt sum_j ae_j LU_j (BGK conserves them)
    if (flags & BDGFS_ARS_MOMU) {
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            double s = U0[i];
            for (int j = 0; j < ar; ++j) {
                const double lu = (j == ar - 1 && (flags & BDGFS_ARS_MOML)) ? LUl[i] : g.LU[j][dof * 5 + i];
                s += g.dt * g.ae[j] * lu;
            }
            Uar[i] = s;
        }
        if (threadIdx.x == 0)
            for (int i = 0; i < 5; ++i) g.U[ar][dof * 5 + i] = Uar[i];
    }
    if (!(flags & BDGFS_ARS_DIST)) return;

    // ---- Maxwellians M_1..M_ar and collision frequencies of U_1..U_ar
    for (int j = 1; j <= ar; ++j) {
        double u[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) u[i] = (j == ar && (flags & BDGFS_ARS_MOMU)) ? Uar[i] : g.U[j][dof * 5 + i];
        double rho, ux, uy, uz, Tt;
        row_state(u, rho, ux, uy, uz, Tt);
        if (threadIdx.x == 0) {
            am[j - 1] = rho / pow(kPi * Tt, 1.5);
            nu[j - 1] = g.prefac * rho * pow(Tt, 1.0 - g.omega);
        }
        const double it = 1.0 / Tt;
        for (int i = threadIdx.x; i < 3 * Nv; i += blockDim.x) {
            const int d = i / Nv, k = i - d * Nv;
            const double c = cs[k] - (d == 0 ? ux : d == 1 ? uy : uz);
            ex[j - 1][d][k] = exp(-c * c * it);
        }
    }
    __syncthreads();
    const double dt = g.dt;
    const double aii = g.ai[ar - 1] * dt * nu[ar - 1];
    const double inv = 1.0 / (1.0 + aii);
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        double acc[VEC];
        Chunk<T, VEC> c;
        c.load(static_cast<const T*>(g.f[0]) + off + v);
#pragma unroll
        for (int q = 0; q < VEC; ++q) acc[q] = double(c.v[q]);
        for (int j = 0; j < ar; ++j) {
            c.load(static_cast<const T*>(g.L[j]) + off + v);
            const double w = g.ae[j] * dt;
#pragma unroll
            for (int q = 0; q < VEC; ++q) acc[q] += w * double(c.v[q]);
        }
        for (int j = 1; j < ar; ++j) {
            c.load(static_cast<const T*>(g.f[j]) + off + v);
            const double w = g.ai[j - 1] * dt * nu[j - 1];
            const double axy = am[j - 1] * ex[j - 1][0][ix] * ex[j - 1][1][iy];
#pragma unroll
            for (int q = 0; q < VEC; ++q) acc[q] += w * (axy * ex[j - 1][2][iz + q] - double(c.v[q]));
        }
        const double axy = am[ar - 1] * ex[ar - 1][0][ix] * ex[ar - 1][1][iy];
        Chunk<T, VEC> o;
#pragma unroll
        for (int q = 0; q < VEC; ++q) o.v[q] = T((acc[q] + aii * axy * ex[ar - 1][2][iz + q]) * inv);
        o.store(static_cast<T*>(g.fout) + off + v);
    }
}

}  // namespace bdgfs

using namespace bdgfs;

namespace {

bool a16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <typename K4, typename K1, typename... Args>
int32_t launch_rows(bool v4, K4 k4, K1 k1, int64_t ndof, cudaStream_t st, Args... args)
{
    if (v4)
        k4<<<unsigned(ndof), 256, 0, st>>>(args...);
    else
        k1<<<unsigned(ndof), 256, 0, st>>>(args...);
    return cuda_status(cudaGetLastError());
}

}  // namespace

extern "C" int32_t bdgfs_bgk_moments(const void* f, int64_t ndof, int32_t Nv, int32_t fp64, const double* c0,
                                     double cw, double* U, void* stream)
{
    if (!f || !c0 || !U || ndof < 0 || ndof > 2147483647LL || Nv < 1 || Nv > kMaxNv) return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = Nv % 4 == 0 && a16(f);
    if (fp64)
        return launch_rows(v4, bgk_moments_kernel<double, 4>, bgk_moments_kernel<double, 1>, ndof, st,
                           static_cast<const double*>(f), int(Nv), c0, cw, U);
    return launch_rows(v4, bgk_moments_kernel<float, 4>, bgk_moments_kernel<float, 1>, ndof, st,
                       static_cast<const float*>(f), int(Nv), c0, cw, U);
}

extern "C" int32_t bdgfs_bgk_maxwellian(const double* U, int64_t ndof, int32_t Nv, int32_t fp64,
                                        const double* c0, void* M, void* stream)
{
    if (!U || !c0 || !M || ndof < 0 || ndof > 2147483647LL || Nv < 1 || Nv > kMaxNv) return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = Nv % 4 == 0 && a16(M);
    if (fp64)
        return launch_rows(v4, bgk_maxwellian_kernel<double, 4>, bgk_maxwellian_kernel<double, 1>, ndof, st, U,
                           int(Nv), c0, static_cast<double*>(M));
    return launch_rows(v4, bgk_maxwellian_kernel<float, 4>, bgk_maxwellian_kernel<float, 1>, ndof, st, U,
                       int(Nv), c0, static_cast<float*>(M));
}

extern "C" int32_t bdgfs_ars_stage(const bdgfs_ars_args* a, void* stream)
{
    if (!a || !a->c0 || a->ndof < 0 || a->ndof > 2147483647LL || a->Nv < 1 || a->Nv > kMaxNv ||
        a->stage < 1 || a->stage > 4 || (a->flags & ~15))
        return BDGFS_EINVAL;
    const int ar = a->stage, fl = a->flags;
    bool ok = true, v4 = a->Nv % 4 == 0;
    if (fl & BDGFS_ARS_MOM0) ok = ok && a->f[0] && a->U[0];
    if (fl & BDGFS_ARS_MOML) ok = ok && a->L[ar - 1] && a->LU[ar - 1];
    if (fl & BDGFS_ARS_MOMU) {
        ok = ok && a->U[0] && a->U[ar];
        for (int j = 0; j < ar; ++j) ok = ok && a->LU[j];
    }
    if (fl & BDGFS_ARS_DIST) {
        ok = ok && a->fout && a->f[0];
        for (int j = 0; j < ar; ++j) ok = ok && a->L[j] && (j == 0 || a->f[j]);
        for (int j = 1; j <= ar; ++j) ok = ok && a->U[j];
        v4 = v4 && a16(a->fout);
    }
    if (!ok) return BDGFS_EINVAL;
    for (int j = 0; j < ar; ++j) {
        if (a->f[j]) v4 = v4 && a16(a->f[j]);
        if (a->L[j]) v4 = v4 && a16(a->L[j]);
    }
    if (a->ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (a->fp64) return launch_rows(v4, ars_kernel<double, 4>, ars_kernel<double, 1>, a->ndof, st, *a);
    return launch_rows(v4, ars_kernel<float, 4>, ars_kernel<float, 1>, a->ndof, st, *a);
}
