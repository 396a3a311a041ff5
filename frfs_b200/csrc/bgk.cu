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
//
// ES-BGK ('esbgk-direct-gll': ADGFSESBGKDirectGLLScatteringModel, kernels
// momentNorm / cmaxwellian / updateMom{q}_ARS of esbgk-direct-gll.mako)
// uses 11 moment rows (the five conserved ones and the six raw second
// moments cx^2, cy^2, cz^2, cx cy, cy cz, cz cx) and relaxes to the
// anisotropic Gaussian of the ES tensor; the Gaussian is not separable and
// is evaluated per velocity.
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

// FP64 moments {1, c, |c|^2, cx^2, cy^2, cz^2, cx cy, cy cz, cz cx} . f of a
// row (NA = 11), followed by {|c|^2 c} (NA = 14); block-wide partial sums
// per thread
template <typename T, int VEC, int NA>
__device__ __forceinline__ void row_moments_hi(const T* __restrict__ row, int n, int Nv, const double* cs,
                                               double (&m)[NA])
{
    static_assert(NA == 11 || NA == 14, "11 or 14 moment rows");
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        Chunk<T, VEC> c;
        c.load(row + v);
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        const double cx = cs[ix], cy = cs[iy];
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            const double x = double(c.v[j]), cz = cs[iz + j];
            const double c2x = (cx * cx + cy * cy + cz * cz) * x;
            m[0] += x;
            m[1] += cx * x;
            m[2] += cy * x;
            m[3] += cz * x;
            m[4] += c2x;
            m[5] += cx * cx * x;
            m[6] += cy * cy * x;
            m[7] += cz * cz * x;
            m[8] += cx * cy * x;
            m[9] += cy * cz * x;
            m[10] += cz * cx * x;
            if constexpr (NA == 14) {
                m[11] += cx * c2x;
                m[12] += cy * c2x;
                m[13] += cz * c2x;
            }
        }
    }
}

// ES Gaussian of an 11-moment row: G(c) = g[0] exp(-q(c - u)), u = g[1..3],
// q(d) = g[4] dx^2 + g[5] dy^2 + g[6] dz^2 + g[7] dx dy + g[8] dy dz + g[9] dz dx
// (the inverse of T_ij = T/Pr delta_ij + 2 (1 - 1/Pr)(P_ij/rho - u_i u_j)).
__device__ __forceinline__ void es_params(const double* U, double Pr, double (&g)[10])
{
    const double rho = U[0], ux = U[1] / rho, uy = U[2] / rho, uz = U[3] / rho;
    const double T = (U[4] - rho * (ux * ux + uy * uy + uz * uz)) / (1.5 * rho);
    const double k = 2.0 * (1.0 - 1.0 / Pr);
    const double txx = T / Pr + k * (U[5] / rho - ux * ux);
    const double tyy = T / Pr + k * (U[6] / rho - uy * uy);
    const double tzz = T / Pr + k * (U[7] / rho - uz * uz);
    const double txy = k * (U[8] / rho - ux * uy);
    const double tyz = k * (U[9] / rho - uy * uz);
    const double tzx = k * (U[10] / rho - uz * ux);
    const double det = txx * (tyy * tzz - tyz * tyz) - txy * (txy * tzz - tyz * tzx)
                       + tzx * (txy * tyz - tyy * tzx);
    const double id = 1.0 / det;
    g[0] = rho / (pow(kPi, 1.5) * sqrt(det));
    g[1] = ux;
    g[2] = uy;
    g[3] = uz;
    g[4] = (tyy * tzz - tyz * tyz) * id;
    g[5] = (txx * tzz - tzx * tzx) * id;
    g[6] = (txx * tyy - txy * txy) * id;
    g[7] = 2.0 * (tyz * tzx - tzz * txy) * id;
    g[8] = 2.0 * (txy * tzx - txx * tyz) * id;
    g[9] = 2.0 * (txy * tyz - tzx * tyy) * id;
}

__device__ __forceinline__ double es_eval(const double* g, double cx, double cy, double cz)
{
    const double dx = cx - g[1], dy = cy - g[2], dz = cz - g[3];
    const double q = g[4] * dx * dx + g[5] * dy * dy + g[6] * dz * dz + g[7] * dx * dy + g[8] * dy * dz
                     + g[9] * dz * dx;
    return g[0] * exp(-q);
}

template <typename T, int VEC, int NA>
__global__ void __launch_bounds__(256) hi_moments_kernel(const T* __restrict__ f, int Nv, const double* c0,
                                                         double cw, double* __restrict__ U)
{
    __shared__ double red[NA * 8];
    __shared__ double cs[kMaxNv];
    const int64_t dof = blockIdx.x;
    const int n = Nv * Nv * Nv;
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = c0[i];
    __syncthreads();
    double m[NA];
#pragma unroll
    for (int i = 0; i < NA; ++i) m[i] = 0.0;
    row_moments_hi<T, VEC, NA>(f + dof * int64_t(n), n, Nv, cs, m);
    block_sum<NA>(m, red);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < NA; ++i) U[dof * NA + i] = m[i] * cw;
    }
}

// Shakov target of a 14-moment row: S(c) = M(c) (1 + (k q . d)(2 |d|^2 / T - 5)),
// d = c - u, k = 2 (1 - Pr) / (5 rho T^2), q the heat flux
// q_i = Q_i - 2 P_ij u_j + rho u_i |u|^2 - 1.5 rho T u_i; s = {u, 1/T, k q}
__device__ __forceinline__ void shakov_params(const double* U, double Pr, double (&s)[7])
{
    const double rho = U[0], ux = U[1] / rho, uy = U[2] / rho, uz = U[3] / rho;
    const double u2 = ux * ux + uy * uy + uz * uz;
    const double T = (U[4] - rho * u2) / (1.5 * rho);
    const double qx = U[11] - 2.0 * (U[5] * ux + U[8] * uy + U[10] * uz) + rho * ux * u2 - 1.5 * rho * T * ux;
    const double qy = U[12] - 2.0 * (U[8] * ux + U[6] * uy + U[9] * uz) + rho * uy * u2 - 1.5 * rho * T * uy;
    const double qz = U[13] - 2.0 * (U[10] * ux + U[9] * uy + U[7] * uz) + rho * uz * u2 - 1.5 * rho * T * uz;
    const double k = 2.0 * (1.0 - Pr) / (5.0 * rho * T * T);
    s[0] = ux;
    s[1] = uy;
    s[2] = uz;
    s[3] = 1.0 / T;
    s[4] = k * qx;
    s[5] = k * qy;
    s[6] = k * qz;
}

// the Shakov factor 1 + (k q . d)(2 |d|^2 / T - 5) at velocity c
__device__ __forceinline__ double shakov_factor(const double* s, double cx, double cy, double cz)
{
    const double dx = cx - s[0], dy = cy - s[1], dz = cz - s[2];
    return 1.0 + (s[4] * dx + s[5] * dy + s[6] * dz) * (2.0 * (dx * dx + dy * dy + dz * dz) * s[3] - 5.0);
}

template <typename T, int VEC>
__global__ void __launch_bounds__(256) shakov_target_kernel(const double* __restrict__ U, int Nv,
                                                            const double* c0, double Pr, T* __restrict__ S)
{
    __shared__ double cs[kMaxNv];
    __shared__ double ex[3][kMaxNv];
    const int64_t dof = blockIdx.x;
    const int n = Nv * Nv * Nv;
    const double* u = U + dof * 14;
    double sp[7];
    shakov_params(u, Pr, sp);
    const double am = u[0] / pow(kPi / sp[3], 1.5);
    for (int i = threadIdx.x; i < 3 * Nv; i += blockDim.x) {
        const int d = i / Nv, k = i - d * Nv;
        if (d == 0) cs[k] = c0[k];
        const double c = c0[k] - sp[d];
        ex[d][k] = exp(-c * c * sp[3]);
    }
    __syncthreads();
    T* row = S + dof * int64_t(n);
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        Chunk<T, VEC> c;
#pragma unroll
        for (int j = 0; j < VEC; ++j)
            c.v[j] = T(am * ex[0][ix] * ex[1][iy] * ex[2][iz + j] * shakov_factor(sp, cs[ix], cs[iy], cs[iz + j]));
        c.store(row + v);
    }
}

template <typename T, int VEC>
__global__ void __launch_bounds__(256) esbgk_gaussian_kernel(const double* __restrict__ U, int Nv,
                                                             const double* c0, double Pr, T* __restrict__ M)
{
    __shared__ double cs[kMaxNv];
    const int64_t dof = blockIdx.x;
    const int n = Nv * Nv * Nv;
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = c0[i];
    double g[10];
    es_params(U + dof * 11, Pr, g);
    __syncthreads();
    T* row = M + dof * int64_t(n);
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        Chunk<T, VEC> c;
#pragma unroll
        for (int j = 0; j < VEC; ++j) c.v[j] = T(es_eval(g, cs[ix], cs[iy], cs[iz + j]));
        c.store(row + v);
    }
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

// second moments of the Maxwellian of a moment row: rho T/2 + rho u_i^2, rho u_i u_j
__device__ __forceinline__ void maxwell_second(const double* u, double (&t)[6])
{
    double rho, ux, uy, uz, Tt;
    double u5[5] = {u[0], u[1], u[2], u[3], u[4]};
    row_state(u5, rho, ux, uy, uz, Tt);
    t[0] = 0.5 * rho * Tt + rho * ux * ux;
    t[1] = 0.5 * rho * Tt + rho * uy * uy;
    t[2] = 0.5 * rho * Tt + rho * uz * uz;
    t[3] = rho * ux * uy;
    t[4] = rho * uy * uz;
    t[5] = rho * uz * ux;
}

// explicit heat-flux relaxation target of a 14-moment row (Shakov):
// Q(M)_i + (1 - Pr)(q_i - Q_i), Q(M)_i = rho u_i |u|^2 + 2.5 rho T u_i,
// q_i - Q_i = -2 P_ij u_j + rho u_i |u|^2 - 1.5 rho T u_i
__device__ __forceinline__ void shakov_heat(const double* u, double Pr, double (&h)[3])
{
    double rho, ux, uy, uz, Tt;
    double u5[5] = {u[0], u[1], u[2], u[3], u[4]};
    row_state(u5, rho, ux, uy, uz, Tt);
    const double u2 = ux * ux + uy * uy + uz * uz;
    const double v[3] = {ux, uy, uz};
    const double Pu[3] = {u[5] * ux + u[8] * uy + u[10] * uz, u[8] * ux + u[6] * uy + u[9] * uz,
                          u[10] * ux + u[9] * uy + u[7] * uz};
#pragma unroll
    for (int i = 0; i < 3; ++i)
        h[i] = rho * v[i] * u2 + 2.5 * rho * Tt * v[i]
               + (1.0 - Pr) * (-2.0 * Pu[i] + rho * v[i] * u2 - 1.5 * rho * Tt * v[i]);
}

// NA = 5: BGK (separable Maxwellians); NA = 11: ES-BGK (second moments
// relaxed implicitly at nu/Pr, Gaussians evaluated per velocity); NA = 14:
// Shakov (second moments at nu, heat flux at nu Pr, separable Maxwellians
// times the heat-flux polynomial).
template <typename T, int VEC, int NA>
__global__ void __launch_bounds__(256) ars_kernel(const bdgfs_ars_args g)
{
    __shared__ double red[NA * 8];
    __shared__ double cs[kMaxNv];
    __shared__ double ex[NA == 11 ? 1 : 4][3][kMaxNv];
    __shared__ double gp[NA == 5 ? 1 : 4][10];
    __shared__ double am[4], nu[4];
    const int64_t dof = blockIdx.x;
    const int Nv = g.Nv, ar = g.stage, flags = g.flags;
    const int n = Nv * Nv * Nv;
    const int64_t off = dof * int64_t(n);
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = g.c0[i];
    __syncthreads();

    auto moments = [&](const T* row, double (&m)[NA]) {
#pragma unroll
        for (int i = 0; i < NA; ++i) m[i] = 0.0;
        if constexpr (NA == 5) {
            row_moments<T, VEC>(row, n, Nv, cs, m);
        } else {
            row_moments_hi<T, VEC, NA>(row, n, Nv, cs, m);
        }
        block_sum<NA>(m, red);
#pragma unroll
        for (int i = 0; i < NA; ++i) m[i] *= g.cw;
    };
    // temperature-dependent collision frequency of a moment row
    auto rate = [&](const double* u) {
        double rho, ux, uy, uz, Tt;
        double u5[5] = {u[0], u[1], u[2], u[3], u[4]};
        row_state(u5, rho, ux, uy, uz, Tt);
        return g.prefac * rho * pow(Tt, 1.0 - g.omega);
    };

    double U0[NA], LUl[NA], Uar[NA];
    // ---- moments of f_0 (updateMom / moment)
    if (flags & BDGFS_ARS_MOM0) {
        moments(static_cast<const T*>(g.f[0]) + off, U0);
        if (threadIdx.x == 0)
            for (int i = 0; i < NA; ++i) g.U[0][dof * NA + i] = U0[i];
    } else if (flags & BDGFS_ARS_MOMU) {
#pragma unroll
        for (int i = 0; i < NA; ++i) U0[i] = g.U[0][dof * NA + i];
    }
    // ---- moments of the newest explicit part L_{ar-1}
    if (flags & BDGFS_ARS_MOML) {
        moments(static_cast<const T*>(g.L[ar - 1]) + off, LUl);
        if (threadIdx.x == 0)
            for (int i = 0; i < NA; ++i) g.LU[ar - 1][dof * NA + i] = LUl[i];
    }
    // ---- stage moments: U_ar = U_0 + dt sum_j ae_j LU_j (the relaxation
    // conserves the first five); higher moments relax implicitly
    if (flags & BDGFS_ARS_MOMU) {
#pragma unroll
        for (int i = 0; i < NA; ++i) {
            double s = U0[i];
            for (int j = 0; j < ar; ++j) {
                const double lu = (j == ar - 1 && (flags & BDGFS_ARS_MOML)) ? LUl[i] : g.LU[j][dof * NA + i];
                s += g.dt * g.ae[j] * lu;
            }
            Uar[i] = s;
        }
        if constexpr (NA >= 11) {
            // second moments: rate nu/Pr (ES-BGK) or nu (Shakov) towards the Maxwellian's
            const double s2 = NA == 11 ? 1.0 / g.Pr : 1.0;
            double num[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) num[k] = Uar[5 + k];
            for (int j = 1; j < ar; ++j) {
                const double* uj = g.U[j] + dof * NA;
                double t[6];
                maxwell_second(uj, t);
                const double w = g.ai[j - 1] * g.dt * rate(uj) * s2;
#pragma unroll
                for (int k = 0; k < 6; ++k) num[k] += w * (t[k] - uj[5 + k]);
            }
            double t[6];
            maxwell_second(Uar, t);
            const double w = g.ai[ar - 1] * g.dt * rate(Uar) * s2;
#pragma unroll
            for (int k = 0; k < 6; ++k) Uar[5 + k] = (num[k] + w * t[k]) / (1.0 + w);
        }
        if constexpr (NA == 14) {
            // heat flux: dQ/dt = nu (Q(M) + (1 - Pr)(q - Q) - Pr Q), -Pr Q implicit
            double num[3] = {Uar[11], Uar[12], Uar[13]};
            for (int j = 1; j < ar; ++j) {
                const double* uj = g.U[j] + dof * NA;
                double h[3];
                shakov_heat(uj, g.Pr, h);
                const double w = g.ai[j - 1] * g.dt * rate(uj);
#pragma unroll
                for (int k = 0; k < 3; ++k) num[k] += w * (h[k] - g.Pr * uj[11 + k]);
            }
            double h[3];
            shakov_heat(Uar, g.Pr, h);
            const double w = g.ai[ar - 1] * g.dt * rate(Uar);
#pragma unroll
            for (int k = 0; k < 3; ++k) Uar[11 + k] = (num[k] + w * h[k]) / (1.0 + g.Pr * w);
        }
        if (threadIdx.x == 0)
            for (int i = 0; i < NA; ++i) g.U[ar][dof * NA + i] = Uar[i];
    }
    if (!(flags & BDGFS_ARS_DIST)) return;

    // ---- relaxation targets of U_1..U_ar (Maxwellians, ES Gaussians or
    // Shakov distributions) and their collision frequencies
    for (int j = 1; j <= ar; ++j) {
        double u[NA];
#pragma unroll
        for (int i = 0; i < NA; ++i) u[i] = (j == ar && (flags & BDGFS_ARS_MOMU)) ? Uar[i] : g.U[j][dof * NA + i];
        if (threadIdx.x == 0) nu[j - 1] = rate(u);
        if constexpr (NA == 11) {
            if (threadIdx.x == 0) {
                double gj[10];
                es_params(u, g.Pr, gj);
#pragma unroll
                for (int i = 0; i < 10; ++i) gp[j - 1][i] = gj[i];
            }
        } else {
            double rho, ux, uy, uz, Tt;
            double u5[5] = {u[0], u[1], u[2], u[3], u[4]};
            row_state(u5, rho, ux, uy, uz, Tt);
            if (threadIdx.x == 0) am[j - 1] = rho / pow(kPi * Tt, 1.5);
            const double it = 1.0 / Tt;
            for (int i = threadIdx.x; i < 3 * Nv; i += blockDim.x) {
                const int d = i / Nv, k = i - d * Nv;
                const double c = cs[k] - (d == 0 ? ux : d == 1 ? uy : uz);
                ex[j - 1][d][k] = exp(-c * c * it);
            }
            if constexpr (NA == 14) {
                if (threadIdx.x == 0) {
                    double sj[7];
                    shakov_params(u, g.Pr, sj);
#pragma unroll
                    for (int i = 0; i < 7; ++i) gp[j - 1][i] = sj[i];
                }
            }
        }
    }
    __syncthreads();
    auto target = [&](int j, uint32_t ix, uint32_t iy, uint32_t izq) -> double {
        if constexpr (NA == 11) {
            return es_eval(gp[j], cs[ix], cs[iy], cs[izq]);
        } else {
            const double m = am[j] * ex[j][0][ix] * ex[j][1][iy] * ex[j][2][izq];
            if constexpr (NA == 14) return m * shakov_factor(gp[j], cs[ix], cs[iy], cs[izq]);
            else return m;
        }
    };
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
#pragma unroll
            for (int q = 0; q < VEC; ++q) acc[q] += w * (target(j - 1, ix, iy, iz + q) - double(c.v[q]));
        }
        Chunk<T, VEC> o;
#pragma unroll
        for (int q = 0; q < VEC; ++q) o.v[q] = T((acc[q] + aii * target(ar - 1, ix, iy, iz + q)) * inv);
        o.store(static_cast<T*>(g.fout) + off + v);
    }
}

// One IMEX-BDF step (updateMom{q}_BDF + constructMaxwellian +
// updateDistribution{q}_BDF): with N = -sum_i (a_i X_i + g_i dt LX_i),
//   U  = N / a_q for the conserved five; higher moments relax implicitly
//        (ES-BGK second moments at b nu/Pr, Shakov second moments at b nu and
//        the heat flux with denominator a_q + Pr b dt nu)
//   f  = (N_f + b dt nu M[U]) / (a_q + b dt nu).
// One CTA per distribution; the newest moment rows (of f_{q-1} and of
// L_{q-1}) are reduced in the same launch when BDGFS_BDF_MOMN is set.
template <typename T, int VEC, int NA>
__global__ void __launch_bounds__(256) bdf_kernel(const bdgfs_bdf_args g)
{
    __shared__ double red[NA * 8];
    __shared__ double cs[kMaxNv];
    __shared__ double ex[3][kMaxNv];
    __shared__ double gp[10];
    __shared__ double am, nu;
    const int64_t dof = blockIdx.x;
    const int Nv = g.Nv, q = g.q, flags = g.flags;
    const int n = Nv * Nv * Nv;
    const int64_t off = dof * int64_t(n);
    for (int i = threadIdx.x; i < Nv; i += blockDim.x) cs[i] = g.c0[i];
    __syncthreads();

    auto moments = [&](const T* row, double (&m)[NA]) {
#pragma unroll
        for (int i = 0; i < NA; ++i) m[i] = 0.0;
        if constexpr (NA == 5) {
            row_moments<T, VEC>(row, n, Nv, cs, m);
        } else {
            row_moments_hi<T, VEC, NA>(row, n, Nv, cs, m);
        }
        block_sum<NA>(m, red);
#pragma unroll
        for (int i = 0; i < NA; ++i) m[i] *= g.cw;
    };
    auto rate = [&](const double* u) {
        double rho, ux, uy, uz, Tt;
        double u5[5] = {u[0], u[1], u[2], u[3], u[4]};
        row_state(u5, rho, ux, uy, uz, Tt);
        return g.prefac * rho * pow(Tt, 1.0 - g.omega);
    };

    double Un[NA], LUn[NA], U[NA];
    if (flags & BDGFS_BDF_MOMN) {
        moments(static_cast<const T*>(g.f[q - 1]) + off, Un);
        moments(static_cast<const T*>(g.L[q - 1]) + off, LUn);
        if (threadIdx.x == 0)
            for (int i = 0; i < NA; ++i) {
                g.U[q - 1][dof * NA + i] = Un[i];
                g.LU[q - 1][dof * NA + i] = LUn[i];
            }
    }
    const double aq = g.a[q];
    if (flags & BDGFS_BDF_MOMU) {
        double N[NA];
#pragma unroll
        for (int k = 0; k < NA; ++k) {
            double s = 0.0;
            for (int i = 0; i < q; ++i) {
                const bool fresh = i == q - 1 && (flags & BDGFS_BDF_MOMN);
                const double ui = fresh ? Un[k] : g.U[i][dof * NA + k];
                const double li = fresh ? LUn[k] : g.LU[i][dof * NA + k];
                s -= g.a[i] * ui + g.g[i] * g.dt * li;
            }
            N[k] = s;
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) U[k] = N[k] / aq;
        if constexpr (NA >= 11) {
            const double w = g.b * g.dt * rate(U) * (NA == 11 ? 1.0 / g.Pr : 1.0);
            double t[6];
            maxwell_second(U, t);
#pragma unroll
            for (int k = 0; k < 6; ++k) U[5 + k] = (N[5 + k] + w * t[k]) / (aq + w);
        }
        if constexpr (NA == 14) {
            const double w = g.b * g.dt * rate(U);
            double h[3];
            shakov_heat(U, g.Pr, h);
#pragma unroll
            for (int k = 0; k < 3; ++k) U[11 + k] = (N[11 + k] + w * h[k]) / (aq + g.Pr * w);
        }
        if (threadIdx.x == 0)
            for (int i = 0; i < NA; ++i) g.Unew[dof * NA + i] = U[i];
    } else {
#pragma unroll
        for (int i = 0; i < NA; ++i) U[i] = g.Unew[dof * NA + i];
    }
    if (!(flags & BDGFS_BDF_DIST)) return;

    // relaxation target of U and its collision frequency
    if (threadIdx.x == 0) nu = rate(U);
    if constexpr (NA == 11) {
        if (threadIdx.x == 0) {
            double gj[10];
            es_params(U, g.Pr, gj);
#pragma unroll
            for (int i = 0; i < 10; ++i) gp[i] = gj[i];
        }
    } else {
        double rho, ux, uy, uz, Tt;
        double u5[5] = {U[0], U[1], U[2], U[3], U[4]};
        row_state(u5, rho, ux, uy, uz, Tt);
        if (threadIdx.x == 0) am = rho / pow(kPi * Tt, 1.5);
        const double it = 1.0 / Tt;
        for (int i = threadIdx.x; i < 3 * Nv; i += blockDim.x) {
            const int d = i / Nv, k = i - d * Nv;
            const double c = cs[k] - (d == 0 ? ux : d == 1 ? uy : uz);
            ex[d][k] = exp(-c * c * it);
        }
        if constexpr (NA == 14) {
            if (threadIdx.x == 0) {
                double sj[7];
                shakov_params(U, g.Pr, sj);
#pragma unroll
                for (int i = 0; i < 7; ++i) gp[i] = sj[i];
            }
        }
    }
    __syncthreads();
    auto target = [&](uint32_t ix, uint32_t iy, uint32_t izq) -> double {
        if constexpr (NA == 11) {
            return es_eval(gp, cs[ix], cs[iy], cs[izq]);
        } else {
            const double m = am * ex[0][ix] * ex[1][iy] * ex[2][izq];
            if constexpr (NA == 14) return m * shakov_factor(gp, cs[ix], cs[iy], cs[izq]);
            else return m;
        }
    };
    const double bdn = g.b * g.dt * nu;
    const double inv = 1.0 / (aq + bdn);
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        uint32_t ix, iy, iz;
        vsplit(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        double acc[VEC];
#pragma unroll
        for (int j = 0; j < VEC; ++j) acc[j] = 0.0;
        for (int i = 0; i < q; ++i) {
            Chunk<T, VEC> cf, cl;
            cf.load(static_cast<const T*>(g.f[i]) + off + v);
            cl.load(static_cast<const T*>(g.L[i]) + off + v);
            const double wa = g.a[i], wg = g.g[i] * g.dt;
#pragma unroll
            for (int j = 0; j < VEC; ++j) acc[j] -= wa * double(cf.v[j]) + wg * double(cl.v[j]);
        }
        Chunk<T, VEC> o;
#pragma unroll
        for (int j = 0; j < VEC; ++j) o.v[j] = T((acc[j] + bdn * target(ix, iy, iz + j)) * inv);
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
        a->stage < 1 || a->stage > 4 || (a->flags & ~15) ||
        (a->model != BDGFS_ARS_BGK && a->model != BDGFS_ARS_ESBGK && a->model != BDGFS_ARS_SHAKOV) ||
        (a->model != BDGFS_ARS_BGK && !(a->Pr > 0.0)))
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
    if (a->model == BDGFS_ARS_SHAKOV) {
        if (a->fp64) return launch_rows(v4, ars_kernel<double, 4, 14>, ars_kernel<double, 1, 14>, a->ndof, st, *a);
        return launch_rows(v4, ars_kernel<float, 4, 14>, ars_kernel<float, 1, 14>, a->ndof, st, *a);
    }
    if (a->model == BDGFS_ARS_ESBGK) {
        if (a->fp64) return launch_rows(v4, ars_kernel<double, 4, 11>, ars_kernel<double, 1, 11>, a->ndof, st, *a);
        return launch_rows(v4, ars_kernel<float, 4, 11>, ars_kernel<float, 1, 11>, a->ndof, st, *a);
    }
    if (a->fp64) return launch_rows(v4, ars_kernel<double, 4, 5>, ars_kernel<double, 1, 5>, a->ndof, st, *a);
    return launch_rows(v4, ars_kernel<float, 4, 5>, ars_kernel<float, 1, 5>, a->ndof, st, *a);
}

extern "C" int32_t bdgfs_esbgk_moments(const void* f, int64_t ndof, int32_t Nv, int32_t fp64,
                                       const double* c0, double cw, double* U, void* stream)
{
    if (!f || !c0 || !U || ndof < 0 || ndof > 2147483647LL || Nv < 1 || Nv > kMaxNv) return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = Nv % 4 == 0 && a16(f);
    if (fp64)
        return launch_rows(v4, hi_moments_kernel<double, 4, 11>, hi_moments_kernel<double, 1, 11>, ndof, st,
                           static_cast<const double*>(f), int(Nv), c0, cw, U);
    return launch_rows(v4, hi_moments_kernel<float, 4, 11>, hi_moments_kernel<float, 1, 11>, ndof, st,
                       static_cast<const float*>(f), int(Nv), c0, cw, U);
}

extern "C" int32_t bdgfs_esbgk_gaussian(const double* U, int64_t ndof, int32_t Nv, int32_t fp64,
                                        const double* c0, double Pr, void* M, void* stream)
{
    if (!U || !c0 || !M || ndof < 0 || ndof > 2147483647LL || Nv < 1 || Nv > kMaxNv || !(Pr > 0.0))
        return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = Nv % 4 == 0 && a16(M);
    if (fp64)
        return launch_rows(v4, esbgk_gaussian_kernel<double, 4>, esbgk_gaussian_kernel<double, 1>, ndof, st, U,
                           int(Nv), c0, Pr, static_cast<double*>(M));
    return launch_rows(v4, esbgk_gaussian_kernel<float, 4>, esbgk_gaussian_kernel<float, 1>, ndof, st, U,
                       int(Nv), c0, Pr, static_cast<float*>(M));
}

extern "C" int32_t bdgfs_shakov_moments(const void* f, int64_t ndof, int32_t Nv, int32_t fp64,
                                        const double* c0, double cw, double* U, void* stream)
{
    if (!f || !c0 || !U || ndof < 0 || ndof > 2147483647LL || Nv < 1 || Nv > kMaxNv) return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = Nv % 4 == 0 && a16(f);
    if (fp64)
        return launch_rows(v4, hi_moments_kernel<double, 4, 14>, hi_moments_kernel<double, 1, 14>, ndof, st,
                           static_cast<const double*>(f), int(Nv), c0, cw, U);
    return launch_rows(v4, hi_moments_kernel<float, 4, 14>, hi_moments_kernel<float, 1, 14>, ndof, st,
                       static_cast<const float*>(f), int(Nv), c0, cw, U);
}

extern "C" int32_t bdgfs_shakov_target(const double* U, int64_t ndof, int32_t Nv, int32_t fp64,
                                       const double* c0, double Pr, void* S, void* stream)
{
    if (!U || !c0 || !S || ndof < 0 || ndof > 2147483647LL || Nv < 1 || Nv > kMaxNv || !(Pr > 0.0))
        return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool v4 = Nv % 4 == 0 && a16(S);
    if (fp64)
        return launch_rows(v4, shakov_target_kernel<double, 4>, shakov_target_kernel<double, 1>, ndof, st, U,
                           int(Nv), c0, Pr, static_cast<double*>(S));
    return launch_rows(v4, shakov_target_kernel<float, 4>, shakov_target_kernel<float, 1>, ndof, st, U,
                       int(Nv), c0, Pr, static_cast<float*>(S));
}

extern "C" int32_t bdgfs_bdf_step(const bdgfs_bdf_args* a, void* stream)
{
    if (!a || a->ndof < 0 || a->ndof > 2147483647LL || a->Nv < 1 || a->Nv > kMaxNv || !a->c0 ||
        a->q < 1 || a->q > 3 || (a->flags & ~7) || !a->Unew ||
        (a->model != BDGFS_ARS_BGK && a->model != BDGFS_ARS_ESBGK && a->model != BDGFS_ARS_SHAKOV) ||
        (a->model != BDGFS_ARS_BGK && !(a->Pr > 0.0)) || a->a[a->q] == 0.0)
        return BDGFS_EINVAL;
    const int q = a->q;
    if (a->flags & BDGFS_BDF_MOMN) {
        if (!a->f[q - 1] || !a->L[q - 1] || !a->U[q - 1] || !a->LU[q - 1]) return BDGFS_EINVAL;
    }
    if (a->flags & BDGFS_BDF_MOMU) {
        for (int i = 0; i < q; ++i)
            if (!a->U[i] || !a->LU[i]) return BDGFS_EINVAL;
    }
    bool v4 = a->Nv % 4 == 0;
    if (a->flags & BDGFS_BDF_DIST) {
        if (!a->fout) return BDGFS_EINVAL;
        v4 = v4 && a16(a->fout);
        for (int i = 0; i < q; ++i) {
            if (!a->f[i] || !a->L[i]) return BDGFS_EINVAL;
            v4 = v4 && a16(a->f[i]) && a16(a->L[i]);
        }
    } else if (a->flags & BDGFS_BDF_MOMN) {
        v4 = v4 && a16(a->f[q - 1]) && a16(a->L[q - 1]);
    }
    if (a->ndof == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define BDF_GO(NA)                                                                                         \
    return a->fp64 ? launch_rows(v4, bdf_kernel<double, 4, NA>, bdf_kernel<double, 1, NA>, a->ndof, st, *a) \
                   : launch_rows(v4, bdf_kernel<float, 4, NA>, bdf_kernel<float, 1, NA>, a->ndof, st, *a);
    if (a->model == BDGFS_ARS_SHAKOV) { BDF_GO(14) }
    if (a->model == BDGFS_ARS_ESBGK) { BDF_GO(11) }
    BDF_GO(5)
#undef BDF_GO
}
