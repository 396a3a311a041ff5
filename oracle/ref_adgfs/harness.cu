// Test infrastructure: one step of the reference's ARS IMEX stepper for the
// BGK-family relaxation models, with the model's own kernels (rendered from
// frfs/solvers/adgfs/kernels/scattering/<model>-direct-gll.mako into the
// file named by REF_KERNELS, FP64) and the explicit part L given (the same
// array at every stage).  Call sequence restated from
// ARSabcAstdStepper.step (frfs/integrators/std/steppers.py:538-585):
//   U0 = moment(f0)
//   stage ar = 1..s:  L_{ar-1} given, LU_{ar-1} = moment(L_{ar-1}),
//                     updateMom{ar}_ARS(prefac, lda, dt, _A[ar][0..ar-1],
//                       A[ar][1..ar], LU_0..LU_{ar-1}, U_0..U_{ar-1}, U_ar),
//                     M_{ar-1} = constructMaxwellian(U_ar),
//                     updateDistribution{ar}_ARS(prefac, nupts, ldim, nvars,
//                       neles, dt, _A.., A.., L_0.., U_0..U_ar, M_0..M_{ar-1},
//                       f_0..f_{ar-1}, f_ar)
// with constructMaxwellian = cmaxwellian (BGK) or momentNorm + cmaxwellian
// (ES-BGK, Shakov; frfs/solvers/adgfs/scattering.py:297-306) and moment =
// the rows of f times the model's moment matrix (scattering.py:85-96,
// 163-172; cuBLAS there, FP64 loops on the host here).  Blocks of 256
// threads and get_grid_for_block's grid.  The 32 distributions are the 32
// elements of one AoSoA block at one solution point (SOA_IX with soasz 32:
// velocity v of element e at v*32 + e), as the reference's kernels index.
#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include REF_KERNELS

namespace {

constexpr int kElems = 32;

int ok(cudaError_t e)
{
    return e == cudaSuccess ? 0 : -2;
}

template <typename K, size_t... I>
void mom_ars(K k, dim3 g, dim3 b, double prefac, int lda, double dt, const double* a_, const double* a,
             double* const* LU, double* const* U, double* Uq, std::index_sequence<I...>)
{
    k<<<g, b>>>(prefac, lda, dt, a_[I]..., a[I]..., LU[I]..., U[I]..., Uq);
}

template <typename K, size_t... I>
void dist_ars(K k, dim3 g, dim3 b, double prefac, int nupts, int ldim, int nvars, int neles, double dt,
              const double* a_, const double* a, double* const* L, double* const* U, double* Uq,
              double* const* M, double* const* F, double* Fq, std::index_sequence<I...>)
{
    k<<<g, b>>>(prefac, nupts, ldim, nvars, neles, dt, a_[I]..., a[I]..., L[I]..., U[I]..., Uq, M[I]...,
                F[I]..., Fq);
}

}  // namespace

// mat: [nalph][nv] moment matrix (times cw); c: [3][nv] velocities;
// f0, L, out: [32][nv]; At, Ai: the (s+1)x(s+1) explicit and implicit ARS
// tables, row-major; 1 <= s <= 4.  Returns 0, -1 (arguments) or -2 (CUDA).
extern "C" int ref_ars_step(int s, const double* At, const double* Ai, double dt, double prefac,
                            int nalph, int nv, const double* mat, const double* c, const double* f0,
                            const double* L, double* out)
{
    if (s < 1 || s > 4 || nalph != NALPH || nv < 1 || !At || !Ai || !mat || !c || !f0 || !L || !out)
        return -1;
    const int nupts = 1, neles = kElems, nvars = nv, ldim = kElems * nv, lda = nupts * neles;
    const size_t nf = size_t(kElems) * nv, nu = size_t(kElems) * NALPH;
    const dim3 block(256), gridf(unsigned((nf + 255) / 256)), gridu(unsigned((lda + 255) / 256));
    std::vector<double> h(nf), hu(nu);
    // device arrays: F[0..s], Lb (one, reused), M[0..s-1], U[0..s], LU (one), Ut, c
    double *dF[5] = {}, *dM[4] = {}, *dU[5] = {}, *dLU = nullptr, *dL = nullptr, *dUt = nullptr,
           *dc = nullptr;
    int rc = 0;
    auto moment = [&](const double* dsrc, double* ddst) -> int {
        int r = ok(cudaMemcpy(h.data(), dsrc, nf * sizeof(double), cudaMemcpyDeviceToHost));
        if (r) return r;
        for (int e = 0; e < kElems; ++e)
            for (int k = 0; k < NALPH; ++k) {
                double acc = 0.0;
                for (int v = 0; v < nv; ++v) acc += h[size_t(v) * kElems + e] * mat[size_t(k) * nv + v];
                hu[size_t(e) * NALPH + k] = acc;
            }
        return ok(cudaMemcpy(ddst, hu.data(), nu * sizeof(double), cudaMemcpyHostToDevice));
    };
    do {
        for (int i = 0; i <= s && !rc; ++i) {
            rc = ok(cudaMalloc(&dF[i], nf * sizeof(double)));
            if (!rc) rc = ok(cudaMalloc(&dU[i], nu * sizeof(double)));
            if (!rc && i < s) rc = ok(cudaMalloc(&dM[i], nf * sizeof(double)));
        }
        if (rc) break;
        if ((rc = ok(cudaMalloc(&dL, nf * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dLU, 4 * nu * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dUt, nu * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dc, 3 * size_t(nv) * sizeof(double))))) break;
        if ((rc = ok(cudaMemcpy(dc, c, 3 * size_t(nv) * sizeof(double), cudaMemcpyHostToDevice)))) break;
        // f0 and L into the AoSoA layout
        for (int e = 0; e < kElems; ++e)
            for (int v = 0; v < nv; ++v) h[size_t(v) * kElems + e] = f0[size_t(e) * nv + v];
        if ((rc = ok(cudaMemcpy(dF[0], h.data(), nf * sizeof(double), cudaMemcpyHostToDevice)))) break;
        for (int e = 0; e < kElems; ++e)
            for (int v = 0; v < nv; ++v) h[size_t(v) * kElems + e] = L[size_t(e) * nv + v];
        if ((rc = ok(cudaMemcpy(dL, h.data(), nf * sizeof(double), cudaMemcpyHostToDevice)))) break;
        if ((rc = moment(dF[0], dU[0]))) break;
        double* LUs[4];
        double* Ls[4];
        for (int i = 0; i < 4; ++i) {
            LUs[i] = dLU + size_t(i) * nu;
            Ls[i] = dL;
        }
        for (int i = 0; i < s && !rc; ++i) {
            const int ar = i + 1;
            if ((rc = moment(Ls[i], LUs[i]))) break;
            double a_[4], a[4];
            for (int j = 0; j < ar; ++j) {
                a_[j] = At[ar * (s + 1) + j];
                a[j] = Ai[ar * (s + 1) + j + 1];
            }
            switch (ar) {
            case 1: mom_ars(updateMom1_ARS, gridu, block, prefac, lda, dt, a_, a, LUs, dU, dU[1], std::make_index_sequence<1>{}); break;
            case 2: mom_ars(updateMom2_ARS, gridu, block, prefac, lda, dt, a_, a, LUs, dU, dU[2], std::make_index_sequence<2>{}); break;
            case 3: mom_ars(updateMom3_ARS, gridu, block, prefac, lda, dt, a_, a, LUs, dU, dU[3], std::make_index_sequence<3>{}); break;
            default: mom_ars(updateMom4_ARS, gridu, block, prefac, lda, dt, a_, a, LUs, dU, dU[4], std::make_index_sequence<4>{}); break;
            }
#ifdef HAS_MOMENT_NORM
            momentNorm<<<gridu, block>>>(lda, dU[ar], dUt);
            cmaxwellian<<<gridf, block>>>(nupts, ldim, nvars, neles, dc, dc + nv, dc + 2 * nv, dM[i], dUt);
#else
            cmaxwellian<<<gridf, block>>>(nupts, ldim, nvars, neles, dc, dc + nv, dc + 2 * nv, dM[i], dU[ar]);
#endif
            switch (ar) {
            case 1: dist_ars(updateDistribution1_ARS, gridf, block, prefac, nupts, ldim, nvars, neles, dt, a_, a, Ls, dU, dU[1], dM, dF, dF[1], std::make_index_sequence<1>{}); break;
            case 2: dist_ars(updateDistribution2_ARS, gridf, block, prefac, nupts, ldim, nvars, neles, dt, a_, a, Ls, dU, dU[2], dM, dF, dF[2], std::make_index_sequence<2>{}); break;
            case 3: dist_ars(updateDistribution3_ARS, gridf, block, prefac, nupts, ldim, nvars, neles, dt, a_, a, Ls, dU, dU[3], dM, dF, dF[3], std::make_index_sequence<3>{}); break;
            default: dist_ars(updateDistribution4_ARS, gridf, block, prefac, nupts, ldim, nvars, neles, dt, a_, a, Ls, dU, dU[4], dM, dF, dF[4], std::make_index_sequence<4>{}); break;
            }
            rc = ok(cudaGetLastError());
        }
        if (rc) break;
        if ((rc = ok(cudaMemcpy(h.data(), dF[s], nf * sizeof(double), cudaMemcpyDeviceToHost)))) break;
        for (int e = 0; e < kElems; ++e)
            for (int v = 0; v < nv; ++v) out[size_t(e) * nv + v] = h[size_t(v) * kElems + e];
    } while (false);
    for (int i = 0; i < 5; ++i) {
        cudaFree(dF[i]);
        cudaFree(dU[i]);
        if (i < 4) cudaFree(dM[i]);
    }
    cudaFree(dL);
    cudaFree(dLU);
    cudaFree(dUt);
    cudaFree(dc);
    return rc;
}

// One update of the reference's IMEX-BDF stepper (BDF2AstdStepper.step,
// frfs/integrators/std/steppers.py:700-760; BDF3 likewise) for q = 2 or 3
// histories, oldest first: Us, LUs = moments of fs, Ls;
// updateMom{q}_BDF(prefac, lda, dt, a_0, U_0, g_0, LU_0, ..., a_q, U, b);
// constructMaxwellian(U); updateDistribution{q}_BDF(prefac, nupts, ldim,
// nvars, neles, dt, a_0, f_0, g_0, L_0, ..., b, M, a_q, U, f).  a[0..q],
// g[0..q-1] as passed to the kernels (g = -G of the stepper's tables).
// fs, Ls: [q][32][nv]; fout: [32][nv]; Uout: [32][nalph].
extern "C" int ref_bdf_update(int q, const double* a, const double* g, double b, double dt, double prefac,
                              int nalph, int nv, const double* mat, const double* c, const double* fs,
                              const double* Ls, double* fout, double* Uout)
{
    if ((q != 2 && q != 3) || nalph != NALPH || nv < 1 || !a || !g || !mat || !c || !fs || !Ls || !fout ||
        !Uout)
        return -1;
    const int nupts = 1, neles = kElems, nvars = nv, ldim = kElems * nv, lda = nupts * neles;
    const size_t nf = size_t(kElems) * nv, nu = size_t(kElems) * NALPH;
    const dim3 block(256), gridf(unsigned((nf + 255) / 256)), gridu(unsigned((lda + 255) / 256));
    std::vector<double> h(nf), hu(nu);
    double *dF[3] = {}, *dL[3] = {}, *dU[3] = {}, *dLU[3] = {}, *dUn = nullptr, *dUt = nullptr, *dM = nullptr,
           *dout = nullptr, *dc = nullptr;
    int rc = 0;
    auto moment = [&](const double* dsrc, double* ddst) -> int {
        int r = ok(cudaMemcpy(h.data(), dsrc, nf * sizeof(double), cudaMemcpyDeviceToHost));
        if (r) return r;
        for (int e = 0; e < kElems; ++e)
            for (int k = 0; k < NALPH; ++k) {
                double acc = 0.0;
                for (int v = 0; v < nv; ++v) acc += h[size_t(v) * kElems + e] * mat[size_t(k) * nv + v];
                hu[size_t(e) * NALPH + k] = acc;
            }
        return ok(cudaMemcpy(ddst, hu.data(), nu * sizeof(double), cudaMemcpyHostToDevice));
    };
    auto upload = [&](const double* src, double* ddst) -> int {
        for (int e = 0; e < kElems; ++e)
            for (int v = 0; v < nv; ++v) h[size_t(v) * kElems + e] = src[size_t(e) * nv + v];
        return ok(cudaMemcpy(ddst, h.data(), nf * sizeof(double), cudaMemcpyHostToDevice));
    };
    do {
        for (int i = 0; i < q && !rc; ++i) {
            rc = ok(cudaMalloc(&dF[i], nf * sizeof(double)));
            if (!rc) rc = ok(cudaMalloc(&dL[i], nf * sizeof(double)));
            if (!rc) rc = ok(cudaMalloc(&dU[i], nu * sizeof(double)));
            if (!rc) rc = ok(cudaMalloc(&dLU[i], nu * sizeof(double)));
        }
        if (rc) break;
        if ((rc = ok(cudaMalloc(&dUn, nu * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dUt, nu * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dM, nf * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dout, nf * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&dc, 3 * size_t(nv) * sizeof(double))))) break;
        if ((rc = ok(cudaMemcpy(dc, c, 3 * size_t(nv) * sizeof(double), cudaMemcpyHostToDevice)))) break;
        for (int i = 0; i < q && !rc; ++i) {
            if ((rc = upload(fs + size_t(i) * nf, dF[i]))) break;
            if ((rc = upload(Ls + size_t(i) * nf, dL[i]))) break;
            if ((rc = moment(dF[i], dU[i]))) break;
            rc = moment(dL[i], dLU[i]);
        }
        if (rc) break;
        if (q == 2)
            updateMom2_BDF<<<gridu, block>>>(prefac, lda, dt, a[0], dU[0], g[0], dLU[0], a[1], dU[1], g[1], dLU[1],
                                             a[2], dUn, b);
        else
            updateMom3_BDF<<<gridu, block>>>(prefac, lda, dt, a[0], dU[0], g[0], dLU[0], a[1], dU[1], g[1], dLU[1],
                                             a[2], dU[2], g[2], dLU[2], a[3], dUn, b);
#ifdef HAS_MOMENT_NORM
        momentNorm<<<gridu, block>>>(lda, dUn, dUt);
        cmaxwellian<<<gridf, block>>>(nupts, ldim, nvars, neles, dc, dc + nv, dc + 2 * nv, dM, dUt);
#else
        cmaxwellian<<<gridf, block>>>(nupts, ldim, nvars, neles, dc, dc + nv, dc + 2 * nv, dM, dUn);
#endif
        if (q == 2)
            updateDistribution2_BDF<<<gridf, block>>>(prefac, nupts, ldim, nvars, neles, dt, a[0], dF[0], g[0],
                                                      dL[0], a[1], dF[1], g[1], dL[1], b, dM, a[2], dUn, dout);
        else
            updateDistribution3_BDF<<<gridf, block>>>(prefac, nupts, ldim, nvars, neles, dt, a[0], dF[0], g[0],
                                                      dL[0], a[1], dF[1], g[1], dL[1], a[2], dF[2], g[2], dL[2],
                                                      b, dM, a[3], dUn, dout);
        if ((rc = ok(cudaGetLastError()))) break;
        if ((rc = ok(cudaMemcpy(h.data(), dout, nf * sizeof(double), cudaMemcpyDeviceToHost)))) break;
        for (int e = 0; e < kElems; ++e)
            for (int v = 0; v < nv; ++v) fout[size_t(e) * nv + v] = h[size_t(v) * kElems + e];
        rc = ok(cudaMemcpy(Uout, dUn, nu * sizeof(double), cudaMemcpyDeviceToHost));
    } while (false);
    for (int i = 0; i < 3; ++i) {
        cudaFree(dF[i]);
        cudaFree(dL[i]);
        cudaFree(dU[i]);
        cudaFree(dLU[i]);
    }
    cudaFree(dUn);
    cudaFree(dUt);
    cudaFree(dM);
    cudaFree(dout);
    cudaFree(dc);
    return rc;
}
