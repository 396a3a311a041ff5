// Test infrastructure: runs the reference's own vss-gll gas-mixture
// collision kernels (rendered from its Mako template into the file named by
// REF_KERNELS, two species) and cuFFT in the order of the reference's host
// code, for a batch of mixture distributions.  Host sequence restated from
// frfs/solvers/dgfsbi/scattering.py:93-202 (perform_precomputation: integer
// wavenumber grid l, precompute_a, precompute_bc_pq per radius and direction
// with fac, fac_b, fac_c, plans), :203-253 (scratch) and :256-330 (Qij and
// fs: per ordered pair (p, q) r2z of f_p and f_q, forward FFTs,
// cosSinMul_pq, two batched inverse FFTs, prod, batched forward FFT,
// computeQG, inverse FFT, ax2, inverse FFT, output_pq, which assigns Q_p for
// q = 0 and accumulates for q > 0).  Blocks of 256 threads and
// get_grid_for_block's grid, as there.  Each species' distribution is placed
// as element 0, solution point 0 of its own AoSoA bank (SOA_IX with soasz
// 32: velocity v at v*32), as the reference's kernels index it.
#include <cstdio>
#include <cufft.h>
#include <cuda_runtime.h>

#include REF_KERNELS

namespace {

constexpr int kSpecies = 2;

int ok(cudaError_t e)
{
    return e == cudaSuccess ? 0 : -2;
}

int ok(cufftResult e)
{
    return e == CUFFT_SUCCESS ? 0 : -3;
}

using BcFn = void (*)(const int, const int, const scalar, const scalar, const scalar, const int*,
                      const int*, const int*, const scalar*, const scalar*, const scalar*, Cplx*,
                      Cplx*);
using CsFn = void (*)(const scalar*, Cplx*, Cplx*, Cplx*, Cplx*);
using OutFn = void (*)(const int, const int, const int, const int, const int, const int,
                       const Cplx*, const Cplx*, scalar*, scalar*);

// the rendered per-pair kernels, pair (p, q) at p*kSpecies + q
const BcFn kBc[] = {precompute_bc_00, precompute_bc_01, precompute_bc_10, precompute_bc_11};
const CsFn kCs[] = {cosSinMul_00, cosSinMul_01, cosSinMul_10, cosSinMul_11};
const OutFn kOut[] = {output_00, output_01, output_10, output_11};

}  // namespace

// sz: the M full-sphere directions [M][3] (the velocity mesh's sz);
// qz, qw: the radial rule [Nrho]; sw = 4 pi / M; swpre = 4 pi / Mpre;
// gamma: [2][2] (gamma_pq = 2 (1 - omega_pq));
// f, Q: host arrays [ndof][2][Nv^3] (FP64, velocity index (x*Nv + y)*Nv + z).
// Returns 0, or -1 (arguments), -2 (CUDA), -3 (cuFFT).
extern "C" int ref_vss_q(int Nv, int Nrho, int M, int nspcs, int ndof, const double* sz,
                         const double* qz, const double* qw, double L, double sw, double swpre,
                         const double* gamma, const double* f, double* Q)
{
    if (Nv < 2 || Nrho < 1 || M < 1 || nspcs != kSpecies || ndof < 0 || !sz || !qz || !qw ||
        !gamma || !f || !Q)
        return -1;
    const int vsize = Nv * Nv * Nv;
    // computeQG stores outside its idx < vsize guard (vss-gll.mako:248): the
    // grid must cover vsize exactly
    if (vsize % 256) return -1;
    const size_t P = size_t(Nrho) * M;
    const dim3 block(256), grid((vsize + 255) / 256);
    int rc = 0;
    int* lx = nullptr;
    double *d_sz = nullptr, *aa = nullptr, *bank = nullptr;
    Cplx *bb1 = nullptr, *bb2 = nullptr, *FTf = nullptr, *t1 = nullptr;
    cufftHandle plan = 0, planMany = 0;
    bool plans = false;
    double* h_bank = nullptr;
    do {
        // l = l0[I], l0[J], l0[K], l0 = [0 .. N/2-1, -N/2 .. -1] (scattering.py:118-131)
        int* h_l = new int[3 * vsize];
        for (int idv = 0; idv < vsize; ++idv) {
            const int I = idv / (Nv * Nv), J = (idv % (Nv * Nv)) / Nv, K = (idv % (Nv * Nv)) % Nv;
            auto l0 = [&](int i) { return i < Nv / 2 ? i : i - Nv; };
            h_l[idv] = l0(I);
            h_l[vsize + idv] = l0(J);
            h_l[2 * vsize + idv] = l0(K);
        }
        if ((rc = ok(cudaMalloc(&lx, 3 * vsize * sizeof(int))))) { delete[] h_l; break; }
        rc = ok(cudaMemcpy(lx, h_l, 3 * vsize * sizeof(int), cudaMemcpyHostToDevice));
        delete[] h_l;
        if (rc) break;
        const int *ly = lx + vsize, *lz = lx + 2 * vsize;
        // sz split into its x, y, z columns (scattering.py:133-136)
        double* h_sz = new double[3 * M];
        for (int y = 0; y < M; ++y)
            for (int c = 0; c < 3; ++c) h_sz[c * M + y] = sz[3 * y + c];
        if ((rc = ok(cudaMalloc(&d_sz, 3 * M * sizeof(double))))) { delete[] h_sz; break; }
        rc = ok(cudaMemcpy(d_sz, h_sz, 3 * M * sizeof(double), cudaMemcpyHostToDevice));
        delete[] h_sz;
        if (rc) break;
        if ((rc = ok(cudaMalloc(&aa, P * vsize * sizeof(double))))) break;
        const int npairs = kSpecies * kSpecies;
        if ((rc = ok(cudaMalloc(&bb1, npairs * P * vsize * sizeof(Cplx))))) break;
        if ((rc = ok(cudaMalloc(&bb2, npairs * size_t(vsize) * sizeof(Cplx))))) break;
        if ((rc = ok(cudaMemset(bb2, 0, npairs * size_t(vsize) * sizeof(Cplx))))) break;
        // FTf, FTg, f1C, f2C, QG
        if ((rc = ok(cudaMalloc(&FTf, 5 * size_t(vsize) * sizeof(Cplx))))) break;
        Cplx *FTg = FTf + vsize, *f1C = FTg + vsize, *f2C = f1C + vsize, *QG = f2C + vsize;
        if ((rc = ok(cudaMalloc(&t1, 3 * P * vsize * sizeof(Cplx))))) break;
        Cplx *t2 = t1 + P * vsize, *t3 = t2 + P * vsize;
        // one bank per species and one per species' Q
        if ((rc = ok(cudaMalloc(&bank, 2 * kSpecies * size_t(vsize) * 32 * sizeof(double))))) break;
        // plans (scattering.py:138-143)
        int n[3] = {Nv, Nv, Nv};
        if ((rc = ok(cufftPlanMany(&planMany, 3, n, nullptr, 1, vsize, nullptr, 1, vsize, CUFFT_Z2Z,
                                   int(P)))))
            break;
        if ((rc = ok(cufftPlan3d(&plan, Nv, Nv, Nv, CUFFT_Z2Z)))) break;
        plans = true;
        precompute_a<<<grid, block>>>(lx, ly, lz, aa);
        for (int pq = 0; pq < npairs && !rc; ++pq) {
            const double g = gamma[pq];
            for (int x = 0; x < Nrho; ++x) {
                const double fac = M_PI / L * qz[x];
                const double fac_b = swpre * pow(qz[x], g + 2);
                const double fac_c = qw[x] * sw * fac_b;
                for (int y = 0; y < M; ++y)
                    kBc[pq]<<<grid, block>>>(x, y, fac, fac_b, fac_c, lx, ly, lz, d_sz, d_sz + M,
                                             d_sz + 2 * M, bb1 + pq * P * vsize, bb2 + pq * vsize);
            }
            rc = ok(cudaGetLastError());
        }
        if (rc) break;
        // element 0, point 0 of each bank: nrow 1, ldim 0, ncola = vsize
        const int nrow = 1, ldim = 0, ncola = vsize, ncolb = 1, elem = 0, upt = 0;
        const size_t bsz = size_t(vsize) * 32;
        h_bank = new double[bsz];
        for (int d = 0; d < ndof && !rc; ++d) {
            for (int p = 0; p < kSpecies && !rc; ++p) {
                for (int v = 0; v < vsize; ++v)
                    h_bank[size_t(v) * 32] = f[(size_t(d) * kSpecies + p) * vsize + v];
                rc = ok(cudaMemcpy(bank + p * bsz, h_bank, bsz * sizeof(double),
                                   cudaMemcpyHostToDevice));
            }
            for (int p = 0; p < kSpecies && !rc; ++p) {
                for (int q = 0; q < kSpecies && !rc; ++q) {
                    const int pq = p * kSpecies + q;
                    double *fp = bank + p * bsz, *fq = bank + q * bsz,
                           *Qp = bank + (kSpecies + p) * bsz;
                    r2z<<<grid, block>>>(nrow, ldim, ncola, ncolb, elem, upt, fp, f1C);
                    r2z<<<grid, block>>>(nrow, ldim, ncola, ncolb, elem, upt, fq, f2C);
                    if ((rc = ok(cufftExecZ2Z(plan, f1C, FTf, CUFFT_FORWARD)))) break;
                    if ((rc = ok(cufftExecZ2Z(plan, f2C, FTg, CUFFT_FORWARD)))) break;
                    kCs[pq]<<<grid, block>>>(aa, FTf, FTg, t1, t2);
                    if ((rc = ok(cufftExecZ2Z(planMany, t1, t3, CUFFT_INVERSE)))) break;
                    if ((rc = ok(cufftExecZ2Z(planMany, t2, t1, CUFFT_INVERSE)))) break;
                    prod<<<grid, block>>>(t3, t1, t2);
                    if ((rc = ok(cufftExecZ2Z(planMany, t2, t1, CUFFT_FORWARD)))) break;
                    computeQG<<<grid, block>>>(bb1 + pq * P * vsize, t1, f1C);
                    if ((rc = ok(cufftExecZ2Z(plan, f1C, QG, CUFFT_INVERSE)))) break;
                    ax2<<<grid, block>>>(bb2 + pq * vsize, FTg, FTf);
                    if ((rc = ok(cufftExecZ2Z(plan, FTf, f2C, CUFFT_INVERSE)))) break;
                    kOut[pq]<<<grid, block>>>(nrow, ldim, ncola, ncolb, elem, upt, QG, f2C, fp, Qp);
                    rc = ok(cudaGetLastError());
                }
            }
            for (int p = 0; p < kSpecies && !rc; ++p) {
                if ((rc = ok(cudaMemcpy(h_bank, bank + (kSpecies + p) * bsz, bsz * sizeof(double),
                                        cudaMemcpyDeviceToHost))))
                    break;
                for (int v = 0; v < vsize; ++v)
                    Q[(size_t(d) * kSpecies + p) * vsize + v] = h_bank[size_t(v) * 32];
            }
        }
    } while (false);
    delete[] h_bank;
    if (plans) {
        cufftDestroy(plan);
        cufftDestroy(planMany);
    }
    cudaFree(lx);
    cudaFree(d_sz);
    cudaFree(aa);
    cudaFree(bb1);
    cudaFree(bb2);
    cudaFree(FTf);
    cudaFree(t1);
    cudaFree(bank);
    return rc;
}
