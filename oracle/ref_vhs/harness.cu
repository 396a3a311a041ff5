// Test infrastructure: runs the reference's own vhs-gll collision kernels
// (rendered from its Mako template into the file named by REF_KERNELS) and
// cuFFT in the order of the reference's host code, for a batch of
// distributions.  Host sequence restated from
// frfs/solvers/dgfs/scattering.py:67-224 (perform_precomputation: wavenumber
// grid l, precompute_aa / precompute_bb, plans) and :227-286 (fs: r2z,
// forward FFT, cosSinMul, two batched inverse FFTs, magSqr, batched forward
// FFT, computeQG, inverse FFT, ax, inverse FFT, output).  Blocks of 256
// threads and get_grid_for_block's grid, as there.  Each distribution is
// placed as element 0, solution point 0 of an AoSoA bank (SOA_IX with
// soasz 32: velocity v at v*32), as the reference's kernels index it.
#include <cstdio>
#include <cufft.h>
#include <cuda_runtime.h>

#include REF_KERNELS

namespace {

int ok(cudaError_t e)
{
    return e == cudaSuccess ? 0 : -2;
}

int ok(cufftResult e)
{
    return e == CUFFT_SUCCESS ? 0 : -3;
}

}  // namespace

// f, Q: host arrays [ndof][Nv^3] (FP64, velocity index (x*Nv + y)*Nv + z).
// Returns 0, or -1 (arguments), -2 (CUDA), -3 (cuFFT).
extern "C" int ref_vhs_q(int Nv, int Nrho, int M, int ndof, const double* f, double* Q)
{
    if (Nv < 2 || Nrho < 1 || M < 1 || ndof < 0 || !f || !Q) return -1;
    const int vsize = Nv * Nv * Nv;
    // computeQG stores outside its idx < vsize guard (vhs-gll.mako:205): the
    // grid must cover vsize exactly
    if (vsize % 256) return -1;
    const dim3 block(256), grid((vsize + 255) / 256);
    int rc = 0;
    double *lx = nullptr, *ly = nullptr, *lz = nullptr, *aa = nullptr, *bb1 = nullptr, *bb2 = nullptr;
    double *bank_in = nullptr, *bank_out = nullptr;
    Cplx *FTf = nullptr, *fC = nullptr, *QG = nullptr, *t1 = nullptr, *t2 = nullptr, *t3 = nullptr,
         *t4 = nullptr;
    cufftHandle plan = 0, planMany = 0;
    bool plans = false;
    do {
        // l = l0[I], l0[J], l0[K] with l0 = [0 .. N/2-1, -N/2 .. -1] (scattering.py:79-89)
        double* h_l = new double[3 * vsize];
        for (int idv = 0; idv < vsize; ++idv) {
            const int I = idv / (Nv * Nv), J = (idv % (Nv * Nv)) / Nv, K = (idv % (Nv * Nv)) % Nv;
            auto l0 = [&](int i) { return i < Nv / 2 ? double(i) : double(i - Nv); };
            h_l[idv] = l0(I);
            h_l[vsize + idv] = l0(J);
            h_l[2 * vsize + idv] = l0(K);
        }
        const size_t P = size_t(Nrho) * M;
        if ((rc = ok(cudaMalloc(&lx, 3 * vsize * sizeof(double))))) { delete[] h_l; break; }
        ly = lx + vsize;
        lz = ly + vsize;
        rc = ok(cudaMemcpy(lx, h_l, 3 * vsize * sizeof(double), cudaMemcpyHostToDevice));
        delete[] h_l;
        if (rc) break;
        if ((rc = ok(cudaMalloc(&aa, P * vsize * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&bb1, size_t(Nrho) * vsize * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&bb2, vsize * sizeof(double))))) break;
        if ((rc = ok(cudaMalloc(&FTf, 3 * vsize * sizeof(Cplx))))) break;
        fC = FTf + vsize;
        QG = fC + vsize;
        if ((rc = ok(cudaMalloc(&t1, 4 * P * vsize * sizeof(Cplx))))) break;
        t2 = t1 + P * vsize;
        t3 = t2 + P * vsize;
        t4 = t3 + P * vsize;
        if ((rc = ok(cudaMalloc(&bank_in, 2 * size_t(vsize) * 32 * sizeof(double))))) break;
        bank_out = bank_in + size_t(vsize) * 32;
        // plans (scattering.py:146-150)
        int n[3] = {Nv, Nv, Nv};
        if ((rc = ok(cufftPlanMany(&planMany, 3, n, nullptr, 1, vsize, nullptr, 1, vsize, CUFFT_Z2Z,
                                   int(P)))))
            break;
        if ((rc = ok(cufftPlan3d(&plan, Nv, Nv, Nv, CUFFT_Z2Z)))) break;
        plans = true;
        precompute_aa<<<grid, block>>>(lx, ly, lz, aa);
        precompute_bb<<<grid, block>>>(lx, ly, lz, bb1, bb2);
        if ((rc = ok(cudaGetLastError()))) break;
        // element 0, point 0 of the bank: nrow 1, ldim 0, ncola = vsize
        const int nrow = 1, ldim = 0, ncola = vsize, ncolb = 1, elem = 0, upt = 0;
        double* h_bank = new double[size_t(vsize) * 32];
        for (int d = 0; d < ndof && !rc; ++d) {
            for (int v = 0; v < vsize; ++v) h_bank[size_t(v) * 32] = f[size_t(d) * vsize + v];
            if ((rc = ok(cudaMemcpy(bank_in, h_bank, size_t(vsize) * 32 * sizeof(double),
                                    cudaMemcpyHostToDevice))))
                break;
            r2z<<<grid, block>>>(nrow, ldim, ncola, ncolb, elem, upt, bank_in, fC);
            if ((rc = ok(cufftExecZ2Z(plan, fC, FTf, CUFFT_FORWARD)))) break;
            cosSinMul<<<grid, block>>>(aa, FTf, t1, t2);
            if ((rc = ok(cufftExecZ2Z(planMany, t1, t3, CUFFT_INVERSE)))) break;
            if ((rc = ok(cufftExecZ2Z(planMany, t2, t4, CUFFT_INVERSE)))) break;
            magSqr<<<grid, block>>>(t3, t4, t2);
            if ((rc = ok(cufftExecZ2Z(planMany, t2, t1, CUFFT_FORWARD)))) break;
            computeQG<<<grid, block>>>(bb1, t1, fC);
            if ((rc = ok(cufftExecZ2Z(plan, fC, QG, CUFFT_INVERSE)))) break;
            ax<<<grid, block>>>(bb2, FTf);
            if ((rc = ok(cufftExecZ2Z(plan, FTf, fC, CUFFT_INVERSE)))) break;
            output<<<grid, block>>>(nrow, ldim, ncola, ncolb, elem, upt, QG, fC, bank_in, bank_out);
            if ((rc = ok(cudaGetLastError()))) break;
            if ((rc = ok(cudaMemcpy(h_bank, bank_out, size_t(vsize) * 32 * sizeof(double),
                                    cudaMemcpyDeviceToHost))))
                break;
            for (int v = 0; v < vsize; ++v) Q[size_t(d) * vsize + v] = h_bank[size_t(v) * 32];
        }
        delete[] h_bank;
    } while (false);
    if (plans) {
        cufftDestroy(plan);
        cufftDestroy(planMany);
    }
    cudaFree(lx);
    cudaFree(aa);
    cudaFree(bb1);
    cudaFree(bb2);
    cudaFree(FTf);
    cudaFree(t1);
    cudaFree(bank_in);
    return rc;
}
