// Fast-spectral VHS collision operator Q(f, f) for a batch of velocity
// cubes, one persistent launch.
//
// Reference algorithm: DGFSVHSGLLScatteringModel.fs
// (frfs/solvers/dgfs/scattering.py:227-286) with the kernels of
// frfs/solvers/dgfs/kernels/scattering/vhs-gll.mako:103-266.  Per
// distribution it does 3 + 3*M*Nrho complex FFTs through HBM scratch.
//
// This kernel computes the same quantity with M*Nrho + Nrho + 2 FFTs, all
// inside one CTA, with f read from HBM once:
//
//   Fh   = FFT(f) / n                                  (real input, kx <= N/2)
//   for p: S_p = sum_q Re(w_pq^2),  w_pq = IFFT(m_pq * Fh)
//          Gh += gw_p * FFT(S_p)                       (Hermitian half)
//   QG + i*fC = IFFT(Gh + i * bb2 * Fh)
//   Q = prefac * (QG - f * fC)
//
// where m_pq = [cos a + sin a + cos abar - sin abar] / 2, a = a_pq(l),
// abar = a_pq evaluated at the Hermitian partner index of l.  Off the
// Nyquist planes abar = -a and m = cos a + sin a; then
// Re(w^2) = IFFT(cos a Fh)^2 + IFFT(sin a Fh)^2 (the reference's magSqr)
// exactly, because IFFT(cos a Fh) is real and IFFT(sin a Fh) imaginary.  On
// the Nyquist planes the reference's phase is not odd and m keeps the
// first-order terms exactly; the remaining term is second order in the
// Nyquist content (measured <= 2e-6 relative).  Summing over q before the
// forward FFT uses linearity; the final packed inverse uses that Gh and
// bb2*Fh are both Hermitian.
//
// Data layout per CTA: the work cube W[i][j][k] lives in shared memory with
// the innermost dimension padded to N+1 (odd), so that the three pencil
// passes (z: thread per (i,j); y: per (i,k); x: per (j,k)) are free of bank
// conflicts; Fh (kx <= N/2) likewise.  S_p stays in registers (thread owns
// the x-pencil (y,z) in the last pass), Gh accumulates in per-CTA global
// scratch (L2 resident).  For Nv = 32 the complex work cube (256 KiB) does
// not fit in shared memory and W and S_p live in per-CTA global scratch.
#include <cstdio>

#include "common.cuh"
#include "cpx.cuh"
#include "fft_codelets.cuh"
#include "vhs_p2_tables.cuh"
#include "tcgen05.cuh"

namespace bdgfs {

template <typename T>
__device__ __forceinline__ cpx<T> cmul(cpx<T> a, cpx<T> b)
{
    return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename T>
__device__ __forceinline__ cpx<T> conjc(cpx<T> a) { return {a.x, -a.y}; }

// z-pencil (kx, ky) of the spectrum m_pq * Fh (tr = 0), or of the Nyquist
// correction term i * m_s * Fh (tr = 1).  Fh holds kx <= N/2 at innermost
// stride FS; kx > N/2 follows from Hermitian symmetry.  ep: the direction's
// phase factors [Ex | Ey | Ez]; ab[kz] = (Ez.x + Ez.y, Ez.x - Ez.y).
template <typename T, int N, int FS>
__device__ __forceinline__ void pencil_spectrum(int kx, int ky, int tr, const cpx<T>* ep,
                                                const cpx<T>* ab, const cpx<T>* Fh,
                                                cpx<T> (&v)[N])
{
    constexpr int NH = N / 2 + 1;
    const cpx<T> Ex = ep[kx], Ey = ep[N + ky];
    const cpx<T> Pxy = cmul(Ex, Ey);
    const bool direct = kx < NH;
    const int pkx = direct ? kx : N - kx;
    const int pky = direct ? ky : (N - ky) % N;
    const cpx<T>* fp = Fh + (pkx * N + pky) * FS;
    const bool nyq = (kx == N / 2) || (ky == N / 2);
    if (tr == 1) {
        // second-order Nyquist term: spectrum i * m_s * Fh with
        // m_s = [sin a + sin abar - cos a + cos abar] / 2
        const cpx<T> Ebx = (kx == N / 2) ? Ex : conjc(Ex);
        const cpx<T> Eby = (ky == N / 2) ? Ey : conjc(Ey);
        const cpx<T> Pb = cmul(Ebx, Eby);
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            cpx<T> F = direct ? fp[kz] : conjc(fp[(N - kz) % N]);
            const cpx<T> Ez = ep[2 * N + kz];
            const cpx<T> Ebz = (kz == N / 2) ? Ez : conjc(Ez);
            const cpx<T> E = cmul(Pxy, Ez);
            const cpx<T> Eb = cmul(Pb, Ebz);
            const T ms = T(0.5) * (E.y + Eb.y - E.x + Eb.x);
            v[kz] = {-ms * F.y, ms * F.x};
        }
    } else if (!nyq) {
        // off the Nyquist planes m = Re(E) + Im(E), E = Pxy * Ez,
        // = Pxy.x (Ez.x + Ez.y) + Pxy.y (Ez.x - Ez.y)
        const cpx<T> Pb = conjc(Pxy);
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            cpx<T> F = direct ? fp[kz] : conjc(fp[(N - kz) % N]);
            T m;
            if (kz == N / 2) {
                const cpx<T> Ez = ep[2 * N + kz];
                const cpx<T> E = cmul(Pxy, Ez);
                const cpx<T> Eb = cmul(Pb, Ez);
                m = T(0.5) * (E.x + E.y + Eb.x - Eb.y);
            } else {
                const cpx<T> w = ab[kz];
                m = Pxy.x * w.x + Pxy.y * w.y;
            }
            v[kz] = {m * F.x, m * F.y};
        }
    } else {
        const cpx<T> Ebx = (kx == N / 2) ? Ex : conjc(Ex);
        const cpx<T> Eby = (ky == N / 2) ? Ey : conjc(Ey);
        const cpx<T> Pb = cmul(Ebx, Eby);
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            cpx<T> F = direct ? fp[kz] : conjc(fp[(N - kz) % N]);
            const cpx<T> Ez = ep[2 * N + kz];
            const cpx<T> Ebz = (kz == N / 2) ? Ez : conjc(Ez);
            const cpx<T> E = cmul(Pxy, Ez);
            const cpx<T> Eb = cmul(Pb, Ebz);
            const T m = T(0.5) * (E.x + E.y + Eb.x - Eb.y);
            v[kz] = {m * F.x, m * F.y};
        }
    }
}

template <typename T, int N, int NT, bool WG, bool SG, bool SL = false>
struct QLayout {
    static constexpr int NH = N / 2 + 1;
    static constexpr int n = N * N * N;
    static constexpr int WS = WG ? N : N + 1;   // innermost stride of W
    static constexpr int FS = N + 1;            // innermost stride of Fh
    static constexpr size_t w_elems = size_t(N) * N * WS;
    static constexpr size_t fh_elems = size_t(NH) * N * FS;
    static constexpr size_t slab_elems = SL ? size_t(NT / 32) * N * (N + 1) : 0;
    // shared memory: [W (if smem)] [Fh] [phase M*3*N] [phab M*N] [warp slabs]
    // [reduction]
    static size_t smem_bytes(int M)
    {
        size_t b = 0;
        if (!WG) b += w_elems * sizeof(cpx<T>);
        b += fh_elems * sizeof(cpx<T>);
        b += size_t(M) * 3 * N * sizeof(cpx<T>);
        b += size_t(M) * N * sizeof(cpx<T>);      // (Ez.x + Ez.y, Ez.x - Ez.y) per direction
        b += slab_elems * sizeof(cpx<T>);
        b += 10 * (NT / 32) * sizeof(double) + 16;
        return b;
    }
    // global scratch per CTA: [Gh N*NH*N] [W N^3 (if WG)] [S N^3 (if SG)]
    static size_t scratch_bytes()
    {
        size_t b = size_t(N) * NH * N * sizeof(cpx<T>);
        if (WG) b += size_t(n) * sizeof(cpx<T>);
        if (SG) b += size_t(n) * sizeof(T);
        return (b + 255) & ~size_t(255);
    }
};

// GR > 0: the z- and y-passes of each inverse transform are done by GR
// groups of NT/GR threads, group g owning the kx-slabs [g*N/GR, (g+1)*N/GR);
// the two passes then only synchronise within the group (named barrier).
// SL (W in global scratch, N = 32): warp w owns the kx-slabs w, w + NT/32, ...
// of each inverse transform and does their z- and y-passes in a private
// shared-memory slab (lane = pencil, no CTA barrier); only the finished slab
// goes to the global W, which the x-pass then reads.  Per transform the
// global traffic is one write and one read of W instead of two of each.
template <typename T, int N, int NT, bool WG, bool SG, int GR = 0, bool SL = false>
__device__ void collide_one(const bdgfs_vhs_grid& g, const T* __restrict__ f,
                            T* __restrict__ Qout, double* mom, int flags,
                            unsigned char* smem, unsigned char* scratch)
{
    const int project = flags & BDGFS_PROJECT;
    const int ntr = (flags & BDGFS_EXACT) ? 2 : 1;
    using L = QLayout<T, N, NT, WG, SG, SL>;
    static_assert(!SL || (WG && N == 32 && GR == 0), "warp slabs: W in global scratch, N = 32");
    constexpr int NH = L::NH;
    constexpr int WS = L::WS;
    constexpr int FS = L::FS;
    constexpr int NP = N * N;                 // pencils per pass
    constexpr int NPT = (NP + NT - 1) / NT;   // pencils per thread
    // register S_p: thread tid owns x-pencils tid + r*NT (r < NPT; the last
    // round is partial when NT does not divide N*N)
    const int tid = threadIdx.x;
    const int M = g.M, Nrho = g.Nrho;

    // ---- carve shared memory and scratch ----
    unsigned char* sp = smem;
    cpx<T>* Ws;
    if constexpr (!WG) {
        Ws = reinterpret_cast<cpx<T>*>(sp);
        sp += L::w_elems * sizeof(cpx<T>);
    }
    cpx<T>* Fh = reinterpret_cast<cpx<T>*>(sp);
    sp += L::fh_elems * sizeof(cpx<T>);
    cpx<T>* ph = reinterpret_cast<cpx<T>*>(sp);
    sp += size_t(M) * 3 * N * sizeof(cpx<T>);
    cpx<T>* phab = reinterpret_cast<cpx<T>*>(sp);       // [q][kz]: (Ez.x + Ez.y, Ez.x - Ez.y)
    sp += size_t(M) * N * sizeof(cpx<T>);
    cpx<T>* slab = reinterpret_cast<cpx<T>*>(sp);       // [warp][ky][z], stride N+1
    sp += L::slab_elems * sizeof(cpx<T>);
    (void)slab;
    double* red = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(sp) + 15) & ~uintptr_t(15));

    cpx<T>* Gh = reinterpret_cast<cpx<T>*>(scratch);   // [kz][kx<NH][ky]
    unsigned char* gp = scratch + size_t(N) * NH * N * sizeof(cpx<T>);
    cpx<T>* W;
    if constexpr (WG) {
        W = reinterpret_cast<cpx<T>*>(gp);
        gp += size_t(L::n) * sizeof(cpx<T>);
    } else {
        W = Ws;
    }
    T* Sg = reinterpret_cast<T*>(gp);                    // [x][y][z] if SG
    (void)Sg;

    auto widx = [](int i, int j, int k) { return (i * N + j) * WS + k; };
    // pencil mapping of the first two inverse passes (kx-major pencils)
    static_assert(GR == 0 || (N % GR == 0 && NT % GR == 0 && (NT / GR) % 32 == 0
                              && ((N / GR) * N) % (NT / GR) == 0), "bad slab groups");
    constexpr int TG = GR ? NT / GR : NT;
    constexpr int P12 = GR ? (N / GR) * N / TG : (NP + NT - 1) / NT;
    const int grp = GR ? tid / TG : 0, lt = GR ? tid % TG : tid;
    auto pencil12 = [&](int r, int& a, int& b) -> bool {
        const int pl = lt + r * TG;
        if (GR) {
            a = grp * (N / (GR ? GR : 1)) + pl / N;
            b = pl % N;
            return true;
        }
        if (pl >= NP) return false;
        a = pl / N;
        b = pl % N;
        return true;
    };
    auto sync12 = [&]() {
        if constexpr (GR > 0)
            asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(TG) : "memory");
        else
            __syncthreads();
    };
    const T inv_n = T(1) / T(L::n);

    // ---- Fh = FFT(f) / n, stored for kx <= N/2 ----
    for (int pid = tid; pid < NP; pid += NT) {           // x-pass, real input
        const int y = pid / N, z = pid % N;
        cpx<T> v[N];
#pragma unroll
        for (int x = 0; x < N; ++x) v[x] = {f[(x * N + y) * N + z], T(0)};
        dft<N, -1>(v);
#pragma unroll
        for (int kx = 0; kx < NH; ++kx) W[widx(kx, y, z)] = v[kx];
    }
    __syncthreads();
    for (int pid = tid; pid < NH * N; pid += NT) {       // y-pass
        const int kx = pid / N, z = pid % N;
        cpx<T> v[N];
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] = W[widx(kx, j, z)];
        dft<N, -1>(v);
#pragma unroll
        for (int j = 0; j < N; ++j) W[widx(kx, j, z)] = v[j];
    }
    __syncthreads();
    for (int pid = tid; pid < NH * N; pid += NT) {       // z-pass -> Fh
        const int kx = pid / N, ky = pid % N;
        cpx<T> v[N];
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = W[widx(kx, ky, k)];
        dft<N, -1>(v);
#pragma unroll
        for (int k = 0; k < N; ++k)
            Fh[(kx * N + ky) * FS + k] = {v[k].x * inv_n, v[k].y * inv_n};
    }
    // (the first phase staging below is followed by a barrier)

    const cpx<T>* phase = static_cast<const cpx<T>*>(g.phase);
    const T* gw = static_cast<const T*>(g.gw);

    T S[SG ? 1 : NPT][SG ? 1 : N];
    if constexpr (!SG) {
#pragma unroll
        for (int r = 0; r < NPT; ++r)
#pragma unroll
            for (int x = 0; x < N; ++x) S[r][x] = T(0);
    }

    for (int p = 0; p < Nrho; ++p) {
        for (int e = tid; e < M * 3 * N; e += NT) {
            const cpx<T> v = phase[size_t(p) * M * 3 * N + e];
            ph[e] = v;
            const int q = e / (3 * N), r = e - q * 3 * N;
            if (r >= 2 * N) phab[q * N + (r - 2 * N)] = {v.x + v.y, v.x - v.y};
        }
        __syncthreads();

        for (int qt = 0; qt < M * ntr; ++qt) {
            const int q = qt / ntr, tr = qt % ntr;   // tr = 1: Nyquist term
            const cpx<T>* ep = ph + q * 3 * N;
            if constexpr (SL) {
                // ---- passes 1 and 2 per kx-slab in the warp's shared slab ----
                const int lane = tid & 31;
                cpx<T>* sl = slab + (tid >> 5) * N * (N + 1);
#pragma unroll 1
                for (int kx = tid >> 5; kx < N; kx += NT / 32) {
                    cpx<T> v[N];
                    pencil_spectrum<T, N, FS>(kx, lane, tr, ep, phab + q * N, Fh, v);
                    dft<N, +1>(v);
#pragma unroll
                    for (int z = 0; z < N; ++z) sl[lane * (N + 1) + z] = v[z];
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < N; ++j) v[j] = sl[j * (N + 1) + lane];
                    dft<N, +1>(v);
#pragma unroll
                    for (int j = 0; j < N; ++j) W[widx(kx, j, lane)] = v[j];
                    __syncwarp();
                }
            } else {
                // ---- pass 1: spectrum * m_pq, inverse along z ----
#pragma unroll 1
                for (int r = 0; r < P12; ++r) {
                    int kx, ky;
                    if (!pencil12(r, kx, ky)) break;
                    cpx<T> v[N];
                    pencil_spectrum<T, N, FS>(kx, ky, tr, ep, phab + q * N, Fh, v);
                    dft<N, +1>(v);
#pragma unroll
                    for (int z = 0; z < N; ++z) W[widx(kx, ky, z)] = v[z];
                }
                sync12();
                // ---- pass 2: inverse along y ----
#pragma unroll 1
                for (int r = 0; r < P12; ++r) {
                    int kx, z;
                    if (!pencil12(r, kx, z)) break;
                    cpx<T> v[N];
#pragma unroll
                    for (int j = 0; j < N; ++j) v[j] = W[widx(kx, j, z)];
                    dft<N, +1>(v);
#pragma unroll
                    for (int j = 0; j < N; ++j) W[widx(kx, j, z)] = v[j];
                }
            }
            __syncthreads();
            // ---- pass 3: inverse along x, S_p += Re(w^2) ----
            if constexpr (SG) {
                for (int pid = tid; pid < NP; pid += NT) {
                    const int y = pid / N, z = pid % N;
                    cpx<T> v[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) v[i] = W[widx(i, y, z)];
                    dft<N, +1>(v);
                    const T sgn = tr ? T(-1) : T(1);
#pragma unroll
                    for (int x = 0; x < N; ++x) {
                        T& s = Sg[(x * N + y) * N + z];
                        const T t = sgn * (v[x].x * v[x].x - v[x].y * v[x].y);
                        s = (qt == 0) ? t : s + t;
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < NPT; ++r) {
                    const int pid = tid + r * NT;
                    if (NP % NT != 0 && pid >= NP) break;
                    const int y = pid / N, z = pid % N;
                    cpx<T> v[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) v[i] = W[widx(i, y, z)];
                    dft<N, +1>(v);
                    if (tr == 0) {
#pragma unroll
                        for (int x = 0; x < N; ++x)
                            S[r][x] += v[x].x * v[x].x - v[x].y * v[x].y;
                    } else {
#pragma unroll
                        for (int x = 0; x < N; ++x)
                            S[r][x] -= v[x].x * v[x].x - v[x].y * v[x].y;
                    }
                }
            }
            __syncthreads();
        }

        // ---- Gh += gw_p * FFT(S_p) (Hermitian half kx <= N/2) ----
        if constexpr (SG) {
            for (int pid = tid; pid < NP; pid += NT) {   // x-pass, real input
                const int y = pid / N, z = pid % N;
                cpx<T> v[N];
#pragma unroll
                for (int x = 0; x < N; ++x) v[x] = {Sg[(x * N + y) * N + z], T(0)};
                dft<N, -1>(v);
#pragma unroll
                for (int kx = 0; kx < NH; ++kx) W[widx(kx, y, z)] = v[kx];
            }
        } else {
#pragma unroll
            for (int r = 0; r < NPT; ++r) {
                const int pid = tid + r * NT;
                if (NP % NT != 0 && pid >= NP) break;
                const int y = pid / N, z = pid % N;
                cpx<T> v[N];
#pragma unroll
                for (int x = 0; x < N; ++x) { v[x] = {S[r][x], T(0)}; S[r][x] = T(0); }
                dft<N, -1>(v);
#pragma unroll
                for (int kx = 0; kx < NH; ++kx) W[widx(kx, y, z)] = v[kx];
            }
        }
        __syncthreads();
        for (int pid = tid; pid < NH * N; pid += NT) {   // y-pass
            const int kx = pid / N, z = pid % N;
            cpx<T> v[N];
#pragma unroll
            for (int j = 0; j < N; ++j) v[j] = W[widx(kx, j, z)];
            dft<N, -1>(v);
#pragma unroll
            for (int j = 0; j < N; ++j) W[widx(kx, j, z)] = v[j];
        }
        __syncthreads();
        for (int pid = tid; pid < NH * N; pid += NT) {   // z-pass, accumulate
            const int kx = pid / N, ky = pid % N;
            cpx<T> v[N];
#pragma unroll
            for (int k = 0; k < N; ++k) v[k] = W[widx(kx, ky, k)];
            dft<N, -1>(v);
            const T* gwp = gw + size_t(p) * N * NH * N + kx * N + ky;
#pragma unroll
            for (int kz = 0; kz < N; ++kz) {
                const T w = ldg(gwp + kz * NH * N);
                cpx<T>& G = Gh[(kz * NH + kx) * N + ky];
                if (p == 0) G = {w * v[kz].x, w * v[kz].y};
                else G = {G.x + w * v[kz].x, G.y + w * v[kz].y};
            }
        }
        // the next iteration's phase staging ends with a barrier
    }
    __syncthreads();

    // ---- QG + i*fC = IFFT(Gh + i*bb2*Fh) ----
    const T* bb2 = static_cast<const T*>(g.bb2);
    for (int pid = tid; pid < NP; pid += NT) {
        const int kx = pid / N, ky = pid % N;
        const bool direct = kx < NH;
        const int pkx = direct ? kx : N - kx;
        const int pky = direct ? ky : (N - ky) % N;
        const cpx<T>* fp = Fh + (pkx * N + pky) * FS;
        cpx<T> v[N];
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            const int pkz = direct ? kz : (N - kz) % N;
            cpx<T> G = Gh[(pkz * NH + pkx) * N + pky];
            cpx<T> F = fp[pkz];
            if (!direct) { G.y = -G.y; F.y = -F.y; }
            const T b = ldg(bb2 + (kz * N + kx) * N + ky);
            v[kz] = {G.x - b * F.y, G.y + b * F.x};
        }
        dft<N, +1>(v);
#pragma unroll
        for (int z = 0; z < N; ++z) W[widx(kx, ky, z)] = v[z];
    }
    __syncthreads();
    for (int pid = tid; pid < NP; pid += NT) {
        const int kx = pid / N, z = pid % N;
        cpx<T> v[N];
#pragma unroll
        for (int j = 0; j < N; ++j) v[j] = W[widx(kx, j, z)];
        dft<N, +1>(v);
#pragma unroll
        for (int j = 0; j < N; ++j) W[widx(kx, j, z)] = v[j];
    }
    __syncthreads();

    const T prefac = T(g.prefac);
    const bool need_m = project || mom;
    T* Qs = reinterpret_cast<T*>(Fh);          // Fh is free from here on
    double m[5] = {0, 0, 0, 0, 0};
    for (int pid = tid; pid < NP; pid += NT) {
        const int y = pid / N, z = pid % N;
        cpx<T> v[N];
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = W[widx(i, y, z)];
        dft<N, +1>(v);
        const double cy = need_m ? g.c0[y] : 0.0, cz = need_m ? g.c0[z] : 0.0;
#pragma unroll
        for (int x = 0; x < N; ++x) {
            const int idx = (x * N + y) * N + z;
            const T qv = prefac * (v[x].x - f[idx] * v[x].y);
            if (project) {
                Qs[idx] = qv;
            } else {
                __stcs(Qout + idx, qv);           // streaming: keep L2 for the scratch
            }
            if (need_m) {
                const double cx = g.c0[x], dq = double(qv);
                m[0] += dq;
                m[1] += cx * dq;
                m[2] += cy * dq;
                m[3] += cz * dq;
                m[4] += (cx * cx + cy * cy + cz * cz) * dq;
            }
        }
    }
    if (!need_m) return;
    block_sum<5>(m, red);
    double m2[5] = {0, 0, 0, 0, 0};
    if (project) {
        double lam[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 5; ++j) s += g.ginv[i * 5 + j] * m[j];
            lam[i] = s;
        }
        for (int pid = tid; pid < NP; pid += NT) {
            const int y = pid / N, z = pid % N;
            const double cy = g.c0[y], cz = g.c0[z];
            for (int x = 0; x < N; ++x) {
                const int idx = (x * N + y) * N + z;
                const double cx = g.c0[x];
                const double c2 = cx * cx + cy * cy + cz * cz;
                const double qc = double(Qs[idx]) - (lam[0] + lam[1] * cx + lam[2] * cy
                                                     + lam[3] * cz + lam[4] * c2);
                __stcs(Qout + idx, T(qc));
                m2[0] += qc;
                m2[1] += cx * qc;
                m2[2] += cy * qc;
                m2[3] += cz * qc;
                m2[4] += c2 * qc;
            }
        }
        if (mom) block_sum<5>(m2, red);
    }
    if (mom && tid == 0) {
        for (int j = 0; j < 5; ++j) {
            mom[j] = m[j] * g.cw;
            mom[5 + j] = project ? m2[j] * g.cw : m[j] * g.cw;
        }
    }
    __syncthreads();   // Qs/red reuse by the next distribution
}

// ---------------------------------------------------------------------------
// Packed variant, Nv = 24, FP32, 288 threads.
//
// Every thread carries two pencils through each pass as float2 pairs: re[k]
// holds the real parts of both pencils' k-th element, im[k] the imaginary
// parts, and the DFT codelets (dft_p2) issue one sm_100 f32x2 instruction
// per operation on both pencils.  The FP32 pipe does the same work as with
// scalar code; the instruction stream halves.  576 pencils per pass are
// exactly 288 pairs (no idle second round), and the work cube lives as two
// float planes Wr/Wi (element (i, j, k) at i*PS + j*RS + k), so that the y-
// and x-passes, which pair pencils along k, load and store 8-byte pairs.
//
// z-passes (first pass of each inverse transform, the spectrum built from
// the Hermitian half Fh) pair pencil A = (kx, ky), kx <= N/2, with its
// conjugate partner B = (N - kx, N - ky): F_B(kz) = conj(F_A(N - kz)), so one
// Fh pencil feeds both.  The multiplier of either pencil, Nyquist planes
// included, is m(kz) = al*Ez.x + be*Ez.y (be2 at kz = N/2), with per-pencil
// al, be, be2 from Ex(kx), Ey(ky) and their Hermitian-partner counterparts:
// no per-pencil branches.  Lane tables (vhs_p2_tables.cuh) order the pencil
// pairs so that shared-memory accesses spread over the banks.
//
// S_p (48 floats per thread) lives in tensor memory: with 9 warps per CTA
// three share an SM sub-partition, which caps registers at 168, and the
// x-pass needs 96 for its two pencils.  Warp w owns TMEM lanes
// 32*(w%4).. and columns 48*(w/4).. of a 256-column allocation; the
// spectra-in-TMEM variant allocates 512 columns and keeps the z-pass
// spectra in the upper 256 (see collide_one_p2).
namespace p2 {
constexpr int N = p2tab::N, NH = N / 2 + 1, NP2 = N / 2, NT = 288;
constexpr uint32_t TMEM_COLS = 256;
static_assert(2 * N * ((NT / 32 + 3) / 4) <= int(TMEM_COLS), "TMEM columns");
constexpr int PS = p2tab::PS, RS = p2tab::RS, FS = p2tab::FS;
constexpr int WF = N * PS;                      // floats per plane set
static_assert(NT == N * NP2 && PS >= N * RS && PS % 2 == 0 && RS % 2 == 0, "packed layout");
}  // namespace p2

struct QLayoutP2 {
    static size_t smem_bytes(int M)
    {
        size_t b = 2 * size_t(p2::WF) * sizeof(float);                     // Wr, Wi
        b += size_t(p2::NH) * p2::N * p2::FS * sizeof(cpx<float>);        // Fh
        b += size_t(M) * 3 * p2::N * sizeof(cpx<float>);                  // phase
        b += size_t(M) * p2::N * sizeof(float4);                          // (Ez.x, Ez.x, Ez.y, Ez.y)
        b += 10 * 10 * sizeof(double) + 16;                                // up to 10 warps
        return b;
    }
    // global scratch per CTA: Gh as two float planes [kz][kx <= N/2][ky]
    static size_t scratch_bytes()
    {
        const size_t b = 2 * size_t(p2::N) * p2::NH * p2::N * sizeof(float);
        return (b + 255) & ~size_t(255);
    }
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, float2 v) { *reinterpret_cast<float2*>(p) = v; }

// Multiplier coefficients of pencil (kx, ky) for direction phases ep:
// m(kz) = a*Ez.x + b*Ez.y (kz != N/2), a*Ez.x + b2*Ez.y (kz = N/2); tr = 1
// gives those of the Nyquist correction term m_s.  Derived from
// m = [E.x + E.y + Eb.x - Eb.y]/2, m_s = [E.y + Eb.y - E.x + Eb.x]/2 with
// E = Ex Ey Ez and Eb the same product at the Hermitian-partner wavenumber.
__device__ __forceinline__ void p2_coef(const cpx<float>* ep, int kx, int ky, int tr, float& a,
                                        float& b, float& b2)
{
    constexpr int N = p2::N;
    const cpx<float> Ex = ep[kx], Ey = ep[N + ky];
    const cpx<float> P = cmul(Ex, Ey);
    const cpx<float> Pb = cmul(kx == N / 2 ? Ex : conjc(Ex), ky == N / 2 ? Ey : conjc(Ey));
    if (tr == 0) {
        a = 0.5f * ((P.x + P.y) + (Pb.x - Pb.y));
        b = 0.5f * ((P.x - P.y) + (Pb.x + Pb.y));
        b2 = 0.5f * ((P.x - P.y) - (Pb.x + Pb.y));
    } else {
        a = 0.5f * ((P.y - P.x) + (Pb.x + Pb.y));
        b = 0.5f * ((P.x + P.y) + (Pb.y - Pb.x));
        b2 = 0.5f * ((P.x + P.y) + (Pb.x - Pb.y));
    }
}

// Spectrum of the pencil pair at kz for multipliers m = (m_A, m_B):
// m * F (tr = 0) or i * m * F (tr = 1).
__device__ __forceinline__ void p2_spec(int tr, float2 m, cpx<float> FA, cpx<float> FB, float2& vr,
                                        float2& vi)
{
    if (tr == 0) {
        vr = f2(m.x * FA.x, m.y * FB.x);
        vi = f2(m.x * FA.y, m.y * FB.y);
    } else {
        vr = f2(-m.x * FA.y, -m.y * FB.y);
        vi = f2(m.x * FA.x, m.y * FB.x);
    }
}

// z-pass spectrum of the thread's pencil pair; SINGLES: some lanes of this
// warp own two self-conjugate pencils (B read from its own Fh pencil).
template <bool SINGLES>
__device__ __forceinline__ void p2_pass1_spectrum(int tr, const float4* ez, float2 al, float2 be,
                                                  float2 be2, const cpx<float>* fa,
                                                  const cpx<float>* fb, bool single,
                                                  float2 (&vr)[p2::N], float2 (&vi)[p2::N])
{
    constexpr int N = p2::N;
    auto mval = [&](int kz) {
        const float4 e = ez[kz];
        return __ffma2_rn(al, f2(e.x, e.y), __fmul2_rn(kz == N / 2 ? be2 : be, f2(e.z, e.w)));
    };
#pragma unroll
    for (int kz = 0; kz <= N / 2; ++kz) {
        const int kn = (N - kz) % N;
        const cpx<float> F0 = fa[kz], F1 = fa[kn];
        cpx<float> B0 = conjc(F1), B1 = conjc(F0);
        if constexpr (SINGLES) {
            if (single) {
                B0 = fb[kz];
                B1 = fb[kn];
            }
        }
        p2_spec(tr, mval(kz), F0, B0, vr[kz], vi[kz]);
        if (kn != kz) p2_spec(tr, mval(kn), F1, B1, vr[kn], vi[kn]);
    }
}

// p2_pass1_spectrum from tensor memory: the thread's pencil spectra A[kz]
// (columns ft..ft+47, re/im interleaved) and B[kz] (ft+48..ft+95): the
// same values p2_pass1_spectrum reads from Fh (B = the conjugate partner,
// or the own pencil of a self-conjugate pair) and the same operations; the
// result agrees to rounding (the compiler may contract the spectrum
// products into the DFT's first additions differently).
__device__ __forceinline__ void p2_pass1_spectrum_tm(int tr, const float4* ez, float2 al, float2 be,
                                                     float2 be2, uint32_t ft, float2 (&vr)[p2::N],
                                                     float2 (&vi)[p2::N])
{
    constexpr int N = p2::N;
#pragma unroll
    for (int c = 0; c < N / 8; ++c) {
        uint32_t ra[16], rb[16];
        tc::tmem_ld16_issue(ft + 16 * c, ra);
        tc::tmem_ld16_issue(ft + 48 + 16 * c, rb);
        tc::tmem_wait();
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int kz = 8 * c + k;
            const float4 e = ez[kz];
            const float2 m = __ffma2_rn(al, f2(e.x, e.y), __fmul2_rn(kz == N / 2 ? be2 : be, f2(e.z, e.w)));
            const cpx<float> A = {__uint_as_float(ra[2 * k]), __uint_as_float(ra[2 * k + 1])};
            const cpx<float> B = {__uint_as_float(rb[2 * k]), __uint_as_float(rb[2 * k + 1])};
            p2_spec(tr, m, A, B, vr[kz], vi[kz]);
        }
    }
}

// SPLIT: the barrier that frees the work cube after the x-pass loads is an
// mbarrier (arrive right after the loads, wait just before the next z-pass
// stores), so the x-pass DFT, the S_p update and the next z-pass spectrum and
// DFT of a warp overlap the other warps' loads instead of waiting at a CTA
// barrier; two CTA barriers per transform remain (z stored, y stored).
// wfree: that mbarrier (NT arrivals per phase), wpar: this thread's phase
// parity, counter: the work counter, whose bit 62 a timed-out wait sets.
// BAL (with SPLIT, 320 threads): in the transform loop warps 0-7 carry the
// pencil pairs 0..255 on f32x2 arithmetic and warps 8-9 the remaining 32
// pairs as 64 single pencils on scalar arithmetic (thread 256 + 2e + s:
// pencil s of pair 256 + e).  With 9 pair-warps one SM sub-partition runs
// three of them and the others two, so its FP32 pipe bounds the kernel at
// 3/4 of the SM's; here the sub-partitions carry 5, 5, 4 and 4 pipe units
// of work (a pair warp 2, a scalar warp 1): a bound of 9/10.  The other
// stages run on threads 0..287 as without BAL.
template <bool SPLIT, bool BAL = false, bool FHT = false>
__device__ void collide_one_p2(const bdgfs_vhs_grid& g, const float* __restrict__ f,
                               float* __restrict__ Qout, double* mom, int flags,
                               unsigned char* smem, unsigned char* scratch, uint32_t tmem,
                               uint64_t* wfree, uint32_t& wpar, unsigned long long* counter)
{
    using namespace p2;
    const int project = flags & BDGFS_PROJECT;
    const int ntr = (flags & BDGFS_EXACT) ? 2 : 1;
    const int tid = threadIdx.x, M = g.M, Nrho = g.Nrho;

    float* Wr = reinterpret_cast<float*>(smem);
    float* Wi = Wr + WF;
    cpx<float>* Fh = reinterpret_cast<cpx<float>*>(Wi + WF);
    cpx<float>* ph = Fh + NH * N * FS;
    float4* ezz = reinterpret_cast<float4*>(ph + M * 3 * N);
    double* red = reinterpret_cast<double*>(ezz + M * N);
    float* Ghr = reinterpret_cast<float*>(scratch);       // [kz][kx <= N/2][ky]
    float* Ghi = Ghr + N * NH * N;

    // lane tables: z-pass pencil pair, y-pass pair (natural), x-pass pair
    // (threads beyond the 288 pairs -- BAL -- read the last entry and take
    // no part in the stages that use them)
    const int te = tid < NT ? tid : NT - 1;
    const bool pt = tid < NT;                              // a pair thread outside the loop
    const int kxA = p2tab::zpen[te][0], kyA = p2tab::zpen[te][1];
    const int kxB = p2tab::zpen[te][2], kyB = p2tab::zpen[te][3];
    const bool single = tid == p2tab::SINGLE_AT || tid == p2tab::SINGLE_AT + 1;
    const bool single_warp = (tid >> 5) == p2tab::SINGLE_AT / 32;
    static_assert(p2tab::SINGLE_AT % 32 < 31, "self-conjugate pairs in one warp");
    const int offA = kxA * PS + kyA * RS, offB = kxB * PS + kyB * RS;
    const cpx<float>* fa = Fh + (kxA * N + kyA) * FS;
    const cpx<float>* fb = Fh + (kxB < NH ? kxB * N + kyB : 0) * FS;
    const int ybase = (te / NP2) * PS + 2 * (te % NP2);        // + j*RS
    const int xbase = p2tab::xpen[te][0] * RS + 2 * p2tab::xpen[te][1];     // + i*PS
    // BAL: the transform loop's single-pencil threads
    static_assert(!BAL || SPLIT, "balanced split needs the split barrier");
    static_assert(p2tab::SINGLE_AT + 1 < 256, "self-conjugate pairs among the pair threads");
    const bool sc = BAL && tid >= 256;                      // single-pencil thread
    const int es = sc ? 256 + ((tid - 256) >> 1) : 0, ss = sc ? ((tid - 256) & 1) : 0;
    const int s_kx = ss ? p2tab::zpen[es][2] : p2tab::zpen[es][0];
    const int s_ky = ss ? p2tab::zpen[es][3] : p2tab::zpen[es][1];
    const int s_off = s_kx * PS + s_ky * RS;
    const cpx<float>* s_fa = Fh + (p2tab::zpen[es][0] * N + p2tab::zpen[es][1]) * FS;
    const int s_ybase = (es / NP2) * PS + 2 * (es % NP2) + ss;
    const int s_xbase = p2tab::xpen[es][0] * RS + 2 * p2tab::xpen[es][1] + ss;
    const bool lp = !BAL || tid < 256;                      // a pair thread in the loop
    const float inv_n = 1.f / float(N * N * N);
    const int warp = tid >> 5;
    const uint32_t ts = tmem + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(2 * N * (warp >> 2));
    // FHT: the z-pass spectra in the upper 256 columns: pair warps 96 columns
    // each (A and B), the single-pencil warps 48
    static_assert(!FHT || (SPLIT && BAL), "spectra in tensor memory with the balanced split variant");
    const uint32_t ft = tmem + (uint32_t(32 * (warp & 3)) << 16) +
                        (lp ? TMEM_COLS + uint32_t(4 * N * (warp >> 2)) : TMEM_COLS + uint32_t(8 * N));

    // ---- Fh = FFT(f) / n (kx <= N/2) ----
    if (pt) {
        const int y = tid / NP2, z = 2 * (tid % NP2);      // x-pass, real input
        float2 vr[N], vi[N];
#pragma unroll
        for (int x = 0; x < N; ++x) {
            const float* fp = f + (x * N + y) * N + z;
            vr[x] = f2(fp[0], fp[1]);
            vi[x] = f2(0.f, 0.f);
        }
        dft_p2<N, -1>(vr, vi);
#pragma unroll
        for (int kx = 0; kx < NH; ++kx) {
            st2(Wr + kx * PS + y * RS + z, vr[kx]);
            st2(Wi + kx * PS + y * RS + z, vi[kx]);
        }
    }
    __syncthreads();
    if (tid < NH * NP2) {                                   // y-pass
        float2 vr[N], vi[N];
#pragma unroll
        for (int j = 0; j < N; ++j) { vr[j] = ld2(Wr + ybase + j * RS); vi[j] = ld2(Wi + ybase + j * RS); }
        dft_p2<N, -1>(vr, vi);
#pragma unroll
        for (int j = 0; j < N; ++j) { st2(Wr + ybase + j * RS, vr[j]); st2(Wi + ybase + j * RS, vi[j]); }
    }
    __syncthreads();
    if (tid < NH * NP2) {                                   // z-pass -> Fh
        const int kx = tid / NP2, ky = 2 * (tid % NP2);
        const int b0 = kx * PS + ky * RS;
        float2 vr[N], vi[N];
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            vr[kz] = f2(Wr[b0 + kz], Wr[b0 + RS + kz]);
            vi[kz] = f2(Wi[b0 + kz], Wi[b0 + RS + kz]);
        }
        dft_p2<N, -1>(vr, vi);
        cpx<float>* F0 = Fh + (kx * N + ky) * FS;
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            F0[kz] = {vr[kz].x * inv_n, vi[kz].x * inv_n};
            F0[FS + kz] = {vr[kz].y * inv_n, vi[kz].y * inv_n};
        }
    }
    // (the first phase staging below is followed by a barrier)

    const cpx<float>* phase = static_cast<const cpx<float>*>(g.phase);
    const float* gw = static_cast<const float*>(g.gw);

    for (int p = 0; p < Nrho; ++p) {
        for (int e = tid; e < M * 3 * N; e += int(blockDim.x)) {
            const cpx<float> v = phase[size_t(p) * M * 3 * N + e];
            ph[e] = v;
            const int q = e / (3 * N), r = e - q * 3 * N;
            if (r >= 2 * N) ezz[q * N + (r - 2 * N)] = make_float4(v.x, v.x, v.y, v.y);
        }
        __syncthreads();

        if constexpr (SPLIT) {
            const int nq = M * ntr;
            // pass 1 of transform qt: spectrum and inverse DFT along z (registers)
            auto zpass = [&](int qt, float2 (&vr)[N], float2 (&vi)[N]) {
                const int q = qt / ntr, tr = qt % ntr;
                const cpx<float>* ep = ph + q * 3 * N;
                float aA, bA, cA, aB, bB, cB;
                p2_coef(ep, kxA, kyA, tr, aA, bA, cA);
                p2_coef(ep, kxB, kyB, tr, aB, bB, cB);
                if constexpr (FHT)
                    p2_pass1_spectrum_tm(tr, ezz + q * N, f2(aA, aB), f2(bA, bB), f2(cA, cB), ft, vr, vi);
                else if (single_warp)
                    p2_pass1_spectrum<true>(tr, ezz + q * N, f2(aA, aB), f2(bA, bB), f2(cA, cB),
                                            fa, fb, single, vr, vi);
                else
                    p2_pass1_spectrum<false>(tr, ezz + q * N, f2(aA, aB), f2(bA, bB), f2(cA, cB),
                                             fa, fb, single, vr, vi);
                dft_p2<N, +1>(vr, vi);
            };
            auto zstore = [&](const float2 (&vr)[N], const float2 (&vi)[N]) {
#pragma unroll
                for (int z = 0; z < N; z += 2) {
                    st2(Wr + offA + z, f2(vr[z].x, vr[z + 1].x));
                    st2(Wi + offA + z, f2(vi[z].x, vi[z + 1].x));
                    st2(Wr + offB + z, f2(vr[z].y, vr[z + 1].y));
                    st2(Wi + offB + z, f2(vi[z].y, vi[z + 1].y));
                }
            };
            // the same for one pencil (BAL single-pencil threads): pencil B of
            // a pair is the conjugate partner, F_B(kz) = conj(F_A(-kz))
            auto zpass_s = [&](int qt, cpx<float> (&v)[N]) {
                const int q = qt / ntr, tr = qt % ntr;
                float a, b, c;
                p2_coef(ph + q * 3 * N, s_kx, s_ky, tr, a, b, c);
                const float4* ez = ezz + q * N;
                if constexpr (FHT) {
#pragma unroll
                    for (int cc = 0; cc < N / 8; ++cc) {
                        uint32_t r[16];
                        tc::tmem_ld16_issue(ft + 16 * cc, r);
                        tc::tmem_wait();
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const int kz = 8 * cc + k;
                            const float4 e = ez[kz];
                            const float m = fmaf(a, e.x, (kz == N / 2 ? c : b) * e.z);
                            const cpx<float> F = {__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1])};
                            v[kz] = tr == 0 ? cpx<float>{m * F.x, m * F.y} : cpx<float>{-m * F.y, m * F.x};
                        }
                    }
                } else {
#pragma unroll
                    for (int kz = 0; kz < N; ++kz) {
                        const float4 e = ez[kz];
                        const float m = fmaf(a, e.x, (kz == N / 2 ? c : b) * e.z);
                        const cpx<float> F = ss ? conjc(s_fa[(N - kz) % N]) : s_fa[kz];
                        v[kz] = tr == 0 ? cpx<float>{m * F.x, m * F.y} : cpx<float>{-m * F.y, m * F.x};
                    }
                }
                dft<N, +1>(v);
            };
            auto zstore_s = [&](const cpx<float> (&v)[N]) {
#pragma unroll
                for (int z = 0; z < N; ++z) {
                    Wr[s_off + z] = v[z].x;
                    Wi[s_off + z] = v[z].y;
                }
            };
            // every thread's x-pass loads done: W is free (bounded wait; on
            // expiry bit 62 of the work counter ends the launch)
            auto wait_free = [&]() {
                uint32_t spins = 0;
                while (!tc::mbar_try(wfree, wpar)) {
                    if (++spins == (1u << 22)) {
                        atomicOr(counter, 1ull << 62);
                        break;
                    }
                }
                wpar ^= 1u;
            };
            if constexpr (FHT) {
                if (p == 0) {
                    // the distribution's spectra, once: A[kz] = Fh of the pencil,
                    // B[kz] = its partner's (see p2_pass1_spectrum)
#pragma unroll
                    for (int cc = 0; cc < N / 8; ++cc) {
                        uint32_t r[16], rb[16];
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const int kz = 8 * cc + k, kn = (N - kz) % N;
                            cpx<float> A, B;
                            if (lp) {
                                A = fa[kz];
                                B = (single_warp && single) ? fb[kz] : conjc(fa[kn]);
                            } else {
                                A = ss ? conjc(s_fa[kn]) : s_fa[kz];
                                B = A;
                            }
                            r[2 * k] = __float_as_uint(A.x);
                            r[2 * k + 1] = __float_as_uint(A.y);
                            rb[2 * k] = __float_as_uint(B.x);
                            rb[2 * k + 1] = __float_as_uint(B.y);
                        }
                        tc::tmem_st16(ft + 16 * cc, r);
                        if (lp) tc::tmem_st16(ft + 48 + 16 * cc, rb);
                    }
                    tc::tmem_wait_st();
                }
            }
            if (lp) {
                float2 vr[N], vi[N];
                zpass(0, vr, vi);
                zstore(vr, vi);
            } else {
                cpx<float> v[N];
                zpass_s(0, v);
                zstore_s(v);
            }
            for (int qt = 0; qt < nq; ++qt) {
                const int tr = qt % ntr;
                __syncthreads();                            // z-pass of qt stored
                if (lp) {                                   // pass 2: inverse along y
                    float2 vr[N], vi[N];
#pragma unroll
                    for (int j = 0; j < N; ++j) { vr[j] = ld2(Wr + ybase + j * RS); vi[j] = ld2(Wi + ybase + j * RS); }
                    dft_p2<N, +1>(vr, vi);
#pragma unroll
                    for (int j = 0; j < N; ++j) { st2(Wr + ybase + j * RS, vr[j]); st2(Wi + ybase + j * RS, vi[j]); }
                } else {
                    cpx<float> v[N];
#pragma unroll
                    for (int j = 0; j < N; ++j) v[j] = {Wr[s_ybase + j * RS], Wi[s_ybase + j * RS]};
                    dft<N, +1>(v);
#pragma unroll
                    for (int j = 0; j < N; ++j) { Wr[s_ybase + j * RS] = v[j].x; Wi[s_ybase + j * RS] = v[j].y; }
                }
                __syncthreads();                            // y-pass stored
                const bool more = qt + 1 < nq;
                if (lp) {                                   // pass 3: inverse along x, S_p += Re(w^2)
                    float2 vr[N], vi[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) { vr[i] = ld2(Wr + i * PS + xbase); vi[i] = ld2(Wi + i * PS + xbase); }
                    if (more) tc::mbar_arrive(wfree);       // this thread is done reading W
                    dft_p2<N, +1>(vr, vi);
                    const float2 m1 = f2(-1.f, -1.f);
                    tc::tmem_wait_st();
#pragma unroll
                    for (int c = 0; c < N / 8; ++c) {
                        uint32_t r[16];
                        if (qt > 0) {
                            tc::tmem_ld16_issue(ts + 16 * c, r);
                            tc::tmem_wait();
                        } else {
#pragma unroll
                            for (int k = 0; k < 16; ++k) r[k] = 0u;
                        }
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const int x = 8 * c + k;
                            const float2 d = tr == 0 ? __ffma2_rn(vi[x], m1, vr[x]) : __ffma2_rn(vr[x], m1, vi[x]);
                            const float2 sv = __ffma2_rn(__fadd2_rn(vr[x], vi[x]), d,
                                                         f2(__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1])));
                            r[2 * k] = __float_as_uint(sv.x);
                            r[2 * k + 1] = __float_as_uint(sv.y);
                        }
                        tc::tmem_st16(ts + 16 * c, r);
                    }
                } else {                                    // one pencil: 24 S_p values, 2 x 16 columns
                    cpx<float> v[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) v[i] = {Wr[i * PS + s_xbase], Wi[i * PS + s_xbase]};
                    if (more) tc::mbar_arrive(wfree);
                    dft<N, +1>(v);
                    tc::tmem_wait_st();
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        uint32_t r[16];
                        if (qt > 0) {
                            tc::tmem_ld16_issue(ts + 16 * c, r);
                            tc::tmem_wait();
                        } else {
#pragma unroll
                            for (int k = 0; k < 16; ++k) r[k] = 0u;
                        }
#pragma unroll
                        for (int k = 0; k < 16; ++k) {
                            const int x = 16 * c + k;
                            if (x < N) {
                                const float d = tr == 0 ? fmaf(v[x].y, -1.f, v[x].x) : fmaf(v[x].x, -1.f, v[x].y);
                                r[k] = __float_as_uint(fmaf(v[x].x + v[x].y, d, __uint_as_float(r[k])));
                            }
                        }
                        tc::tmem_st16(ts + 16 * c, r);
                    }
                }
                if (more) {                                 // pass 1 of the next transform
                    if (lp) {
                        float2 vr[N], vi[N];
                        zpass(qt + 1, vr, vi);
                        wait_free();
                        zstore(vr, vi);
                    } else {
                        cpx<float> v[N];
                        zpass_s(qt + 1, v);
                        wait_free();
                        zstore_s(v);
                    }
                }
            }
            __syncthreads();                                // last x-pass loads done
        } else {
            for (int qt = 0; qt < M * ntr; ++qt) {
                const int q = qt / ntr, tr = qt % ntr;
                const cpx<float>* ep = ph + q * 3 * N;
                // ---- pass 1: spectrum, inverse along z (pencil pairs of the table) ----
                {
                    float aA, bA, cA, aB, bB, cB;
                    p2_coef(ep, kxA, kyA, tr, aA, bA, cA);
                    p2_coef(ep, kxB, kyB, tr, aB, bB, cB);
                    float2 vr[N], vi[N];
                    if (single_warp)
                        p2_pass1_spectrum<true>(tr, ezz + q * N, f2(aA, aB), f2(bA, bB), f2(cA, cB),
                                                fa, fb, single, vr, vi);
                    else
                        p2_pass1_spectrum<false>(tr, ezz + q * N, f2(aA, aB), f2(bA, bB), f2(cA, cB),
                                                 fa, fb, single, vr, vi);
                    dft_p2<N, +1>(vr, vi);
#pragma unroll
                    for (int z = 0; z < N; z += 2) {
                        st2(Wr + offA + z, f2(vr[z].x, vr[z + 1].x));
                        st2(Wi + offA + z, f2(vi[z].x, vi[z + 1].x));
                        st2(Wr + offB + z, f2(vr[z].y, vr[z + 1].y));
                        st2(Wi + offB + z, f2(vi[z].y, vi[z + 1].y));
                    }
                }
                __syncthreads();
                // ---- pass 2: inverse along y ----
                {
                    float2 vr[N], vi[N];
#pragma unroll
                    for (int j = 0; j < N; ++j) { vr[j] = ld2(Wr + ybase + j * RS); vi[j] = ld2(Wi + ybase + j * RS); }
                    dft_p2<N, +1>(vr, vi);
#pragma unroll
                    for (int j = 0; j < N; ++j) { st2(Wr + ybase + j * RS, vr[j]); st2(Wi + ybase + j * RS, vi[j]); }
                }
                __syncthreads();
                // ---- pass 3: inverse along x, S_p += Re(w^2) = (re + im)(re - im) ----
                {
                    float2 vr[N], vi[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) { vr[i] = ld2(Wr + i * PS + xbase); vi[i] = ld2(Wi + i * PS + xbase); }
                    dft_p2<N, +1>(vr, vi);
                    const float2 m1 = f2(-1.f, -1.f);
                    tc::tmem_wait_st();
#pragma unroll
                    for (int c = 0; c < N / 8; ++c) {
                        uint32_t r[16];
                        if (qt > 0) {
                            tc::tmem_ld16_issue(ts + 16 * c, r);
                            tc::tmem_wait();
                        } else {
#pragma unroll
                            for (int k = 0; k < 16; ++k) r[k] = 0u;
                        }
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const int x = 8 * c + k;
                            const float2 d = tr == 0 ? __ffma2_rn(vi[x], m1, vr[x]) : __ffma2_rn(vr[x], m1, vi[x]);
                            const float2 sv = __ffma2_rn(__fadd2_rn(vr[x], vi[x]), d,
                                                         f2(__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1])));
                            r[2 * k] = __float_as_uint(sv.x);
                            r[2 * k + 1] = __float_as_uint(sv.y);
                        }
                        tc::tmem_st16(ts + 16 * c, r);
                    }
                }
                __syncthreads();
            }
        }

        // ---- Gh += gw_p * FFT(S_p) (kx <= N/2) ----
        if (lp) {
            float2 vr[N], vi[N];                            // x-pass, real input
            tc::tmem_wait_st();
#pragma unroll
            for (int c = 0; c < N / 8; ++c) {
                uint32_t r[16];
                tc::tmem_ld16_issue(ts + 16 * c, r);
                tc::tmem_wait();
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    vr[8 * c + k] = f2(__uint_as_float(r[2 * k]), __uint_as_float(r[2 * k + 1]));
                    vi[8 * c + k] = f2(0.f, 0.f);
                }
            }
            dft_p2<N, -1>(vr, vi);
#pragma unroll
            for (int kx = 0; kx < NH; ++kx) { st2(Wr + kx * PS + xbase, vr[kx]); st2(Wi + kx * PS + xbase, vi[kx]); }
        } else {                                            // BAL single pencil
            cpx<float> v[N];
            tc::tmem_wait_st();
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                uint32_t r[16];
                tc::tmem_ld16_issue(ts + 16 * c, r);
                tc::tmem_wait();
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (16 * c + k < N) v[16 * c + k] = {__uint_as_float(r[k]), 0.f};
            }
            dft<N, -1>(v);
#pragma unroll
            for (int kx = 0; kx < NH; ++kx) { Wr[kx * PS + s_xbase] = v[kx].x; Wi[kx * PS + s_xbase] = v[kx].y; }
        }
        __syncthreads();
        if (tid < NH * NP2) {                               // y-pass
            float2 vr[N], vi[N];
#pragma unroll
            for (int j = 0; j < N; ++j) { vr[j] = ld2(Wr + ybase + j * RS); vi[j] = ld2(Wi + ybase + j * RS); }
            dft_p2<N, -1>(vr, vi);
#pragma unroll
            for (int j = 0; j < N; ++j) { st2(Wr + ybase + j * RS, vr[j]); st2(Wi + ybase + j * RS, vi[j]); }
        }
        __syncthreads();
        if (tid < NH * NP2) {                               // z-pass, accumulate
            const int kx = tid / NP2, ky = 2 * (tid % NP2);
            const int b0 = kx * PS + ky * RS;
            float2 vr[N], vi[N];
#pragma unroll
            for (int kz = 0; kz < N; ++kz) {
                vr[kz] = f2(Wr[b0 + kz], Wr[b0 + RS + kz]);
                vi[kz] = f2(Wi[b0 + kz], Wi[b0 + RS + kz]);
            }
            dft_p2<N, -1>(vr, vi);
            const float* gwp = gw + size_t(p) * N * NH * N + kx * N + ky;
#pragma unroll
            for (int kz = 0; kz < N; ++kz) {
                const float2 w = __ldg(reinterpret_cast<const float2*>(gwp + kz * NH * N));
                const int gi = (kz * NH + kx) * N + ky;
                if (p == 0) {
                    st2(Ghr + gi, __fmul2_rn(w, vr[kz]));
                    st2(Ghi + gi, __fmul2_rn(w, vi[kz]));
                } else {
                    st2(Ghr + gi, __ffma2_rn(w, vr[kz], ld2(Ghr + gi)));
                    st2(Ghi + gi, __ffma2_rn(w, vi[kz], ld2(Ghi + gi)));
                }
            }
        }
        // the next iteration's phase staging ends with a barrier
    }
    __syncthreads();

    // ---- QG + i*fC = IFFT(Gh + i*bb2*Fh) ----
    const float* bb2 = static_cast<const float*>(g.bb2);
    if (pt) {
        auto spec = [&](int kx, int ky, int kz) -> cpx<float> {
            const bool direct = kx < NH;
            const int pkx = direct ? kx : N - kx;
            const int pky = direct ? ky : (N - ky) % N;
            const int pkz = direct ? kz : (N - kz) % N;
            const int gi = (pkz * NH + pkx) * N + pky;
            cpx<float> G = {Ghr[gi], Ghi[gi]};
            cpx<float> F = Fh[(pkx * N + pky) * FS + pkz];
            if (!direct) { G.y = -G.y; F.y = -F.y; }
            const float b = ldg(bb2 + (kz * N + kx) * N + ky);
            return {G.x - b * F.y, G.y + b * F.x};
        };
        float2 vr[N], vi[N];
#pragma unroll
        for (int kz = 0; kz < N; ++kz) {
            const cpx<float> a = spec(kxA, kyA, kz), b = spec(kxB, kyB, kz);
            vr[kz] = f2(a.x, b.x);
            vi[kz] = f2(a.y, b.y);
        }
        dft_p2<N, +1>(vr, vi);
#pragma unroll
        for (int z = 0; z < N; z += 2) {
            st2(Wr + offA + z, f2(vr[z].x, vr[z + 1].x));
            st2(Wi + offA + z, f2(vi[z].x, vi[z + 1].x));
            st2(Wr + offB + z, f2(vr[z].y, vr[z + 1].y));
            st2(Wi + offB + z, f2(vi[z].y, vi[z + 1].y));
        }
    }
    __syncthreads();
    if (pt) {
        float2 vr[N], vi[N];
#pragma unroll
        for (int j = 0; j < N; ++j) { vr[j] = ld2(Wr + ybase + j * RS); vi[j] = ld2(Wi + ybase + j * RS); }
        dft_p2<N, +1>(vr, vi);
#pragma unroll
        for (int j = 0; j < N; ++j) { st2(Wr + ybase + j * RS, vr[j]); st2(Wi + ybase + j * RS, vi[j]); }
    }
    __syncthreads();

    const float prefac = float(g.prefac);
    const bool need_m = project || mom;
    float* Qs = reinterpret_cast<float*>(Fh);          // Fh is free from here on
    double m[5] = {0, 0, 0, 0, 0};
    if (pt) {
        const int y = tid / NP2, z = 2 * (tid % NP2);
        float2 vr[N], vi[N];
#pragma unroll
        for (int i = 0; i < N; ++i) { vr[i] = ld2(Wr + i * PS + y * RS + z); vi[i] = ld2(Wi + i * PS + y * RS + z); }
        dft_p2<N, +1>(vr, vi);
        const double cy = need_m ? g.c0[y] : 0.0;
        const double cz0 = need_m ? g.c0[z] : 0.0, cz1 = need_m ? g.c0[z + 1] : 0.0;
#pragma unroll
        for (int x = 0; x < N; ++x) {
            const int idx = (x * N + y) * N + z;
            const float q0 = prefac * (vr[x].x - f[idx] * vi[x].x);
            const float q1 = prefac * (vr[x].y - f[idx + 1] * vi[x].y);
            float* dst = project ? Qs : Qout;
            dst[idx] = q0;
            dst[idx + 1] = q1;
            if (need_m) {
                const double cx = g.c0[x], d0 = double(q0), d1 = double(q1);
                m[0] += d0 + d1;
                m[1] += cx * (d0 + d1);
                m[2] += cy * (d0 + d1);
                m[3] += cz0 * d0 + cz1 * d1;
                m[4] += (cx * cx + cy * cy + cz0 * cz0) * d0 + (cx * cx + cy * cy + cz1 * cz1) * d1;
            }
        }
    }
    if (!need_m) return;
    block_sum<5>(m, red);
    double m2[5] = {0, 0, 0, 0, 0};
    if (project) {
        double lam[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 5; ++j) s += g.ginv[i * 5 + j] * m[j];
            lam[i] = s;
        }
        for (int pid = tid; pid < N * N; pid += int(blockDim.x)) {
            const int y = pid / N, z = pid % N;
            const double cy = g.c0[y], cz = g.c0[z];
            for (int x = 0; x < N; ++x) {
                const int idx = (x * N + y) * N + z;
                const double cx = g.c0[x];
                const double c2 = cx * cx + cy * cy + cz * cz;
                const double qc = double(Qs[idx]) - (lam[0] + lam[1] * cx + lam[2] * cy
                                                     + lam[3] * cz + lam[4] * c2);
                __stcs(Qout + idx, float(qc));   // streaming: keep L2 for the scratch
                m2[0] += qc;
                m2[1] += cx * qc;
                m2[2] += cy * qc;
                m2[3] += cz * qc;
                m2[4] += c2 * qc;
            }
        }
        if (mom) block_sum<5>(m2, red);
    }
    if (mom && tid == 0) {
        for (int j = 0; j < 5; ++j) {
            mom[j] = m[j] * g.cw;
            mom[5 + j] = project ? m2[j] * g.cw : m[j] * g.cw;
        }
    }
    __syncthreads();   // Qs/red reuse by the next distribution
}

struct KArgs {
    bdgfs_vhs_grid grids[2];
    bdgfs_vhs_batch batches[4];
    int64_t start[5];       // prefix sums of ndof over batches
    int32_t nbatch;
    int32_t flags;
    unsigned char* scratch;
    size_t scratch_per_cta;
    unsigned long long* counter;
};

template <typename T, int N, int NT, bool WG, bool SG, int GR = 0, bool SL = false>
struct Variant {
    using L = QLayout<T, N, NT, WG, SG, SL>;
    static constexpr int n = N;
    static constexpr bool wg = WG, sg = SG, sl = SL, pk = false, split = false, bal = false, fht = false;
    static constexpr int gr = GR;
};

// packed Nv = 24 FP32 variant (288 threads); SPLIT: split work-cube barrier;
// FHT: each thread's z-pass spectra held in tensor memory (see collide_one_p2)
template <bool SPLIT = false, bool BAL = false, bool FHT = false>
struct VariantP2 {
    using L = QLayoutP2;
    static constexpr int n = p2::N;
    static constexpr bool wg = false, sg = false, sl = false, pk = true, split = SPLIT, bal = BAL, fht = FHT;
    static constexpr int gr = 0;
};

// Kernel over a set of grid variants; a distribution of a batch on a grid
// with Nv == V::n is processed by that variant's code path.
template <typename T, int NT, typename V0, typename V1>
__global__ void __launch_bounds__(NT, 1) __maxnreg__(65536 / NT / 8 * 8 > 255 ? 255 : 65536 / NT / 8 * 8) vhs_collide_kernel(const KArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int64_t s_item;
    __shared__ int64_t s_start[5];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_wfree;
    constexpr bool kPacked = V0::pk || V1::pk;
    constexpr uint32_t kTmemCols = (V0::fht || V1::fht) ? 2 * p2::TMEM_COLS : p2::TMEM_COLS;
    if constexpr (kPacked) {
        if (threadIdx.x < 32) tc::tmem_alloc(&s_tmem, kTmemCols);
        if (threadIdx.x == 0) tc::mbar_init(&s_wfree, NT);
        tc::tc_fence_before();
    }
    uint32_t wpar = 0;
    unsigned char* scratch = a.scratch + size_t(blockIdx.x) * a.scratch_per_cta;
    if (threadIdx.x == 0) {
        // per-batch counts: the host size, or a device count when given
        s_start[0] = 0;
        for (int b = 0; b < a.nbatch; ++b) {
            int64_t c = a.batches[b].ndof;
            if (a.batches[b].count) {
                const int64_t d = *a.batches[b].count;
                c = d < 0 ? 0 : (d < c ? d : c);
            }
            s_start[b + 1] = s_start[b] + c;
        }
    }
    __syncthreads();
    uint32_t tmem = 0;
    if constexpr (kPacked) {
        tc::tc_fence_after();
        tmem = s_tmem;
    }
    const int64_t total = s_start[a.nbatch];
    for (;;) {
        if (threadIdx.x == 0) s_item = int64_t(atomicAdd(a.counter, 1ull));
        __syncthreads();
        const int64_t item = s_item;
        __syncthreads();
        if (item >= total) break;
        int b = 0;
        while (item >= s_start[b + 1]) ++b;
        const bdgfs_vhs_batch& bt = a.batches[b];
        const bdgfs_vhs_grid& g = a.grids[bt.grid];
        const int64_t pos = item - s_start[b];
        const int64_t dof = bt.index ? int64_t(bt.index[pos]) : pos;
        if (dof < 0 || dof >= bt.ndof) continue;   // malformed index list: skip
        const int64_t n3 = int64_t(g.Nv) * g.Nv * g.Nv;
        const T* f = static_cast<const T*>(bt.f) + dof * n3;
        T* Q = static_cast<T*>(bt.Q) + dof * n3;
        double* mom = bt.moments ? bt.moments + dof * 10 : nullptr;
        if (g.Nv == V0::n) {
            if constexpr (V0::pk)
                collide_one_p2<V0::split, V0::bal, V0::fht>(g, f, Q, mom, a.flags, smem, scratch, tmem, &s_wfree, wpar,
                                          a.counter);
            else
                collide_one<T, V0::n, NT, V0::wg, V0::sg, V0::gr, V0::sl>(
                    g, f, Q, mom, a.flags, smem, scratch);
        } else if constexpr (V1::n > 0) {
            if (g.Nv == V1::n) {
                if constexpr (V1::pk)
                    collide_one_p2<V1::split, V1::bal, V1::fht>(g, f, Q, mom, a.flags, smem, scratch, tmem, &s_wfree,
                                              wpar, a.counter);
                else
                    collide_one<T, V1::n, NT, V1::wg, V1::sg, V1::gr, V1::sl>(
                        g, f, Q, mom, a.flags, smem, scratch);
            }
        }
    }
    if constexpr (kPacked) {
        tc::tmem_wait_st();
        tc::tc_fence_before();
        __syncthreads();
        if (threadIdx.x < 32) {
            tc::tc_fence_after();
            tc::tmem_dealloc(tmem, kTmemCols);
        }
    }
}

struct NoVariant {
    static constexpr int n = 0;
    static constexpr bool wg = false, sg = false, sl = false, pk = false, split = false, bal = false,
                          fht = false;
    static constexpr int gr = 0;
    struct L {
        static constexpr int WS = 0;
        static size_t smem_bytes(int) { return 0; }
        static size_t scratch_bytes() { return 0; }
    };
};

// Variant table: each entry is one compiled (precision, grid set, CTA size)
// combination; the tile field of the first grid picks among the entries that
// match the grid set (tile 0 = first match).
template <typename T, int NT, typename V0, typename V1>
static int launch(const bdgfs_vhs_grid* grids, int ngrids, const bdgfs_vhs_batch* batches,
                  int nbatch, int flags, void* scratch, size_t scratch_bytes,
                  uint64_t* counter, cudaStream_t st);

template <typename T, int NT, typename V0, typename V1>
static size_t entry_per_cta(int maxM, size_t* smem)
{
    size_t s0 = V0::L::smem_bytes(maxM), s1 = V1::L::smem_bytes(maxM);
    *smem = s0 > s1 ? s0 : s1;
    size_t p0 = V0::L::scratch_bytes(), p1 = V1::L::scratch_bytes();
    return p0 > p1 ? p0 : p1;
}

struct Entry {
    int fp64, n0, n1, threads;
    int (*run)(const bdgfs_vhs_grid*, int, const bdgfs_vhs_batch*, int, int, void*, size_t,
               uint64_t*, cudaStream_t);
    size_t (*per)(int, size_t*);
};

#define VARIANT(T, N, NT, WG, SG) Variant<T, N, NT, WG, SG>
#define VARIANTG(T, N, NT, GR) Variant<T, N, NT, false, false, GR>
#define VARIANTS(T, NT) Variant<T, 32, NT, true, false, 0, true>
#define ENTRYG(FP, T, NT, N0, GR)                                                            \
    {FP, N0, 0, NT, &launch<T, NT, VARIANTG(T, N0, NT, GR), NoVariant>,                     \
     &entry_per_cta<T, NT, VARIANTG(T, N0, NT, GR), NoVariant>}
#define ENTRY(FP, T, NT, N0, WG0, SG0, N1, WG1, SG1)                                        \
    {FP, N0, N1, NT,                                                                         \
     &launch<T, NT, VARIANT(T, N0, NT, WG0, SG0), VARIANT(T, N1, NT, WG1, SG1)>,             \
     &entry_per_cta<T, NT, VARIANT(T, N0, NT, WG0, SG0), VARIANT(T, N1, NT, WG1, SG1)>}
#define ENTRY1(FP, T, NT, N0, WG0, SG0)                                                      \
    {FP, N0, 0, NT, &launch<T, NT, VARIANT(T, N0, NT, WG0, SG0), NoVariant>,                \
     &entry_per_cta<T, NT, VARIANT(T, N0, NT, WG0, SG0), NoVariant>}

static const Entry kEntries[] = {
    // fp32, one grid
    ENTRY1(0, float, 288, 24, false, false),
    ENTRY1(0, float, 576, 24, false, false),
    ENTRY1(0, float, 192, 24, false, false),
    ENTRYG(0, float, 288, 24, 3),
    ENTRYG(0, float, 576, 24, 6),
    ENTRY1(0, float, 288, 32, true, true),
    ENTRY1(0, float, 576, 32, true, true),
    ENTRY1(0, float, 256, 16, false, false),
    ENTRY1(0, float, 128, 16, false, false),
    ENTRYG(0, float, 256, 16, 2),
    ENTRY1(0, float, 144, 12, false, false),
    ENTRY1(0, float, 64, 8, false, false),
    // fp32, two grids in one launch
    ENTRY(0, float, 288, 24, false, false, 32, true, true),
    ENTRY(0, float, 576, 24, false, false, 32, true, true),
    // fp64
    ENTRY1(1, double, 256, 16, false, false),
    ENTRY1(1, double, 128, 16, false, false),
    ENTRYG(1, double, 256, 16, 2),
    ENTRY1(1, double, 144, 12, false, false),
    ENTRY1(1, double, 64, 8, false, false),
    // appended variants (earlier tile indices stay valid)
    ENTRY1(0, float, 384, 24, false, false),
    // 32^3 with warp slabs in shared memory, S_p in registers
    {0, 32, 0, 256, &launch<float, 256, VARIANTS(float, 256), NoVariant>,
     &entry_per_cta<float, 256, VARIANTS(float, 256), NoVariant>},
    {0, 24, 32, 256,
     &launch<float, 256, VARIANT(float, 24, 256, false, false), VARIANTS(float, 256)>,
     &entry_per_cta<float, 256, VARIANT(float, 24, 256, false, false), VARIANTS(float, 256)>},
    // 24^3 packed: two pencils per thread on f32x2 arithmetic
    {0, 24, 0, 288, &launch<float, 288, VariantP2<>, NoVariant>,
     &entry_per_cta<float, 288, VariantP2<>, NoVariant>},
    // the same with the split work-cube barrier
    {0, 24, 0, 288, &launch<float, 288, VariantP2<true>, NoVariant>,
     &entry_per_cta<float, 288, VariantP2<true>, NoVariant>},
    // split barrier, 8 pair-warps + 2 single-pencil warps in the transform loop
    {0, 24, 0, 320, &launch<float, 320, VariantP2<true, true>, NoVariant>,
     &entry_per_cta<float, 320, VariantP2<true, true>, NoVariant>},
    // the same with each thread's z-pass spectra in tensor memory
    {0, 24, 0, 320, &launch<float, 320, VariantP2<true, true, true>, NoVariant>,
     &entry_per_cta<float, 320, VariantP2<true, true, true>, NoVariant>},
};
static constexpr int kNumEntries = int(sizeof(kEntries) / sizeof(kEntries[0]));

static bool entry_matches(const Entry& e, const bdgfs_vhs_grid* grids, int ngrids)
{
    if (e.fp64 != grids[0].fp64) return false;
    if (ngrids == 1) return e.n1 == 0 && e.n0 == grids[0].Nv;
    if (e.n1 == 0) return false;
    const int a = grids[0].Nv, b = grids[1].Nv;
    return (a == e.n0 || a == e.n1) && (b == e.n0 || b == e.n1);
}

// Entry index for (grids, tile), or -1.
static int choose(const bdgfs_vhs_grid* grids, int ngrids)
{
    if (!grids || ngrids < 1 || ngrids > 2) return -1;
    for (int i = 0; i < ngrids; ++i) {
        if (grids[i].fp64 != grids[0].fp64) return -1;
        if (grids[i].Nrho < 1 || grids[i].M < 1 || grids[i].M > 64) return -1;
    }
    int tile = grids[0].tile, k = 0;
    for (int i = 0; i < kNumEntries; ++i) {
        if (!entry_matches(kEntries[i], grids, ngrids)) continue;
        if (k == tile) return i;
        ++k;
    }
    return -1;
}

template <typename T, int NT, typename V0, typename V1>
static int launch(const bdgfs_vhs_grid* grids, int ngrids, const bdgfs_vhs_batch* batches,
                  int nbatch, int flags, void* scratch, size_t scratch_bytes,
                  uint64_t* counter, cudaStream_t st)
{
    KArgs a{};
    int maxM = 1;
    for (int i = 0; i < ngrids; ++i) {
        a.grids[i] = grids[i];
        maxM = grids[i].M > maxM ? grids[i].M : maxM;
    }
    a.nbatch = nbatch;
    a.flags = flags;
    a.start[0] = 0;
    for (int b = 0; b < nbatch; ++b) {
        a.batches[b] = batches[b];
        a.start[b + 1] = a.start[b] + batches[b].ndof;
    }
    if (a.start[nbatch] == 0) return BDGFS_OK;
    size_t smem = 0;
    const size_t per = entry_per_cta<T, NT, V0, V1>(maxM, &smem);
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return BDGFS_ECUDA;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return BDGFS_ECUDA;
    int64_t nblk = nsm;
    if (nblk > a.start[nbatch]) nblk = a.start[nbatch];
    const int64_t fit = int64_t(scratch_bytes / per);
    if (fit < 1) return BDGFS_ESCRATCH;
    if (nblk > fit) nblk = fit;
    a.scratch = static_cast<unsigned char*>(scratch);
    a.scratch_per_cta = per;
    a.counter = reinterpret_cast<unsigned long long*>(counter);
    auto k = vhs_collide_kernel<T, NT, V0, V1>;
    // per device, once (and again only if a larger M needs more)
    if (const int rc = smem_optin(reinterpret_cast<const void*>(k), smem)) return rc;
    if (cudaMemsetAsync(counter, 0, sizeof(uint64_t), st) != cudaSuccess)
        return BDGFS_ECUDA;
    k<<<unsigned(nblk), NT, smem, st>>>(a);
    return cuda_status(cudaGetLastError());
}

__global__ void fma_probe_kernel(float* out, int iters)
{
    // 8 independent FMA chains per thread; the final sum defeats DCE.
    float a0 = threadIdx.x * 1e-7f, a1 = a0 + 1e-7f, a2 = a0 + 2e-7f, a3 = a0 + 3e-7f;
    float a4 = a0 + 4e-7f, a5 = a0 + 5e-7f, a6 = a0 + 6e-7f, a7 = a0 + 7e-7f;
    const float b = 0.999999f, c = 1e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678f) out[0] = s;   // practically never taken
}

}  // namespace bdgfs

using namespace bdgfs;

extern "C" int32_t bdgfs_vhs_tiles(const bdgfs_vhs_grid* grids, int32_t ngrids,
                                   int32_t* threads, int32_t capacity)
{
    if (!grids || ngrids < 1 || ngrids > 2) return 0;
    int k = 0;
    for (int i = 0; i < kNumEntries; ++i) {
        if (!entry_matches(kEntries[i], grids, ngrids)) continue;
        if (threads && k < capacity) threads[k] = kEntries[i].threads;
        ++k;
    }
    return k;
}

extern "C" size_t bdgfs_vhs_scratch_bytes(const bdgfs_vhs_grid* grids, int32_t ngrids,
                                          int32_t nctas)
{
    const int id = choose(grids, ngrids);
    if (id < 0) return 0;
    int maxM = 1;
    for (int i = 0; i < ngrids; ++i) maxM = grids[i].M > maxM ? grids[i].M : maxM;
    size_t smem = 0;
    const size_t per = kEntries[id].per(maxM, &smem);
    if (nctas <= 0) {
        int dev = 0, nsm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return 0;
        nctas = nsm;
    }
    return per * size_t(nctas);
}

extern "C" int32_t bdgfs_vhs_collide(const bdgfs_vhs_grid* grids, int32_t ngrids,
                                     const bdgfs_vhs_batch* batches, int32_t nbatch,
                                     int32_t flags, void* scratch, size_t scratch_bytes,
                                     uint64_t* work_counter, void* stream)
{
    if (!grids || !batches || nbatch < 1 || nbatch > 4 || !work_counter || !scratch)
        return BDGFS_EINVAL;
    for (int b = 0; b < nbatch; ++b) {
        if (batches[b].grid < 0 || batches[b].grid >= ngrids || batches[b].ndof < 0)
            return BDGFS_EINVAL;
        if (batches[b].ndof > 0 && (!batches[b].f || !batches[b].Q)) return BDGFS_EINVAL;
    }
    const int id = choose(grids, ngrids);
    if (id < 0) return BDGFS_EUNSUPPORTED;
    return kEntries[id].run(grids, ngrids, batches, nbatch, flags, scratch, scratch_bytes,
                            work_counter, static_cast<cudaStream_t>(stream));
}

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot allocate device memory at the point where they need the
// collision operator: a host application whose device memory is owned by
// another allocator (a caching allocator or a fixed arena handed out at
// start-up), a time loop that must not allocate once it is running, or a
// plugin whose host only passes it input and output pointers.  For them
// bdgfs_vhs_collide_static takes its scratch and its work counter from one
// file-scope device array instead of a caller-provided buffer.
//
// Layout of the array: bytes [0, 256) hold the 64-bit work counter, the rest
// is per-CTA scratch.  Its size is fixed (BDGFS_STATIC_SCRATCH_BYTES); every
// GPU that loads this library holds it until the process exits.  When one
// CTA's scratch for the given grids does not fit, the call fails with
// BDGFS_ESCRATCH; when fewer CTAs than SMs fit, fewer run (slower, same
// result).  Calls share the array and it keeps the last call's contents:
// the counter is cleared (stream-ordered) on every call and every other
// scratch word is written before it is read, but calls that overlap on the
// GPU (different streams, or different host threads) race on it.
#define BDGFS_STATIC_SCRATCH_BYTES (size_t(16) << 20)
static __device__ __align__(256) unsigned char g_vhs_static_scratch[BDGFS_STATIC_SCRATCH_BYTES];

// Device address of the array, looked up once per device with that device
// current (the array's name is only a host-side stand-in in host code).  The
// lookup is serialised, so host threads may make their first calls at once.
// The address is kept for the life of the process: after cudaDeviceReset the
// module may load elsewhere, so this entry point must not be used across a
// device reset.
static void* static_scratch_addr(int dev)
{
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    if (dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_vhs_static_scratch) != cudaSuccess) return nullptr;
        addr[dev] = p;
    }
    return addr[dev];
}

extern "C" int32_t bdgfs_vhs_collide_static(const bdgfs_vhs_grid* grids, int32_t ngrids,
                                            const bdgfs_vhs_batch* batches, int32_t nbatch,
                                            int32_t flags, void* stream)
{
    if (!grids || !batches || nbatch < 1 || nbatch > 4) return BDGFS_EINVAL;
    for (int b = 0; b < nbatch; ++b) {
        if (batches[b].grid < 0 || batches[b].grid >= ngrids || batches[b].ndof < 0)
            return BDGFS_EINVAL;
        if (batches[b].ndof > 0 && (!batches[b].f || !batches[b].Q)) return BDGFS_EINVAL;
    }
    const int id = choose(grids, ngrids);
    if (id < 0) return BDGFS_EUNSUPPORTED;
    int maxM = 1;
    for (int i = 0; i < ngrids; ++i) maxM = grids[i].M > maxM ? grids[i].M : maxM;
    size_t smem = 0;
    const size_t per = kEntries[id].per(maxM, &smem);
    const size_t capacity = BDGFS_STATIC_SCRATCH_BYTES - 256;
    if (per > capacity) return BDGFS_ESCRATCH;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return BDGFS_ECUDA;
    unsigned char* base = static_cast<unsigned char*>(static_scratch_addr(dev));
    if (!base) return BDGFS_ECUDA;
    return kEntries[id].run(grids, ngrids, batches, nbatch, flags, base + 256, capacity,
                            reinterpret_cast<uint64_t*>(base), static_cast<cudaStream_t>(stream));
}

extern "C" int32_t bdgfs_fma_probe(float* out, int32_t nblocks, int32_t iters, void* stream)
{
    if (!out || nblocks < 1 || iters < 1) return BDGFS_EINVAL;
    fma_probe_kernel<<<nblocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(out, iters);
    return cuda_status(cudaGetLastError());
}
