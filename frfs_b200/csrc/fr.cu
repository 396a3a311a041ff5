// Flux-reconstruction advection of the distribution function, all Nv^3
// velocities at once (no velocity batching).
//
// Reference path (per velocity batch, frfs/solvers/dgfs/system.py:140-196):
//   disu        u_f = M0 u                       (solvers/dgfs/elements.py:56-59)
//   tdisf       F~_i = smats[i][k] c_k u          (kernels/tflux.mako, flux.mako)
//   tdivtpcorf  R = (M1 - M3 M2) F~               (elements.py:79-82)
//   comm_flux   upwind flux at interfaces / diffuse walls
//               (kernels/intcflux.mako, rsolvers/rusanov.mako, bccflux.mako,
//                bcs/dgfs-wall-diffuse.mako)
//   tdivtconf   R += M3 Fhat                      (elements.py:85-88)
//   negdivconf  R = -R / |J|                      (kernels/negdivconf.mako)
//   axnpby      RK update                         (backends/cuda/kernels/axnpby.mako)
//   update_bc   diffuse-wall mass balance sums    (kernels/bccupdate.mako,
//               bcs/dgfs-wall-diffuse-update.mako)
//
// Layout: state u[e][upt][v], face values uf[e][fpt][v], v = (x*Nv+y)*Nv+z
// contiguous, so every global access below is coalesced across the threads
// of a block (one thread per velocity).  bdgfs_fr_rhs fuses tdisf,
// tdivtpcorf, both comm_flux kernels, tdivtconf, negdivconf and the RK
// combination out = a*u + b*L(u) + c1*x1 + c2*x2 in one pass; the common
// flux of an interior face point is evaluated by both neighbours (each with
// its own outward normal), which equals the reference's lhs-computed value
// with the sign flip of intcflux.mako:21-23.
#include "common.cuh"
#include "fr_tc.cuh"

namespace bdgfs {

template <typename T>
struct FrSmem {
    T* dT;      // [ND*NU][NU]  (M1 - M3 M2) transposed
    T* m3T;     // [NF][NU]
    T* m0;      // [NF][NU]
};

// velocity components of index v
template <typename T>
__device__ __forceinline__ void vel(const T* c0, int Nv, int64_t v, T (&c)[3])
{
    // v < Nv^3 <= 2^18: 32-bit arithmetic
    const uint32_t vv = uint32_t(v), n = uint32_t(Nv);
    const uint32_t q = vv / n, iz = vv - q * n;
    const uint32_t ix = q / n, iy = q - ix * n;
    c[0] = c0[ix];
    c[1] = c0[iy];
    c[2] = c0[iz];
}

// VB consecutive values of a velocity row (one vector access when aligned)
template <typename T, int VB>
struct Vec {
    T v[VB];
    __device__ __forceinline__ void load(const T* __restrict__ p)
    {
        if constexpr (VB == 4 && sizeof(T) == 4) {
            const float4 x = *reinterpret_cast<const float4*>(p);
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
        } else if constexpr (VB == 2 && sizeof(T) == 4) {
            const float2 x = *reinterpret_cast<const float2*>(p);
            v[0] = x.x; v[1] = x.y;
        } else if constexpr (VB == 2 && sizeof(T) == 8) {
            const double2 x = *reinterpret_cast<const double2*>(p);
            v[0] = x.x; v[1] = x.y;
        } else {
#pragma unroll
            for (int q = 0; q < VB; ++q) v[q] = p[q];
        }
    }
    __device__ __forceinline__ void store(T* __restrict__ p) const
    {
        if constexpr (VB == 4 && sizeof(T) == 4) {
            *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        } else if constexpr (VB == 2 && sizeof(T) == 4) {
            *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
        } else if constexpr (VB == 2 && sizeof(T) == 8) {
            *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
        } else {
#pragma unroll
            for (int q = 0; q < VB; ++q) p[q] = v[q];
        }
    }
};

// r[0..N) = p[0..N) from shared memory in one vector load (p aligned to
// N * sizeof(T); N = 2 or 4)
template <typename T, int N>
__device__ __forceinline__ void lds_vec(const T* __restrict__ p, T (&r)[N])
{
    if constexpr (sizeof(T) == 4 && N == 4) {
        const float4 x = *reinterpret_cast<const float4*>(p);
        r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
    } else if constexpr (sizeof(T) == 4 && N == 2) {
        const float2 x = *reinterpret_cast<const float2*>(p);
        r[0] = x.x; r[1] = x.y;
    } else if constexpr (sizeof(T) == 8 && N == 4) {
        const double2 x0 = *reinterpret_cast<const double2*>(p);
        const double2 x1 = *reinterpret_cast<const double2*>(p + 2);
        r[0] = x0.x; r[1] = x0.y; r[2] = x1.x; r[3] = x1.y;
    } else if constexpr (sizeof(T) == 8 && N == 2) {
        const double2 x = *reinterpret_cast<const double2*>(p);
        r[0] = x.x; r[1] = x.y;
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) r[i] = p[i];
    }
}

// Residual accumulators R(q, i) of a thread's VB velocities at the NU
// solution points.  FP32 with an even VB (PK): consecutive solution points
// in float2 pairs, so that the operator columns, read as 16-byte
// broadcasts, feed sm_100 f32x2 FMAs: half the FMA instructions of scalar
// code and the same rounding (each lane is one fused multiply-add).
template <typename T, int NU, int VB, bool PK = false>
struct Racc {
    T r[VB][NU];
    __device__ __forceinline__ T& operator()(int q, int i) { return r[q][i]; }
};
template <int NU, int VB>
struct Racc<float, NU, VB, true> {
    static constexpr int NPR = NU / 2;               // pairs (i, i+1), i even < 2 NPR
    float2 p[VB][NPR];
    float l[VB];                                     // i = NU - 1 when NU is odd
    __device__ __forceinline__ float& operator()(int q, int i)
    {
        return i < 2 * NPR ? ((i & 1) ? p[q][i >> 1].y : p[q][i >> 1].x) : l[q];
    }
};

// R(q, i) += col[i] * s[q] for i < NU, col a shared-memory column padded to
// a multiple of 4 (read as 16-byte broadcasts for float)
template <typename T, int NU, int NUP, int VB, bool PK>
__device__ __forceinline__ void axpy_col(const T* __restrict__ col, const T (&s)[VB], Racc<T, NU, VB, PK>& R)
{
    if constexpr (PK) {
        constexpr int NPR = Racc<T, NU, VB, PK>::NPR;
        float2 s2[VB];
#pragma unroll
        for (int q = 0; q < VB; ++q) s2[q] = make_float2(s[q], s[q]);
#pragma unroll
        for (int i4 = 0; i4 < NUP; i4 += 4) {
            const float4 x = *reinterpret_cast<const float4*>(col + i4);
            const float2 w2[2] = {make_float2(x.x, x.y), make_float2(x.z, x.w)};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = i4 + 2 * h;
                if (i + 1 < 2 * NPR) {
#pragma unroll
                    for (int q = 0; q < VB; ++q) R.p[q][i >> 1] = __ffma2_rn(w2[h], s2[q], R.p[q][i >> 1]);
                } else if (i < NU) {
#pragma unroll
                    for (int q = 0; q < VB; ++q) R(q, i) += w2[h].x * s[q];
                }
            }
        }
    } else {
#pragma unroll
        for (int i4 = 0; i4 < NUP; i4 += 4) {
            T w[4];
            if constexpr (sizeof(T) == 4) {
                const float4 x = *reinterpret_cast<const float4*>(col + i4);
                w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
            } else {
                const double2 x0 = *reinterpret_cast<const double2*>(col + i4);
                const double2 x1 = *reinterpret_cast<const double2*>(col + i4 + 2);
                w[0] = x0.x; w[1] = x0.y; w[2] = x1.x; w[3] = x1.y;
            }
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                if (i4 + t < NU) {
#pragma unroll
                    for (int q = 0; q < VB; ++q) R(q, i4 + t) += w[t] * s[q];
                }
            }
        }
    }
}

// asynchronous global -> shared copies of one thread (Ampere-style
// cp.async; BYTES 4, 8 or 16, both addresses aligned to BYTES)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* sdst, const void* gsrc)
{
    const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(sa), "l"(gsrc), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// u_f = M0 u (gm0 = M0, NF flux points), or any other per-element operator
// with NF rows (the inverse mass matrix: NF = NU).  Each CTA (128 threads)
// owns one element and a chunk of velocities, each thread VB consecutive
// velocities per step.  When every row of the operator is a unit vector
// (flux points on solution points, as with GLL points) the product is a
// gather: uf[f] = u[sel[f]], pure data movement; otherwise the dense product
// with the operator read from shared memory.
template <typename T, int NU, int NF, int VB>
__global__ void __launch_bounds__(128) disu_kernel(const bdgfs_fr_eles el, const T* __restrict__ gm0,
                                                   const T* __restrict__ u, T* __restrict__ uf,
                                                   int64_t chunk)
{
    __shared__ T m0[NF * NU];
    __shared__ int sel[NF];
    __shared__ int gather;
    for (int i = threadIdx.x; i < NF * NU; i += blockDim.x) m0[i] = gm0[i];
    if (threadIdx.x == 0) gather = 1;
    __syncthreads();
    for (int f = threadIdx.x; f < NF; f += blockDim.x) {
        int nz = 0, at = -1;
        bool unit = true;
        for (int i = 0; i < NU; ++i) {
            const T x = m0[f * NU + i];
            if (x != T(0)) {
                ++nz;
                at = i;
                unit = unit && x == T(1);
            }
        }
        sel[f] = at;
        if (nz != 1 || !unit) atomicAnd(&gather, 0);
    }
    __syncthreads();
    const int64_t nv = el.nv;
    const int64_t e = blockIdx.y;
    const int64_t v1 = (int64_t(blockIdx.x) + 1) * chunk < nv ? (int64_t(blockIdx.x) + 1) * chunk : nv;
    const int64_t vs = int64_t(blockIdx.x) * chunk + int64_t(threadIdx.x) * VB;
    if (gather) {
        for (int64_t v0 = vs; v0 < v1; v0 += int64_t(blockDim.x) * VB) {
#pragma unroll 6
            for (int f = 0; f < NF; ++f) {
                Vec<T, VB> x;
                x.load(u + (e * NU + sel[f]) * nv + v0);
                x.store(uf + (e * NF + f) * nv + v0);
            }
        }
        return;
    }
    for (int64_t v0 = vs; v0 < v1; v0 += int64_t(blockDim.x) * VB) {
#pragma unroll
        for (int q = 0; q < VB; ++q) {
            T uu[NU];
#pragma unroll
            for (int i = 0; i < NU; ++i) uu[i] = u[(e * NU + i) * nv + v0 + q];
#pragma unroll 4
            for (int f = 0; f < NF; ++f) {
                T acc = T(0);
#pragma unroll
                for (int i = 0; i < NU; ++i) acc += m0[f * NU + i] * uu[i];
                uf[(e * NF + f) * nv + v0 + q] = acc;
            }
        }
    }
}

// GATHER: no face-value array; the face value of face point f of element e
// is the solution-point row u[e][fsel[f]] (M0 rows are unit vectors, as with
// GLL points), and a neighbour entry e'*NF + f' of nbr reads u[e'][fsel[f']].
// out must not alias u then (other CTAs read u's face rows).
// TPP > 0 (tensor-product points, TPP per line, flux points on solution
// points, own face value of f equal to u[e][fsel[f]]): the residual is
// applied factored, R = M1 F~ + M3 (F^n - M2 F~), with M1 along its lines
// (tp.m1line, TPP nonzeros per column at compile-time rows) and M2 a
// selection (row f: tp.fsgn[f] at column tp.fdim[f]*NU + fsel[f]), instead of
// the dense M1 - M3 M2.
// first velocity of the chunk of VB velocities that holds the mirror
// images of v0 .. v0 + VB - 1 under c_d -> -c_d (the grid is symmetric:
// c0[Nv - 1 - i] = -c0[i]); for the z axis the chunk holds them reversed.
// Chunks never straddle a z line (VB divides Nv when a y or z mirror is
// in use, checked on the host).
__device__ __forceinline__ int64_t mirror_chunk(int64_t v0, int Nv, int kind, int VB)
{
    const int64_t N = Nv, N2 = N * N;
    if (kind == BDGFS_BC_SPECULAR_X) return v0 + (N - 1 - 2 * (v0 / N2)) * N2;
    if (kind == BDGFS_BC_SPECULAR_Y) return v0 + (N - 1 - 2 * ((v0 / N) % N)) * N;
    const int64_t iz = v0 % N;
    return v0 - iz + (N - iz - VB);
}


template <typename T, int ND, int NU, int NF, int VB, bool GATHER = false, int RING = 8, int TPP = 0>
__global__ void __launch_bounds__(128, (NU <= 16 && sizeof(T) == 4) ? 4 : 3) rhs_kernel(const bdgfs_fr_eles el, const bdgfs_fr_walls wl,
                                                  const T* __restrict__ u, const T* __restrict__ uf,
                                                  const int32_t* __restrict__ fsel,
                                                  const bdgfs_fr_tensor tp,
                                                  T* out, T a, T b, const T* x1, T c1, const T* x2,
                                                  T c2, int64_t chunk)
{
    constexpr int NUP = (NU + 3) / 4 * 4;
    constexpr bool PK = sizeof(T) == 4 && VB % 2 == 0 && TPP > 0;    // f32x2 accumulation
    extern __shared__ __align__(16) unsigned char smraw[];
    // [RING][128][VB] row ring (see below), then the operators
    // (M1 - M3 M2) is read only by the dense residual (TPP == 0)
    constexpr int NDT = TPP ? 0 : ND * NU * NUP;
    T* dT = reinterpret_cast<T*>(smraw) + RING * 128 * VB;   // [ND*NU][NUP]  (M1 - M3 M2) transposed
    // rows of the metric terms, the normals and M1's line values are padded
    // to 4 (2 for smats in 2-D) entries, read with one vector load each
    constexpr int SR = ND == 3 ? 4 : ND;
    T* m3T = dT + NDT;                                  // [NF][NUP]
    T* sm = m3T + NF * NUP;                             // [NU][ND][SR]  smats
    T* pn = sm + NU * ND * SR;                          // [NF][4]: unit normal (ND), |n| at 3
    T* m1l = pn + NF * 4;                               // [ND][NU][4] (TPP)
    T* fsg = m1l + (TPP ? ND * NU * 4 : 0);             // [NF] (TPP)
    T* rj = fsg + (TPP ? NF : 0);                       // [NU]
    int* nb = reinterpret_cast<int*>(rj + NU);          // [NF]
    int* fs = nb + NF;                                  // [NF] (GATHER)
    int* fdm = fs + NF;                                 // [NF] (TPP)
    const int64_t e = blockIdx.y;
    {
        for (int i = threadIdx.x; i < NDT + NF * NUP; i += blockDim.x) dT[i] = T(0);
        __syncthreads();
        if constexpr (NDT > 0) {
            const T* gd = static_cast<const T*>(el.dcorr);   // [NU][ND*NU], read coalesced
            for (int i = threadIdx.x; i < NU * ND * NU; i += blockDim.x) {
                const int row = i / (ND * NU), col = i - row * (ND * NU);
                dT[col * NUP + row] = gd[i];
            }
        }
        const T* gm3 = static_cast<const T*>(el.m3);     // [NU][NF]
        for (int i = threadIdx.x; i < NU * NF; i += blockDim.x) {
            const int row = i / NF, f = i - row * NF;
            m3T[f * NUP + row] = gm3[i];
        }
        const T* gs = static_cast<const T*>(el.smats) + e * NU * ND * ND;
        for (int i = threadIdx.x; i < NU * ND * SR; i += blockDim.x) {
            const int row = i / SR, k = i - row * SR;
            sm[i] = k < ND ? gs[row * ND + k] : T(0);
        }
        const T* gr = static_cast<const T*>(el.rcpdjac) + e * NU;
        for (int i = threadIdx.x; i < NU; i += blockDim.x) rj[i] = gr[i];
        const T* gp = static_cast<const T*>(el.pnorm) + e * NF * ND;
        const T* gg = static_cast<const T*>(el.magn) + e * NF;
        for (int i = threadIdx.x; i < NF * 4; i += blockDim.x) {
            const int f = i >> 2, k = i & 3;
            pn[i] = k < ND ? gp[f * ND + k] : (k == 3 ? gg[f] : T(0));
        }
        for (int i = threadIdx.x; i < NF; i += blockDim.x) {
            nb[i] = el.nbr[e * NF + i];
            // table entries clamped into range (a malformed table gives wrong
            // values, never an out-of-range access)
            if constexpr (GATHER || TPP > 0) fs[i] = min(max(fsel[i], 0), NU - 1);
            if constexpr (TPP > 0) {
                fdm[i] = min(max(tp.fdim[i], 0), ND - 1);
                fsg[i] = static_cast<const T*>(tp.fsgn)[i];
            }
        }
        if constexpr (TPP > 0) {
            const T* gl = static_cast<const T*>(tp.m1line);
            for (int i = threadIdx.x; i < ND * NU * 4; i += blockDim.x) m1l[i] = gl[i];
        }
    }
    __syncthreads();
    const int64_t nv = el.nv;
    const T* c0 = static_cast<const T*>(el.c0);
    const T* uw = static_cast<const T*>(wl.uwall);
    const T* fw = static_cast<const T*>(wl.fw);
    const T* bcv = static_cast<const T*>(wl.bcv);
    // Every row the thread reads in one velocity step, in order, goes through
    // a per-thread ring of RING slots in shared memory, filled by cp.async
    // RING - 1 rows ahead (no registers held for the prefetch):
    //   k < NU              u_k (volume)
    //   k < NU + 2 NF       face f = (k - NU) / 2: own value, then the
    //                       neighbour's (or the wall Maxwellian's)
    //   k < NU + 2 NF + 3 NU  combination row i: u_i, x1_i, x2_i
    constexpr int NR = NU + 2 * NF + 3 * NU;
    T* ring = reinterpret_cast<T*>(smraw) + size_t(threadIdx.x) * VB;   // slot r at ring + r*128*VB
    auto lsrc = [&](int f, int64_t v0) -> const T* {
        if constexpr (GATHER) return u + (e * NU + fs[f]) * nv + v0;
        else return uf + (e * NF + f) * nv + v0;
    };
    auto rsrc = [&](int f, int64_t v0) -> const T* {
        const int n = nb[f];
        if (n < 0) {
            const int bid = wl.bcid[-1 - n];
            const int kd = wl.kind ? wl.kind[bid] : BDGFS_BC_DIFFUSE;
            // specular: this face's own row at the mirrored velocities
            if (kd >= BDGFS_BC_SPECULAR_X) return lsrc(f, mirror_chunk(v0, el.Nv, kd, VB));
            return fw + int64_t(bid) * nv + v0;
        }
        if constexpr (GATHER) {
            const int en = n / NF;
            if (en >= el.neles) return lsrc(f, v0);     // outside this state: no flux
            return u + (int64_t(en) * NU + fs[n - en * NF]) * nv + v0;
        } else {
            return uf + int64_t(n) * nv + v0;
        }
    };
    auto rowptr = [&](int k, int64_t v0) -> const T* {
        if (k < NU) return u + (e * NU + k) * nv + v0;
        k -= NU;
        if (k < 2 * NF) return (k & 1) ? rsrc(k >> 1, v0) : lsrc(k >> 1, v0);
        k -= 2 * NF;
        const int i = k / 3, w = k - 3 * (k / 3);
        const T* base = w == 0 ? u : (w == 1 ? (x1 ? x1 : u) : (x2 ? x2 : u));
        return base + (e * NU + i) * nv + v0;
    };
    // Sources of the rows past the volume rows (k >= NU) are the same for
    // every thread of the CTA and are looked up once: rowp, the row at
    // velocity 0, and rowm, 0 or 1 + the mirrored axis of a specular wall
    // (that row is read at the mirrored velocity chunk).  moff[m][thread]
    // holds the thread's velocity offset for kind m (128 threads per CTA):
    // 0 for m = 0, the others set per velocity step when a specular wall is
    // present.  The volume rows are addressed directly.
    __shared__ const T* rowp[NR - NU];
    __shared__ unsigned char rowm[NR - NU];
    __shared__ int64_t moff[4][128];
    for (int k = NU + int(threadIdx.x); k < NR; k += int(blockDim.x)) {
        const int kk = k - NU;
        unsigned char m = 0;
        if (kk < 2 * NF && (kk & 1) && nb[kk >> 1] < 0) {
            const int bid = wl.bcid[-1 - nb[kk >> 1]];
            const int kd = wl.kind ? wl.kind[bid] : BDGFS_BC_DIFFUSE;
            if (kd >= BDGFS_BC_SPECULAR_X) m = static_cast<unsigned char>(1 + kd - BDGFS_BC_SPECULAR_X);
        }
        rowp[kk] = m ? lsrc(kk >> 1, 0) : rowptr(k, 0);
        rowm[kk] = m;
    }
    moff[0][threadIdx.x] = 0;
    const bool mirrors = wl.kind && (wl.kinds_used & ((1 << BDGFS_BC_SPECULAR_X) | (1 << BDGFS_BC_SPECULAR_Y) |
                                                      (1 << BDGFS_BC_SPECULAR_Z)));
    __syncthreads();
    auto issue = [&](int k, int64_t v0) {
        if (k < NR) {
            const T* src;
            if (k < NU) {
                src = u + (e * NU + k) * nv + v0;
            } else {
                src = rowp[k - NU] + v0 + moff[rowm[k - NU]][threadIdx.x];
            }
            cp_async<VB * sizeof(T)>(ring + size_t(k % RING) * 128 * VB, src);
        }
        cp_async_commit();
    };
    auto take = [&](int k) {
        cp_async_wait<RING - 1>();
        Vec<T, VB> r;
        r.load(ring + size_t(k % RING) * 128 * VB);
        return r;
    };
    const int64_t v1 = (int64_t(blockIdx.x) + 1) * chunk < nv ? (int64_t(blockIdx.x) + 1) * chunk : nv;
    for (int64_t v0 = int64_t(blockIdx.x) * chunk + int64_t(threadIdx.x) * VB; v0 < v1;
         v0 += int64_t(blockDim.x) * VB) {
        T c[VB][3];
#pragma unroll
        for (int q = 0; q < VB; ++q) vel(c0, el.Nv, v0 + q, c[q]);
        if (mirrors) {                                   // the thread's own slots only
#pragma unroll
            for (int a = 0; a < 3; ++a)
                moff[1 + a][threadIdx.x] = mirror_chunk(v0, el.Nv, BDGFS_BC_SPECULAR_X + a, VB) - v0;
        }
        Racc<T, NU, VB, PK> R;
#pragma unroll
        for (int q = 0; q < VB; ++q)
#pragma unroll
            for (int i = 0; i < NU; ++i) R(q, i) = T(0);
#pragma unroll
        for (int k = 0; k < RING - 1; ++k) issue(k, v0);
        if constexpr (TPP > 0) {
            // volume: R += M1 F~ along the lines of M1 (rows known at compile time)
#pragma unroll
            for (int j = 0; j < NU; ++j) {
                issue(j + RING - 1, v0);
                const Vec<T, VB> uj = take(j);
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    // scalar reads here: this loop is unrolled over every (j, d)
                    // and vector reads of the padded rows measured slower
                    const T* srow = sm + (j * ND + d) * SR;
                    const T* w = m1l + (d * NU + j) * 4;
                    T ft[VB];
#pragma unroll
                    for (int q = 0; q < VB; ++q) {
                        T al = T(0);
#pragma unroll
                        for (int k = 0; k < ND; ++k) al += srow[k] * c[q][k];
                        ft[q] = al * uj.v[q];
                    }
                    const int st = d == 0 ? 1 : (d == 1 ? TPP : TPP * TPP);
                    const int base = j - ((j / st) % TPP) * st;
#pragma unroll
                    for (int t = 0; t < TPP; ++t) {
                        const T wt = w[t];
#pragma unroll
                        for (int q = 0; q < VB; ++q) R(q, base + t * st) += wt * ft[q];
                    }
                }
            }
        } else {
        // volume: R += (M1 - M3 M2) F~,  F~[d][j] = (sum_k smats[j][d][k] c_k) u_j
#pragma unroll 1
        for (int j = 0; j < NU; ++j) {
            issue(j + RING - 1, v0);
            const Vec<T, VB> uj = take(j);
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                T srow[SR];
                lds_vec<T, SR>(sm + (j * ND + d) * SR, srow);
                T ft[VB];
#pragma unroll
                for (int q = 0; q < VB; ++q) {
                    T al = T(0);
#pragma unroll
                    for (int k = 0; k < ND; ++k) al += srow[k] * c[q][k];
                    ft[q] = al * uj.v[q];
                }
                axpy_col<T, NU, NUP, VB, PK>(dT + (d * NU + j) * NUP, ft, R);
            }
        }
        }
        // surface: common normal flux at each face point, lifted by M3
#pragma unroll 1
        for (int f = 0; f < NF; ++f) {
            const int k = NU + 2 * f;
            issue(k + RING - 1, v0);
            const Vec<T, VB> ul = take(k);
            issue(k + RING, v0);
            Vec<T, VB> ur = take(k + 1);
            const int n = nb[f];
            T prow[4];                                       // unit normal, |n| at 3
            lds_vec<T, 4>(pn + f * 4, prow);
            T nc[VB];
#pragma unroll
            for (int q = 0; q < VB; ++q) {
                nc[q] = T(0);
#pragma unroll
                for (int d = 0; d < ND; ++d) nc[q] += prow[d] * c[q][d];
            }
            if (n < 0) {                                     // boundary: ur holds f_w or the mirrored row
                const int w = -1 - n;
                const int bid = wl.bcid[w];
                const int kd = wl.kind ? wl.kind[bid] : BDGFS_BC_DIFFUSE;
                if (kd == BDGFS_BC_OUTLET) {
                    ur = ul;
                } else if (kd == BDGFS_BC_SPECULAR_Z) {      // mirrored chunk comes reversed
#pragma unroll
                    for (int q = 0; q < VB / 2; ++q) {
                        const T t = ur.v[q];
                        ur.v[q] = ur.v[VB - 1 - q];
                        ur.v[VB - 1 - q] = t;
                    }
                } else if (kd < BDGFS_BC_SPECULAR_X) {       // diffuse wall or inlet
                    const T sc = kd == BDGFS_BC_DIFFUSE ? -bcv[2 * w] / bcv[2 * w + 1] : T(1);
#pragma unroll
                    for (int q = 0; q < VB; ++q) {
                        T fac = T(0);
#pragma unroll
                        for (int d = 0; d < ND; ++d) fac += (c[q][d] - uw[bid * 3 + d]) * prow[d];
                        ur.v[q] = (fac < T(0)) ? ur.v[q] * sc : ul.v[q];
                    }
                }
            }
            T fh[VB];
#pragma unroll
            for (int q = 0; q < VB; ++q) {
                const T fn = T(0.5) * nc[q] * (ul.v[q] + ur.v[q]) + T(0.5) * fabs(nc[q]) * (ul.v[q] - ur.v[q]);
                fh[q] = prow[3] * fn;
            }
            if constexpr (TPP > 0) {                         // F^n - M2 F~ (ul is u at fsel[f])
                const int jf = fs[f], df = fdm[f];
                const T sg = fsg[f];
                T srow[SR];
                lds_vec<T, SR>(sm + (jf * ND + df) * SR, srow);
#pragma unroll
                for (int q = 0; q < VB; ++q) {
                    T al = T(0);
#pragma unroll
                    for (int k = 0; k < ND; ++k) al += srow[k] * c[q][k];
                    fh[q] -= sg * al * ul.v[q];
                }
            }
            axpy_col<T, NU, NUP, VB, PK>(m3T + f * NUP, fh, R);
        }
        // combination rows u, x1, x2: out = a u + b L(u) + c1 x1 + c2 x2
#pragma unroll
        for (int i = 0; i < NU; ++i) {
            const int k = NU + 2 * NF + 3 * i;
            issue(k + RING - 1, v0);
            const Vec<T, VB> ui = take(k);
            issue(k + RING, v0);
            const Vec<T, VB> y1 = take(k + 1);
            issue(k + RING + 1, v0);
            const Vec<T, VB> y2 = take(k + 2);
            Vec<T, VB> o;
#pragma unroll
            for (int q = 0; q < VB; ++q) o.v[q] = a * ui.v[q] + b * (-rj[i] * R(q, i));
            if (x1) {
#pragma unroll
                for (int q = 0; q < VB; ++q) o.v[q] += c1 * y1.v[q];
            }
            if (x2) {
#pragma unroll
                for (int q = 0; q < VB; ++q) o.v[q] += c2 * y2.v[q];
            }
            o.store(out + (e * NU + i) * nv + v0);
        }
    }
}

// uf: face-value rows [E][NF]; or, with fsel, the solution-point rows of u
// ([E][NU]) read at row fsel[f] (GATHER, M0 rows unit vectors)
template <typename T>
__global__ void __launch_bounds__(256) bc_update_kernel(const bdgfs_fr_eles el,
                                                        const bdgfs_fr_walls wl,
                                                        const T* __restrict__ uf,
                                                        const int32_t* __restrict__ fsel)
{
    __shared__ double red[2 * 8];
    __shared__ T cs[1024];                                    // cell-centre velocities (Nv <= 1024)
    const int w = blockIdx.x;
    const int e = wl.fpt[2 * w], f = wl.fpt[2 * w + 1];
    const int bid = wl.bcid[w];
    if (wl.kind && wl.kind[bid] != BDGFS_BC_DIFFUSE) {        // nothing to balance
        if (threadIdx.x == 0) {
            T* out = static_cast<T*>(wl.bcv);
            out[2 * w] = T(0);
            out[2 * w + 1] = T(-1);
        }
        return;
    }
    const int ND = el.ndims;
    const T* pn = static_cast<const T*>(el.pnorm) + (int64_t(e) * el.nfpts + f) * ND;
    const T* uw = static_cast<const T*>(wl.uwall) + bid * 3;
    const T* fw = static_cast<const T*>(wl.fw) + int64_t(bid) * el.nv;
    const T* ul = fsel ? uf + (int64_t(e) * el.nupts + fsel[f]) * el.nv
                       : uf + (int64_t(e) * el.nfpts + f) * el.nv;
    const T* c0 = static_cast<const T*>(el.c0);
    for (int i = threadIdx.x; i < el.Nv; i += blockDim.x) cs[i] = c0[i];
    __syncthreads();
    double s0 = 0.0, s1 = 0.0;
    // four velocities per step (16-byte loads) when rows are aligned; with
    // Nv % 4 == 0 the four share one z line (one index split per step)
    const bool v4 = sizeof(T) == 4 && el.nv % 4 == 0 && (reinterpret_cast<uintptr_t>(ul) & 15u) == 0 &&
                    (reinterpret_cast<uintptr_t>(fw) & 15u) == 0;
    const bool zline = el.Nv % 4 == 0;
    const int64_t nv4 = v4 ? el.nv : 0;
    for (int64_t v0 = int64_t(threadIdx.x) * 4; v0 < nv4; v0 += int64_t(blockDim.x) * 4) {
        Vec<T, 4> a, b;
        a.load(ul + v0);
        b.load(fw + v0);
        const uint32_t vv = uint32_t(v0), nn = uint32_t(el.Nv);    // v < Nv^3 <= 2^30
        const uint32_t qq = vv / nn, iz0 = vv - qq * nn;
        const uint32_t ix = qq / nn, iy = qq - ix * nn;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            T c[3];
            if (zline) {
                c[0] = cs[ix];
                c[1] = cs[iy];
                c[2] = cs[iz0 + q];
            } else {
                vel(cs, el.Nv, v0 + q, c);
            }
            T fac = T(0);
            for (int d = 0; d < ND; ++d) fac += (c[d] - uw[d]) * pn[d];
            if (fac >= T(0)) s0 += double(fac * a.v[q]);
            else s1 += double(fac * b.v[q]);
        }
    }
    for (int64_t v = nv4 + threadIdx.x; v < el.nv; v += blockDim.x) {
        T c[3];
        vel(cs, el.Nv, v, c);
        T fac = T(0);
        for (int d = 0; d < ND; ++d) fac += (c[d] - uw[d]) * pn[d];
        if (fac >= T(0)) s0 += double(fac * ul[v]);
        else s1 += double(fac * fw[v]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[2 * warp] = s0; red[2 * warp + 1] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int i = 0; i < int(blockDim.x >> 5); ++i) { a0 += red[2 * i]; a1 += red[2 * i + 1]; }
        T* out = static_cast<T*>(wl.bcv);
        out[2 * w] = T(a0 * wl.cw);
        out[2 * w + 1] = T(a1 * wl.cw);
    }
}

// raw FP64 velocity moments of each distribution:
// sum f, sum c f (3), sum c_i c_j f (6: xx xy xz yy yz zz), sum |c|^2 c f (3)
template <typename T>
__global__ void __launch_bounds__(256) moments_kernel(const T* __restrict__ f, int Nv,
                                                      const double* __restrict__ c0, double cw,
                                                      double* __restrict__ out)
{
    __shared__ double red[13 * 8];
    const int64_t n = int64_t(Nv) * Nv * Nv;
    const T* fd = f + int64_t(blockIdx.x) * n;
    double m[13];
#pragma unroll
    for (int j = 0; j < 13; ++j) m[j] = 0.0;
    for (int64_t v = threadIdx.x; v < n; v += blockDim.x) {
        const double cx = c0[v / (int64_t(Nv) * Nv)], cy = c0[(v / Nv) % Nv], cz = c0[v % Nv];
        const double fv = double(fd[v]);
        const double c2 = cx * cx + cy * cy + cz * cz;
        m[0] += fv;
        m[1] += cx * fv; m[2] += cy * fv; m[3] += cz * fv;
        m[4] += cx * cx * fv; m[5] += cx * cy * fv; m[6] += cx * cz * fv;
        m[7] += cy * cy * fv; m[8] += cy * cz * fv; m[9] += cz * cz * fv;
        m[10] += c2 * cx * fv; m[11] += c2 * cy * fv; m[12] += c2 * cz * fv;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 13; ++j) {
        double x = m[j];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp * 13 + j] = x;
    }
    __syncthreads();
    if (threadIdx.x < 13) {
        double s = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += red[w * 13 + threadIdx.x];
        out[int64_t(blockIdx.x) * 13 + threadIdx.x] = s * cw;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) residual_kernel(const T* __restrict__ a,
                                                       const T* __restrict__ b, int64_t n,
                                                       double* out)
{
    __shared__ double red[2 * 8];
    double s0 = 0.0, s1 = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const double x = double(a[i]), y = double(b[i]);
        s0 += (x - y) * (x - y);
        s1 += y * y;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { red[2 * warp] = s0; red[2 * warp + 1] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0;
        for (int i = 0; i < int(blockDim.x >> 5); ++i) { a0 += red[2 * i]; a1 += red[2 * i + 1]; }
        atomicAdd(out, a0);
        atomicAdd(out + 1, a1);
    }
}

// status word check: any non-finite or negative-density flag set by the
// scan below (NaN/Inf detection of the state, read back after graph replay)
template <typename T>
__global__ void __launch_bounds__(256) status_kernel(const T* __restrict__ a, int64_t n,
                                                     int32_t* status)
{
    int bad = 0;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const T x = a[i];
        if (!isfinite(x)) bad |= 1;
    }
    bad = __reduce_or_sync(0xffffffffu, bad);
    if (bad && (threadIdx.x & 31) == 0) atomicOr(status, bad);
}

// Velocity chunk per CTA (a multiple of 128*VB).
static int64_t fr_chunk(int64_t nv, int neles, int VB)
{
    // one 128*VB velocity step per CTA: staging the operators costs ~40
    // instructions per thread against ~20k of work, and short CTAs balance
    // the waves; longer chunks only when the grid's x extent would overflow
    const int64_t step = 128 * int64_t(VB);
    int64_t chunk = step;
    while ((nv + chunk - 1) / chunk > 65535) chunk *= 2;
    (void)neles;
    return chunk;
}

static int grid_v(int64_t nv, int neles, int64_t chunk, dim3* g)
{
    const int64_t bx = (nv + chunk - 1) / chunk;
    if (bx > 65535 || neles > 65535 || neles < 1) return BDGFS_EINVAL;
    *g = dim3(unsigned(bx), unsigned(neles));
    return BDGFS_OK;
}

// VB velocities per thread when every row is VB-aligned
template <typename T>
static int vec_width(int64_t nv, const void* const* ptrs, int n)
{
    const int VB = sizeof(T) == 4 ? 4 : 2;
    if (nv % VB) return 1;
    for (int i = 0; i < n; ++i)
        if (ptrs[i] && (reinterpret_cast<uintptr_t>(ptrs[i]) % (VB * sizeof(T)))) return 1;
    return VB;
}

template <typename T, int ND, int NU, int NF, int VB, int TPP = 0>
static int rhs_launch_vb(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl, const void* u,
                         const void* uf, const int32_t* fsel, const bdgfs_fr_tensor* tp, void* out,
                         double a, double b, const void* x1, double c1, const void* x2, double c2,
                         cudaStream_t st)
{
    constexpr int NUP = (NU + 3) / 4 * 4;
    const int64_t chunk = fr_chunk(el->nv, el->neles, VB);
    dim3 g;
    if (grid_v(el->nv, el->neles, chunk, &g) != BDGFS_OK) return BDGFS_EINVAL;
    constexpr int RING = 8;
    constexpr int SR = ND == 3 ? 4 : ND;
    const size_t smem = sizeof(T) * (size_t(RING) * 128 * VB + ((TPP ? 0 : ND * NU) + NF) * NUP + NU * ND * SR
                                     + NF * 4 + (TPP ? ND * NU * 4 + NF : 0) + NU)
                        + sizeof(int) * 3 * NF + 16;
    auto k = TPP ? (uf ? rhs_kernel<T, ND, NU, NF, VB, false, RING, TPP>
                       : rhs_kernel<T, ND, NU, NF, VB, true, RING, TPP>)
                 : (fsel ? rhs_kernel<T, ND, NU, NF, VB, true, RING> : rhs_kernel<T, ND, NU, NF, VB, false, RING>);
    if (const int rc = smem_optin(reinterpret_cast<const void*>(k), smem)) return rc;
    bdgfs_fr_walls w0{};
    const bdgfs_fr_tensor t0{};
    k<<<g, 128, smem, st>>>(*el, wl ? *wl : w0, static_cast<const T*>(u), static_cast<const T*>(uf),
                            fsel, tp ? *tp : t0, static_cast<T*>(out), T(a), T(b),
                            static_cast<const T*>(x1), T(c1), static_cast<const T*>(x2), T(c2), chunk);
    return cuda_status(cudaGetLastError());
}

template <typename T, int ND, int NU, int NF, int TPP = 0>
static int rhs_launch(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl, const void* u,
                      const void* uf, const int32_t* fsel, const bdgfs_fr_tensor* tp, void* out,
                      double a, double b, const void* x1, double c1, const void* x2, double c2,
                      cudaStream_t st)
{
    const void* ptrs[] = {u, uf, out, x1, x2, wl ? wl->fw : nullptr};
    // 4 velocities per thread for float (each operator column read from
    // shared memory feeds 4 x 4 FMAs; measured faster than 2 also for NU = 27)
    constexpr int VBW = sizeof(T) == 4 ? 4 : 2;
    const int ymask = (1 << BDGFS_BC_SPECULAR_Y) | (1 << BDGFS_BC_SPECULAR_Z);
    const bool mirror_ok = !(wl && wl->kind && (wl->kinds_used & ymask)) || el->Nv % VBW == 0;
    if (mirror_ok && vec_width<T>(el->nv, ptrs, 6) >= VBW)
        return rhs_launch_vb<T, ND, NU, NF, VBW, TPP>(el, wl, u, uf, fsel, tp, out, a, b, x1, c1, x2, c2, st);
    return rhs_launch_vb<T, ND, NU, NF, 1, TPP>(el, wl, u, uf, fsel, tp, out, a, b, x1, c1, x2, c2, st);
}

template <typename T, int NU, int NF, int VB>
static int disu_launch_vb(const bdgfs_fr_eles* el, const void* op, const void* u, void* uf,
                          cudaStream_t st)
{
    const int64_t chunk = fr_chunk(el->nv, el->neles, VB);
    dim3 g;
    if (grid_v(el->nv, el->neles, chunk, &g) != BDGFS_OK) return BDGFS_EINVAL;
    disu_kernel<T, NU, NF, VB><<<g, 128, 0, st>>>(*el, static_cast<const T*>(op), static_cast<const T*>(u),
                                                  static_cast<T*>(uf), chunk);
    return cuda_status(cudaGetLastError());
}

// op: [NF][NU] operator (M0 for disu, the inverse mass matrix for invmass)
template <typename T, int NU, int NF>
static int disu_launch(const bdgfs_fr_eles* el, const void* op, const void* u, void* uf, cudaStream_t st)
{
    const void* ptrs[] = {u, uf};
    constexpr int VBW = sizeof(T) == 4 ? 4 : 2;
    if (vec_width<T>(el->nv, ptrs, 2) == VBW) return disu_launch_vb<T, NU, NF, VBW>(el, op, u, uf, st);
    return disu_launch_vb<T, NU, NF, 1>(el, op, u, uf, st);
}

#define BDGFS_FR_SHAPES(X)                                                          \
    X(2, 4, 8) X(2, 9, 12) X(2, 16, 16) X(2, 25, 20) X(3, 8, 24) X(3, 27, 54)

static bool shape_ok(const bdgfs_fr_eles* el)
{
#define CHK(D, U, F) if (el->ndims == D && el->nupts == U && el->nfpts == F) return true;
    BDGFS_FR_SHAPES(CHK)
#undef CHK
    return false;
}

static int check_eles(const bdgfs_fr_eles* el)
{
    if (!el || el->nv < 1 || el->neles < 1 || el->Nv < 1 || el->Nv > 1024 ||
        int64_t(el->Nv) * el->Nv * el->Nv != el->nv)
        return BDGFS_EINVAL;
    if (!el->m0 || !el->dcorr || !el->m3 || !el->smats || !el->rcpdjac || !el->pnorm ||
        !el->magn || !el->nbr || !el->c0)
        return BDGFS_EINVAL;
    return shape_ok(el) ? BDGFS_OK : BDGFS_EUNSUPPORTED;
}

}  // namespace bdgfs

using namespace bdgfs;

extern "C" int32_t bdgfs_fr_disu(const bdgfs_fr_eles* el, const void* u, void* uf, void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!u || !uf) return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define GO(D, U, F)                                                                         \
    if (el->ndims == D && el->nupts == U && el->nfpts == F)                                 \
        return el->fp64 ? disu_launch<double, U, F>(el, el->m0, u, uf, st)                 \
                        : disu_launch<float, U, F>(el, el->m0, u, uf, st);
    BDGFS_FR_SHAPES(GO)
#undef GO
    return BDGFS_EUNSUPPORTED;
}

extern "C" int32_t bdgfs_fr_invmass(const bdgfs_fr_eles* el, const void* minv, const void* u, void* out,
                                    void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!minv || !u || !out || u == out) return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define GO(D, U, F)                                                                         \
    if (el->ndims == D && el->nupts == U && el->nfpts == F)                                 \
        return el->fp64 ? disu_launch<double, U, U>(el, minv, u, out, st)                   \
                        : disu_launch<float, U, U>(el, minv, u, out, st);
    BDGFS_FR_SHAPES(GO)
#undef GO
    return BDGFS_EUNSUPPORTED;
}

extern "C" int32_t bdgfs_fr_bc_update(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                                      const void* uf, void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!wl || !uf) return BDGFS_EINVAL;
    if (wl->nwall == 0) return BDGFS_OK;
    if (wl->nwall < 0 || !wl->fpt || !wl->bcid || !wl->uwall || !wl->fw || !wl->bcv)
        return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (el->fp64)
        bc_update_kernel<double><<<wl->nwall, 256, 0, st>>>(*el, *wl, static_cast<const double*>(uf),
                                                            nullptr);
    else
        bc_update_kernel<float><<<wl->nwall, 256, 0, st>>>(*el, *wl, static_cast<const float*>(uf),
                                                           nullptr);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_fr_bc_update_gather(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                                             const int32_t* fsel, const void* u, void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!wl || !u || !fsel) return BDGFS_EINVAL;
    if (wl->nwall == 0) return BDGFS_OK;
    if (wl->nwall < 0 || !wl->fpt || !wl->bcid || !wl->uwall || !wl->fw || !wl->bcv)
        return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (el->fp64)
        bc_update_kernel<double><<<wl->nwall, 256, 0, st>>>(*el, *wl, static_cast<const double*>(u), fsel);
    else
        bc_update_kernel<float><<<wl->nwall, 256, 0, st>>>(*el, *wl, static_cast<const float*>(u), fsel);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_fr_rhs(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl, const void* u,
                                const void* uf, void* out, double a, double b, const void* x1,
                                double c1, const void* x2, double c2, void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!u || !uf || !out) return BDGFS_EINVAL;
    if (wl && wl->nwall > 0 && (!wl->bcid || !wl->uwall || !wl->fw || !wl->bcv))
        return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!el->fp64 && el->engine == 1) {          // tensor-core engine when the shape has one
        const bdgfs_fr_walls w0{};
        const int tc = fr_rhs_tc(*el, wl ? *wl : w0, u, uf, out, a, b, x1, c1, x2, c2, st);
        if (tc != BDGFS_EUNSUPPORTED) return tc;
    }
#define GO(D, U, F)                                                                          \
    if (el->ndims == D && el->nupts == U && el->nfpts == F)                                  \
        return el->fp64 ? rhs_launch<double, D, U, F>(el, wl, u, uf, nullptr, nullptr, out, a, b, x1, c1, x2, c2, st) \
                        : rhs_launch<float, D, U, F>(el, wl, u, uf, nullptr, nullptr, out, a, b, x1, c1, x2, c2, st);
    BDGFS_FR_SHAPES(GO)
#undef GO
    return BDGFS_EUNSUPPORTED;
}

extern "C" int32_t bdgfs_fr_rhs_gather(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                                       const int32_t* fsel, const void* u, void* out, double a,
                                       double b, const void* x1, double c1, const void* x2,
                                       double c2, void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!u || !out || !fsel || out == u) return BDGFS_EINVAL;
    if (wl && wl->nwall > 0 && (!wl->bcid || !wl->uwall || !wl->fw || !wl->bcv))
        return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define GO(D, U, F)                                                                          \
    if (el->ndims == D && el->nupts == U && el->nfpts == F)                                  \
        return el->fp64 ? rhs_launch<double, D, U, F>(el, wl, u, nullptr, fsel, nullptr, out, a, b, x1, c1, x2, c2, st) \
                        : rhs_launch<float, D, U, F>(el, wl, u, nullptr, fsel, nullptr, out, a, b, x1, c1, x2, c2, st);
    BDGFS_FR_SHAPES(GO)
#undef GO
    return BDGFS_EUNSUPPORTED;
}

extern "C" int32_t bdgfs_fr_rhs_tensor(const bdgfs_fr_eles* el, const bdgfs_fr_walls* wl,
                                       const bdgfs_fr_tensor* tp, const void* u, const void* uf,
                                       void* out, double a, double b, const void* x1, double c1,
                                       const void* x2, double c2, void* stream)
{
    int rc = check_eles(el);
    if (rc != BDGFS_OK) return rc;
    if (!tp || !tp->fsel || !tp->fdim || !tp->fsgn || !tp->m1line || !u || !out || (!uf && out == u))
        return BDGFS_EINVAL;
    if (wl && wl->nwall > 0 && (!wl->bcid || !wl->uwall || !wl->fw || !wl->bcv))
        return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
#define GO(D, U, F, P)                                                                        \
    if (el->ndims == D && el->nupts == U && el->nfpts == F && tp->p == P)                     \
        return el->fp64 ? rhs_launch<double, D, U, F, P>(el, wl, u, uf, tp->fsel, tp, out, a, b, x1, c1, x2, c2, st) \
                        : rhs_launch<float, D, U, F, P>(el, wl, u, uf, tp->fsel, tp, out, a, b, x1, c1, x2, c2, st);
    GO(2, 4, 8, 2) GO(2, 9, 12, 3) GO(2, 16, 16, 4) GO(3, 8, 24, 2) GO(3, 27, 54, 3)
#undef GO
    return BDGFS_EUNSUPPORTED;
}

extern "C" int32_t bdgfs_moments(const void* f, int64_t ndof, int32_t Nv, int32_t fp64,
                                 const double* c0, double cw, double* out, void* stream)
{
    if (!f || !c0 || !out || ndof < 0 || Nv < 1) return BDGFS_EINVAL;
    if (ndof == 0) return BDGFS_OK;
    if (ndof > 2147483647LL) return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (fp64)
        moments_kernel<double><<<unsigned(ndof), 256, 0, st>>>(static_cast<const double*>(f), Nv, c0, cw, out);
    else
        moments_kernel<float><<<unsigned(ndof), 256, 0, st>>>(static_cast<const float*>(f), Nv, c0, cw, out);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_residual(const void* a, const void* b, int64_t n, int32_t fp64,
                                  double* out2, void* stream)
{
    if (!a || !b || !out2 || n < 0) return BDGFS_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(out2, 0, 2 * sizeof(double), st) != cudaSuccess) return BDGFS_ECUDA;
    if (n == 0) return BDGFS_OK;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (fp64)
        residual_kernel<double><<<unsigned(blocks), 256, 0, st>>>(static_cast<const double*>(a),
                                                                  static_cast<const double*>(b), n, out2);
    else
        residual_kernel<float><<<unsigned(blocks), 256, 0, st>>>(static_cast<const float*>(a),
                                                                 static_cast<const float*>(b), n, out2);
    return cuda_status(cudaGetLastError());
}

extern "C" int32_t bdgfs_status_check(const void* a, int64_t n, int32_t fp64, int32_t* status,
                                      void* stream)
{
    if (!a || !status || n < 0) return BDGFS_EINVAL;
    if (n == 0) return BDGFS_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int64_t blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (fp64)
        status_kernel<double><<<unsigned(blocks), 256, 0, st>>>(static_cast<const double*>(a), n, status);
    else
        status_kernel<float><<<unsigned(blocks), 256, 0, st>>>(static_cast<const float*>(a), n, status);
    return cuda_status(cudaGetLastError());
}
