// Per-distribution row helpers shared by the hybrid and BGK kernels: one
// CTA walks one velocity cube f[v], v = (ix*Nv + iy)*Nv + iz.
#pragma once
#include <cstdint>

namespace bdgfs {

constexpr int kMaxNv = 64;

// velocity index v = (ix*Nv + iy)*Nv + iz, 32-bit arithmetic; NVC > 0: Nv
// known at compile time (the divisions become multiplications)
template <int NVC = 0>
__device__ __forceinline__ void vsplit(uint32_t v, uint32_t Nv, uint32_t& ix, uint32_t& iy, uint32_t& iz)
{
    const uint32_t N = NVC > 0 ? uint32_t(NVC) : Nv;
    const uint32_t q = v / N;
    iz = v - q * N;
    ix = q / N;
    iy = q - ix * N;
}

// Four consecutive values (same x, y; z..z+3) of a row: one 16-byte load
// for float, two for double (VEC = 4), or one scalar (VEC = 1).
template <typename T, int VEC>
struct Chunk {
    T v[VEC];
    __device__ __forceinline__ void load(const T* p)
    {
        if constexpr (VEC == 4 && sizeof(T) == 4) {
            const float4 x = *reinterpret_cast<const float4*>(p);
            v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
        } else if constexpr (VEC == 4) {
            const double2 a = reinterpret_cast<const double2*>(p)[0];
            const double2 b = reinterpret_cast<const double2*>(p)[1];
            v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
        } else {
            v[0] = *p;
        }
    }
    __device__ __forceinline__ void store(T* p) const
    {
        if constexpr (VEC == 4 && sizeof(T) == 4) {
            *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        } else if constexpr (VEC == 4) {
            reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
            reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
        } else {
            *p = v[0];
        }
    }
};

// FP64 raw moments {sum x, sum c x, sum |c|^2 x} of one row (block-wide)
template <typename T, int VEC, int NVC = 0>
__device__ __forceinline__ void row_moments(const T* __restrict__ row, int n, int Nv, const double* cs,
                                            double (&m)[5])
{
#pragma unroll 2
    for (int v = threadIdx.x * VEC; v < n; v += blockDim.x * VEC) {
        Chunk<T, VEC> c;
        c.load(row + v);
        uint32_t ix, iy, iz;
        vsplit<NVC>(uint32_t(v), uint32_t(Nv), ix, iy, iz);
        const double cx = cs[ix], cy = cs[iy], b = cx * cx + cy * cy;
#pragma unroll
        for (int j = 0; j < VEC; ++j) {
            const double x = double(c.v[j]), cz = cs[iz + j];
            m[0] += x;
            m[1] += cx * x;
            m[2] += cy * x;
            m[3] += cz * x;
            m[4] += (b + cz * cz) * x;
        }
    }
}

}  // namespace bdgfs
