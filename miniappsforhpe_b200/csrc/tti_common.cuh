// Shared definitions for the B200 TTI/VTI pseudo-acoustic RTM kernels.
//
// Volume layout (reference contract, utils/volume_index.h:20-23 and
// infrastructure/axis.cpp:78-99): FP32, x fastest,
//   idx = (iz*ldimy + iy)*ldimx + ix,
// a radius-4 halo on every axis, the interior is [ibeg, iend] per axis and
// ldimx is padded to a multiple of 32 floats (128 bytes).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/tti_capi.h"

namespace tti {

constexpr int kRadius = 4;

// Least-squares 8th-order coefficients used by every launcher of the path.
// Staggered first derivative: kernels/fd_coef.h:464-470 (DF_order8_1..4).
__host__ __device__ __forceinline__ float c1(int i)
{
    constexpr float c[5] = {0.0f, 1.19628906250000e+00f, -7.97526041666667e-02f, 9.57031250000000e-03f,
                            -6.97544642857143e-04f};
    return c[i];
}
// Centred second-derivative set, used along the diagonals for the mixed
// derivatives: kernels/fd_coef.h:516-521 (DF2_order8_0..4).
__host__ __device__ __forceinline__ float c2(int i)
{
    constexpr float c[5] = {-0.2903117E+1f, 0.1645351E+1f, -0.2236606E+0f, 0.3265851E-1f, -0.2790073E-2f};
    return c[i];
}
// stg_d1<8> (kernels/fd_coefficients.h:28-31); equal to c1(i+1) in float.
__host__ __device__ __forceinline__ float cs(int r)
{
    constexpr float c[4] = {1.1962891e+0f, -7.9752604e-2f, 9.5703125e-3f, -6.9754464e-4f};
    return c[r];
}
// Tap k (0..7) of the staggered operator written as consecutive points:
// -c4,-c3,-c2,-c1,+c1,+c2,+c3,+c4 (kernel_type2_fwd.cu:104-115).
__host__ __device__ __forceinline__ float tap(int k) { return (k < 4) ? -c1(4 - k) : c1(k - 3); }

struct Layout {
    int ldimx, ldimy, ldimz;
    int ixbeg, ixend, iybeg, iyend, izbeg, izend;
    __host__ __device__ int64_t idx(int ix, int iy, int iz) const
    {
        return ((int64_t)iz * ldimy + iy) * (int64_t)ldimx + ix;
    }
    __host__ __device__ int64_t zstride() const { return (int64_t)ldimx * ldimy; }
    __host__ __device__ int nx() const { return ixend - ixbeg + 1; }
    __host__ __device__ int ny() const { return iyend - iybeg + 1; }
    __host__ __device__ int nz() const { return izend - izbeg + 1; }
};

// Snapshot storage precision: FP32, or FP16/BF16 holding value*scale with a
// per-snapshot, per-field power-of-two scale.
enum SnapPrec { SNAP_F32 = 0, SNAP_F16 = 1, SNAP_BF16 = 2 };
inline size_t snap_elt_bytes(int prec) { return prec == SNAP_F32 ? 4 : 2; }

// Store v (already scaled) at element i; returns true if it had to saturate.
__device__ __forceinline__ bool snap_store(void* base, int64_t i, float v, int prec)
{
    if (prec == SNAP_F32) {
        static_cast<float*>(base)[i] = v;
        return false;
    }
    if (prec == SNAP_F16) {
        const bool sat = fabsf(v) > 65504.0f;
        static_cast<__half*>(base)[i] = __float2half_rn(fminf(fmaxf(v, -65504.0f), 65504.0f));
        return sat;
    }
    static_cast<__nv_bfloat16*>(base)[i] = __float2bfloat16_rn(v);
    return false;
}
// Reduced-precision wavefields: p and q leave each step rounded to FP16 or
// BF16 of value*scale and read back exactly (the scale a power of two taken
// from the largest |p|, |q| of the step before, target 2^11 below the FP16
// limit; FP16 values beyond its range are clamped, and the maxima pass
// flags them); the values stay in FP32 arrays.  prec and scale are kernel
// parameters, so the FP32 path carries no extra registers.
__device__ __forceinline__ float wave_round(int prec, float v, float s)
{
    const float w = v * s;
    const float r = prec == 1 ? __half2float(__float2half_rn(fminf(fmaxf(w, -65504.0f), 65504.0f)))
                              : __bfloat162float(__float2bfloat16_rn(w));
    return r / s;  // a power of two: exact
}
__device__ __forceinline__ void wave_apply(int prec, const float* scale, float& p, float& q)
{
    if (!prec) return;
    p = wave_round(prec, p, __ldg(scale));
    q = wave_round(prec, q, __ldg(scale + 1));
}

// a12: model1..model7 of one cell from (vp, eps, delta, vs, theta, phi),
// simulator2SetUp.cu:10-29 (init_cijs_kernel).
__device__ __forceinline__ void init_cij_cell(float v, float e, float d, float s, float th, float ph, float& m1,
                                              float& m2, float& m3, float& m4, float& m5, float& m6, float& m7)
{
    m1 = v * v * (1 + 2 * e);
    m2 = sqrtf((v * v - s * s) * (v * v * (1 + 2 * d) - s * s));
    m3 = v * v;
    m4 = s * s;
    m5 = sinf(th) * cosf(ph);
    m6 = sinf(th) * sinf(ph);
    m7 = cosf(th);
}

template <typename T> __device__ __forceinline__ float to_f32(T v);
template <> __device__ __forceinline__ float to_f32<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f32<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f32<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// Host-side check of a launcher's index ranges against the radius-4 halo
// contract.  ldimz is not part of the reference launcher signatures, so the
// z extent is the caller's responsibility (izend + 4 < ldimz).
inline bool ranges_ok(int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy)
{
    return ixbeg >= kRadius && iybeg >= kRadius && izbeg >= kRadius && ixend >= ixbeg && iyend >= iybeg &&
           izend >= izbeg && ldimx >= ixend + 1 + kRadius && ldimy >= iyend + 1 + kRadius;
}

inline int launch_status()
{
    cudaError_t e = cudaPeekAtLastError();
    if (e == cudaSuccess) return TTI_OK;
    if (e == cudaErrorMemoryAllocation) return TTI_ENOMEM;
    return TTI_ELAUNCH;
}

} // namespace tti
