// Type1 discretisation of the TTI p/q system (kernels/kernel_type1_gpu_*.cu):
// constant density, centred second derivatives (DF2 least-squares
// coefficients, kernels/fd_coef.h:516-521) on the normal directions and the
// same diagonal form for the mixed ones, applied directly to p and q with no
// first-derivative stage.  Drop-in launchers for the reference's three type1
// entry points:
//   fwd_main_loop_2_1_inner_gpu::launch  (kernel_type1_gpu_fwd.h:6-9)
//   adj_main_loop_2_inner_gpu::launch    (kernel_type1_gpu_adj.h:6-9)
//   launch_update_grad_loop_kernel       (kernel_type1_gpu_grad.h:4-7)
// One thread per cell; the adjoint first forms the point-wise transposed
// model (lap/hz of both fields) in the library's four-float scratch, then
// differentiates it.  The arithmetic follows the launchers' default
// (optimised) kernels: the derivative sums of compute_z_contributions /
// compute_xy_contributions (kernel_type1_gpu_fwd.cu:150-232,
// kernel_type1_gpu_adj.cu:162-217) and the V/H combination of
// compute_result (kernel_type1_gpu_fwd.cu:122-146).
#include <cuda_runtime.h>

#include <cstdint>

#include "tti_common.cuh"
#include "tti_internal.cuh"

namespace tti {
namespace {

constexpr int T1X = 32, T1Y = 8;

struct R6 {
    int ixbeg, ixend, iybeg, iyend, izbeg, izend;
};

inline dim3 t1_grid(const R6& r)
{
    return dim3((r.ixend - r.ixbeg + T1X) / T1X, (r.iyend - r.iybeg + T1Y) / T1Y, r.izend - r.izbeg + 1);
}

struct FdConst {
    float xx, yy, zz, xy, yz, zx;
};

// kernel_utils::compute_fd_const (kernels/kernel_utils.h:89-101)
FdConst fd_const(double dx, double dy, double dz)
{
    return FdConst{(float)(1.0 / (dx * dx)), (float)(1.0 / (dy * dy)), (float)(1.0 / (dz * dz)),
                   (float)(1.0 / (4 * dx * dy)), (float)(1.0 / (4 * dy * dz)), (float)(1.0 / (4 * dx * dz))};
}

struct Drv {
    float xx, yy, zz, xy, yz, zx;
};

__device__ __forceinline__ Drv centred(const float* __restrict__ f, int64_t i, int64_t sy, int64_t sz, FdConst k)
{
    float zz = 0.0f, zx = 0.0f, yz = 0.0f;
#pragma unroll
    for (int ir = -4; ir <= 4; ++ir) {
        const float c = c2(ir < 0 ? -ir : ir);
        const int64_t j = i + ir * sz;
        zz = zz + c * __ldg(f + j);
        if (ir != 0) {
            zx = zx + c * (__ldg(f + j + ir) - __ldg(f + j - ir));
            yz = yz + c * (__ldg(f + j + ir * sy) - __ldg(f + j - ir * sy));
        }
    }
    const float f0 = __ldg(f + i);
    float xx = c2(0) * f0, yy = c2(0) * f0, xy = 0.0f;
#pragma unroll
    for (int q = 1; q <= 4; ++q) {
        const float c = c2(q);
        xx += c * (__ldg(f + i + q) + __ldg(f + i - q));
        yy += c * (__ldg(f + i + q * sy) + __ldg(f + i - q * sy));
        xy += c * (__ldg(f + i + q * sy + q) - __ldg(f + i + q * sy - q) + __ldg(f + i - q * sy - q) -
                   __ldg(f + i - q * sy + q));
    }
    return Drv{xx * k.xx, yy * k.yy, zz * k.zz, xy * k.xy, yz * k.yz, zx * k.zx};
}

// MODE 0: f3,f4 += rhs*dt;  1: f = A f + B rhs dt (sponge);  2: rhs into
// halo-free outputs (calc_snap).
template <int MODE>
__global__ void __launch_bounds__(T1X* T1Y)
    k_t1_fwd(float* __restrict__ f3, float* __restrict__ f4, const float* __restrict__ f1,
             const float* __restrict__ f2, const float* __restrict__ m1, const float* __restrict__ m2,
             const float* __restrict__ m3, const float* __restrict__ m4, const float* __restrict__ m5,
             const float* __restrict__ m6, const float* __restrict__ m7, const float2* __restrict__ abx,
             const float2* __restrict__ aby, const float2* __restrict__ abz, R6 r, int ldimx, int ldimy, int ldox,
             int ldoy, float dt, FdConst k)
{
    const int ix = r.ixbeg + blockIdx.x * T1X + threadIdx.x;
    const int iy = r.iybeg + blockIdx.y * T1Y + threadIdx.y;
    const int iz = r.izbeg + blockIdx.z;
    if (ix > r.ixend || iy > r.iyend) return;
    const int64_t sy = ldimx, sz = (int64_t)ldimx * ldimy;
    const int64_t i = iz * sz + (int64_t)iy * sy + ix;
    const Drv a = centred(f1, i, sy, sz, k);
    const Drv b = centred(f2, i, sy, sz, k);
    const float rx = __ldg(m5 + i), ry = __ldg(m6 + i), rz = __ldg(m7 + i);
    const float rxx = rx * rx, ryy = ry * ry, rzz = rz * rz;
    const float rxy = 2.0f * rx * ry, ryz = 2.0f * ry * rz, rzx = 2.0f * rz * rx;
    const float V1 = rxx * a.xx + ryy * a.yy + rzz * a.zz + rxy * a.xy + rzx * a.zx + ryz * a.yz;
    const float H1 = a.xx + a.yy + a.zz - V1;
    const float V2 = rxx * b.xx + ryy * b.yy + rzz * b.zz + rxy * b.xy + rzx * b.zx + ryz * b.yz;
    const float H2 = b.xx + b.yy + b.zz - V2;
    const float r3 = __ldg(m1 + i) * H1 + __ldg(m4 + i) * V1 + __ldg(m2 + i) * V2;
    const float r4 = __ldg(m2 + i) * H1 + __ldg(m3 + i) * V2 + __ldg(m4 + i) * H2;
    if constexpr (MODE == 2) {
        const int64_t o = ((int64_t)(iz - r.izbeg) * ldoy + (iy - r.iybeg)) * ldox + (ix - r.ixbeg);
        f3[o] = r3;
        f4[o] = r4;
    } else {
        // output base offset with the input dimensions, then the output strides
        // (kernel_type1_gpu_fwd.cu:488-492 and :283)
        const int64_t o = ((int64_t)r.izbeg * ldimy + r.iybeg) * ldimx +
                          ((int64_t)(iz - r.izbeg) * ldoy + (iy - r.iybeg)) * ldox + ix;
        if constexpr (MODE == 1) {
            const float A = fminf(abx[ix].x, fminf(aby[iy].x, abz[iz].x));
            const float B = fminf(abx[ix].y, fminf(aby[iy].y, abz[iz].y));
            f3[o] = A * f3[o] + B * r3 * dt;
            f4[o] = A * f4[o] + B * r4 * dt;
        } else {
            f3[o] += r3 * dt;
            f4[o] += r4 * dt;
        }
    }
}

// Transposed-model temporary of one derivative at cell j: field 3 and 4 of
// lap*[with_lap] + w*hz, from the scratch (lap_x, hz_x, lap_z, hz_z).
__device__ __forceinline__ float2 t1_temp(const float4* __restrict__ base, int64_t j, float w, bool with_lap)
{
    const float4 b = __ldg(base + j);
    return make_float2((with_lap ? b.x : 0.0f) + w * b.y, (with_lap ? b.z : 0.0f) + w * b.w);
}

template <bool SPONGE>
__global__ void __launch_bounds__(T1X* T1Y)
    k_t1_adj(float* __restrict__ f3, float* __restrict__ f4, const float4* __restrict__ base,
             const float* __restrict__ rx, const float* __restrict__ ry, const float* __restrict__ rz,
             const float2* __restrict__ abx, const float2* __restrict__ aby, const float2* __restrict__ abz, R6 r,
             int ldimx, int ldimy, float dt, FdConst k)
{
    const int ix = r.ixbeg + blockIdx.x * T1X + threadIdx.x;
    const int iy = r.iybeg + blockIdx.y * T1Y + threadIdx.y;
    const int iz = r.izbeg + blockIdx.z;
    if (ix > r.ixend || iy > r.iyend) return;
    const int64_t sy = ldimx, sz = (int64_t)ldimx * ldimy;
    const int64_t i = iz * sz + (int64_t)iy * sy + ix;
    float s3 = 0.0f, s4 = 0.0f;
#pragma unroll
    for (int ir = -4; ir <= 4; ++ir) {
        const float c = c2(ir < 0 ? -ir : ir);
        const int64_t j = i + ir * sz;
        const float rzj = __ldg(rz + j);
        const float2 tz = t1_temp(base, j, rzj * rzj, true);
        float a3 = k.zz * c * tz.x, a4 = k.zz * c * tz.y;
        if (ir != 0) {
            int64_t jp = j + ir * sy, jm = j - ir * sy;
            float2 tp = t1_temp(base, jp, 2.0f * __ldg(ry + jp) * __ldg(rz + jp), false);
            float2 tm = t1_temp(base, jm, 2.0f * __ldg(ry + jm) * __ldg(rz + jm), false);
            a3 = a3 + k.yz * c * (tp.x - tm.x);
            a4 = a4 + k.yz * c * (tp.y - tm.y);
            jp = j + ir;
            jm = j - ir;
            tp = t1_temp(base, jp, 2.0f * __ldg(rz + jp) * __ldg(rx + jp), false);
            tm = t1_temp(base, jm, 2.0f * __ldg(rz + jm) * __ldg(rx + jm), false);
            a3 = a3 + k.zx * c * (tp.x - tm.x);
            a4 = a4 + k.zx * c * (tp.y - tm.y);
        }
        s3 = s3 + a3;
        s4 = s4 + a4;
    }
    const float rxi = __ldg(rx + i), ryi = __ldg(ry + i);
    float2 t = t1_temp(base, i, rxi * rxi, true);
    float xx3 = c2(0) * t.x, xx4 = c2(0) * t.y;
    t = t1_temp(base, i, ryi * ryi, true);
    float yy3 = c2(0) * t.x, yy4 = c2(0) * t.y;
    float xy3 = 0.0f, xy4 = 0.0f;
#pragma unroll
    for (int q = 1; q <= 4; ++q) {
        const float c = c2(q);
        int64_t jp = i + q, jm = i - q;
        float rp = __ldg(rx + jp), rm = __ldg(rx + jm);
        float2 tp = t1_temp(base, jp, rp * rp, true), tm = t1_temp(base, jm, rm * rm, true);
        xx3 += c * (tp.x + tm.x);
        xx4 += c * (tp.y + tm.y);
        jp = i + q * sy;
        jm = i - q * sy;
        rp = __ldg(ry + jp);
        rm = __ldg(ry + jm);
        tp = t1_temp(base, jp, rp * rp, true);
        tm = t1_temp(base, jm, rm * rm, true);
        yy3 += c * (tp.x + tm.x);
        yy4 += c * (tp.y + tm.y);
        const int64_t jpp = i + q * sy + q, jpm = i + q * sy - q, jmm = i - q * sy - q, jmp = i - q * sy + q;
        const float2 p = t1_temp(base, jpp, 2.0f * __ldg(rx + jpp) * __ldg(ry + jpp), false);
        const float2 u = t1_temp(base, jpm, 2.0f * __ldg(rx + jpm) * __ldg(ry + jpm), false);
        const float2 v = t1_temp(base, jmm, 2.0f * __ldg(rx + jmm) * __ldg(ry + jmm), false);
        const float2 w = t1_temp(base, jmp, 2.0f * __ldg(rx + jmp) * __ldg(ry + jmp), false);
        xy3 += c * (p.x - u.x + v.x - w.x);
        xy4 += c * (p.y - u.y + v.y - w.y);
    }
    s3 += k.xx * xx3 + k.yy * yy3 + k.xy * xy3;
    s4 += k.xx * xx4 + k.yy * yy4 + k.xy * xy4;
    if constexpr (SPONGE) {
        const float A = fminf(abx[ix].x, fminf(aby[iy].x, abz[iz].x));
        const float B = fminf(abx[ix].y, fminf(aby[iy].y, abz[iz].y));
        f3[i] = A * f3[i] + B * s3 * dt;
        f4[i] = A * f4[i] + B * s4 * dt;
    } else {
        f3[i] += s3 * dt;
        f4[i] += s4 * dt;
    }
}

__global__ void __launch_bounds__(T1X* T1Y)
    k_t1_grad(const float* __restrict__ snap_x, const float* __restrict__ snap_z, float* __restrict__ grad,
              const float* __restrict__ adj_x, const float* __restrict__ adj_z, R6 r, int sldx, int sldy, int ldimx,
              int ldimy)
{
    const int ix = r.ixbeg + blockIdx.x * T1X + threadIdx.x;
    const int iy = r.iybeg + blockIdx.y * T1Y + threadIdx.y;
    const int iz = r.izbeg + blockIdx.z;
    if (ix > r.ixend || iy > r.iyend) return;
    const int64_t d = ((int64_t)(iz - r.izbeg) * sldy + (iy - r.iybeg)) * sldx + (ix - r.ixbeg);
    const int64_t i = ((int64_t)iz * ldimy + iy) * ldimx + ix;
    grad[d] += adj_x[i] * snap_x[d] + adj_z[i] * snap_z[d];
}

inline cudaStream_t S(tti_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

bool t1_ranges_ok(int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy, int ldimz)
{
    return ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy) && ldimz >= izend + 1 + kRadius;
}

} // namespace
} // namespace tti

using namespace tti;

extern "C" {

int tti_launch_type1_fwd(float* field3, float* field4, const float* field1, const float* field2, const float* model1,
                         const float* model2, const float* model3, const float* model4, const float* model5,
                         const float* model6, const float* model7, const float* ABx, const float* ABy,
                         const float* ABz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                         int ldimx_in, int ldimy_in, int ldimz_in, int ldimx_out, int ldimy_out, int ldimz_out,
                         float dt, double dx, double dy, double dz, int order, tti_stream_t stream, int calc_snap,
                         int use_sponge, int simple)
{
    (void)simple;
    (void)ldimz_out;
    if (order != 8 || (calc_snap && use_sponge)) return TTI_EINVAL;
    if (!t1_ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx_in, ldimy_in, ldimz_in)) return TTI_EINVAL;
    if (!field3 || !field4 || !field1 || !field2 || !model1 || !model2 || !model3 || !model4 || !model5 ||
        !model6 || !model7)
        return TTI_EINVAL;
    if (use_sponge && (!ABx || !ABy || !ABz)) return TTI_EINVAL;
    if (calc_snap ? (ldimx_out < ixend - ixbeg + 1 || ldimy_out < iyend - iybeg + 1)
                  : (ldimx_out < ixend + 1 || ldimy_out < iyend - iybeg + 1))
        return TTI_EINVAL;
    const R6 r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    const FdConst k = fd_const(dx, dy, dz);
    const float2* ax = reinterpret_cast<const float2*>(ABx);
    const float2* ay = reinterpret_cast<const float2*>(ABy);
    const float2* az = reinterpret_cast<const float2*>(ABz);
    const dim3 g = t1_grid(r), b(T1X, T1Y);
    if (calc_snap)
        k_t1_fwd<2><<<g, b, 0, S(stream)>>>(field3, field4, field1, field2, model1, model2, model3, model4, model5,
                                            model6, model7, ax, ay, az, r, ldimx_in, ldimy_in, ldimx_out, ldimy_out,
                                            dt, k);
    else if (use_sponge)
        k_t1_fwd<1><<<g, b, 0, S(stream)>>>(field3, field4, field1, field2, model1, model2, model3, model4, model5,
                                            model6, model7, ax, ay, az, r, ldimx_in, ldimy_in, ldimx_out, ldimy_out,
                                            dt, k);
    else
        k_t1_fwd<0><<<g, b, 0, S(stream)>>>(field3, field4, field1, field2, model1, model2, model3, model4, model5,
                                            model6, model7, ax, ay, az, r, ldimx_in, ldimy_in, ldimx_out, ldimy_out,
                                            dt, k);
    return launch_status();
}

int tti_launch_type1_adj(float* field3, float* field4, const float* field1, const float* field2, const float* model1,
                         const float* model2, const float* model3, const float* model4, const float* model5,
                         const float* model6, const float* model7, const float* ABx, const float* ABy,
                         const float* ABz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                         int ldimx, int ldimy, int ldimz, float dt, double dx, double dy, double dz, int order,
                         tti_stream_t stream, int use_sponge, int simple)
{
    (void)simple;
    if (order != 8) return TTI_EINVAL;
    if (!t1_ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy, ldimz)) return TTI_EINVAL;
    if (!field3 || !field4 || !field1 || !field2 || !model1 || !model2 || !model3 || !model4 || !model5 ||
        !model6 || !model7)
        return TTI_EINVAL;
    if (use_sponge && (!ABx || !ABy || !ABz)) return TTI_EINVAL;
    const size_t nelem = (size_t)ldimx * ldimy * (size_t)(izend + 1 + kRadius);
    cudaStream_t st = S(stream);
    const tti::CallScratch scratch(nelem, st);
    float4* base = scratch.get();
    if (!base) return TTI_ENOMEM;
    int rc = launch_base(field1, field2, model1, model2, model3, model4, base, ixbeg, ixend, iybeg, iyend, izbeg,
                         izend, ldimx, ldimy, st);
    if (rc) return rc;
    const R6 r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    const FdConst k = fd_const(dx, dy, dz);
    const float2* ax = reinterpret_cast<const float2*>(ABx);
    const float2* ay = reinterpret_cast<const float2*>(ABy);
    const float2* az = reinterpret_cast<const float2*>(ABz);
    if (use_sponge)
        k_t1_adj<true><<<t1_grid(r), dim3(T1X, T1Y), 0, st>>>(field3, field4, base, model5, model6, model7, ax, ay,
                                                             az, r, ldimx, ldimy, dt, k);
    else
        k_t1_adj<false><<<t1_grid(r), dim3(T1X, T1Y), 0, st>>>(field3, field4, base, model5, model6, model7, ax, ay,
                                                              az, r, ldimx, ldimy, dt, k);
    return launch_status();
}

int tti_launch_type1_update_grad(const float* snap_x, const float* snap_z, float* grad_Vp, const float* adj_x,
                                 const float* adj_z, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                                 int snap_ldimx, int snap_ldimy, int ldimx, int ldimy, tti_stream_t stream)
{
    if (ixend < ixbeg || iyend < iybeg || izend < izbeg || ixbeg < 0 || iybeg < 0 || izbeg < 0) return TTI_EINVAL;
    if (ldimx < ixend + 1 || ldimy < iyend + 1) return TTI_EINVAL;
    if (snap_ldimx < ixend - ixbeg + 1 || snap_ldimy < iyend - iybeg + 1) return TTI_EINVAL;
    if (!snap_x || !snap_z || !grad_Vp || !adj_x || !adj_z) return TTI_EINVAL;
    const R6 r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_t1_grad<<<t1_grid(r), dim3(T1X, T1Y), 0, S(stream)>>>(snap_x, snap_z, grad_Vp, adj_x, adj_z, r, snap_ldimx,
                                                             snap_ldimy, ldimx, ldimy);
    return launch_status();
}

} // extern "C"
