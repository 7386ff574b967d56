// Per-kernel launchers: the reference's kernel sequence on B200.
//
// One entry point per reference launcher (include/tti_capi.h section 1), each
// computing exactly what the reference kernel computes, in the reference's
// accumulation order (tap order, where 1/h and the buoyancy are applied), so
// that the FP32 results agree with the reference kernels to rounding.  These
// kernels are the drop-in boundary and the simulator's non-fused path; the
// fused step kernels live in tti_fused.cu.
//
// Every kernel maps one thread to one output cell: blocks of 32x8 cells in
// XY, one Z plane per grid row, neighbours read through the L1/texture path.

#include <cuda_runtime.h>

#include <vector>

#include "tti_common.cuh"
#include "tti_internal.cuh"

namespace tti {
namespace {

constexpr int BX = 32, BY = 8;

struct Ranges {
    int ixbeg, ixend, iybeg, iyend, izbeg, izend;
};

inline dim3 grid_for(const Ranges& r)
{
    return dim3((r.ixend - r.ixbeg + BX) / BX, (r.iyend - r.iybeg + BY) / BY, r.izend - r.izbeg + 1);
}

__device__ __forceinline__ bool thread_cell(const Ranges& r, int& ix, int& iy, int& iz)
{
    ix = r.ixbeg + blockIdx.x * BX + threadIdx.x;
    iy = r.iybeg + blockIdx.y * BY + threadIdx.y;
    iz = r.izbeg + blockIdx.z;
    return ix <= r.ixend && iy <= r.iyend;
}

// ---------------------------------------------------------------------------
// a1  kernel_base.cu:82-104
__global__ void __launch_bounds__(BX* BY)
    k_loop2(float* __restrict__ f1, float* __restrict__ f2, const float* __restrict__ f3,
            const float* __restrict__ f4, Ranges r, int ldimx, int ldimy, const float2* __restrict__ abx,
            const float2* __restrict__ aby, const float2* __restrict__ abz, float dt)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    float2 ax = abx[ix], ay = aby[iy], az = abz[iz];
    float A = fminf(ax.x, fminf(ay.x, az.x));
    float B = fminf(ax.y, fminf(ay.y, az.y));
    int64_t i = ((int64_t)iz * ldimy + iy) * ldimx + ix;
    float r1 = A * f1[i] + B * f3[i] * dt;
    float r2 = A * f2[i] + B * f4[i] * dt;
    f1[i] = r1;
    f2[i] = r2;
}

// a2  kernel_base.cu:142-162 (whole XY planes, iz <= izbeg)
__global__ void k_loop4(float* __restrict__ f1, float* __restrict__ f2, int64_t plane, int izbeg)
{
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int iz = blockIdx.y;
    if (j >= plane) return;
    int64_t i = iz * plane + j;
    if (iz == izbeg) {
        f1[i] = 0.0f;
        f2[i] = 0.0f;
    } else {
        int64_t m = (int64_t)(2 * izbeg - iz) * plane + j;
        float a = -f1[m], b = -f2[m];
        f1[i] = a;
        f2[i] = b;
    }
}

// a3  kernel_type2_fwd_drv.cu:36-116 (compute_dz_negative_shift,
// compute_dx_dy_negative_shift, multiply_inv_model10)
__global__ void __launch_bounds__(BX* BY)
    k_fwd_drv(const float* __restrict__ f1, const float* __restrict__ f2, const float* __restrict__ irho,
              float* __restrict__ d1x, float* __restrict__ d1y, float* __restrict__ d1z, float* __restrict__ d2x,
              float* __restrict__ d2y, float* __restrict__ d2z, Ranges r, int ldimx, int ldimy, float invdx,
              float invdy, float invdz)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t ys = ldimx, zs = (int64_t)ldimx * ldimy;
    const int64_t i = iz * zs + iy * ys + ix;
    float z1 = 0.0f, z2 = 0.0f;
#pragma unroll
    for (int ir = -4; ir <= 3; ++ir) {
        float a = __ldg(f1 + i + ir * zs), b = __ldg(f2 + i + ir * zs);
        if (ir >= 0) {
            z1 = z1 + c1(ir + 1) * a;
            z2 = z2 + c1(ir + 1) * b;
        } else {
            z1 = z1 - c1(-ir) * a;
            z2 = z2 - c1(-ir) * b;
        }
    }
    z1 *= invdz;
    z2 *= invdz;
    float x1 = 0.0f, y1 = 0.0f, x2 = 0.0f, y2 = 0.0f;
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        x1 += c1(k) * (__ldg(f1 + i + (k - 1)) - __ldg(f1 + i - k));
        y1 += c1(k) * (__ldg(f1 + i + (k - 1) * ys) - __ldg(f1 + i - k * ys));
        x2 += c1(k) * (__ldg(f2 + i + (k - 1)) - __ldg(f2 + i - k));
        y2 += c1(k) * (__ldg(f2 + i + (k - 1) * ys) - __ldg(f2 + i - k * ys));
    }
    x1 *= invdx;
    y1 *= invdy;
    x2 *= invdx;
    y2 *= invdy;
    const float rho = __ldg(irho + i);
    d1x[i] = x1 * rho;
    d1y[i] = y1 * rho;
    d1z[i] = z1 * rho;
    d2x[i] = x2 * rho;
    d2y[i] = y2 * rho;
    d2z[i] = z2 * rho;
}

// a4  kernel_type2_small.cu:5-40
__global__ void k_loop4_derivatives(float* __restrict__ d1x, float* __restrict__ d1y, float* __restrict__ d1z,
                                    float* __restrict__ d2x, float* __restrict__ d2y, float* __restrict__ d2z,
                                    int64_t plane, int izbeg)
{
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int iz = blockIdx.y;
    if (j >= plane) return;
    int64_t i = iz * plane + j;
    if (iz == izbeg) {
        d1x[i] = 0.0f;
        d1y[i] = 0.0f;
        d2x[i] = 0.0f;
        d2y[i] = 0.0f;
    } else {
        int64_t m = (int64_t)(2 * izbeg - iz) * plane + j;
        d1x[i] = -d1x[m];
        d1y[i] = -d1y[m];
        d2x[i] = -d2x[m];
        d2y[i] = -d2y[m];
    }
    int64_t mz = (int64_t)(2 * izbeg + 1 - iz) * plane + j;
    d1z[i] = d1z[mz];
    d2z[i] = d2z[mz];
}

// a5  kernel_type2_fwd.cu:98-235 and the accumulation of :360-539
__global__ void __launch_bounds__(BX* BY)
    k_fwd_update(float* __restrict__ f3, float* __restrict__ f4, const float* __restrict__ d1x,
                 const float* __restrict__ d2x, const float* __restrict__ d1y, const float* __restrict__ d2y,
                 const float* __restrict__ d1z, const float* __restrict__ d2z, const float* __restrict__ f1,
                 const float* __restrict__ f2, const float* __restrict__ irho, const float* __restrict__ m1,
                 const float* __restrict__ m2, const float* __restrict__ m3, const float* __restrict__ m4,
                 const float* __restrict__ rx, const float* __restrict__ ry, const float* __restrict__ rz, Ranges r,
                 int ldimx, int ldimy, float invdx, float invdy, float invdz, float invdxdy, float invdydz,
                 float invdzdx, float dt)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t ys = ldimx, zs = (int64_t)ldimx * ldimy;
    const int64_t i = iz * zs + iy * ys + ix;
    float xx1 = 0.0f, xx2 = 0.0f, yy1 = 0.0f, yy2 = 0.0f, zz1 = 0.0f, zz2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        xx1 += tap(k) * __ldg(d1x + i + (k - 3));
        xx2 += tap(k) * __ldg(d2x + i + (k - 3));
        yy1 += tap(k) * __ldg(d1y + i + (k - 3) * ys);
        yy2 += tap(k) * __ldg(d2y + i + (k - 3) * ys);
        zz1 = zz1 + tap(k) * __ldg(d1z + i + (k - 3) * zs);
        zz2 = zz2 + tap(k) * __ldg(d2z + i + (k - 3) * zs);
    }
    xx1 *= invdx;
    xx2 *= invdx;
    yy1 *= invdy;
    yy2 *= invdy;
    zz1 *= invdz;
    zz2 *= invdz;
    float zx1 = 0.0f, zx2 = 0.0f, yz1 = 0.0f, yz2 = 0.0f;
#pragma unroll
    for (int m = -4; m <= 4; ++m) {
        if (m == 0) continue;
        const float c = c2(m < 0 ? -m : m);
        const int64_t p = i + m * zs;
        zx1 += c * (__ldg(f1 + p + m) - __ldg(f1 + p - m));
        yz1 += c * (__ldg(f1 + p + m * ys) - __ldg(f1 + p - m * ys));
        zx2 += c * (__ldg(f2 + p + m) - __ldg(f2 + p - m));
        yz2 += c * (__ldg(f2 + p + m * ys) - __ldg(f2 + p - m * ys));
    }
    yz1 *= invdydz;
    zx1 *= invdzdx;
    yz2 *= invdydz;
    zx2 *= invdzdx;
    float xy1 = 0.0f, xy2 = 0.0f;
#pragma unroll
    for (int k = -4; k <= 4; ++k) {
        if (k == 0) continue;
        const float c = c2(k < 0 ? -k : k);
        xy1 += c * (__ldg(f1 + i + k * ys + k) - __ldg(f1 + i - k * ys + k));
        xy2 += c * (__ldg(f2 + i + k * ys + k) - __ldg(f2 + i - k * ys + k));
    }
    xy1 *= invdxdy;
    xy2 *= invdxdy;

    const float rho = 1.0f / __ldg(irho + i);
    const float vrx = __ldg(rx + i), vry = __ldg(ry + i), vrz = __ldg(rz + i);
    const float rx2 = vrx * vrx, ry2 = vry * vry, rz2 = vrz * vrz;
    const float rxy = 2.0f * vrx * vry, ryz = 2.0f * vry * vrz, rzx = 2.0f * vrz * vrx;
    xx1 *= rho;
    yy1 *= rho;
    zz1 *= rho;
    xx2 *= rho;
    yy2 *= rho;
    zz2 *= rho;
    const float V1 = rx2 * xx1 + ry2 * yy1 + rz2 * zz1 + rxy * xy1 + rzx * zx1 + ryz * yz1;
    const float H1 = xx1 + yy1 + zz1 - V1;
    const float V2 = rx2 * xx2 + ry2 * yy2 + rz2 * zz2 + rxy * xy2 + rzx * zx2 + ryz * yz2;
    const float H2 = xx2 + yy2 + zz2 - V2;
    const float a1 = __ldg(m1 + i), a2 = __ldg(m2 + i), a3 = __ldg(m3 + i), a4 = __ldg(m4 + i);
    const float r3 = a1 * H1 + a4 * V1 + a2 * V2;
    const float r4 = a2 * H1 + a3 * V2 + a4 * H2;
    f3[i] += r3 * dt;
    f4[i] += r4 * dt;
}

// Point-wise transposed model shared by the adjoint-derivative and the
// density-gradient kernels (kernel_type2_grad_snap.cu:98-102,
// kernel_type2_grad.cu:156-157,201-205):
//   s1 = m1 p + m2 q,  h1 = (m4 - m1) p - m2 q,  s2 = m4 q,  h2 = m2 p + (m3 - m4) q
// stored as four scratch volumes over the halo'd range.
__global__ void __launch_bounds__(BX* BY)
    k_adj_base(const float* __restrict__ f1, const float* __restrict__ f2, const float* __restrict__ m1,
               const float* __restrict__ m2, const float* __restrict__ m3, const float* __restrict__ m4,
               float4* __restrict__ base, Ranges r, int ldimx, int ldimy)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t i = ((int64_t)iz * ldimy + iy) * ldimx + ix;
    const float p = f1[i], q = f2[i], a1 = m1[i], a2 = m2[i], a3 = m3[i], a4 = m4[i];
    float4 b;
    b.x = a1 * p + a2 * q;
    b.y = (-a1 + a4) * p - a2 * q;
    b.z = a4 * q;
    b.w = a2 * p + (-a4 + a3) * q;
    base[i] = b;
}

struct AdjT {
    float xx1, xx2, yy1, yy2, zz1, zz2;
};

// Temporaries of compute_temp_arrays (kernel_type2_grad_snap.cu:66-132) at one cell.
__device__ __forceinline__ float2 t_norm(const float4* __restrict__ base, const float* __restrict__ irho,
                                         const float* __restrict__ ra, int64_t j)
{
    const float4 b = __ldg(base + j);
    const float rho = 1.0f / __ldg(irho + j);
    const float a = __ldg(ra + j);
    const float rr = a * a;
    return make_float2(rho * (b.x + rr * b.y), rho * (b.z + rr * b.w));
}
__device__ __forceinline__ float2 t_mixed(const float4* __restrict__ base, const float* __restrict__ ra,
                                          const float* __restrict__ rb, int64_t j)
{
    const float4 b = __ldg(base + j);
    const float w = 2.0f * __ldg(ra + j) * __ldg(rb + j);
    return make_float2(w * b.y, w * b.w);
}

// a6  kernel_type2_grad_snap.cu:134-240,242-427
__global__ void __launch_bounds__(BX* BY)
    k_adj_drv(float* __restrict__ d1x, float* __restrict__ d2x, float* __restrict__ d1y, float* __restrict__ d2y,
              float* __restrict__ d1z, float* __restrict__ d2z, float* __restrict__ rhs3, float* __restrict__ rhs4,
              const float4* __restrict__ base, const float* __restrict__ irho, const float* __restrict__ rx,
              const float* __restrict__ ry, const float* __restrict__ rz, Ranges r, int ldimx, int ldimy,
              float invdxy, float invdyz, float invdzx, float invdx, float invdy, float invdz)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t ys = ldimx, zs = (int64_t)ldimx * ldimy;
    const int64_t i = iz * zs + iy * ys + ix;
    const float ir_ = __ldg(irho + i);
    float z1 = 0.0f, z2 = 0.0f;
#pragma unroll
    for (int ir = -4; ir <= 3; ++ir) {
        const float alpha = (ir < 0) ? -invdz * c1(-ir) : invdz * c1(ir + 1);
        const float2 t = t_norm(base, irho, rz, i + ir * zs);
        z1 = z1 + alpha * t.x;
        z2 = z2 + alpha * t.y;
    }
    float x1 = 0.0f, x2 = 0.0f, y1 = 0.0f, y2 = 0.0f, s3 = 0.0f, s4 = 0.0f;
#pragma unroll
    for (int ir = -4; ir <= -1; ++ir) {
        const float c = c2(-ir);
        const int64_t p = i + ir * zs;
        const float2 yp = t_mixed(base, ry, rz, p + ir * ys), ym = t_mixed(base, ry, rz, p - ir * ys);
        const float2 xp = t_mixed(base, rz, rx, p + ir), xm = t_mixed(base, rz, rx, p - ir);
        s3 = s3 + (invdyz * c * (yp.x - ym.x)) + (invdzx * c * (xp.x - xm.x));
        s4 = s4 + (invdyz * c * (yp.y - ym.y)) + (invdzx * c * (xp.y - xm.y));
    }
#pragma unroll
    for (int k = 1; k <= 4; ++k) {
        const float ax = invdx * c1(k);
        const float2 xp = t_norm(base, irho, rx, i + (k - 1)), xm = t_norm(base, irho, rx, i - k);
        x1 += ax * (xp.x - xm.x) * ir_;
        x2 += ax * (xp.y - xm.y) * ir_;
        const float ay = invdy * c1(k);
        const float2 yp = t_norm(base, irho, ry, i + (k - 1) * ys), ym = t_norm(base, irho, ry, i - k * ys);
        y1 += ay * (yp.x - ym.x) * ir_;
        y2 += ay * (yp.y - ym.y) * ir_;
        const float axy = invdxy * c2(k);
        const float2 pp = t_mixed(base, rx, ry, i + k * ys + k), pm = t_mixed(base, rx, ry, i + k * ys - k);
        const float2 mm = t_mixed(base, rx, ry, i - k * ys - k), mp = t_mixed(base, rx, ry, i - k * ys + k);
        s3 += axy * (pp.x - pm.x + mm.x - mp.x);
        s4 += axy * (pp.y - pm.y + mm.y - mp.y);
    }
#pragma unroll
    for (int ir = 1; ir <= 4; ++ir) {
        const float c = c2(ir);
        const int64_t p = i + ir * zs;
        const float2 yp = t_mixed(base, ry, rz, p + ir * ys), ym = t_mixed(base, ry, rz, p - ir * ys);
        const float2 xp = t_mixed(base, rz, rx, p + ir), xm = t_mixed(base, rz, rx, p - ir);
        s3 = s3 + (invdyz * c * (yp.x - ym.x)) + (invdzx * c * (xp.x - xm.x));
        s4 = s4 + (invdyz * c * (yp.y - ym.y)) + (invdzx * c * (xp.y - xm.y));
    }
    rhs3[i] = s3;
    rhs4[i] = s4;
    d1x[i] = x1;
    d1y[i] = y1;
    d1z[i] = z1 * ir_;
    d2x[i] = x2;
    d2y[i] = y2;
    d2z[i] = z2 * ir_;
}

// a7  kernel_type2_adj.cu:85-98 (dfdx_stg_right), :196-239
__device__ __forceinline__ float stg_right(const float* __restrict__ f, int64_t i, int64_t s, float h)
{
    float out = 0.0f;
#pragma unroll
    for (int k = 1; k <= 4; ++k) out += c1(k) * (__ldg(f + i + k * s) - __ldg(f + i + (1 - k) * s));
    out *= h;
    return out;
}

template <bool SPONGE>
__global__ void __launch_bounds__(BX* BY)
    k_adj_update(float* __restrict__ f3, float* __restrict__ f4, const float* __restrict__ d1x,
                 const float* __restrict__ d2x, const float* __restrict__ d1y, const float* __restrict__ d2y,
                 const float* __restrict__ d1z, const float* __restrict__ d2z, const float* __restrict__ rhs3,
                 const float* __restrict__ rhs4, const float2* __restrict__ abx, const float2* __restrict__ aby,
                 const float2* __restrict__ abz, Ranges r, int ldimx, int ldimy, float dt, float invdx, float invdy,
                 float invdz)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t ys = ldimx, zs = (int64_t)ldimx * ldimy;
    const int64_t i = iz * zs + iy * ys + ix;
    float r3 = stg_right(d1x, i, 1, invdx) + stg_right(d1y, i, ys, invdy) + stg_right(d1z, i, zs, invdz);
    float r4 = stg_right(d2x, i, 1, invdx) + stg_right(d2y, i, ys, invdy) + stg_right(d2z, i, zs, invdz);
    r3 += rhs3[i];
    r4 += rhs4[i];
    if constexpr (!SPONGE) {
        f3[i] += r3 * dt;
        f4[i] += r4 * dt;
    } else {
        const float2 ax = abx[ix], ay = aby[iy], az = abz[iz];
        const float A = fminf(fminf(ax.x, ay.x), az.x);
        const float B = fminf(fminf(ax.y, ay.y), az.y) * dt;
        f3[i] = A * f3[i] + B * r3;
        f4[i] = A * f4[i] + B * r4;
    }
}

// a8  kernel_type2_small.cu:42-59
__global__ void __launch_bounds__(BX* BY)
    k_vp_gradient(const float* __restrict__ snap3, const float* __restrict__ snap4, float* __restrict__ grad,
                  const float* __restrict__ adj3, const float* __restrict__ adj4, Ranges r, int snx, int sny,
                  int ldimx, int ldimy)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t g = ((int64_t)(iz - r.izbeg) * sny + (iy - r.iybeg)) * snx + (ix - r.ixbeg);
    const int64_t i = ((int64_t)iz * ldimy + iy) * ldimx + ix;
    const float s3 = snap3[g], s4 = snap4[g];
    grad[g] += adj3[i] * s3 + adj4[i] * s4;
}

// a11  kernel_type2_small.cu:61-74
__global__ void __launch_bounds__(BX* BY)
    k_finalize_vp(const float* __restrict__ model3, float* __restrict__ grad, Ranges r, int snx, int sny, int ldimx,
                  int ldimy, float dt_xcorr)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t g = ((int64_t)(iz - r.izbeg) * sny + (iy - r.iybeg)) * snx + (ix - r.ixbeg);
    const float vp = sqrtf(model3[((int64_t)iz * ldimy + iy) * ldimx + ix]);
    grad[g] *= -dt_xcorr * 2.0 / vp;
}

// a10  kernel_type2_grad.cu:188-260 (adj, stg) and :344-509 (accumulation)
__device__ __forceinline__ float2 rho_t(const float4* __restrict__ base, const float* __restrict__ irho,
                                        const float* __restrict__ ra, int64_t j)
{
    const float4 b = __ldg(base + j);
    const float rho = 1.0f / __ldg(irho + j);
    const float a = __ldg(ra + j);
    const float rr = a * a;
    return make_float2(rho * (b.x + rr * b.y), rho * (b.z + rr * b.w));
}

__device__ __forceinline__ float stg_plus(const float* __restrict__ t, int64_t i, int64_t s, float h)
{
    float d = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) d += cs(q) * (__ldg(t + i + (q + 1) * s) - __ldg(t + i - q * s));
    return d * h;
}

__global__ void __launch_bounds__(BX* BY)
    k_rho_gradient(float* __restrict__ grad, const float* __restrict__ fd1x, const float* __restrict__ fd2x,
                   const float* __restrict__ fd1y, const float* __restrict__ fd2y, const float* __restrict__ fd1z,
                   const float* __restrict__ fd2z, const float4* __restrict__ base, const float* __restrict__ irho,
                   const float* __restrict__ rx, const float* __restrict__ ry, const float* __restrict__ rz,
                   Ranges r, int ldimx, int ldimy, int gldx, int gldy, float hx, float hy, float hz)
{
    int ix, iy, iz;
    if (!thread_cell(r, ix, iy, iz)) return;
    const int64_t ys = ldimx, zs = (int64_t)ldimx * ldimy;
    const int64_t i = iz * zs + iy * ys + ix;
    const float2 ax = rho_t(base, irho, rx, i), ay = rho_t(base, irho, ry, i), az = rho_t(base, irho, rz, i);
    float dax1 = 0.0f, dax2 = 0.0f, day1 = 0.0f, day2 = 0.0f, daz1 = 0.0f, daz2 = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float c = cs(q);
        float2 p = rho_t(base, irho, rx, i + q), m = rho_t(base, irho, rx, i - (q + 1));
        dax1 += c * (p.x - m.x);
        dax2 += c * (p.y - m.y);
        p = rho_t(base, irho, ry, i + q * ys);
        m = rho_t(base, irho, ry, i - (q + 1) * ys);
        day1 += c * (p.x - m.x);
        day2 += c * (p.y - m.y);
        p = rho_t(base, irho, rz, i + q * zs);
        m = rho_t(base, irho, rz, i - (q + 1) * zs);
        daz1 += c * (p.x - m.x);
        daz2 += c * (p.y - m.y);
    }
    dax1 *= hx;
    dax2 *= hx;
    day1 *= hy;
    day2 *= hy;
    daz1 *= hz;
    daz2 *= hz;
    const float dfx1 = stg_plus(fd1x, i, 1, hx), dfx2 = stg_plus(fd2x, i, 1, hx);
    const float dfy1 = stg_plus(fd1y, i, ys, hy), dfy2 = stg_plus(fd2y, i, ys, hy);
    const float dfz1 = stg_plus(fd1z, i, zs, hz), dfz2 = stg_plus(fd2z, i, zs, hz);
    const float rxy = ax.x * dfx1 + ax.y * dfx2 + ay.x * dfy1 + ay.y * dfy2 + dax1 * __ldg(fd1x + i) +
                      dax2 * __ldg(fd2x + i) + day1 * __ldg(fd1y + i) + day2 * __ldg(fd2y + i);
    const float rhs = rxy + az.x * dfz1 + az.y * dfz2 + daz1 * __ldg(fd1z + i) + daz2 * __ldg(fd2z + i);
    const int64_t g = ((int64_t)(iz - r.izbeg) * gldy + (iy - r.iybeg)) * gldx + (ix - r.ixbeg);
    grad[g] += -__ldg(irho + i) * rhs;
}

// a12  simulator2SetUp.cu:10-29 per cell
__global__ void k_init_cijs(const float* __restrict__ vp, const float* __restrict__ eps,
                            const float* __restrict__ delta, const float* __restrict__ vs,
                            const float* __restrict__ theta, const float* __restrict__ phi, float* __restrict__ m1,
                            float* __restrict__ m2, float* __restrict__ m3, float* __restrict__ m4,
                            float* __restrict__ m5, float* __restrict__ m6, float* __restrict__ m7, int64_t n)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    init_cij_cell(vp[i], eps[i], delta[i], vs[i], theta[i], phi[i], m1[i], m2[i], m3[i], m4[i], m5[i], m6[i], m7[i]);
}

// a16  simulator2SetUp.cu:31-42
__global__ void k_pressure(float* __restrict__ out, const float* __restrict__ f1, const float* __restrict__ f2,
                           int64_t n)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = -(2 * f1[i] + f2[i]) / 3;
}

inline cudaStream_t S(tti_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

} // namespace

// Launch helpers used by the simulator (same kernels as the C ABI).
int launch_base(const float* f1, const float* f2, const float* m1, const float* m2, const float* m3,
                const float* m4, float4* base, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                int ldimx, int ldimy, cudaStream_t st)
{
    Ranges h{ixbeg - kRadius, ixend + kRadius, iybeg - kRadius, iyend + kRadius, izbeg - kRadius, izend + kRadius};
    k_adj_base<<<grid_for(h), dim3(BX, BY), 0, st>>>(f1, f2, m1, m2, m3, m4, base, h, ldimx, ldimy);
    return launch_status();
}

int launch_adj_drv_with_base(float* d1x, float* d2x, float* d1y, float* d2y, float* d1z, float* d2z, float* rhs3,
                             float* rhs4, const float4* base, const float* irho, const float* rx, const float* ry,
                             const float* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                             int ldimx, int ldimy, float invdxy, float invdyz, float invdzx, float invdx, float invdy,
                             float invdz, cudaStream_t st)
{
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_adj_drv<<<grid_for(r), dim3(BX, BY), 0, st>>>(d1x, d2x, d1y, d2y, d1z, d2z, rhs3, rhs4, base, irho, rx, ry, rz,
                                                   r, ldimx, ldimy, invdxy, invdyz, invdzx, invdx, invdy, invdz);
    return launch_status();
}

int launch_rho_gradient_with_base(float* grad, const float* fd1x, const float* fd2x, const float* fd1y,
                                  const float* fd2y, const float* fd1z, const float* fd2z, const float4* base,
                                  const float* irho, const float* rx, const float* ry, const float* rz, int ixbeg,
                                  int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy,
                                  int gldx, int gldy, double dx, double dy, double dz, cudaStream_t st)
{
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    float hx = 1.0 / dx, hy = 1.0 / dy, hz = 1.0 / dz;
    k_rho_gradient<<<grid_for(r), dim3(BX, BY), 0, st>>>(grad, fd1x, fd2x, fd1y, fd2y, fd1z, fd2z, base, irho, rx,
                                                        ry, rz, r, ldimx, ldimy, gldx, gldy, hx, hy, hz);
    return launch_status();
}

} // namespace tti

using namespace tti;

extern "C" {

const char* tti_status_string(int status)
{
    switch (status) {
    case TTI_OK: return "ok";
    case TTI_EINVAL: return "invalid argument";
    case TTI_ENOMEM: return "out of memory";
    case TTI_ELAUNCH: return "kernel launch or CUDA error";
    case TTI_ETIMEOUT: return "timed out";
    case TTI_ESTATE: return "call out of order";
    case TTI_ERANGE: return "reduced-precision snapshot saturated";
    case TTI_ETOOBIG: return "request exceeds a fixed-capacity buffer";
    default: return "unknown status";
    }
}

const char* tti_version(void) { return "0.1.0"; }

int tti_launch_fwd_kernel2_drv(const float* field1, const float* field2, const float* Model11, float* dfield1dx,
                               float* dfield1dy, float* dfield1dz, float* dfield2dx, float* dfield2dy,
                               float* dfield2dz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                               float invdx, float invdy, float invdz, int ldimx, int ldimy, int order,
                               tti_stream_t stream)
{
    if (order != 8 || !ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (!field1 || !field2 || !Model11 || !dfield1dx || !dfield1dy || !dfield1dz || !dfield2dx || !dfield2dy ||
        !dfield2dz)
        return TTI_EINVAL;
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_fwd_drv<<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(field1, field2, Model11, dfield1dx, dfield1dy, dfield1dz,
                                                          dfield2dx, dfield2dy, dfield2dz, r, ldimx, ldimy, invdx,
                                                          invdy, invdz);
    return launch_status();
}

int tti_launch_update_rho_fwd_main_loop_2_1(
    float* field3, float* field4, const float* field1_dx, const float* field2_dx, const float* field1_dy,
    const float* field2_dy, const float* field1_dz, const float* field2_dz, const float* field1, const float* field2,
    const float* irho, const float* model1, const float* model2, const float* model3, const float* model4,
    const float* rx, const float* ry, const float* rz, float* pml_field1_xx, float* pml_field2_xx,
    float* pml_field1_yy, float* pml_field2_yy, float* pml_field1_zz, float* pml_field2_zz, const float* pml_ab_x,
    const float* pml_ab_y, const float* pml_ab_z, const float* sponge_ab_xx, const float* sponge_ab_yy,
    const float* sponge_ab_zz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx,
    int ldimy, float dt, double dx, double dy, double dz, int sponge_active, int order, int pml_x, int pml_y,
    int pml_z, tti_stream_t stream)
{
    (void)sponge_ab_xx;
    (void)sponge_ab_yy;
    (void)sponge_ab_zz;
    (void)sponge_active;
    if (order != 8 || pml_x || pml_y || pml_z || pml_field1_xx || pml_field2_xx || pml_field1_yy || pml_field2_yy ||
        pml_field1_zz || pml_field2_zz || pml_ab_x || pml_ab_y || pml_ab_z)
        return TTI_EINVAL;
    if (!ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (!field3 || !field4 || !field1_dx || !field2_dx || !field1_dy || !field2_dy || !field1_dz || !field2_dz ||
        !field1 || !field2 || !irho || !model1 || !model2 || !model3 || !model4 || !rx || !ry || !rz)
        return TTI_EINVAL;
    // kernel_utils.h:89-101: reciprocals formed in double, stored as float.
    float invdx = 1.0 / dx, invdy = 1.0 / dy, invdz = 1.0 / dz;
    float invdxdy = 1.0 / (4 * dx * dy), invdydz = 1.0 / (4 * dy * dz), invdzdx = 1.0 / (4 * dx * dz);
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_fwd_update<<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(field3, field4, field1_dx, field2_dx, field1_dy,
                                                             field2_dy, field1_dz, field2_dz, field1, field2, irho,
                                                             model1, model2, model3, model4, rx, ry, rz, r, ldimx,
                                                             ldimy, invdx, invdy, invdz, invdxdy, invdydz, invdzdx,
                                                             dt);
    return launch_status();
}

int tti_launch_adj_kernel2_drv(float* dfield1dx, float* dfield2dx, float* dfield1dy, float* dfield2dy,
                               float* dfield1dz, float* dfield2dz, float* field3_rhs, float* field4_rhs,
                               const float* field1, const float* field2, const float* Model11, const float* model1,
                               const float* model2, const float* model3, const float* model4, const float* model5,
                               const float* model6, const float* model7, int ixbeg, int ixend, int iybeg,
                               int iyend, int izbeg, int izend, float invdxx, float invdyy, float invdzz,
                               float invdxy, float invdyz, float invdzx, int ldimx, int ldimy, int order, float dt,
                               float invdx, float invdy, float invdz, tti_stream_t stream)
{
    (void)invdxx;
    (void)invdyy;
    (void)invdzz;
    (void)dt;
    if (order != 8 || !ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (!dfield1dx || !dfield2dx || !dfield1dy || !dfield2dy || !dfield1dz || !dfield2dz || !field3_rhs ||
        !field4_rhs || !field1 || !field2 || !Model11 || !model1 || !model2 || !model3 || !model4 || !model5 ||
        !model6 || !model7)
        return TTI_EINVAL;
    const size_t nelem = (size_t)ldimx * ldimy * (size_t)(izend + 1 + kRadius);
    cudaStream_t st = S(stream);
    const tti::CallScratch scratch(nelem, st);
    float4* base = scratch.get();
    if (!base) return TTI_ENOMEM;
    int rc = launch_base(field1, field2, model1, model2, model3, model4, base, ixbeg, ixend, iybeg, iyend, izbeg,
                         izend, ldimx, ldimy, st);
    if (rc) return rc;
    return launch_adj_drv_with_base(dfield1dx, dfield2dx, dfield1dy, dfield2dy, dfield1dz, dfield2dz, field3_rhs,
                                    field4_rhs, base, Model11, model5, model6, model7, ixbeg, ixend, iybeg, iyend,
                                    izbeg, izend, ldimx, ldimy, invdxy, invdyz, invdzx, invdx, invdy, invdz, st);
}

int tti_launch_update_adj_kernel_main_3(float* field3, float* field4, const float* field1_dx,
                                        const float* field2_dx, const float* field1_dy, const float* field2_dy,
                                        const float* field1_dz, const float* field2_dz, const float* field3_rhs,
                                        const float* field4_rhs, const float* ab_xx, const float* ab_yy,
                                        const float* ab_zz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                                        int izend, int ldimx, int ldimy, float dt, double dx, double dy, double dz,
                                        int pmlx, int pmly, int pmlz, int order, int sponge_active,
                                        tti_stream_t stream)
{
    if (order != 8 || pmlx || pmly || pmlz) return TTI_EINVAL;
    if (!ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (!field3 || !field4 || !field1_dx || !field2_dx || !field1_dy || !field2_dy || !field1_dz || !field2_dz ||
        !field3_rhs || !field4_rhs)
        return TTI_EINVAL;
    if (sponge_active && (!ab_xx || !ab_yy || !ab_zz)) return TTI_EINVAL;
    float invdx = 1.0 / dx, invdy = 1.0 / dy, invdz = 1.0 / dz;
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    const float2* ax = reinterpret_cast<const float2*>(ab_xx);
    const float2* ay = reinterpret_cast<const float2*>(ab_yy);
    const float2* az = reinterpret_cast<const float2*>(ab_zz);
    if (sponge_active)
        k_adj_update<true><<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(field3, field4, field1_dx, field2_dx,
                                                                       field1_dy, field2_dy, field1_dz, field2_dz,
                                                                       field3_rhs, field4_rhs, ax, ay, az, r, ldimx,
                                                                       ldimy, dt, invdx, invdy, invdz);
    else
        k_adj_update<false><<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(field3, field4, field1_dx, field2_dx,
                                                                        field1_dy, field2_dy, field1_dz, field2_dz,
                                                                        field3_rhs, field4_rhs, ax, ay, az, r,
                                                                        ldimx, ldimy, dt, invdx, invdy, invdz);
    return launch_status();
}

int tti_launch_update_rho_gradient_rho(float* grad, const float* fwd_field1_dx, const float* fwd_field2_dx,
                                       const float* fwd_field1_dy, const float* fwd_field2_dy,
                                       const float* fwd_field1_dz, const float* fwd_field2_dz, const float* field1,
                                       const float* field2, const float* irho, const float* model1,
                                       const float* model2, const float* model3, const float* model4,
                                       const float* rx, const float* ry, const float* rz, int ixbeg, int ixend,
                                       int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy,
                                       int grad_ldimx, int grad_ldimy, double dx, double dy, double dz, int order,
                                       int simple_gradient, tti_stream_t stream)
{
    (void)simple_gradient;
    if (order != 8) return TTI_EINVAL;
    // kernel_type2_grad.cu:624-625: an empty range is a no-op.
    if (ixend < ixbeg || iyend < iybeg || izend < izbeg) return TTI_OK;
    if (!ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (grad_ldimx < ixend - ixbeg + 1 || grad_ldimy < iyend - iybeg + 1) return TTI_EINVAL;
    if (!grad || !fwd_field1_dx || !fwd_field2_dx || !fwd_field1_dy || !fwd_field2_dy || !fwd_field1_dz ||
        !fwd_field2_dz || !field1 || !field2 || !irho || !model1 || !model2 || !model3 || !model4 || !rx || !ry ||
        !rz)
        return TTI_EINVAL;
    const size_t nelem = (size_t)ldimx * ldimy * (size_t)(izend + 1 + kRadius);
    cudaStream_t st = S(stream);
    const tti::CallScratch scratch(nelem, st);
    float4* base = scratch.get();
    if (!base) return TTI_ENOMEM;
    int rc = launch_base(field1, field2, model1, model2, model3, model4, base, ixbeg, ixend, iybeg, iyend, izbeg,
                         izend, ldimx, ldimy, st);
    if (rc) return rc;
    return launch_rho_gradient_with_base(grad, fwd_field1_dx, fwd_field2_dx, fwd_field1_dy, fwd_field2_dy,
                                         fwd_field1_dz, fwd_field2_dz, base, irho, rx, ry, rz, ixbeg, ixend, iybeg,
                                         iyend, izbeg, izend, ldimx, ldimy, grad_ldimx, grad_ldimy, dx, dy, dz, st);
}

int tti_launch_kernel_loop4_derivatives(float* dfield1dx, float* dfield1dy, float* dfield1dz, float* dfield2dx,
                                        float* dfield2dy, float* dfield2dz, int xtot, int ytot, int izbeg,
                                        tti_stream_t stream)
{
    if (xtot <= 0 || ytot <= 0 || izbeg < 0) return TTI_EINVAL;
    if (!dfield1dx || !dfield1dy || !dfield1dz || !dfield2dx || !dfield2dy || !dfield2dz) return TTI_EINVAL;
    int64_t plane = (int64_t)xtot * ytot;
    dim3 grid((unsigned)((plane + 255) / 256), izbeg + 1);
    k_loop4_derivatives<<<grid, 256, 0, S(stream)>>>(dfield1dx, dfield1dy, dfield1dz, dfield2dx, dfield2dy,
                                                     dfield2dz, plane, izbeg);
    return launch_status();
}

int tti_launch_update_Vp_gradient(const float* snap_field3, const float* snap_field4, float* grad_Vp,
                                  const float* adj_field3, const float* adj_field4, int ixbeg, int ixend, int iybeg,
                                  int iyend, int izbeg, int izend, int snx, int sny, int ldimx, int ldimy,
                                  tti_stream_t stream)
{
    if (!ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (snx < ixend - ixbeg + 1 || sny < iyend - iybeg + 1) return TTI_EINVAL;
    if (!snap_field3 || !snap_field4 || !grad_Vp || !adj_field3 || !adj_field4) return TTI_EINVAL;
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_vp_gradient<<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(snap_field3, snap_field4, grad_Vp, adj_field3,
                                                              adj_field4, r, snx, sny, ldimx, ldimy);
    return launch_status();
}

int tti_launch_finalize_Vp_gradient(const float* model3, float* grad_Vp, int ixbeg, int ixend, int iybeg,
                                    int iyend, int izbeg, int izend, int snx, int sny, int ldimx, int ldimy,
                                    float dt_xcorr, tti_stream_t stream)
{
    if (!ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (snx < ixend - ixbeg + 1 || sny < iyend - iybeg + 1 || !model3 || !grad_Vp) return TTI_EINVAL;
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_finalize_vp<<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(model3, grad_Vp, r, snx, sny, ldimx, ldimy,
                                                              dt_xcorr);
    return launch_status();
}

int tti_launch_kernel_loop2(float* field1, float* field2, const float* field3, const float* field4, int ldimx,
                            int ldimy, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                            const float* ab_x, const float* ab_y, const float* ab_z, float dt, tti_stream_t stream)
{
    if (ixbeg < 0 || iybeg < 0 || izbeg < 0 || ixend < ixbeg || iyend < iybeg || izend < izbeg || ldimx <= ixend ||
        ldimy <= iyend)
        return TTI_EINVAL;
    if (!field1 || !field2 || !field3 || !field4 || !ab_x || !ab_y || !ab_z) return TTI_EINVAL;
    Ranges r{ixbeg, ixend, iybeg, iyend, izbeg, izend};
    k_loop2<<<grid_for(r), dim3(BX, BY), 0, S(stream)>>>(field1, field2, field3, field4, r, ldimx, ldimy,
                                                        reinterpret_cast<const float2*>(ab_x),
                                                        reinterpret_cast<const float2*>(ab_y),
                                                        reinterpret_cast<const float2*>(ab_z), dt);
    return launch_status();
}

int tti_launch_kernel_loop4(float* field1, float* field2, int ldimx, int ldimy, int izbeg, tti_stream_t stream)
{
    if (ldimx <= 0 || ldimy <= 0 || izbeg < 0 || !field1 || !field2) return TTI_EINVAL;
    int64_t plane = (int64_t)ldimx * ldimy;
    dim3 grid((unsigned)((plane + 255) / 256), izbeg + 1);
    k_loop4<<<grid, 256, 0, S(stream)>>>(field1, field2, plane, izbeg);
    return launch_status();
}

int tti_launch_init_cijs(const float* vp, const float* eps, const float* delta, const float* vs,
                         const float* theta, const float* phi, float* model1, float* model2, float* model3,
                         float* model4, float* model5, float* model6, float* model7, int64_t n,
                         tti_stream_t stream)
{
    if (n < 0 || !vp || !eps || !delta || !vs || !theta || !phi || !model1 || !model2 || !model3 || !model4 ||
        !model5 || !model6 || !model7)
        return TTI_EINVAL;
    if (n == 0) return TTI_OK;
    k_init_cijs<<<(unsigned)((n + 255) / 256), 256, 0, S(stream)>>>(vp, eps, delta, vs, theta, phi, model1, model2,
                                                                   model3, model4, model5, model6, model7, n);
    return launch_status();
}

int tti_launch_compute_pressure(float* pressure, const float* field1, const float* field2, int64_t n,
                                tti_stream_t stream)
{
    if (n < 0 || !pressure || !field1 || !field2) return TTI_EINVAL;
    if (n == 0) return TTI_OK;
    k_pressure<<<(unsigned)((n + 255) / 256), 256, 0, S(stream)>>>(pressure, field1, field2, n);
    return launch_status();
}

} // extern "C"
