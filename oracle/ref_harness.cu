// Reference-kernel harness: TEST INFRASTRUCTURE ONLY.
//
// Thin extern "C" wrappers around the reference's own launchers for the TTI
// p/q path, so the tests can run the reference kernels (compiled unmodified
// from the reference sources for sm_100a, see oracle/Makefile) on the same
// device buffers as the product kernels.  Nothing here is linked into the
// product.  All pointers are device pointers to full halo'd volumes in the
// reference layout; every wrapper launches on the legacy default stream, as
// the reference simulator does (kernel_base.h:32-40).
//
// The reference aborts on a CUDA error (CUDA_TRY, utils/cuda_utils.h:20-28);
// the wrappers check the arguments first so that only in-bounds launches are
// ever issued: every axis must carry a radius-4 halo, ixbeg must be 4 and
// ldimx a multiple of 32 (the layout of infrastructure/axis.cpp:78-99).

#include <cuda_runtime.h>
#include <cstdio>

#include "kernel_type1_gpu_adj.h"
#include "kernel_type1_gpu_fwd.h"
#include "kernel_type1_gpu_grad.h"
#include "kernel_type2_adj.h"
#include "kernel_type2_fwd.h"
#include "kernel_type2_fwd_drv.h"
#include "kernel_type2_grad.h"
#include "kernel_type2_grad_snap.h"
#include "kernel_type2_small.h"
#include "volume_index.h"

// Defined in kernels/kernel_base.cu:82 and :142 (no header declares them).
__global__ void kernel_loop2_inner_kernel(float* field1_, float* field2_, const float* field3_, const float* field4_,
                                          volume_index idx, int ixbeg, int ixend, int iybeg, int izbeg,
                                          const float2* ABx, const float2* ABy, const float2* ABz, const float dt);
__global__ void kernel_loop4_kernel(float* field1, float* field2, int stride, int izbeg);

namespace {
bool layout_ok(int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy)
{
    bool ok = ixbeg == 4 && iybeg == 4 && izbeg == 4 && ixend >= ixbeg && iyend >= iybeg && izend >= izbeg &&
              ldimx % 32 == 0 && ldimx >= ixend + 5 && ldimy == iyend + 5;
    if (!ok) std::fprintf(stderr, "ref_harness: unsupported layout\n");
    return ok;
}
int status() { return cudaPeekAtLastError() == cudaSuccess ? 0 : 1; }
} // namespace

extern "C" {

int ref_fwd_drv(const float* f1, const float* f2, const float* irho, float* d1x, float* d1y, float* d1z, float* d2x,
                float* d2y, float* d2z, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, float invdx,
                float invdy, float invdz, int ldimx, int ldimy)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    kernel3_gpu_kernels::launch_fwd_kernel2_drv(f1, f2, irho, d1x, d1y, d1z, d2x, d2y, d2z, ixbeg, ixend, iybeg, iyend,
                                               izbeg, izend, invdx, invdy, invdz, ldimx, ldimy, 8, 0);
    return status();
}

int ref_fwd_update(float* f3, float* f4, const float* d1x, const float* d2x, const float* d1y, const float* d2y,
                   const float* d1z, const float* d2z, const float* f1, const float* f2, const float* irho,
                   const float* m1, const float* m2, const float* m3, const float* m4, const float* rx,
                   const float* ry, const float* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                   int ldimx, int ldimy, float dt, double dx, double dy, double dz)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    launch_update_rho_fwd_main_loop_2_1(f3, f4, d1x, d2x, d1y, d2y, d1z, d2z, f1, f2, irho, m1, m2, m3, m4, rx, ry, rz,
                                        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, nullptr, nullptr, ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx,
                                        ldimy, dt, dx, dy, dz, false, 8, false, false, false, 0);
    return status();
}

int ref_adj_drv(float* d1x, float* d2x, float* d1y, float* d2y, float* d1z, float* d2z, float* rhs3, float* rhs4,
                float* f1, float* f2, float* irho, float* m1, float* m2, float* m3, float* m4, float* rx, float* ry,
                float* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, double dx, double dy,
                double dz, int ldimx, int ldimy, float dt)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    // kernel_type2.cu:467-480: constants from compute_fd_const (kernel_utils.h:89-101).
    float invdx = 1.0 / dx, invdy = 1.0 / dy, invdz = 1.0 / dz;
    float invdxx = 1.0 / (dx * dx), invdyy = 1.0 / (dy * dy), invdzz = 1.0 / (dz * dz);
    float invdxy = 1.0 / (4 * dx * dy), invdyz = 1.0 / (4 * dy * dz), invdzx = 1.0 / (4 * dx * dz);
    adj_kernel3_derivatives::launch_adj_kernel2_drv(d1x, d2x, d1y, d2y, d1z, d2z, rhs3, rhs4, f1, f2, irho, m1, m2, m3,
                                                   m4, rx, ry, rz, ixbeg, ixend, iybeg, iyend, izbeg, izend, invdxx,
                                                   invdyy, invdzz, invdxy, invdyz, invdzx, ldimx, ldimy, 8, dt, invdx,
                                                   invdy, invdz, 0);
    return status();
}

int ref_adj_update(float* f3, float* f4, const float* d1x, const float* d2x, const float* d1y, const float* d2y,
                   const float* d1z, const float* d2z, const float* rhs3, const float* rhs4, const float* abx,
                   const float* aby, const float* abz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                   int izend, int ldimx, int ldimy, float dt, double dx, double dy, double dz, int sponge_active)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    kernel3_gpu_kernels::launch_update_adj_kernel_main_3(
        f3, f4, d1x, d2x, d1y, d2y, d1z, d2z, rhs3, rhs4, reinterpret_cast<const float2*>(abx),
        reinterpret_cast<const float2*>(aby), reinterpret_cast<const float2*>(abz), ixbeg, ixend, iybeg, iyend, izbeg,
        izend, ldimx, ldimy, dt, dx, dy, dz, false, false, false, 8, sponge_active != 0, 0);
    return status();
}

int ref_rho_gradient(float* grad, const float* fd1x, const float* fd2x, const float* fd1y, const float* fd2y,
                     const float* fd1z, const float* fd2z, const float* f1, const float* f2, const float* irho,
                     const float* m1, const float* m2, const float* m3, const float* m4, const float* rx,
                     const float* ry, const float* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                     int izend, int ldimx, int ldimy, int grad_ldimx, int grad_ldimy, double dx, double dy, double dz,
                     int simple)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    launch_update_rho_gradient_rho(grad, fd1x, fd2x, fd1y, fd2y, fd1z, fd2z, f1, f2, irho, m1, m2, m3, m4, rx, ry, rz,
                                   ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy, grad_ldimx, grad_ldimy, dx,
                                   dy, dz, 8, simple != 0, 0);
    return status();
}

// Launch shape of kernel_type2::kernel_loop4_derivative_impl (kernel_type2.cu:278-293).
int ref_loop4_derivatives(float* d1x, float* d1y, float* d1z, float* d2x, float* d2y, float* d2z, int ldimx, int ldimy,
                          int izbeg)
{
    dim3 threads(32, 32, 1);
    dim3 blocks((ldimx + 31) / 32, (ldimy + 31) / 32, izbeg + 1);
    kernel3_gpu_kernels::kernel_loop4_derivatives<<<blocks, threads>>>(d1x, d1y, d1z, d2x, d2y, d2z, ldimx, ldimy,
                                                                        izbeg);
    return status();
}

// Launch shape of kernel_type2::update_grad_loop_1_impl (kernel_type2.cu:305-330).
int ref_update_vp_gradient(const float* snap3, const float* snap4, float* grad, const float* adj3, const float* adj4,
                           int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int snx, int sny,
                           int ldimx, int ldimy)
{
    volume_index idx(snx, sny);
    volume_index idx_adj(ldimx, ldimy);
    int nx = ixend - ixbeg + 1, ny = iyend - iybeg + 1, nz = izend - izbeg + 1;
    dim3 threads(32, 32, 1);
    dim3 blocks((nx + 31) / 32, (ny + 31) / 32, nz);
    kernel3_gpu_kernels::update_Vp_gradient<<<blocks, threads, 0>>>(
        idx, idx_adj, const_cast<float*>(snap3), const_cast<float*>(snap4), grad, const_cast<float*>(adj3),
        const_cast<float*>(adj4), ixbeg, ixend, iybeg, iyend, izbeg, izend);
    return status();
}

// Launch shape of kernel_base::kernel_loop2_inner (kernel_base.cu:106-140).
int ref_loop2(float* f1, float* f2, const float* f3, const float* f4, int ldimx, int ldimy, int ixbeg, int ixend,
              int iybeg, int iyend, int izbeg, int izend, const float* abx, const float* aby, const float* abz,
              float dt)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    volume_index idx(ldimx, ldimy);
    dim3 threads(128, 1, 1);
    dim3 blocks(ixend / 128 + 1, iyend - iybeg + 1, izend - izbeg + 1);
    kernel_loop2_inner_kernel<<<blocks, threads>>>(f1, f2, f3, f4, idx, ixbeg, ixend, iybeg, izbeg,
                                                   reinterpret_cast<const float2*>(abx),
                                                   reinterpret_cast<const float2*>(aby),
                                                   reinterpret_cast<const float2*>(abz), dt);
    return status();
}

// Launch shape of kernel_base::kernel_loop4_inner (kernel_base.cu:164-187).
int ref_loop4(float* f1, float* f2, int ldimx, int ldimy, int izbeg)
{
    int stride = ldimx * ldimy;
    dim3 threads(1024, 1, 1);
    dim3 blocks((stride - 1) / 1024 + 1, 1, izbeg + 1);
    kernel_loop4_kernel<<<blocks, threads>>>(f1, f2, stride, izbeg);
    return status();
}

// Type1 launchers (kernels/kernel_type1_gpu_{fwd,adj,grad}.cu), default
// (optimised) kernels, standard layout only (ldimz = izend + 5).
int ref_t1_fwd(float* f3, float* f4, const float* f1, const float* f2, const float* m1, const float* m2,
               const float* m3, const float* m4, const float* m5, const float* m6, const float* m7, const float* abx,
               const float* aby, const float* abz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
               int ldimx, int ldimy, int ldimz, int ldimx_out, int ldimy_out, int ldimz_out, float dt, double dx,
               double dy, double dz, int calc_snap, int use_sponge)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy) || ldimz != izend + 5) return 2;
    if (calc_snap && use_sponge) return 2;
    if (!calc_snap && (ldimx_out != ldimx || ldimy_out != ldimy)) return 2;
    fwd_main_loop_2_1_inner_gpu::launch(f3, f4, f1, f2, m1, m2, m3, m4, m5, m6, m7,
                                        reinterpret_cast<const float2*>(abx), reinterpret_cast<const float2*>(aby),
                                        reinterpret_cast<const float2*>(abz), ixbeg, ixend, iybeg, iyend, izbeg,
                                        izend, ldimx, ldimy, ldimz, ldimx_out, ldimy_out, ldimz_out, dt, dx, dy, dz, 8,
                                        0, calc_snap != 0, use_sponge != 0, false);
    return status();
}

int ref_t1_adj(float* f3, float* f4, const float* f1, const float* f2, const float* m1, const float* m2,
               const float* m3, const float* m4, const float* m5, const float* m6, const float* m7, const float* abx,
               const float* aby, const float* abz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
               int ldimx, int ldimy, int ldimz, float dt, double dx, double dy, double dz, int use_sponge)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy) || ldimz != izend + 5) return 2;
    adj_main_loop_2_inner_gpu::launch(f3, f4, f1, f2, m1, m2, m3, m4, m5, m6, m7,
                                      reinterpret_cast<const float2*>(abx), reinterpret_cast<const float2*>(aby),
                                      reinterpret_cast<const float2*>(abz), ixbeg, ixend, iybeg, iyend, izbeg, izend,
                                      ldimx, ldimy, ldimz, dt, dx, dy, dz, 8, 0, use_sponge != 0, false);
    return status();
}

int ref_t1_grad(float* snap_x, float* snap_z, float* grad, float* adj_x, float* adj_z, int ixbeg, int ixend,
                int iybeg, int iyend, int izbeg, int izend, int snx, int sny, int ldimx, int ldimy)
{
    if (!layout_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return 2;
    launch_update_grad_loop_kernel(volume_index(snx, sny), volume_index(ldimx, ldimy), snap_x, snap_z, grad, adj_x,
                                   adj_z, ixbeg, ixend, iybeg, iyend, izbeg, izend);
    return status();
}

int ref_sync() { return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1; }

} // extern "C"
