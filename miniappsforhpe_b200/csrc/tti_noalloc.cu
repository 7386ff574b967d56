// Adjoint derivatives with a fixed, statically allocated scratch volume.
//
// tti_launch_adj_kernel2_drv takes its four-float-per-cell scratch (the
// point-wise transposed model) from the device's stream-ordered allocator on
// every call.  Some callers cannot let a library allocate:
//   * a host framework that owns the device memory through its own pool and
//     has reserved most of HBM for it, so an allocation behind its back fails
//     or pushes the pool out of memory;
//   * a caller whose device memory pool is configured for its own use (a
//     release threshold, access flags, a pool it does not want the library's
//     blocks mixed into);
//   * a caller that must know its full device footprint up front, before the
//     first step runs.
// tti_launch_adj_kernel2_drv_noalloc serves them: its scratch is a
// file-scope __device__ array of fixed size that is part of the loaded
// module, so the call itself never allocates.  Its limits:
//   * the volume range it can take is bounded by the array's capacity
//     (TTI_NOALLOC_SCRATCH_CELLS cells); larger requests return TTI_ETOOBIG;
//   * the first call on a device looks up the array's address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture;
//   * every call on a device shares the one array; calls whose kernels
//     overlap on the GPU (different streams, no ordering between them) race
//     on it and give wrong results.  Order them on one stream or with events.
// Nothing in the array has to start at zero: the first kernel of a call
// writes every cell the second kernel reads (the interior range widened by
// the radius-4 halo on every axis), so the previous call's contents never
// reach an output.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "tti_common.cuh"
#include "tti_internal.cuh"

namespace {

using tti::kRadius;

__device__ __align__(256) float4 g_adj_scratch[TTI_NOALLOC_SCRATCH_CELLS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
float4* g_addr[kMaxDevices];  // address of g_adj_scratch per device, set once

// Address of the scratch array on the current device (nullptr on failure).
float4* scratch_address()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_adj_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_addr[dev] = static_cast<float4*>(p);
    }
    return g_addr[dev];
}

} // namespace

extern "C" int tti_launch_adj_kernel2_drv_noalloc(
    float* dfield1dx, float* dfield2dx, float* dfield1dy, float* dfield2dy, float* dfield1dz, float* dfield2dz,
    float* field3_rhs, float* field4_rhs, const float* field1, const float* field2, const float* Model11,
    const float* model1, const float* model2, const float* model3, const float* model4, const float* model5,
    const float* model6, const float* model7, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
    float invdxx, float invdyy, float invdzz, float invdxy, float invdyz, float invdzx, int ldimx, int ldimy,
    int order, float dt, float invdx, float invdy, float invdz, tti_stream_t stream)
{
    (void)invdxx;
    (void)invdyy;
    (void)invdzz;
    (void)dt;
    if (order != 8 || !tti::ranges_ok(ixbeg, ixend, iybeg, iyend, izbeg, izend, ldimx, ldimy)) return TTI_EINVAL;
    if (!dfield1dx || !dfield2dx || !dfield1dy || !dfield2dy || !dfield1dz || !dfield2dz || !field3_rhs ||
        !field4_rhs || !field1 || !field2 || !Model11 || !model1 || !model2 || !model3 || !model4 || !model5 ||
        !model6 || !model7)
        return TTI_EINVAL;
    // The scratch is indexed like the volumes; the highest cell written is
    // (izend + 4, iyend + 4, ixend + 4), below ldimx * ldimy * (izend + 5).
    const int64_t cells = (int64_t)ldimx * ldimy * ((int64_t)izend + 1 + kRadius);
    if (cells > (int64_t)TTI_NOALLOC_SCRATCH_CELLS) return TTI_ETOOBIG;
    float4* base = scratch_address();
    if (!base) return TTI_ELAUNCH;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int rc = tti::launch_base(field1, field2, model1, model2, model3, model4, base, ixbeg, ixend, iybeg, iyend, izbeg,
                              izend, ldimx, ldimy, st);
    if (rc) return rc;
    return tti::launch_adj_drv_with_base(dfield1dx, dfield2dx, dfield1dy, dfield2dy, dfield1dz, dfield2dz,
                                         field3_rhs, field4_rhs, base, Model11, model5, model6, model7, ixbeg, ixend,
                                         iybeg, iyend, izbeg, izend, ldimx, ldimy, invdxy, invdyz, invdzx, invdx,
                                         invdy, invdz, st);
}
