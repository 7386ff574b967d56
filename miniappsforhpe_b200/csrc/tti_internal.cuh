// Internal launch helpers shared by the simulator, the C ABI and the fused
// kernels.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <vector>

#include "tti_common.cuh"

namespace tti {

// Scratch of nelem float4 cells for one launcher call, allocated and freed
// in stream order on that call's stream (cudaMallocAsync / cudaFreeAsync):
// nothing is kept between calls, calls on different streams never share
// memory, and no call synchronizes the device.  get() is nullptr when the
// allocation failed.
class CallScratch {
public:
    CallScratch(size_t nelem, cudaStream_t st) : st_(st)
    {
        if (cudaMallocAsync(reinterpret_cast<void**>(&p_), nelem * sizeof(float4), st) != cudaSuccess) {
            cudaGetLastError();
            p_ = nullptr;
        }
    }
    ~CallScratch()
    {
        if (p_) cudaFreeAsync(p_, st_);
    }
    CallScratch(const CallScratch&) = delete;
    CallScratch& operator=(const CallScratch&) = delete;
    float4* get() const { return p_; }

private:
    float4* p_ = nullptr;
    cudaStream_t st_;
};

int launch_base(const float* f1, const float* f2, const float* m1, const float* m2, const float* m3,
                const float* m4, float4* base, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                int ldimx, int ldimy, cudaStream_t st);
int launch_adj_drv_with_base(float* d1x, float* d2x, float* d1y, float* d2y, float* d1z, float* d2z, float* rhs3,
                             float* rhs4, const float4* base, const float* irho, const float* rx, const float* ry,
                             const float* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                             int ldimx, int ldimy, float invdxy, float invdyz, float invdzx, float invdx, float invdy,
                             float invdz, cudaStream_t st);
int launch_rho_gradient_with_base(float* grad, const float* fd1x, const float* fd2x, const float* fd1y,
                                  const float* fd2y, const float* fd1z, const float* fd2z, const float4* base,
                                  const float* irho, const float* rx, const float* ry, const float* rz, int ixbeg,
                                  int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx, int ldimy,
                                  int gldx, int gldy, double dx, double dy, double dz, cudaStream_t st);

// Receiver cells for the step kernels: the receivers lie on nz planes with
// halo'd z index z[k]; plane k's table of receiver numbers per interior cell
// (-1: none) starts at off[k] in xy.  Passed by value, so the plane check of
// an output plane is a block-uniform comparison with kernel parameters.
constexpr int kRecPlanesFolded = 8;
struct RecMap {
    const int* xy = nullptr;
    int nz = 0;
    int zlo = 1, zhi = 0;  // range of the z[k] (empty when nz = 0)
    int z[kRecPlanesFolded] = {};
    int off[kRecPlanesFolded] = {};
};

// Model volumes in the reference layout, all halo'd; the fused adjoint also
// reads them interleaved per cell: ma = (m1, m2, m3, m4), mb = (irho, rx,
// ry, rz), in the same layout with float4 cells.
struct Model {
    const float *irho, *m1, *m2, *m3, *m4, *rx, *ry, *rz;
    const float4* ma = nullptr;
    const float4* mb = nullptr;
};

// Fused forward step (tti_fused.cu).  Reads p,q at time n from pin/qin
// (free surface already applied), updates pdot/qdot in place with the TTI
// operator plus the point source, writes p,q at time n+1 (loop2 + free
// surface) to pout/qout, and optionally stores the snapshot of this step.
struct FwdStepArgs {
    const float* pin;
    const float* qin;
    float* pout;
    float* qout;
    float* f3;
    float* f4;
    Model m;
    const float2 *abx, *aby, *abz;
    int64_t src_index;  // -1: no source
    float src_term;     // w[n]*dt
    void* snap;                 // nullptr or 4 interior volumes: pdot, qdot, p, q
    int snap_prec;              // SnapPrec of the store
    const float* snap_scale;    // 4 multipliers applied before storing (reduced precision)
    unsigned int* snap_amax;    // 4 running max |value| (float bits) of this snapshot
    int free_surface;
    int vti;            // 1: rx=ry=0, rz=1 are not read
    float dt;
    double dx, dy, dz;
    int* err = nullptr;  // error word of the bounded waits (nullptr: the device's)
    int bz = 0;          // planes per CTA of the tile-major (tile, z) work (0: tuned or modelled)
    int ztop = 0;        // > 0: column tops of ztop planes, bz planes per CTA of the bottoms
    int wave_prec = 0;                 // p/q leave the step rounded to FP16 (1) or BF16 (2)
    const float* wave_scale = nullptr; // 2 power-of-two scales (p, q) of the output
    // receivers sampled inside the step: trace[r] = -(2p + q)/3 of the
    // incoming p, q at receiver r's cell (nullptr: not sampled here)
    float* trace = nullptr;
    RecMap rec{};
};
int launch_fused_forward(const Layout& L, const FwdStepArgs& a, cudaStream_t st);

// Fused adjoint step (tti_fused.cu): the reference's adjoint sequence
// adj_drv, loop4_derivatives, adj_update, loop2, loop4 in one pass.
struct AdjStepArgs {
    const float* pin;
    const float* qin;
    float* pout;
    float* qout;
    float* f3;
    float* f4;
    Model m;
    const float2 *abx, *aby, *abz;
    int sponge_active;
    int free_surface;
    int vti;
    float dt;
    double dx, dy, dz;
    int* err = nullptr;
    int bz = 0;
    int ztop = 0;
    int wave_prec = 0;
    const float* wave_scale = nullptr;
    // folded into the step: residual injection pdot += -2/3 v, qdot += -1/3 v
    // at receiver r's cell, v = res[r] (- obs[r] if obs), before the update;
    // and the source trace *srctr = p + q of the incoming state at src_index
    const float* res = nullptr;
    const float* obs = nullptr;
    RecMap rec{};
    float* srctr = nullptr;
    int64_t src_index = -1;
};
int launch_fused_adjoint(const Layout& L, const AdjStepArgs& a, cudaStream_t st);

// Fused imaging at a snapshot step (tti_fused.cu): Vp image from the adjoint
// pdot/qdot and the stored pdot/qdot, density gradient from the stored p/q
// (forward derivatives formed on the fly) and the adjoint p/q.  The store is
// nsnap slots of four dense interior volumes (pdot, qdot, p, q).
struct ImageArgs {
    const float* adj1;
    const float* adj2;
    const float* adj3;
    const float* adj4;
    const void* store;
    int snap_prec;
    const float* snap_scale;  // 4 multipliers the slot was stored with
    int nsnap;
    int slot;
    Model m;
    float* grad_vp;   // dense nx*ny*nz
    float* grad_rho;  // dense nx*ny*nz
    int free_surface;
    int vti;
    double dx, dy, dz;
    int* err = nullptr;
    int bz = 0;
    int ztop = 0;
};
bool fused_image_supported(const Layout& L);
int launch_fused_image(const Layout& L, const ImageArgs& a, cudaStream_t st);

// Status of the bounded waits inside the fused kernels since the last call
// (TTI_ETIMEOUT if any gave up, TTI_ERANGE if a reduced-precision snapshot
// saturated); synchronizes the stream and clears the word.  word = nullptr
// reads the device's shared word.
int fused_wait_status(cudaStream_t st, int* word = nullptr);

// Work split of a fused kernel on this grid.  ztop = 0: each CTA takes bz
// consecutive planes of the grid's (tile, z) planes in tile-major order.
// ztop > 0 (grids with fewer tile columns than SMs): CTA t < tiles takes the
// top ztop planes of column t, and the remaining CTAs share the columns'
// bottoms (planes ztop .. nz-1, tile-major) bz planes each, so that every SM
// has work while the CTAs that run side by side stay at the same depth.
// kernel kinds of the work-split table: the staggered scheme's three fused
// kernels, then the centred (type1) forward and adjoint step kernels
enum { KIND_FWD = 0, KIND_ADJ = 1, KIND_IMG = 2, KIND_T1F = 3, KIND_T1A = 4, KIND_COUNT = 5 };
struct Split {
    int bz = 0;
    int ztop = 0;
    bool operator==(const Split& o) const { return bz == o.bz && ztop == o.ztop; }
};
bool split_valid(const Layout& L, Split s);
// The autotuned split if one was recorded, else the wave-count model's.
Split choose_split(const Layout& L, int kind);
void record_tuned_split(const Layout& L, int kind, Split s);  // bz = 0 clears
Split tuned_split(const Layout& L, int kind);                 // bz = 0 if none recorded
Split model_split(const Layout& L, int kind);
// Candidates the tuner tries: whole-column chunks ceil(nz/n), equal shares
// of the work for 1..8 CTAs per SM (each at least 8 planes), and top/bottom
// splits around the balance point of the kind's pipeline fill.
std::vector<Split> split_candidates(const Layout& L, int kind);

// Type1 scheme (constant density, centred second derivatives): fused forward
// step (pdot update with the sponge form when sponge = 1, as the type1
// launcher's use_sponge), fused adjoint step (sponge per a.sponge_active), and
// the Vp imaging of a store slot.  m.irho is not read.
int launch_t1_fused_forward(const Layout& L, const FwdStepArgs& a, int sponge, cudaStream_t st);
int launch_t1_fused_adjoint(const Layout& L, const AdjStepArgs& a, cudaStream_t st);
int launch_t1_image(const Layout& L, const ImageArgs& a, cudaStream_t st);

// Sets the fused kernels' attributes and allocates the error word on the
// current device (done by the first launch otherwise); call before a stream
// capture that contains fused launches.
int prepare_fused_kernels();

// Runs the bounded-wait path on a barrier that never completes; returns
// TTI_ETIMEOUT when the wait gave up and reported as it should.
int wait_selfcheck(cudaStream_t st, long long limit_cycles);

} // namespace tti
