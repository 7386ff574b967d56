// Simulator object: the simulator2SetUp call surface on one B200.
//
// Mirrors simulator2/simulator2SetUp.{h,cu}: model setup (init_cijs plus the
// buoyancy volume the reference never fills, simulator2SetUp.cu:476-502,
// kernel_type2.cu:136-141), the forward time loop with snapshots every
// xcorr_step steps (:530-651), the adjoint loop with the imaging condition
// at snapshot steps (:654-782), and image readback.  Differences from the
// reference, all deliberate:
//   * one domain on one GPU: no zones, no halo exchange, no MPI;
//   * snapshots stay in HBM (interior only; p/q halos are re-derived);
//   * a point source injected every step and receivers sampled every step
//     (the reference only seeds an impulse, simulator2SetUp.cu:44-49);
//   * the adjoint starts from rest and is driven by residual traces;
//   * the density gradient is stored interior-only at its own cells.
// Every call returns a status code; nothing aborts.

#include <cuda_runtime.h>

#include <cmath>
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "tti_common.cuh"
#include "tti_internal.cuh"
#include "tti_shot.cuh"

using namespace tti;

namespace {

// Model set-up in one pass over the halo'd volumes: every cell takes the
// parameters of the nearest interior cell (edge extension on every axis,
// the x padding included), applies init_cijs (simulator2SetUp.cu:10-29) and
// writes the buoyancy irho = 1/rho (IEEE division; the reference never sets
// Model11, kernel_type2.cu:136-141).  par holds the dense interior arrays
// vp, eps, delta, vs, theta, phi, rho; a null entry takes its default (0,
// rho 1).  Any theta != 0 marks the model TTI in *tti_flag.
struct ModelOut {
    float* v[8];        // irho, model1..model4, rx, ry, rz
    float4* pack[2];    // nullptr, or (m1, m2, m3, m4) and (irho, rx, ry, rz) per cell
};
struct ModelIn {
    const float* p[7];
};
__global__ void k_model_setup(ModelOut out, ModelIn par, Layout L, int* __restrict__ tti_flag)
{
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;  // ldimx is a multiple of 32: whole warps leave
    const int iy = blockIdx.y, iz = blockIdx.z;
    if (ix >= L.ldimx) return;
    const int nx = L.nx(), ny = L.ny(), nz = L.nz();
    const int jx = min(max(ix - L.ixbeg, 0), nx - 1);
    const int jy = min(max(iy - L.iybeg, 0), ny - 1);
    const int jz = min(max(iz - L.izbeg, 0), nz - 1);
    const int64_t d = ((int64_t)jz * ny + jy) * nx + jx;
    const float dflt[7] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 1.0f};
    float v[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = par.p[k] ? __ldg(par.p[k] + d) : dflt[k];
    const int64_t g = L.idx(ix, iy, iz);
    float m[7];
    init_cij_cell(v[0], v[1], v[2], v[3], v[4], v[5], m[0], m[1], m[2], m[3], m[4], m[5], m[6]);
    const float irho = 1.0f / v[6];
    out.v[0][g] = irho;
#pragma unroll
    for (int k = 0; k < 7; ++k) out.v[k + 1][g] = m[k];
    if (out.pack[0]) {
        out.pack[0][g] = make_float4(m[0], m[1], m[2], m[3]);
        out.pack[1][g] = make_float4(irho, m[4], m[5], m[6]);
    }
    if (__any_sync(0xffffffffu, v[4] != 0.0f) && (threadIdx.x & 31) == 0) atomicOr(tti_flag, 1);
}

// Interior copy between a halo'd volume and a dense interior array.
template <bool TO_DENSE>
__global__ void k_interior_copy(float* __restrict__ vol, float* __restrict__ dense, Layout L)
{
    int jx = blockIdx.x * blockDim.x + threadIdx.x;
    int jy = blockIdx.y;
    int jz = blockIdx.z;
    int nx = L.nx();
    if (jx >= nx) return;
    int64_t d = ((int64_t)jz * L.ny() + jy) * nx + jx;
    int64_t v = L.idx(jx + L.ixbeg, jy + L.iybeg, jz + L.izbeg);
    if (TO_DENSE)
        dense[d] = vol[v];
    else
        vol[v] = dense[d];
}

// Snapshot of one forward step: pdot, qdot, p, q interior -> slot.
__global__ void k_snapshot_save(float* __restrict__ slot, const float* __restrict__ f3, const float* __restrict__ f4,
                                const float* __restrict__ f1, const float* __restrict__ f2, Layout L)
{
    int jx = blockIdx.x * blockDim.x + threadIdx.x;
    int jy = blockIdx.y;
    int jz = blockIdx.z;
    int nx = L.nx();
    if (jx >= nx) return;
    int64_t n = (int64_t)nx * L.ny() * L.nz();
    int64_t d = ((int64_t)jz * L.ny() + jy) * nx + jx;
    int64_t v = L.idx(jx + L.ixbeg, jy + L.iybeg, jz + L.izbeg);
    slot[d] = f3[v];
    slot[n + d] = f4[v];
    if (f1) {  // two-field slots (centred scheme) keep pdot and qdot only
        slot[2 * n + d] = f1[v];
        slot[3 * n + d] = f2[v];
    }
}

__global__ void k_add_source(float* f3, float* f4, int64_t i, float term)
{
    f3[i] += term;
    f4[i] += term;
}

__global__ void k_receivers(float* __restrict__ out, const float* __restrict__ f1, const float* __restrict__ f2,
                            const int64_t* __restrict__ rec, int nrec)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    int64_t i = rec[r];
    out[r] = -(2 * f1[i] + f2[i]) / 3;
}

// Adjoint p+q at the source cell: dt times this is the gradient of the
// receiver misfit with respect to the source wavelet sample of that step.
__global__ void k_source_trace(float* __restrict__ out, const float* __restrict__ f1, const float* __restrict__ f2,
                               int64_t i)
{
    *out = f1[i] + f2[i];
}

// Residual injection: (-2/3, -1/3) times the residual, the transpose of the
// pressure receiver -(2p+q)/3.  With obs != nullptr the residual is the
// recorded synthetic trace minus the observed one.
__global__ void k_inject_residual(float* __restrict__ f3, float* __restrict__ f4, const int64_t* __restrict__ rec,
                                  const float* __restrict__ res, const float* __restrict__ obs, int nrec)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    int64_t i = rec[r];
    float v = obs ? res[r] - obs[r] : res[r];
    f3[i] += (-2.0f / 3.0f) * v;
    f4[i] += (-1.0f / 3.0f) * v;
}

// Per-field power-of-two scale of the next reduced-precision snapshot from
// the running max |value| of the previous one: max*scale ~ 2^11, leaving a
// factor 32 of growth before FP16 saturates; the running max is reset.
__global__ void k_snap_scale(float* __restrict__ scale, unsigned int* __restrict__ amax, int nfield)
{
    const int f = threadIdx.x;
    if (f >= nfield) return;
    const float m = __uint_as_float(amax[f]);
    float sc = 1.0f;
    if (m > 0.0f && isfinite(m)) {
        int e = 0;
        frexpf(m, &e);  // m = g * 2^e, g in [0.5, 1)
        e = max(-100, min(100, 11 - e));
        sc = ldexpf(1.0f, e);
    }
    scale[f] = sc;
    amax[f] = 0u;
}

// Interior-only Vp image scaling g *= -2*dt_xcorr/vp (kernel_type2_small.cu:61-74).
__global__ void k_finalize_dense(float* __restrict__ g, const float* __restrict__ m3, Layout L, float dt_xcorr)
{
    int jx = blockIdx.x * blockDim.x + threadIdx.x;
    int jy = blockIdx.y;
    int jz = blockIdx.z;
    int nx = L.nx();
    if (jx >= nx) return;
    int64_t d = ((int64_t)jz * L.ny() + jy) * nx + jx;
    float vp = sqrtf(m3[L.idx(jx + L.ixbeg, jy + L.iybeg, jz + L.izbeg)]);
    g[d] *= -dt_xcorr * 2.0 / vp;
}

inline int cuda_rc(cudaError_t e)
{
    if (e == cudaSuccess) return TTI_OK;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? TTI_ENOMEM : TTI_ELAUNCH;
}

// Fields per snapshot slot: pdot, qdot, p, q for the staggered scheme (its
// density image differentiates the stored p/q); pdot and qdot alone for the
// centred scheme, whose Vp image is all it makes.
inline int snap_fields(const tti_sim_config& c) { return c.scheme == 1 ? 2 : 4; }

} // namespace

// Device state of one wavefield: p, q (read buffer), pdot, qdot, and the
// second p, q buffer the fused kernels write the next step into.
struct WaveState {
    float *p = nullptr, *q = nullptr, *pd = nullptr, *qd = nullptr, *p2 = nullptr, *q2 = nullptr;
    // reduced-precision wavefields: scales (p, q) of the next step's output
    // and the maxima of |p|, |q| of the current state
    float* wscale = nullptr;
    unsigned* wamax = nullptr;
    void swap()
    {
        std::swap(p, p2);
        std::swap(q, q2);
    }
};

struct tti_sim {
    tti_sim_config cfg{};
    Layout L{};
    cudaStream_t stream = nullptr;
    std::vector<void*> allocs;
    WaveState w;   // forward wavefield, then the adjoint one
    WaveState rw;  // forward wavefield recomputed from checkpoints
    // reference kernel sequence only (fused = 0, or imaging on grids the fused
    // imaging kernel does not take)
    float* d[6] = {};
    float *rhs3 = nullptr, *rhs4 = nullptr;
    float4* base = nullptr;
    float *snp = nullptr, *snq = nullptr;  // halo'd p/q restored from a snapshot
    bool aux = false;
    float* mv[8] = {};  // irho, m1..m4, rx, ry, rz
    float4* mpack[2] = {};  // the same interleaved: (m1, m2, m3, m4), (irho, rx, ry, rz) (fused staggered path)
    float2 *abx = nullptr, *aby = nullptr, *abz = nullptr;
    // snapshot store: nslot slots of 4 interior volumes (pdot, qdot, p, q)
    void* snaps = nullptr;
    float* snap_scale = nullptr;        // nslot x 4 storage multipliers
    unsigned int* snap_amax = nullptr;  // 4 running max |value| (float bits)
    int nsnap = 0;                      // snapshot steps in the shot
    int nslot = 0;                      // slots held (nsnap, or one segment with checkpoints)
    // checkpoints: ncp FP32 states (p, q, pdot, qdot interior) every ckpt steps
    float* ckpts = nullptr;
    unsigned int* ckpt_amax = nullptr;  // running snapshot max at each checkpoint
    int ckpt = 0, ncp = 0;
    float *grad_vp = nullptr, *grad_rho = nullptr;
    int* err = nullptr;  // error word of this simulator's fused kernels
    int64_t src_index = -1;
    std::vector<float> wavelet;
    int nrec = 0;
    int64_t* rec = nullptr;
    float* traces = nullptr;  // nt*nrec device
    float* resid = nullptr;   // nt*nrec device
    float* srctr = nullptr;   // nt device: adjoint p+q at the source
    // receiver cells as per-plane tables for the fused staggered step kernels,
    // which then sample the receivers and inject the residual themselves
    int* rec_xy = nullptr;  // receiver number per cell of the receiver planes, -1 elsewhere
    RecMap recmap{};        // the planes and their table offsets (kernel parameters)
    bool rec_fold = false;
    bool model_set = false, forward_done = false;
    bool sponge_active = false;
    bool vti = false;
    bool profiling = false;
    bool capturing = false;
    cudaGraphExec_t gexec[3] = {};  // cached graphs: forward, adjoint (last segment), recompute segment
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<int, size_t>> ev_marks;  // (kind, index of start event)
    double kind_ms[3] = {0, 0, 0};
    int64_t kind_n[3] = {0, 0, 0};
    int64_t launches = 0;
    int64_t ninterior = 0;
    // resumable shot: phase 0 idle, 1 forward, 2 adjoint, 3 done
    int sh_phase = 0, sh_n = 0, sh_seg = 0;
    bool sh_recomp = false;
    // step-level cursor: 0 idle, 1 forward (next step st_n), 2 adjoint (next
    // step st_n, last adjoint step st_last, imaged st_imaged)
    int st_mode = 0, st_n = 0, st_last = -1, st_imaged = -1;

    cudaMemPool_t pool = nullptr;  // nullptr: the device's default pool
    // stream-ordered: creating and destroying simulators never synchronizes
    // the device
    cudaError_t raw_alloc(void** p, size_t bytes, cudaStream_t st)
    {
        return pool ? cudaMallocFromPoolAsync(p, bytes, pool, st) : cudaMallocAsync(p, bytes, st);
    }
    int alloc(void** p, size_t bytes)
    {
        *p = nullptr;
        if (bytes == 0) return TTI_OK;
        cudaError_t e = raw_alloc(p, bytes, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            return TTI_ENOMEM;
        }
        allocs.push_back(*p);
        return TTI_OK;
    }
    int64_t nvol() const { return (int64_t)L.ldimx * L.ldimy * L.ldimz; }
    dim3 dense_grid() const { return dim3((L.nx() + 127) / 128, L.ny(), L.nz()); }
    size_t slot_bytes() const
    {
        return (size_t)snap_fields(cfg) * ninterior * snap_elt_bytes(cfg.snap_precision);
    }
    void* slot_ptr(int k) const { return static_cast<unsigned char*>(snaps) + (size_t)k * slot_bytes(); }
};

namespace {

Layout layout_of(const tti_sim_config& c)
{
    Layout L{};
    L.ldimx = 32 * ((c.nx + 2 * kRadius - 1) / 32 + 1);
    L.ldimy = c.ny + 2 * kRadius;
    L.ldimz = c.nz + 2 * kRadius;
    L.ixbeg = L.iybeg = L.izbeg = kRadius;
    L.ixend = kRadius + c.nx - 1;
    L.iyend = kRadius + c.ny - 1;
    L.izend = kRadius + c.nz - 1;
    return L;
}

int validate(const tti_sim_config& c)
{
    if (c.nx < 1 || c.ny < 1 || c.nz < 1 || c.nt < 1 || c.xcorr_step < 1 || !(c.dx > 0) || !(c.dy > 0) ||
        !(c.dz > 0) || !(c.dt > 0) || c.sponge_width < 0 || (c.nz <= kRadius && c.free_surface))
        return TTI_EINVAL;
    if (c.snap_precision < 0 || c.snap_precision > 2) return TTI_EINVAL;
    if (c.scheme < 0 || c.scheme > 1) return TTI_EINVAL;
    if (c.wave_precision < 0 || c.wave_precision > 2 || (c.wave_precision && !c.fused)) return TTI_EINVAL;
    if (c.snap_precision != 0 && (!c.fused || c.nx % 8 != 0)) return TTI_EINVAL;
    if (c.checkpoint_every < 0) return TTI_EINVAL;
    if (c.checkpoint_every > 0 && (c.checkpoint_every % c.xcorr_step != 0 || !c.fused || !c.save_snapshots))
        return TTI_EINVAL;
    return TTI_OK;
}

// Device memory of a simulator, by the same plan tti_sim_create allocates.
struct Plan {
    size_t core = 0, aux = 0, snaps = 0, ckpts = 0, recompute = 0;
    bool need_aux = false;
    bool packed_model = false;  // interleaved model volumes for the fused staggered adjoint
    int nsnap = 0, nslot = 0, ncp = 0;
    size_t total() const { return core + aux + snaps + ckpts + recompute; }
};

Plan plan_of(const tti_sim_config& c)
{
    Plan pl;
    const Layout L = layout_of(c);
    const size_t vb = (size_t)L.ldimx * L.ldimy * L.ldimz * sizeof(float);
    const size_t nin = (size_t)c.nx * c.ny * c.nz;
    pl.core = 6 * vb + 8 * vb + 2 * nin * sizeof(float) + (size_t)c.nt * sizeof(float) +
              (size_t)(L.ldimx + L.ldimy + L.ldimz) * sizeof(float2) + sizeof(int);
    const size_t wave = c.wave_precision ? 2 * sizeof(float) + 2 * sizeof(unsigned) : 0;  // scales, maxima
    pl.core += wave;
    pl.packed_model = c.scheme == 0 && c.fused;
    if (pl.packed_model) pl.core += 8 * vb;  // two volumes of float4 cells
    // derivative volumes and scratch: only the staggered scheme's kernel sequence
    pl.need_aux = c.scheme == 0 && (!c.fused || (c.save_snapshots && !fused_image_supported(L)));
    if (pl.need_aux) pl.aux = 10 * vb + 4 * vb;  // rhs3, rhs4, snp, snq, six derivatives, 4-float scratch
    if (c.save_snapshots) {
        pl.nsnap = (c.nt - 1) / c.xcorr_step + 1;
        pl.nslot = pl.nsnap;
        if (c.checkpoint_every > 0) {
            pl.ncp = (c.nt - 1) / c.checkpoint_every + 1;
            pl.nslot = c.checkpoint_every / c.xcorr_step;
            pl.ckpts = (size_t)pl.ncp * 4 * nin * sizeof(float) + (size_t)pl.ncp * 4 * sizeof(unsigned int);
            pl.recompute = 6 * vb + wave;
        }
        pl.snaps = (size_t)pl.nslot * snap_fields(c) * nin * snap_elt_bytes(c.snap_precision) +
                   (size_t)pl.nslot * 4 * sizeof(float) +
                   4 * sizeof(unsigned int);
    }
    return pl;
}

int sim_zero(tti_sim* s, void* p, size_t bytes, cudaStream_t st = nullptr)
{
    if (cudaMemsetAsync(p, 0, bytes, st ? st : s->stream) != cudaSuccess) return cuda_rc(cudaGetLastError());
    return TTI_OK;
}

int zero_state(tti_sim* s, WaveState& w, cudaStream_t st = nullptr)
{
    const size_t vb = (size_t)s->nvol() * sizeof(float);
    int rc = TTI_OK;
    for (float* v : {w.p, w.q, w.pd, w.qd, w.p2, w.q2})
        if (!rc && v) rc = sim_zero(s, v, vb, st);
    if (!rc && w.wamax) rc = sim_zero(s, w.wamax, 2 * sizeof(unsigned), st);
    return rc;
}

// Reduced-precision wavefields: the size of the p, q the next step will
// write, estimated from the state it starts from (run just before the step,
// after any injection into pdot, qdot): max over the interior of
// |p| + dt*|pdot| (and the same for q), since the step writes about
// A*p + B*dt*pdot.  The output scales come from it, so a wavefield that
// starts from rest gets a scale from its first non-zero pdot instead of
// having its first small values flushed to zero.  With FP16, a stored p or q
// at the clamp of the scale it was stored with flags a saturation.
__global__ void k_wave_amax(const float* __restrict__ p, const float* __restrict__ q, const float* __restrict__ pd,
                            const float* __restrict__ qd, float dt, unsigned* amax,
                            const float* __restrict__ used_scale, int prec, int* err, Layout L)
{
    const int64_t n = (int64_t)L.nx() * L.ny() * L.nz();
    unsigned mp = 0u, mq = 0u;    // bits of max |p| + dt|pdot| (non-negative floats order like their bits)
    float sp = 0.0f, sq = 0.0f;   // max |p|, |q| as stored
    for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < n; d += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(d % L.nx()), iy = (int)((d / L.nx()) % L.ny()), iz = (int)(d / ((int64_t)L.nx() * L.ny()));
        const int64_t i = L.idx(ix + L.ixbeg, iy + L.iybeg, iz + L.izbeg);
        const float ap = fabsf(p[i]), aq = fabsf(q[i]);
        sp = fmaxf(sp, ap);
        sq = fmaxf(sq, aq);
        mp = max(mp, __float_as_uint(ap + dt * fabsf(pd[i])));
        mq = max(mq, __float_as_uint(aq + dt * fabsf(qd[i])));
    }
    mp = __reduce_max_sync(0xffffffffu, mp);
    mq = __reduce_max_sync(0xffffffffu, mq);
    sp = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(sp)));
    sq = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(sq)));
    if ((threadIdx.x & 31) == 0) {
        if (mp) atomicMax(amax, mp);
        if (mq) atomicMax(amax + 1, mq);
        if (prec == 1 && used_scale && (sp * used_scale[0] >= 65504.0f || sq * used_scale[1] >= 65504.0f))
            atomicOr(err, 2);
    }
}

// Sponge profile: damping factor G(k) = exp(-(0.3*(W-k)/W)^2) on the k-th cell
// from an absorbing face (k < W), 1 elsewhere; A = B = G.  The reference
// ships only all-ones profiles (simulator2SetUp.cu:334-356); its sponge
// arithmetic (min over axes, A*f + B*dt*rhs) is kept as is.
std::vector<float2> sponge_axis(int n, int ldim, int width, bool absorb_low)
{
    std::vector<float2> ab(ldim, make_float2(1.0f, 1.0f));
    for (int k = 0; k < width && k < n; ++k) {
        float g = std::exp(-std::pow(0.3 * (width - k) / (double)width, 2.0));
        if (absorb_low) ab[kRadius + k] = make_float2(g, g);
        ab[kRadius + n - 1 - k] = make_float2(fminf(g, ab[kRadius + n - 1 - k].x), fminf(g, ab[kRadius + n - 1 - k].y));
    }
    return ab;
}

Model model_of(tti_sim* s)
{
    return Model{s->mv[0], s->mv[1], s->mv[2], s->mv[3], s->mv[4], s->mv[5], s->mv[6], s->mv[7], s->mpack[0], s->mpack[1]};
}

// ---------------------------------------------------------------------------
// Optional per-launch timing of the step kernels (CUDA events on the
// simulator's stream): kind 0 = forward step, 1 = adjoint step, 2 = imaging.
cudaEvent_t next_event(tti_sim* s)
{
    if (s->ev_used == s->ev_pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        s->ev_pool.push_back(e);
    }
    return s->ev_pool[s->ev_used++];
}
void mark_begin(tti_sim* s, int kind, cudaStream_t st)
{
    if (!s->profiling || s->capturing) return;
    size_t k = s->ev_used;
    cudaEvent_t e = next_event(s);
    if (!e) return;
    cudaEventRecord(e, st);
    s->ev_marks.push_back({kind, k});
}
void mark_end(tti_sim* s, cudaStream_t st)
{
    if (!s->profiling || s->capturing || s->ev_marks.empty()) return;
    cudaEvent_t e = next_event(s);
    if (e) cudaEventRecord(e, st);
}
void collect_marks(tti_sim* s)
{
    for (auto& m : s->ev_marks) {
        if (m.second + 1 >= s->ev_used) continue;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, s->ev_pool[m.second], s->ev_pool[m.second + 1]) == cudaSuccess) {
            s->kind_ms[m.first] += ms;
            s->kind_n[m.first] += 1;
        }
    }
    cudaGetLastError();
    s->ev_marks.clear();
    s->ev_used = 0;
}

// ---------------------------------------------------------------------------
// Reference kernel sequence (fused = 0), on the main state in place.
int forward_per_kernel_step(tti_sim* s, int n, cudaStream_t st)
{
    const Layout& L = s->L;
    const tti_sim_config& c = s->cfg;
    WaveState& w = s->w;
    int rc = tti_launch_kernel_loop2(w.p, w.q, w.pd, w.qd, L.ldimx, L.ldimy, L.ixbeg, L.ixend, L.iybeg, L.iyend,
                                     L.izbeg, L.izend, (const float*)s->abx, (const float*)s->aby,
                                     (const float*)s->abz, c.dt, st);
    if (rc) return rc;
    s->launches++;
    if (c.free_surface) {
        if ((rc = tti_launch_kernel_loop4(w.p, w.q, L.ldimx, L.ldimy, L.izbeg, st))) return rc;
        s->launches++;
    }
    if (c.scheme == 1) {  // centred constant-density operator (kernels/kernel_type1_gpu_fwd.cu)
        if ((rc = tti_launch_type1_fwd(w.pd, w.qd, w.p, w.q, s->mv[1], s->mv[2], s->mv[3], s->mv[4], s->mv[5],
                                       s->mv[6], s->mv[7], (const float*)s->abx, (const float*)s->aby,
                                       (const float*)s->abz, L.ixbeg, L.ixend, L.iybeg, L.iyend, L.izbeg, L.izend,
                                       L.ldimx, L.ldimy, L.ldimz, L.ldimx, L.ldimy, L.ldimz, c.dt, c.dx, c.dy, c.dz,
                                       8, st, 0, s->sponge_active ? 1 : 0, 0)))
            return rc;
        s->launches++;
        if (s->src_index >= 0) {
            k_add_source<<<1, 1, 0, st>>>(w.pd, w.qd, s->src_index, s->wavelet[n] * c.dt);
            s->launches++;
        }
        return launch_status();
    }
    if ((rc = tti_launch_fwd_kernel2_drv(w.p, w.q, s->mv[0], s->d[0], s->d[1], s->d[2], s->d[3], s->d[4], s->d[5],
                                         L.ixbeg, L.ixend, L.iybeg, L.iyend, L.izbeg, L.izend, (float)(1.0 / c.dx),
                                         (float)(1.0 / c.dy), (float)(1.0 / c.dz), L.ldimx, L.ldimy, 8, st)))
        return rc;
    s->launches++;
    if (c.free_surface) {
        if ((rc = tti_launch_kernel_loop4_derivatives(s->d[0], s->d[1], s->d[2], s->d[3], s->d[4], s->d[5], L.ldimx,
                                                      L.ldimy, L.izbeg, st)))
            return rc;
        s->launches++;
    }
    // argument order of launch_update_rho_fwd_main_loop_2_1: dx, dx2, dy, dy2, dz, dz2
    if ((rc = tti_launch_update_rho_fwd_main_loop_2_1(
             w.pd, w.qd, s->d[0], s->d[3], s->d[1], s->d[4], s->d[2], s->d[5], w.p, w.q, s->mv[0], s->mv[1],
             s->mv[2], s->mv[3], s->mv[4], s->mv[5], s->mv[6], s->mv[7], nullptr, nullptr, nullptr, nullptr, nullptr,
             nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, L.ixbeg, L.ixend, L.iybeg, L.iyend,
             L.izbeg, L.izend, L.ldimx, L.ldimy, c.dt, c.dx, c.dy, c.dz, 0, 8, 0, 0, 0, st)))
        return rc;
    s->launches++;
    if (s->src_index >= 0) {
        k_add_source<<<1, 1, 0, st>>>(w.pd, w.qd, s->src_index, s->wavelet[n] * c.dt);
        s->launches++;
    }
    return launch_status();
}

int adjoint_per_kernel_step(tti_sim* s, cudaStream_t st)
{
    const Layout& L = s->L;
    const tti_sim_config& c = s->cfg;
    WaveState& w = s->w;
    if (c.scheme == 1) {  // kernels/kernel_type1_gpu_adj.cu, then loop2 and loop4
        int rc = tti_launch_type1_adj(w.pd, w.qd, w.p, w.q, s->mv[1], s->mv[2], s->mv[3], s->mv[4], s->mv[5],
                                      s->mv[6], s->mv[7], (const float*)s->abx, (const float*)s->aby,
                                      (const float*)s->abz, L.ixbeg, L.ixend, L.iybeg, L.iyend, L.izbeg, L.izend,
                                      L.ldimx, L.ldimy, L.ldimz, c.dt, c.dx, c.dy, c.dz, 8, st,
                                      s->sponge_active ? 1 : 0, 0);
        if (rc) return rc;
        s->launches += 2;
        if ((rc = tti_launch_kernel_loop2(w.p, w.q, w.pd, w.qd, L.ldimx, L.ldimy, L.ixbeg, L.ixend, L.iybeg,
                                          L.iyend, L.izbeg, L.izend, (const float*)s->abx, (const float*)s->aby,
                                          (const float*)s->abz, c.dt, st)))
            return rc;
        s->launches++;
        if (c.free_surface) {
            if ((rc = tti_launch_kernel_loop4(w.p, w.q, L.ldimx, L.ldimy, L.izbeg, st))) return rc;
            s->launches++;
        }
        return TTI_OK;
    }
    int rc = launch_base(w.p, w.q, s->mv[1], s->mv[2], s->mv[3], s->mv[4], s->base, L.ixbeg, L.ixend, L.iybeg, L.iyend,
                         L.izbeg, L.izend, L.ldimx, L.ldimy, st);
    if (rc) return rc;
    rc = launch_adj_drv_with_base(s->d[0], s->d[3], s->d[1], s->d[4], s->d[2], s->d[5], s->rhs3, s->rhs4, s->base,
                                  s->mv[0], s->mv[5], s->mv[6], s->mv[7], L.ixbeg, L.ixend, L.iybeg, L.iyend, L.izbeg,
                                  L.izend, L.ldimx, L.ldimy, (float)(1.0 / (4 * c.dx * c.dy)),
                                  (float)(1.0 / (4 * c.dy * c.dz)), (float)(1.0 / (4 * c.dx * c.dz)),
                                  (float)(1.0 / c.dx), (float)(1.0 / c.dy), (float)(1.0 / c.dz), st);
    if (rc) return rc;
    s->launches += 2;
    if (c.free_surface) {
        if ((rc = tti_launch_kernel_loop4_derivatives(s->d[0], s->d[1], s->d[2], s->d[3], s->d[4], s->d[5], L.ldimx,
                                                      L.ldimy, L.izbeg, st)))
            return rc;
        s->launches++;
    }
    if ((rc = tti_launch_update_adj_kernel_main_3(w.pd, w.qd, s->d[0], s->d[3], s->d[1], s->d[4], s->d[2], s->d[5],
                                                  s->rhs3, s->rhs4, (const float*)s->abx, (const float*)s->aby,
                                                  (const float*)s->abz, L.ixbeg, L.ixend, L.iybeg, L.iyend, L.izbeg,
                                                  L.izend, L.ldimx, L.ldimy, c.dt, c.dx, c.dy, c.dz, 0, 0, 0, 8,
                                                  s->sponge_active ? 1 : 0, st)))
        return rc;
    s->launches++;
    if ((rc = tti_launch_kernel_loop2(w.p, w.q, w.pd, w.qd, L.ldimx, L.ldimy, L.ixbeg, L.ixend, L.iybeg, L.iyend,
                                      L.izbeg, L.izend, (const float*)s->abx, (const float*)s->aby,
                                      (const float*)s->abz, c.dt, st)))
        return rc;
    s->launches++;
    if (c.free_surface) {
        if ((rc = tti_launch_kernel_loop4(w.p, w.q, L.ldimx, L.ldimy, L.izbeg, st))) return rc;
        s->launches++;
    }
    return TTI_OK;
}

// Imaging at a snapshot step with the reference kernels
// (simulator2SetUp.cu:753-781): Vp image, forward derivatives of the stored
// p/q, derivative mirror, density gradient with the current adjoint p/q.
int image_per_kernel(tti_sim* s, const float* slot, cudaStream_t st)
{
    const Layout& L = s->L;
    const tti_sim_config& c = s->cfg;
    WaveState& w = s->w;
    int64_t n = s->ninterior;
    if (c.scheme == 1) {  // kernels/kernel_type1_gpu_grad.cu: Vp image only
        int rc = tti_launch_type1_update_grad(slot, slot + n, s->grad_vp, w.pd, w.qd, L.ixbeg, L.ixend, L.iybeg,
                                              L.iyend, L.izbeg, L.izend, L.nx(), L.ny(), L.ldimx, L.ldimy, st);
        s->launches++;
        return rc;
    }
    int rc = tti_launch_update_Vp_gradient(slot, slot + n, s->grad_vp, w.pd, w.qd, L.ixbeg, L.ixend, L.iybeg, L.iyend,
                                           L.izbeg, L.izend, L.nx(), L.ny(), L.ldimx, L.ldimy, st);
    if (rc) return rc;
    k_interior_copy<false><<<s->dense_grid(), 128, 0, st>>>(s->snp, const_cast<float*>(slot + 2 * n), L);
    k_interior_copy<false><<<s->dense_grid(), 128, 0, st>>>(s->snq, const_cast<float*>(slot + 3 * n), L);
    s->launches += 3;
    if (c.free_surface) {
        if ((rc = tti_launch_kernel_loop4(s->snp, s->snq, L.ldimx, L.ldimy, L.izbeg, st))) return rc;
        s->launches++;
    }
    if ((rc = tti_launch_fwd_kernel2_drv(s->snp, s->snq, s->mv[0], s->d[0], s->d[1], s->d[2], s->d[3], s->d[4],
                                         s->d[5], L.ixbeg, L.ixend, L.iybeg, L.iyend, L.izbeg, L.izend,
                                         (float)(1.0 / c.dx), (float)(1.0 / c.dy), (float)(1.0 / c.dz), L.ldimx,
                                         L.ldimy, 8, st)))
        return rc;
    s->launches++;
    if (c.free_surface) {
        if ((rc = tti_launch_kernel_loop4_derivatives(s->d[0], s->d[1], s->d[2], s->d[3], s->d[4], s->d[5], L.ldimx,
                                                      L.ldimy, L.izbeg, st)))
            return rc;
        s->launches++;
    }
    if ((rc = launch_base(w.p, w.q, s->mv[1], s->mv[2], s->mv[3], s->mv[4], s->base, L.ixbeg, L.ixend, L.iybeg,
                          L.iyend, L.izbeg, L.izend, L.ldimx, L.ldimy, st)))
        return rc;
    if ((rc = launch_rho_gradient_with_base(s->grad_rho, s->d[0], s->d[3], s->d[1], s->d[4], s->d[2], s->d[5],
                                            s->base, s->mv[0], s->mv[5], s->mv[6], s->mv[7], L.ixbeg, L.ixend,
                                            L.iybeg, L.iyend, L.izbeg, L.izend, L.ldimx, L.ldimy, L.nx(), L.ny(), c.dx,
                                            c.dy, c.dz, st)))
        return rc;
    s->launches += 2;
    return launch_status();
}

// ---------------------------------------------------------------------------
// Fused path.
// p/q of step 0 (loop2 + free surface of the reference step; the fused
// kernel of step n ends with the p/q update of step n+1).
int fused_prologue(tti_sim* s, WaveState& w, cudaStream_t st)
{
    const Layout& L = s->L;
    const tti_sim_config& c = s->cfg;
    int rc = tti_launch_kernel_loop2(w.p, w.q, w.pd, w.qd, L.ldimx, L.ldimy, L.ixbeg, L.ixend, L.iybeg, L.iyend,
                                     L.izbeg, L.izend, (const float*)s->abx, (const float*)s->aby,
                                     (const float*)s->abz, c.dt, st);
    s->launches++;
    if (!rc && c.free_surface) {
        rc = tti_launch_kernel_loop4(w.p, w.q, L.ldimx, L.ldimy, L.izbeg, st);
        s->launches++;
    }
    return rc;
}

// One fused forward step n on state w; the snapshot (if any) goes to slot k.
// Reduced-precision wavefields: just before a step, the estimated size of
// its output from the state it starts from, then the output scales from it
// (the maxima are cleared again).  The scales are a function of the state
// alone, so a forward step recomputed from a checkpoint rounds exactly as
// the first time.
int wave_scale_step(tti_sim* s, WaveState& w, cudaStream_t st)
{
    if (!s->cfg.wave_precision) return TTI_OK;
    const int64_t n = s->ninterior;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 148LL * 8);
    k_wave_amax<<<blocks, 256, 0, st>>>(w.p, w.q, w.pd, w.qd, s->cfg.dt, w.wamax, w.wscale, s->cfg.wave_precision,
                                        s->err, s->L);
    k_snap_scale<<<1, 32, 0, st>>>(w.wscale, w.wamax, 2);
    s->launches += 2;
    return launch_status();
}

int fused_forward_step(tti_sim* s, WaveState& w, int n, int slot, cudaStream_t st, bool record = true)
{
    const tti_sim_config& c = s->cfg;
    int rc0 = TTI_OK;
    FwdStepArgs a{};
    a.pin = w.p;
    a.qin = w.q;
    a.pout = w.p2;
    a.qout = w.q2;
    a.f3 = w.pd;
    a.f4 = w.qd;
    a.m = model_of(s);
    a.abx = s->abx;
    a.aby = s->aby;
    a.abz = s->abz;
    a.src_index = s->src_index;
    a.src_term = s->src_index >= 0 ? s->wavelet[n] * c.dt : 0.0f;
    a.snap = slot >= 0 ? s->slot_ptr(slot) : nullptr;
    a.snap_prec = c.snap_precision;
    if (slot >= 0 && c.snap_precision != SNAP_F32) {
        float* sc = s->snap_scale + (size_t)slot * 4;
        k_snap_scale<<<1, 32, 0, st>>>(sc, s->snap_amax, 4);
        s->launches++;
        a.snap_scale = sc;
        a.snap_amax = s->snap_amax;
    }
    a.free_surface = c.free_surface;
    a.vti = s->vti ? 1 : 0;
    a.dt = c.dt;
    a.dx = c.dx;
    a.dy = c.dy;
    a.dz = c.dz;
    a.err = s->err;
    if (s->rec_fold && record && s->nrec) {  // receivers sampled inside the step
        a.trace = s->traces + (size_t)n * s->nrec;
        a.rec = s->recmap;
    }
    if ((rc0 = wave_scale_step(s, w, st))) return rc0;
    a.wave_prec = c.wave_precision;
    a.wave_scale = w.wscale;
    mark_begin(s, 0, st);
    int rc = c.scheme == 1 ? launch_t1_fused_forward(s->L, a, s->sponge_active ? 1 : 0, st)
                           : launch_fused_forward(s->L, a, st);
    mark_end(s, st);
    if (rc) return rc;
    s->launches++;
    w.swap();
    return TTI_OK;
}

int fused_adjoint_step(tti_sim* s, cudaStream_t st, const float* res = nullptr, const float* obs = nullptr,
                       float* srctr = nullptr)
{
    const tti_sim_config& c = s->cfg;
    WaveState& w = s->w;
    AdjStepArgs a{};
    a.pin = w.p;
    a.qin = w.q;
    a.pout = w.p2;
    a.qout = w.q2;
    a.f3 = w.pd;
    a.f4 = w.qd;
    a.m = model_of(s);
    a.abx = s->abx;
    a.aby = s->aby;
    a.abz = s->abz;
    a.sponge_active = s->sponge_active ? 1 : 0;
    a.free_surface = c.free_surface;
    a.vti = s->vti ? 1 : 0;
    a.dt = c.dt;
    a.dx = c.dx;
    a.dy = c.dy;
    a.dz = c.dz;
    a.err = s->err;
    a.res = res;
    a.obs = obs;
    if (res) a.rec = s->recmap;
    a.srctr = srctr;
    a.src_index = srctr ? s->src_index : -1;
    int rc = wave_scale_step(s, w, st);
    if (rc) return rc;
    a.wave_prec = c.wave_precision;
    a.wave_scale = w.wscale;
    mark_begin(s, 1, st);
    rc = c.scheme == 1 ? launch_t1_fused_adjoint(s->L, a, st) : launch_fused_adjoint(s->L, a, st);
    mark_end(s, st);
    if (rc) return rc;
    s->launches++;
    w.swap();
    return TTI_OK;
}

int image_step(tti_sim* s, int slot, cudaStream_t st)
{
    const tti_sim_config& c = s->cfg;
    int rc;
    mark_begin(s, 2, st);
    if (c.fused && c.scheme == 1) {
        ImageArgs ia{};
        ia.adj3 = s->w.pd;
        ia.adj4 = s->w.qd;
        ia.store = s->snaps;
        ia.snap_prec = c.snap_precision;
        ia.snap_scale = s->snap_scale + (size_t)slot * 4;
        ia.nsnap = s->nslot;
        ia.slot = slot;
        ia.grad_vp = s->grad_vp;
        rc = launch_t1_image(s->L, ia, st);
        s->launches++;
    } else if (c.fused && (c.snap_precision != SNAP_F32 || fused_image_supported(s->L))) {
        ImageArgs ia{};
        ia.adj1 = s->w.p;
        ia.adj2 = s->w.q;
        ia.adj3 = s->w.pd;
        ia.adj4 = s->w.qd;
        ia.store = s->snaps;
        ia.snap_prec = c.snap_precision;
        ia.snap_scale = s->snap_scale + (size_t)slot * 4;
        ia.nsnap = s->nslot;
        ia.slot = slot;
        ia.m = model_of(s);
        ia.grad_vp = s->grad_vp;
        ia.grad_rho = s->grad_rho;
        ia.free_surface = c.free_surface;
        ia.vti = s->vti ? 1 : 0;
        ia.dx = c.dx;
        ia.dy = c.dy;
        ia.dz = c.dz;
        ia.err = s->err;
        rc = launch_fused_image(s->L, ia, st);
        s->launches++;
    } else {
        rc = image_per_kernel(s, static_cast<const float*>(s->slot_ptr(slot)), st);
    }
    mark_end(s, st);
    return rc;
}

int receivers_step(tti_sim* s, WaveState& w, int n, cudaStream_t st)
{
    if (!s->nrec || s->rec_fold) return TTI_OK;  // folded: the fused step samples them
    k_receivers<<<(s->nrec + 255) / 256, 256, 0, st>>>(s->traces + (size_t)n * s->nrec, w.p, w.q, s->rec, s->nrec);
    s->launches++;
    return launch_status();
}

// Checkpoint k: the state at the start of step k*ckpt (interior p, q, pdot,
// qdot in FP32) and the running snapshot max of that moment.
int save_checkpoint(tti_sim* s, WaveState& w, int k, cudaStream_t st)
{
    float* slot = s->ckpts + (size_t)k * 4 * s->ninterior;
    k_snapshot_save<<<s->dense_grid(), 128, 0, st>>>(slot, w.p, w.q, w.pd, w.qd, s->L);
    s->launches++;
    if (cudaMemcpyAsync(s->ckpt_amax + 4 * k, s->snap_amax, 4 * sizeof(unsigned int), cudaMemcpyDeviceToDevice, st) !=
        cudaSuccess)
        return cuda_rc(cudaGetLastError());
    return launch_status();
}

int restore_checkpoint(tti_sim* s, WaveState& w, int k, cudaStream_t st)
{
    const int64_t n = s->ninterior;
    float* slot = s->ckpts + (size_t)k * 4 * n;
    int rc = zero_state(s, w, st);
    if (rc) return rc;
    k_interior_copy<false><<<s->dense_grid(), 128, 0, st>>>(w.p, slot, s->L);
    k_interior_copy<false><<<s->dense_grid(), 128, 0, st>>>(w.q, slot + n, s->L);
    k_interior_copy<false><<<s->dense_grid(), 128, 0, st>>>(w.pd, slot + 2 * n, s->L);
    k_interior_copy<false><<<s->dense_grid(), 128, 0, st>>>(w.qd, slot + 3 * n, s->L);
    s->launches += 4;
    if (s->cfg.free_surface) {  // the halo above the surface is the mirror of the interior
        if ((rc = tti_launch_kernel_loop4(w.p, w.q, s->L.ldimx, s->L.ldimy, s->L.izbeg, st))) return rc;
        s->launches++;
    }
    if (cudaMemcpyAsync(s->snap_amax, s->ckpt_amax + 4 * k, 4 * sizeof(unsigned int), cudaMemcpyDeviceToDevice, st) !=
        cudaSuccess)
        return cuda_rc(cudaGetLastError());
    return launch_status();
}

// One adjoint step n (reference order, simulator2SetUp.cu:654-782): source
// trace, residual injection, the step, and imaging at snapshot steps from
// store slot (n - seg_start) / xcorr_step.  observed: s->resid holds observed
// traces and the residual is formed from the last forward's traces.
int adjoint_unit(tti_sim* s, int n, int seg_start, bool observed, cudaStream_t st, bool with_image = true)
{
    const tti_sim_config& c = s->cfg;
    int r = TTI_OK;
    const float* obs = (s->nrec && observed) ? s->resid + (size_t)n * s->nrec : nullptr;
    const float* res = !s->nrec ? nullptr : observed ? s->traces + (size_t)n * s->nrec : s->resid + (size_t)n * s->nrec;
    if (s->rec_fold) {  // source trace and residual injection inside the fused step
        if ((r = fused_adjoint_step(s, st, res, obs, s->src_index >= 0 ? s->srctr + n : nullptr))) return r;
    } else {
        if (s->src_index >= 0) {
            k_source_trace<<<1, 1, 0, st>>>(s->srctr + n, s->w.p, s->w.q, s->src_index);
            s->launches++;
        }
        if (s->nrec) {
            k_inject_residual<<<(s->nrec + 255) / 256, 256, 0, st>>>(s->w.pd, s->w.qd, s->rec, res, obs, s->nrec);
            s->launches++;
        }
        if (!c.fused) {
            if ((r = adjoint_per_kernel_step(s, st))) return r;
        } else {
            if ((r = fused_adjoint_step(s, st))) return r;
        }
    }
    if (with_image && n % c.xcorr_step == 0 && (r = image_step(s, (n - seg_start) / c.xcorr_step, st))) return r;
    return launch_status();
}

// Run `body` either directly on the simulator's stream or captured into a
// CUDA graph that is then launched once.  The instantiated graph of each kind
// is kept and updated in place when the next capture has the same topology.
template <typename F>
int run_on_stream(tti_sim* s, int kind, F body)
{
    cudaStream_t st = s->stream;
    if (!s->cfg.use_graphs) return body(st);
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return cuda_rc(cudaGetLastError());
    s->capturing = true;
    int rc = body(st);
    s->capturing = false;
    cudaError_t e = cudaStreamEndCapture(st, &g);
    if (!rc && e != cudaSuccess) rc = cuda_rc(e);
    cudaGraphExec_t& ge = s->gexec[kind];
    if (!rc && ge) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(ge, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(ge);
            ge = nullptr;
        }
    }
    if (!rc && !ge && cudaGraphInstantiate(&ge, g, 0) != cudaSuccess) {
        rc = cuda_rc(cudaGetLastError());
        ge = nullptr;
    }
    if (!rc && cudaGraphLaunch(ge, st) != cudaSuccess) rc = cuda_rc(cudaGetLastError());
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return rc;
}

} // namespace

extern "C" {

int tti_sim_footprint_bytes(const tti_sim_config* cfg, int64_t* bytes)
{
    if (!cfg || !bytes) return TTI_EINVAL;
    int rc = validate(*cfg);
    if (rc) return rc;
    *bytes = (int64_t)plan_of(*cfg).total();
    return TTI_OK;
}

int tti_sim_create(const tti_sim_config* cfg, tti_sim** out) { return tti::sim_create_in_pool(cfg, nullptr, out); }

} // extern "C"

int tti::sim_create_in_pool(const tti_sim_config* cfg, cudaMemPool_t pool, tti_sim** out)
{
    if (!cfg || !out) return TTI_EINVAL;
    *out = nullptr;
    const tti_sim_config& c = *cfg;
    int rc = validate(c);
    if (rc) return rc;
    if (c.use_graphs && c.fused) {
        // first launches set kernel attributes and allocate the error word:
        // do that before any capture
        if ((rc = prepare_fused_kernels())) return rc;
    }
    tti_sim* s = new (std::nothrow) tti_sim();
    if (!s) return TTI_ENOMEM;
    s->cfg = c;
    s->L = layout_of(c);
    const Layout& L = s->L;
    s->ninterior = (int64_t)c.nx * c.ny * c.nz;
    const Plan pl = plan_of(c);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return TTI_ELAUNCH;
    }
    s->pool = pool;
    const size_t vb = (size_t)s->nvol() * sizeof(float);
    for (float** v : {&s->w.p, &s->w.q, &s->w.pd, &s->w.qd, &s->w.p2, &s->w.q2})
        if (!rc) rc = s->alloc((void**)v, vb);
    for (int k = 0; k < 8 && !rc; ++k) rc = s->alloc((void**)&s->mv[k], vb);
    if (pl.packed_model)
        for (int k = 0; k < 2 && !rc; ++k) rc = s->alloc((void**)&s->mpack[k], 4 * vb);
    if (!rc && c.wave_precision) {
        rc = s->alloc((void**)&s->w.wscale, 2 * sizeof(float));
        if (!rc) rc = s->alloc((void**)&s->w.wamax, 2 * sizeof(unsigned));
    }
    if (!rc && pl.need_aux) {
        s->aux = true;
        for (float** v : {&s->rhs3, &s->rhs4, &s->snp, &s->snq, &s->d[0], &s->d[1], &s->d[2], &s->d[3], &s->d[4],
                          &s->d[5]})
            if (!rc) rc = s->alloc((void**)v, vb);
        if (!rc) rc = s->alloc((void**)&s->base, (size_t)s->nvol() * sizeof(float4));
    }
    if (!rc) rc = s->alloc((void**)&s->err, sizeof(int));
    if (!rc) rc = sim_zero(s, s->err, sizeof(int));
    if (!rc) rc = s->alloc((void**)&s->grad_vp, s->ninterior * sizeof(float));
    if (!rc) rc = s->alloc((void**)&s->grad_rho, s->ninterior * sizeof(float));
    if (!rc) rc = s->alloc((void**)&s->srctr, (size_t)c.nt * sizeof(float));
    if (!rc) rc = s->alloc((void**)&s->abx, L.ldimx * sizeof(float2));
    if (!rc) rc = s->alloc((void**)&s->aby, L.ldimy * sizeof(float2));
    if (!rc) rc = s->alloc((void**)&s->abz, L.ldimz * sizeof(float2));
    if (!rc && c.save_snapshots) {
        s->nsnap = pl.nsnap;
        s->nslot = pl.nslot;
        rc = s->alloc(&s->snaps, (size_t)s->nslot * s->slot_bytes());
        if (!rc) rc = s->alloc((void**)&s->snap_scale, (size_t)s->nslot * 4 * sizeof(float));
        if (!rc) rc = s->alloc((void**)&s->snap_amax, 4 * sizeof(unsigned int));
        if (!rc && c.checkpoint_every > 0) {
            s->ckpt = c.checkpoint_every;
            s->ncp = pl.ncp;
            rc = s->alloc((void**)&s->ckpts, (size_t)s->ncp * 4 * s->ninterior * sizeof(float));
            if (!rc) rc = s->alloc((void**)&s->ckpt_amax, (size_t)s->ncp * 4 * sizeof(unsigned int));
            for (float** v : {&s->rw.p, &s->rw.q, &s->rw.pd, &s->rw.qd, &s->rw.p2, &s->rw.q2})
                if (!rc) rc = s->alloc((void**)v, vb);
            if (!rc && c.wave_precision) {
                rc = s->alloc((void**)&s->rw.wscale, 2 * sizeof(float));
                if (!rc) rc = s->alloc((void**)&s->rw.wamax, 2 * sizeof(unsigned));
            }
        }
    }
    if (!rc) rc = zero_state(s, s->w);
    if (!rc && s->ckpt) rc = zero_state(s, s->rw);
    if (!rc && s->aux)
        for (float* v : {s->rhs3, s->rhs4, s->snp, s->snq, s->d[0], s->d[1], s->d[2], s->d[3], s->d[4], s->d[5]})
            rc = rc ? rc : sim_zero(s, v, vb);
    if (!rc) rc = sim_zero(s, s->grad_vp, s->ninterior * sizeof(float));
    if (!rc) rc = sim_zero(s, s->grad_rho, s->ninterior * sizeof(float));
    if (!rc && s->snap_amax) rc = sim_zero(s, s->snap_amax, 4 * sizeof(unsigned int));
    if (!rc) {
        auto ax = sponge_axis(c.nx, L.ldimx, c.sponge_width, true);
        auto ay = sponge_axis(c.ny, L.ldimy, c.sponge_width, true);
        auto az = sponge_axis(c.nz, L.ldimz, c.sponge_width, !c.free_surface);
        s->sponge_active = c.sponge_width > 0;
        if (cudaMemcpy(s->abx, ax.data(), ax.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->aby, ay.data(), ay.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(s->abz, az.data(), az.size() * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = cuda_rc(cudaGetLastError());
    }
    if (!rc) rc = cuda_rc(cudaStreamSynchronize(s->stream));
    if (rc) {
        tti_sim_destroy(s);
        return rc;
    }
    *out = s;
    return TTI_OK;
}

extern "C" {

int tti_sim_destroy(tti_sim* s)
{
    if (!s) return TTI_EINVAL;
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    for (cudaGraphExec_t g : s->gexec)
        if (g) cudaGraphExecDestroy(g);
    for (void* p : s->allocs)
        if (p) cudaFreeAsync(p, s->stream);
    if (s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    cudaGetLastError();
    delete s;
    return TTI_OK;
}

int tti_sim_set_model(tti_sim* s, const float* vp, const float* eps, const float* delta, const float* vs,
                      const float* theta, const float* phi, const float* rho)
{
    if (!s || !vp) return TTI_EINVAL;
    const int64_t n = s->ninterior;
    const Layout& L = s->L;
    cudaStream_t st = s->stream;
    // The given host parameter arrays go to one dense device buffer (plus a
    // flag word), one kernel builds every model volume from it, and the
    // stream is synchronized once, to read the flag and release the buffer.
    const float* src[7] = {vp, eps, delta, vs, theta, phi, rho};
    int present = 0;
    for (const float* p : src) present += p ? 1 : 0;
    const size_t bytes = (size_t)present * n * sizeof(float) + 256;
    unsigned char* buf = nullptr;
    if (s->raw_alloc((void**)&buf, bytes, st) != cudaSuccess) {
        cudaGetLastError();
        return TTI_ENOMEM;
    }
    int* flag = reinterpret_cast<int*>(buf);
    float* dense = reinterpret_cast<float*>(buf + 256);
    ModelIn in{};
    ModelOut out{};
    for (int k = 0; k < 8; ++k) out.v[k] = s->mv[k];
    out.pack[0] = s->mpack[0];
    out.pack[1] = s->mpack[1];
    int rc = cuda_rc(cudaMemsetAsync(flag, 0, sizeof(int), st));
    for (int k = 0, j = 0; k < 7 && !rc; ++k) {
        if (!src[k]) continue;
        float* dst = dense + (size_t)j++ * n;
        rc = cuda_rc(cudaMemcpyAsync(dst, src[k], n * sizeof(float), cudaMemcpyHostToDevice, st));
        in.p[k] = dst;
    }
    if (!rc) {
        k_model_setup<<<dim3((L.ldimx + 127) / 128, L.ldimy, L.ldimz), 128, 0, st>>>(out, in, L, flag);
        rc = launch_status();
    }
    int tti_flag = 0;
    if (!rc) rc = cuda_rc(cudaMemcpyAsync(&tti_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    cudaFreeAsync(buf, st);
    const int rs = cuda_rc(cudaStreamSynchronize(st));
    if (!rc) rc = rs;
    if (rc) return rc;
    s->vti = (tti_flag == 0);
    s->model_set = true;
    return TTI_OK;
}

int tti_sim_set_source(tti_sim* s, int ix, int iy, int iz, const float* w, int nt)
{
    if (!s || !w || nt < s->cfg.nt) return TTI_EINVAL;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= s->cfg.nx || iy >= s->cfg.ny || iz >= s->cfg.nz) return TTI_EINVAL;
    s->src_index = s->L.idx(ix + kRadius, iy + kRadius, iz + kRadius);
    s->wavelet.assign(w, w + s->cfg.nt);
    return TTI_OK;
}

int tti_sim_set_receivers(tti_sim* s, int nrec, const int* ixyz)
{
    if (!s || nrec < 0 || (nrec > 0 && !ixyz)) return TTI_EINVAL;
    std::vector<int64_t> idx(nrec);
    for (int r = 0; r < nrec; ++r) {
        int ix = ixyz[3 * r], iy = ixyz[3 * r + 1], iz = ixyz[3 * r + 2];
        if (ix < 0 || iy < 0 || iz < 0 || ix >= s->cfg.nx || iy >= s->cfg.ny || iz >= s->cfg.nz) return TTI_EINVAL;
        idx[r] = s->L.idx(ix + kRadius, iy + kRadius, iz + kRadius);
    }
    std::vector<int64_t> sorted(idx);
    std::sort(sorted.begin(), sorted.end());
    for (int r = 1; r < nrec; ++r)
        if (sorted[r] == sorted[r - 1]) return TTI_EINVAL;
    for (void** p : {(void**)&s->rec, (void**)&s->traces, (void**)&s->resid}) {
        if (*p) {
            cudaFreeAsync(*p, s->stream);
            for (auto& a : s->allocs)
                if (a == *p) a = nullptr;
            *p = nullptr;
        }
    }
    for (void** p : {(void**)&s->rec_xy}) {
        if (*p) {
            cudaFreeAsync(*p, s->stream);
            for (auto& a : s->allocs)
                if (a == *p) a = nullptr;
            *p = nullptr;
        }
    }
    s->rec_fold = false;
    s->recmap = RecMap{};
    s->nrec = nrec;
    if (nrec == 0) return TTI_OK;
    int rc = s->alloc((void**)&s->rec, nrec * sizeof(int64_t));
    // The fused staggered step kernels sample the receivers and inject the
    // residual themselves when the receivers lie on a few planes (a table of
    // nx*ny receiver numbers per plane); otherwise separate kernels do it.
    const tti_sim_config& c = s->cfg;
    std::vector<int> plane_of(c.nz, -1);
    int nplanes = 0;
    for (int r = 0; r < nrec; ++r) {
        int& pl = plane_of[ixyz[3 * r + 2]];
        if (pl < 0) pl = nplanes++;
    }
    if (!rc && c.fused && c.scheme == 0 && nplanes <= kRecPlanesFolded) {
        const size_t plane = (size_t)c.nx * c.ny;
        std::vector<int> xy(nplanes * plane, -1);
        RecMap m{};
        m.nz = nplanes;
        m.zlo = 1 << 30;
        m.zhi = -1;
        for (int iz = 0; iz < c.nz; ++iz)
            if (plane_of[iz] >= 0) {
                m.z[plane_of[iz]] = iz + kRadius;
                m.off[plane_of[iz]] = (int)(plane_of[iz] * plane);
                m.zlo = std::min(m.zlo, iz + kRadius);
                m.zhi = std::max(m.zhi, iz + kRadius);
            }
        for (int r = 0; r < nrec; ++r)
            xy[plane_of[ixyz[3 * r + 2]] * plane + (size_t)ixyz[3 * r + 1] * c.nx + ixyz[3 * r]] = r;
        rc = s->alloc((void**)&s->rec_xy, xy.size() * sizeof(int));
        if (!rc && cudaMemcpy(s->rec_xy, xy.data(), xy.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = cuda_rc(cudaGetLastError());
        m.xy = s->rec_xy;
        s->recmap = m;
        s->rec_fold = !rc;
    }
    if (!rc) rc = s->alloc((void**)&s->traces, (size_t)nrec * s->cfg.nt * sizeof(float));
    if (!rc) rc = s->alloc((void**)&s->resid, (size_t)nrec * s->cfg.nt * sizeof(float));
    if (!rc && cudaMemcpy(s->rec, idx.data(), nrec * sizeof(int64_t), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = cuda_rc(cudaGetLastError());
    return rc;
}

int tti_sim_forward(tti_sim* s, float* traces, int traces_on_device)
{
    if (!s) return TTI_EINVAL;
    if (!s->model_set) return TTI_ESTATE;
    const tti_sim_config& c = s->cfg;
    s->launches = 0;
    s->forward_done = false;
    s->st_mode = 0;
    int rc = zero_state(s, s->w);
    if (!rc && s->snap_amax) rc = sim_zero(s, s->snap_amax, 4 * sizeof(unsigned int));
    if (rc) return rc;
    const bool fused = c.fused != 0;
    // With checkpoints the store holds one segment: every snapshot step still
    // writes its slot (the running max behind the FP16/BF16 scales then
    // evolves exactly as without checkpoints), and the last segment's
    // snapshots are the ones left for the adjoint.
    rc = run_on_stream(s, 0, [&](cudaStream_t st) -> int {
        int r = TTI_OK;
        if (fused && (r = fused_prologue(s, s->w, st))) return r;
        for (int n = 0; n < c.nt; ++n) {
            if (s->ckpt && n % s->ckpt == 0 && (r = save_checkpoint(s, s->w, n / s->ckpt, st))) return r;
            int slot = -1;
            if (c.save_snapshots && n % c.xcorr_step == 0)
                slot = s->ckpt ? (n % s->ckpt) / c.xcorr_step : n / c.xcorr_step;
            if (!fused) {
                if ((r = forward_per_kernel_step(s, n, st))) return r;
                if (slot >= 0) {
                    const bool two = snap_fields(c) == 2;
                    k_snapshot_save<<<s->dense_grid(), 128, 0, st>>>(static_cast<float*>(s->slot_ptr(slot)), s->w.pd,
                                                                     s->w.qd, two ? nullptr : s->w.p,
                                                                     two ? nullptr : s->w.q, s->L);
                    s->launches++;
                }
                if ((r = receivers_step(s, s->w, n, st))) return r;
            } else {
                if ((r = receivers_step(s, s->w, n, st))) return r;
                if ((r = fused_forward_step(s, s->w, n, slot, st))) return r;
            }
            if ((r = launch_status())) return r;
        }
        return TTI_OK;
    });
    if (!rc && traces && s->nrec) {
        size_t bytes = (size_t)s->nrec * c.nt * sizeof(float);
        cudaError_t e = cudaMemcpyAsync(traces, s->traces, bytes,
                                        traces_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s->stream);
        if (e != cudaSuccess) rc = cuda_rc(e);
    }
    if (rc) {
        cudaStreamSynchronize(s->stream);
        return rc;
    }
    rc = cuda_rc(cudaStreamSynchronize(s->stream));
    if (!rc && fused) rc = fused_wait_status(s->stream, s->err);
    collect_marks(s);
    if (!rc) s->forward_done = true;
    return rc;
}

static int sim_adjoint(tti_sim* s, const float* residual, int residual_on_device, bool observed);

int tti_sim_adjoint(tti_sim* s, const float* residual, int residual_on_device)
{
    return sim_adjoint(s, residual, residual_on_device, false);
}

int tti_sim_adjoint_observed(tti_sim* s, const float* observed, int observed_on_device)
{
    if (!s || !observed) return TTI_EINVAL;
    return sim_adjoint(s, observed, observed_on_device, true);
}

static int sim_adjoint(tti_sim* s, const float* residual, int residual_on_device, bool observed)
{
    if (!s) return TTI_EINVAL;
    if (!s->model_set || !s->forward_done || !s->cfg.save_snapshots) return TTI_ESTATE;
    const tti_sim_config& c = s->cfg;
    cudaStream_t st0 = s->stream;
    s->launches = 0;
    s->st_mode = 0;
    int rc = zero_state(s, s->w);
    if (!rc) rc = sim_zero(s, s->grad_vp, s->ninterior * sizeof(float));
    if (!rc) rc = sim_zero(s, s->grad_rho, s->ninterior * sizeof(float));
    if (rc) return rc;
    if (s->nrec && residual) {
        size_t bytes = (size_t)s->nrec * c.nt * sizeof(float);
        cudaError_t e = cudaMemcpyAsync(s->resid, residual, bytes,
                                        residual_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st0);
        if (e != cudaSuccess) return cuda_rc(e);
    } else if (s->nrec) {
        if ((rc = sim_zero(s, s->resid, (size_t)s->nrec * c.nt * sizeof(float)))) return rc;
    }
    const bool fused = c.fused != 0;
    auto adjoint_steps = [&](int hi, int lo, int seg_start, cudaStream_t st) -> int {
        for (int n = hi; n >= lo; --n) {
            int r = adjoint_unit(s, n, seg_start, observed, st);
            if (r) return r;
        }
        return TTI_OK;
    };
    if (!s->ckpt) {
        rc = run_on_stream(s, 1, [&](cudaStream_t st) { return adjoint_steps(c.nt - 1, 0, 0, st); });
    } else {
        // segments from the last to the first; the last one's snapshots are
        // still in the store from the forward pass
        const int nseg = (c.nt - 1) / s->ckpt + 1;
        for (int k = nseg - 1; k >= 0 && !rc; --k) {
            const int a = k * s->ckpt, b = std::min(c.nt, a + s->ckpt);
            rc = run_on_stream(s, k == nseg - 1 ? 1 : 2, [&](cudaStream_t st) -> int {
                int r = TTI_OK;
                if (k != nseg - 1) {
                    if ((r = restore_checkpoint(s, s->rw, k, st))) return r;
                    for (int n = a; n < b; ++n) {
                        const int slot = (n % c.xcorr_step == 0) ? (n - a) / c.xcorr_step : -1;
                        if ((r = fused_forward_step(s, s->rw, n, slot, st, false))) return r;
                    }
                }
                return adjoint_steps(b - 1, a, a, st);
            });
        }
    }
    if (rc) {
        cudaStreamSynchronize(st0);
        return rc;
    }
    k_finalize_dense<<<s->dense_grid(), 128, 0, st0>>>(s->grad_vp, s->mv[3], s->L, c.dt * c.xcorr_step);
    s->launches++;
    rc = cuda_rc(cudaStreamSynchronize(st0));
    if (!rc && fused) rc = fused_wait_status(st0, s->err);
    collect_marks(s);
    return rc;
}

// ---------------------------------------------------------------------------
// Step-level calls (the loop body of simulator2SetUp::execute,
// simulator2SetUp.cu:517-814, one time step per call).
int tti_sim_forward_begin(tti_sim* s)
{
    if (!s) return TTI_EINVAL;
    if (!s->model_set) return TTI_ESTATE;
    if (s->cfg.checkpoint_every > 0 || s->cfg.use_graphs) return TTI_EINVAL;
    s->launches = 0;
    s->forward_done = false;
    s->st_mode = 0;
    int rc = zero_state(s, s->w);
    if (!rc && s->snap_amax) rc = sim_zero(s, s->snap_amax, 4 * sizeof(unsigned int));
    if (!rc && s->cfg.fused) rc = fused_prologue(s, s->w, s->stream);
    if (rc) return rc;
    s->st_mode = 1;
    s->st_n = 0;
    return TTI_OK;
}

int tti_sim_forward_step(tti_sim* s, int n)
{
    if (!s) return TTI_EINVAL;
    if (s->st_mode != 1 || n != s->st_n) return TTI_ESTATE;
    const tti_sim_config& c = s->cfg;
    cudaStream_t st = s->stream;
    const int slot = (c.save_snapshots && n % c.xcorr_step == 0) ? n / c.xcorr_step : -1;
    int r = TTI_OK;
    if (!c.fused) {
        if ((r = forward_per_kernel_step(s, n, st))) return r;
        if (slot >= 0) {
            const bool two = snap_fields(c) == 2;
            k_snapshot_save<<<s->dense_grid(), 128, 0, st>>>(static_cast<float*>(s->slot_ptr(slot)), s->w.pd,
                                                             s->w.qd, two ? nullptr : s->w.p, two ? nullptr : s->w.q,
                                                             s->L);
            s->launches++;
        }
        if ((r = receivers_step(s, s->w, n, st))) return r;
    } else {
        if ((r = receivers_step(s, s->w, n, st))) return r;
        if ((r = fused_forward_step(s, s->w, n, slot, st))) return r;
    }
    if ((r = launch_status())) return r;
    if (++s->st_n == c.nt) {
        s->st_mode = 0;
        s->forward_done = true;
    }
    return TTI_OK;
}

int tti_sim_get_traces(tti_sim* s, float* traces, int on_device)
{
    if (!s || !traces) return TTI_EINVAL;
    if (!s->nrec) return TTI_OK;
    const size_t bytes = (size_t)s->nrec * s->cfg.nt * sizeof(float);
    cudaError_t e = cudaMemcpyAsync(traces, s->traces, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    s->stream);
    if (e != cudaSuccess) return cuda_rc(e);
    return cuda_rc(cudaStreamSynchronize(s->stream));
}

int tti_sim_adjoint_begin(tti_sim* s, const float* residual, int residual_on_device)
{
    if (!s) return TTI_EINVAL;
    if (!s->model_set || !s->forward_done || !s->cfg.save_snapshots) return TTI_ESTATE;
    if (s->cfg.checkpoint_every > 0 || s->cfg.use_graphs) return TTI_EINVAL;
    const tti_sim_config& c = s->cfg;
    s->launches = 0;
    s->st_mode = 0;
    int rc = zero_state(s, s->w);
    if (!rc) rc = sim_zero(s, s->grad_vp, s->ninterior * sizeof(float));
    if (!rc) rc = sim_zero(s, s->grad_rho, s->ninterior * sizeof(float));
    if (!rc && s->nrec) {
        if (residual) {
            const size_t bytes = (size_t)s->nrec * c.nt * sizeof(float);
            cudaError_t e = cudaMemcpyAsync(s->resid, residual, bytes,
                                            residual_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                            s->stream);
            if (e != cudaSuccess) rc = cuda_rc(e);
        } else {
            rc = sim_zero(s, s->resid, (size_t)s->nrec * c.nt * sizeof(float));
        }
    }
    if (rc) return rc;
    s->st_mode = 2;
    s->st_n = c.nt - 1;
    s->st_last = -1;
    s->st_imaged = -1;
    return TTI_OK;
}

int tti_sim_adjoint_step(tti_sim* s, int n)
{
    if (!s) return TTI_EINVAL;
    if (s->st_mode != 2 || n != s->st_n) return TTI_ESTATE;
    const int r = adjoint_unit(s, n, 0, false, s->stream, false);
    if (r) return r;
    s->st_last = n;
    s->st_n = n - 1;
    return TTI_OK;
}

int tti_sim_image_step(tti_sim* s, int n)
{
    if (!s) return TTI_EINVAL;
    if (s->st_mode != 2 || n != s->st_last || s->st_imaged == n) return TTI_ESTATE;
    if (n % s->cfg.xcorr_step != 0) return TTI_EINVAL;
    const int r = image_step(s, n / s->cfg.xcorr_step, s->stream);
    if (r) return r;
    s->st_imaged = n;
    return launch_status();
}

int tti_sim_adjoint_finish(tti_sim* s)
{
    if (!s) return TTI_EINVAL;
    if (s->st_mode != 2 || s->st_n != -1) return TTI_ESTATE;
    cudaStream_t st = s->stream;
    k_finalize_dense<<<s->dense_grid(), 128, 0, st>>>(s->grad_vp, s->mv[3], s->L, s->cfg.dt * s->cfg.xcorr_step);
    s->launches++;
    s->st_mode = 0;
    int rc = cuda_rc(cudaStreamSynchronize(st));
    if (!rc && s->cfg.fused) rc = fused_wait_status(st, s->err);
    collect_marks(s);
    return rc;
}

int tti_sim_sync(tti_sim* s)
{
    if (!s) return TTI_EINVAL;
    int rc = cuda_rc(cudaStreamSynchronize(s->stream));
    if (!rc && s->cfg.fused) rc = fused_wait_status(s->stream, s->err);
    return rc;
}

// ---------------------------------------------------------------------------
// Run-level call: one whole shot from host arrays.
int tti_rtm_shot(const tti_shot_request* r, const tti_sim_config* opts)
{
    if (!r) return TTI_EINVAL;
    tti_sim_config c{};
    c.nx = r->nx;
    c.ny = r->ny;
    c.nz = r->nz;
    c.dx = r->dx;
    c.dy = r->dy;
    c.dz = r->dz;
    c.dt = r->dt;
    c.nt = r->nt;
    c.xcorr_step = r->xcorr_step;
    c.sponge_width = r->sponge_width;
    c.free_surface = r->free_surface;
    c.fused = opts ? opts->fused : 1;
    c.save_snapshots = 1;
    c.snap_precision = opts ? opts->snap_precision : 0;
    c.checkpoint_every = opts ? opts->checkpoint_every : 0;
    c.use_graphs = opts ? opts->use_graphs : 0;
    c.scheme = opts ? opts->scheme : 0;
    c.wave_precision = opts ? opts->wave_precision : 0;
    tti_sim* s = nullptr;
    int rc = tti_sim_create(&c, &s);
    if (!rc) rc = tti_sim_set_model(s, r->vp, r->eps, r->delta, r->vs, r->theta, r->phi, r->rho);
    if (!rc) rc = tti_sim_set_source(s, r->src_ix, r->src_iy, r->src_iz, r->wavelet, r->nt);
    if (!rc) rc = tti_sim_set_receivers(s, r->nrec, r->rec_ixyz);
    if (!rc) rc = tti_sim_forward(s, r->traces, 0);
    if (!rc) {
        if (r->observed)
            rc = tti_sim_adjoint_observed(s, r->observed, 0);
        else  // residual = the synthetic traces themselves
            rc = tti_sim_adjoint(s, s->nrec ? s->traces : nullptr, 1);
    }
    if (!rc && (r->image_vp || r->image_rho)) rc = tti_sim_get_image(s, r->image_vp, r->image_rho, 0);
    if (s) {
        const int rd = tti_sim_destroy(s);
        if (!rc) rc = rd;
    }
    return rc;
}

} // extern "C"

// ---------------------------------------------------------------------------
// A whole shot (forward with receivers, adjoint driven by observed traces,
// imaging, finalisation) as a sequence of work units that can be enqueued a
// few at a time on any stream, or captured.  A unit is one fused step:
// forward, recomputed forward (checkpointed stores) or adjoint (with its
// imaging).  Same kernels and order as tti_sim_forward followed by
// tti_sim_adjoint_observed.
namespace tti {

int shot_upload_observed(tti_sim* s, const float* host_obs)
{
    if (!s) return TTI_EINVAL;
    if (!s->nrec) return TTI_OK;
    const size_t bytes = (size_t)s->nrec * s->cfg.nt * sizeof(float);
    if (!host_obs) return sim_zero(s, s->resid, bytes);
    if (cudaMemcpyAsync(s->resid, host_obs, bytes, cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
        return cuda_rc(cudaGetLastError());
    return TTI_OK;
}

int shot_begin(tti_sim* s)
{
    if (!s) return TTI_EINVAL;
    if (!s->cfg.fused || !s->cfg.save_snapshots) return TTI_EINVAL;
    if (!s->model_set) return TTI_ESTATE;
    s->launches = 0;
    s->forward_done = false;
    int rc = zero_state(s, s->w);
    if (!rc && s->snap_amax) rc = sim_zero(s, s->snap_amax, 4 * sizeof(unsigned int));
    if (rc) return rc;
    s->sh_phase = 1;
    s->sh_n = 0;
    s->sh_seg = 0;
    s->sh_recomp = false;
    return TTI_OK;
}

int64_t shot_units_left(const tti_sim* s)
{
    if (!s || s->sh_phase == 0 || s->sh_phase == 3) return 0;
    const int nt = s->cfg.nt, K = s->ckpt ? s->ckpt : nt;
    const int last_a = ((nt - 1) / K) * K;  // start of the last segment
    if (s->sh_phase == 1) return (int64_t)(nt - s->sh_n) + nt + last_a;
    // adjoint: the rest of this segment, then the earlier segments in full
    const int a = s->sh_seg * K;
    int64_t left = s->sh_recomp ? (int64_t)(std::min(nt, a + K) - s->sh_n) + std::min(nt, a + K) - a
                                : (int64_t)(s->sh_n - a + 1);
    left += 2LL * a;  // segments 0 .. sh_seg-1: recompute + adjoint
    return left;
}

bool shot_done(const tti_sim* s) { return s && s->sh_phase == 3; }

cudaStream_t shot_stream(const tti_sim* s) { return s ? s->stream : nullptr; }

// Enqueue up to max_units units on st.
int shot_advance(tti_sim* s, cudaStream_t st, int64_t max_units, int64_t* done)
{
    if (!s || !done) return TTI_EINVAL;
    *done = 0;
    const tti_sim_config& c = s->cfg;
    const int nt = c.nt, K = s->ckpt ? s->ckpt : nt;
    const int nseg = (nt - 1) / K + 1;
    int rc = TTI_OK;
    while (*done < max_units && (s->sh_phase == 1 || s->sh_phase == 2)) {
        if (s->sh_phase == 1) {
            const int n = s->sh_n;
            if (n == 0 && (rc = fused_prologue(s, s->w, st))) return rc;
            if (s->ckpt && n % s->ckpt == 0 && (rc = save_checkpoint(s, s->w, n / s->ckpt, st))) return rc;
            const int slot = (n % c.xcorr_step == 0) ? (s->ckpt ? (n % s->ckpt) / c.xcorr_step : n / c.xcorr_step) : -1;
            if ((rc = receivers_step(s, s->w, n, st))) return rc;
            if ((rc = fused_forward_step(s, s->w, n, slot, st))) return rc;
            ++*done;
            if (++s->sh_n == nt) {  // into the adjoint: last segment first, its snapshots are in the store
                if ((rc = zero_state(s, s->w, st))) return rc;
                if ((rc = sim_zero(s, s->grad_vp, s->ninterior * sizeof(float), st))) return rc;
                if ((rc = sim_zero(s, s->grad_rho, s->ninterior * sizeof(float), st))) return rc;
                s->sh_phase = 2;
                s->sh_seg = nseg - 1;
                s->sh_recomp = false;
                s->sh_n = nt - 1;
            }
        } else {
            const int a = s->sh_seg * K, b = std::min(nt, a + K);
            if (s->sh_recomp) {
                const int n = s->sh_n;
                if (n == a && (rc = restore_checkpoint(s, s->rw, s->sh_seg, st))) return rc;
                const int slot = (n % c.xcorr_step == 0) ? (n - a) / c.xcorr_step : -1;
                if ((rc = fused_forward_step(s, s->rw, n, slot, st, false))) return rc;
                ++*done;
                if (++s->sh_n == b) {
                    s->sh_recomp = false;
                    s->sh_n = b - 1;
                }
            } else {
                if ((rc = adjoint_unit(s, s->sh_n, a, true, st))) return rc;
                ++*done;
                if (--s->sh_n < a) {
                    if (--s->sh_seg < 0) {
                        k_finalize_dense<<<s->dense_grid(), 128, 0, st>>>(s->grad_vp, s->mv[3], s->L,
                                                                         c.dt * c.xcorr_step);
                        s->launches++;
                        s->sh_phase = 3;
                    } else {
                        s->sh_recomp = true;
                        s->sh_n = s->sh_seg * K;
                    }
                }
            }
        }
        if ((rc = launch_status())) return rc;
    }
    return TTI_OK;
}

int shot_read_traces(tti_sim* s, float* host)
{
    if (!s || !host) return TTI_EINVAL;
    if (!s->nrec) return TTI_OK;
    const size_t bytes = (size_t)s->nrec * s->cfg.nt * sizeof(float);
    if (cudaMemcpyAsync(host, s->traces, bytes, cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
        return cuda_rc(cudaGetLastError());
    return cuda_rc(cudaStreamSynchronize(s->stream));
}

// After the enqueued units have run: status of the shot's kernels.
int shot_end(tti_sim* s)
{
    if (!s) return TTI_EINVAL;
    int rc = cuda_rc(cudaStreamSynchronize(s->stream));
    if (!rc) rc = fused_wait_status(s->stream, s->err);
    if (!rc && s->sh_phase == 3) s->forward_done = true;
    return rc;
}

} // namespace tti

extern "C" {

int tti_sim_get_image(tti_sim* s, float* grad_vp, float* grad_rho, int on_device)
{
    if (!s) return TTI_EINVAL;
    size_t bytes = s->ninterior * sizeof(float);
    cudaMemcpyKind k = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (grad_vp && cudaMemcpyAsync(grad_vp, s->grad_vp, bytes, k, s->stream) != cudaSuccess)
        return cuda_rc(cudaGetLastError());
    if (grad_rho && cudaMemcpyAsync(grad_rho, s->grad_rho, bytes, k, s->stream) != cudaSuccess)
        return cuda_rc(cudaGetLastError());
    return cuda_rc(cudaStreamSynchronize(s->stream));
}

int tti_sim_set_profiling(tti_sim* s, int enable)
{
    if (!s) return TTI_EINVAL;
    s->profiling = enable != 0;
    for (int k = 0; k < 3; ++k) {
        s->kind_ms[k] = 0;
        s->kind_n[k] = 0;
    }
    return TTI_OK;
}

int tti_sim_kernel_times(tti_sim* s, double* ms, int64_t* launches)
{
    if (!s || !ms || !launches) return TTI_EINVAL;
    for (int k = 0; k < 3; ++k) {
        ms[k] = s->kind_ms[k];
        launches[k] = s->kind_n[k];
    }
    return TTI_OK;
}

int tti_sim_autotune(tti_sim* s, int reps, tti_tune_report* out)
{
    if (!s || !out || reps < 1) return TTI_EINVAL;
    if (!s->cfg.fused) return TTI_EINVAL;
    if (!s->model_set) return TTI_ESTATE;
    *out = tti_tune_report{};
    const Layout& L = s->L;
    const tti_sim_config& c = s->cfg;
    const bool t1 = c.scheme == 1;
    // the type1 image is a point-wise kernel with no work split to tune
    const bool img = !t1 && s->snaps && (c.snap_precision != SNAP_F32 || fused_image_supported(L));
    cudaStream_t st = s->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        cudaGetLastError();
        return TTI_ELAUNCH;
    }
    // Each candidate runs on the simulator's own volumes; the wavefield and
    // image contents afterwards are unspecified (forward() and adjoint()
    // start from zero).
    auto launch = [&](int kind, Split sp) -> int {
        WaveState& w = s->w;
        if (kind == KIND_FWD) {
            FwdStepArgs a{};
            a.pin = w.p;
            a.qin = w.q;
            a.pout = w.p2;
            a.qout = w.q2;
            a.f3 = w.pd;
            a.f4 = w.qd;
            a.m = model_of(s);
            a.abx = s->abx;
            a.aby = s->aby;
            a.abz = s->abz;
            a.src_index = -1;
            a.snap_prec = c.snap_precision;
            a.free_surface = c.free_surface;
            a.vti = s->vti ? 1 : 0;
            a.dt = c.dt;
            a.dx = c.dx;
            a.dy = c.dy;
            a.dz = c.dz;
            a.err = s->err;
            a.bz = sp.bz;
            a.ztop = sp.ztop;
            return t1 ? launch_t1_fused_forward(L, a, s->sponge_active ? 1 : 0, st) : launch_fused_forward(L, a, st);
        }
        if (kind == KIND_ADJ) {
            AdjStepArgs a{};
            a.pin = w.p;
            a.qin = w.q;
            a.pout = w.p2;
            a.qout = w.q2;
            a.f3 = w.pd;
            a.f4 = w.qd;
            a.m = model_of(s);
            a.abx = s->abx;
            a.aby = s->aby;
            a.abz = s->abz;
            a.sponge_active = s->sponge_active ? 1 : 0;
            a.free_surface = c.free_surface;
            a.vti = s->vti ? 1 : 0;
            a.dt = c.dt;
            a.dx = c.dx;
            a.dy = c.dy;
            a.dz = c.dz;
            a.err = s->err;
            a.bz = sp.bz;
            a.ztop = sp.ztop;
            return t1 ? launch_t1_fused_adjoint(L, a, st) : launch_fused_adjoint(L, a, st);
        }
        ImageArgs ia{};
        ia.adj1 = w.p;
        ia.adj2 = w.q;
        ia.adj3 = w.pd;
        ia.adj4 = w.qd;
        ia.store = s->snaps;
        ia.snap_prec = c.snap_precision;
        ia.snap_scale = s->snap_scale;
        ia.nsnap = s->nslot;
        ia.slot = 0;
        ia.m = model_of(s);
        ia.grad_vp = s->grad_vp;
        ia.grad_rho = s->grad_rho;
        ia.free_surface = c.free_surface;
        ia.vti = s->vti ? 1 : 0;
        ia.dx = c.dx;
        ia.dy = c.dy;
        ia.dz = c.dz;
        ia.err = s->err;
        ia.bz = sp.bz;
        ia.ztop = sp.ztop;
        return launch_fused_image(L, ia, st);
    };
    int rc = TTI_OK;
    if (s->snap_scale) rc = sim_zero(s, s->snap_scale, (size_t)s->nslot * 4 * sizeof(float));
    for (int kind = 0; kind < 3 && !rc; ++kind) {
        if (kind == KIND_IMG && !img) continue;
        const int table_kind = !t1 ? kind : (kind == KIND_FWD ? KIND_T1F : KIND_T1A);
        const std::vector<Split> cand = split_candidates(L, table_kind);
        const Split modelled = model_split(L, table_kind);
        out->ncand = std::max(out->ncand, (int)cand.size());
        auto time_of = [&](const Split& sp, int n, float* ms) -> int {
            int r = launch(kind, sp);  // warm-up
            if (r) return r;
            cudaEventRecord(e0, st);
            for (int k = 0; k < n && !r; ++k) r = launch(kind, sp);
            cudaEventRecord(e1, st);
            if (r) return r;
            if ((r = cuda_rc(cudaEventSynchronize(e1)))) return r;
            cudaEventElapsedTime(ms, e0, e1);
            *ms /= n;
            return TTI_OK;
        };
        // first pass over every candidate, then the three fastest and the
        // model's choice again with more launches: candidates within a few
        // per cent of each other are ranked on the longer timing
        std::vector<std::pair<float, Split>> timed;
        for (const Split& sp : cand) {
            float ms = 0;
            if ((rc = time_of(sp, reps, &ms))) break;
            timed.push_back({ms, sp});
        }
        if (rc) break;
        std::sort(timed.begin(), timed.end(), [](const auto& x, const auto& y) { return x.first < y.first; });
        std::vector<Split> finalists;
        for (size_t k = 0; k < timed.size() && finalists.size() < 3; ++k) finalists.push_back(timed[k].second);
        if (std::find(finalists.begin(), finalists.end(), modelled) == finalists.end()) finalists.push_back(modelled);
        // the fastest top/bottom candidate too, when it is within 3 % on the
        // first pass (the tie-break below can only prefer a finalist)
        for (const auto& t : timed)
            if (t.second.ztop > 0) {
                if (t.first <= 1.03f * timed.front().first &&
                    std::find(finalists.begin(), finalists.end(), t.second) == finalists.end())
                    finalists.push_back(t.second);
                break;
            }
        std::vector<std::pair<float, Split>> fin;
        for (const Split& sp : finalists) {
            float ms = 0;
            if ((rc = time_of(sp, 2 * reps + 1, &ms))) break;
            if (sp == modelled) out->model_ms[kind] = ms;
            fin.push_back({ms, sp});
        }
        if (rc) break;
        // the fastest; among finalists within 1 % of it a top/bottom split
        // is preferred: it keeps the halo planes that neighbouring columns
        // share in L2 and so moves about half the DRAM bytes of a tile-major
        // split at the same speed
        float best = 1e30f;
        Split best_sp{};
        for (const auto& f : fin)
            if (f.first < best) {
                best = f.first;
                best_sp = f.second;
            }
        if (best_sp.ztop == 0) {
            float alt = 1e30f;
            for (const auto& f : fin)
                if (f.second.ztop > 0 && f.first <= 1.01f * best && f.first < alt) {
                    alt = f.first;
                    best_sp = f.second;
                }
            if (alt < 1e30f) best = alt;
        }
        record_tuned_split(L, table_kind, best_sp);
        out->bz[kind] = best_sp.bz;
        out->ztop[kind] = best_sp.ztop;
        out->ms[kind] = best;
    }
    if (!rc) rc = cuda_rc(cudaStreamSynchronize(st));
    if (!rc) rc = fused_wait_status(st, s->err);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGetLastError();
    return rc;
}

int tti_selfcheck_bounded_wait(double seconds, tti_stream_t stream)
{
    if (!(seconds > 0) || seconds > 10) return TTI_EINVAL;
    int dev = 0, khz = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dev) != cudaSuccess) {
        cudaGetLastError();
        return TTI_ELAUNCH;
    }
    const long long cycles = (long long)(seconds * khz * 1e3);
    return wait_selfcheck(reinterpret_cast<cudaStream_t>(stream), cycles);
}

int tti_tune_set_split(int nx, int ny, int nz, int kind, int bz, int ztop)
{
    if (nx < 1 || ny < 1 || nz < 1 || kind < 0 || kind >= KIND_COUNT || bz < 0) return TTI_EINVAL;
    tti_sim_config c{};
    c.nx = nx;
    c.ny = ny;
    c.nz = nz;
    const Layout L = layout_of(c);
    if (bz > 0 && !split_valid(L, Split{bz, ztop})) return TTI_EINVAL;
    record_tuned_split(L, kind, Split{bz, bz > 0 ? ztop : 0});
    return TTI_OK;
}

int tti_tune_set(int nx, int ny, int nz, int kind, int bz) { return tti_tune_set_split(nx, ny, nz, kind, bz, 0); }

int tti_tune_get_split(int nx, int ny, int nz, int kind, int* bz, int* ztop)
{
    if (nx < 1 || ny < 1 || nz < 1 || kind < 0 || kind >= KIND_COUNT || !bz || !ztop) return TTI_EINVAL;
    tti_sim_config c{};
    c.nx = nx;
    c.ny = ny;
    c.nz = nz;
    const Split sp = choose_split(layout_of(c), kind);
    *bz = sp.bz;
    *ztop = sp.ztop;
    return TTI_OK;
}

int tti_tune_get(int nx, int ny, int nz, int kind)
{
    int bz = 0, ztop = 0;
    const int rc = tti_tune_get_split(nx, ny, nz, kind, &bz, &ztop);
    return rc ? -rc : bz;
}

int tti_sim_source_gradient(tti_sim* s, float* host_out)
{
    if (!s || !host_out) return TTI_EINVAL;
    if (s->src_index < 0) return TTI_ESTATE;
    std::vector<float> tmp(s->cfg.nt);
    if (cudaMemcpyAsync(tmp.data(), s->srctr, s->cfg.nt * sizeof(float), cudaMemcpyDeviceToHost, s->stream) !=
        cudaSuccess)
        return cuda_rc(cudaGetLastError());
    int rc = cuda_rc(cudaStreamSynchronize(s->stream));
    if (rc) return rc;
    for (int n = 0; n < s->cfg.nt; ++n) host_out[n] = tmp[n] * s->cfg.dt;
    return TTI_OK;
}

int tti_sim_volume(tti_sim* s, int which, float** dev_ptr)
{
    if (!s || !dev_ptr || which < 0 || which > 11) return TTI_EINVAL;
    float* v[12] = {s->w.p, s->w.q, s->w.pd, s->w.qd, s->mv[0], s->mv[1], s->mv[2], s->mv[3],
                    s->mv[4], s->mv[5], s->mv[6], s->mv[7]};
    *dev_ptr = v[which];
    return TTI_OK;
}

int tti_sim_read_volume(tti_sim* s, int which, float* host_dst)
{
    float* src = nullptr;
    int rc = tti_sim_volume(s, which, &src);
    if (rc) return rc;
    if (!host_dst) return TTI_EINVAL;
    if (cudaMemcpyAsync(host_dst, src, s->nvol() * sizeof(float), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess)
        return cuda_rc(cudaGetLastError());
    return cuda_rc(cudaStreamSynchronize(s->stream));
}

int tti_sim_layout(tti_sim* s, int* ldimx, int* ldimy, int* ldimz)
{
    if (!s || !ldimx || !ldimy || !ldimz) return TTI_EINVAL;
    *ldimx = s->L.ldimx;
    *ldimy = s->L.ldimy;
    *ldimz = s->L.ldimz;
    return TTI_OK;
}

int64_t tti_sim_launch_count(tti_sim* s) { return s ? s->launches : -1; }

tti_stream_t tti_sim_stream(tti_sim* s) { return s ? (tti_stream_t)s->stream : nullptr; }

} // extern "C"
