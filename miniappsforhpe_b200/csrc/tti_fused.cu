// Fused time-step kernels for the TTI/VTI pseudo-acoustic RTM on B200.
//
// One kernel per forward step and one per adjoint step replace the
// reference's per-step kernel sequences
//   forward  (simulator2SetUp.cu:530-651): loop2, loop4, fwd_drv,
//            loop4_derivatives, fwd_main_loop_2
//   adjoint  (simulator2SetUp.cu:654-720): adj_drv, loop4_derivatives,
//            update_adj_kernel_main_3, loop2, loop4
// so that each step streams every volume through HBM once: p,q are read
// from one buffer and the next p,q are written to a second one; pdot,qdot
// are updated in place; the six buoyancy-scaled derivative volumes and the
// two mixed-derivative volumes of the reference never touch HBM.
//
// Structure (2.5D blocking): a CTA owns a 32x16 column tile and marches
// through a chunk of z.  Halo'd XY planes are staged into shared memory by
// TMA (cp.async.bulk.tensor, zero fill outside the volume) behind a
// multi-stage mbarrier pipeline; the z-direction stencils run in per-thread
// register queues.  The D-z stage of the staggered pair is scattered plane by
// plane as in the reference kernels; the D+z stage keeps the raw buoyancy-
// scaled z-derivatives of the last eight planes so the reference's tap order
// is preserved and the free-surface mirror can be resolved at output time.
// Output for plane z happens when plane z+7 arrives.
//
// The grid's (tile, z) planes are split among CTAs either tile-major (bz
// consecutive planes each) or, on grids with fewer tile columns than SMs,
// top/bottom (a CTA per column top, the others sharing the bottoms); the
// split changes the launch shape only.  The centred (type1) operator has its
// own step kernels here as well (output lag 4; the forward one computes two
// x-neighbouring outputs per thread), and every step kernel can round the
// p, q it writes to FP16/BF16 of a per-field scaled value.
//
// Every mbarrier wait is bounded (clock-based); a wait that gives up sets the
// error word the host reads back, and the kernel stops waiting.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "tti_common.cuh"
#include "tti_internal.cuh"

namespace tti {
namespace {

constexpr int TX = 32, TY = 16, NT = TX * TY;
constexpr int PW = TX + 16, PH = TY + 16;  // p/q tile with a halo of 8
constexpr int IW = TX + 8, IH = TY + 8;    // tile with a halo of 4
constexpr int LAG = 7;                     // output plane = arrival plane - 7

// Packed pairs: the two wavefields of a cell travel together in one float2
// and are updated by the paired FP32 instructions of sm_100 (FFMA2, FADD2,
// FMUL2), one instruction for both fields with per-component rounding the
// same as fmaf / add / mul.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// Reciprocal of a buoyancy (irho in (0, 1]): the hardware approximation,
// within one unit in the last place.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// ---------------------------------------------------------------------------
// TMA / mbarrier primitives (PTX ISA 8.x, sm_90+).
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: about a second of SM clocks, then report and give up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, bool& dead)
{
    if (dead) return false;
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (2LL << 30)) {
            atomicExch(err, 1);
            dead = true;
            return false;
        }
    }
    return true;
}
// Give-up path of a pipelined CTA.  A bounded wait that times out sets the
// error word and the waiting thread's `dead` flag; the CTA agrees to stop at
// its next block barrier (__syncthreads_or of the flags), so no thread
// issues a further load or processes a further plane.  Before exiting,
// thread 0 waits, again with a bound, for every plane it issued from the
// one being waited on when the CTA stopped (global plane g: stage g % ns,
// parity (g / ns) & 1; at most the prefetch distance ahead, so one phase
// per stage) so that no bulk copy it started is left writing into shared
// memory.  If such a copy never completes even then, the CTA exits with it
// in flight; what the copy does afterwards is undefined, and the error word
// already tells the host that the launch's results are invalid.
__device__ __noinline__ void drain_loads(uint64_t* bars, int ns, int g0, int g1)
{
    for (int g = g0; g < g1; ++g) {
        uint64_t* b = &bars[g % ns];
        const uint32_t par = (uint32_t)((g / ns) & 1);
        const long long t0 = clock64();
        while (!mbar_try_wait(b, par))
            if (clock64() - t0 > (2LL << 30)) break;
    }
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(saddr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(saddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(saddr(bar))
        : "memory");
}

// ---------------------------------------------------------------------------
// Work split of one fused step.  The grid's (tile, z) planes are taken in
// tile-major order (all of tile 0's column, then tile 1's, ...) and every CTA
// processes per_cta consecutive planes of that sequence, as one or more
// segments that each lie in one tile column.  A segment costs its planes
// plus the 2*LAG planes of pipeline fill, so per_cta is chosen to balance
// the SMs rather than to cut columns evenly.
struct Segment {
    int x0, y0, zs, len;
};
// With ztop > 0 the sequence is split in two: CTA t < tiles takes the top
// ztop planes of column t; the other CTAs walk the columns' bottoms (planes
// ztop .. nz-1 of every column, tile-major), per_cta planes each.
struct WorkRange {
    long long pos, end;
    int tiles_x, span, zbase, ixbeg, iybeg, izbeg;
    __device__ WorkRange(const Layout& L, int per_cta, int ztop)
    {
        tiles_x = (L.nx() + TX - 1) / TX;
        const long long tiles = (long long)tiles_x * ((L.ny() + TY - 1) / TY);
        ixbeg = L.ixbeg;
        iybeg = L.iybeg;
        izbeg = L.izbeg;
        long long cta = blockIdx.x;
        if (ztop > 0 && cta < tiles) {
            span = ztop;
            zbase = 0;
            per_cta = ztop;
        } else {
            span = L.nz() - ztop;
            zbase = ztop;
            if (ztop > 0) cta -= tiles;
        }
        pos = cta * per_cta;
        end = min(tiles * span, pos + per_cta);
    }
    __device__ bool next(Segment& sg)
    {
        if (pos >= end) return false;
        const long long tile = pos / span;
        const int z0 = (int)(pos - tile * span);
        sg.len = (int)min((long long)(span - z0), end - pos);
        sg.x0 = ixbeg + (int)(tile % tiles_x) * TX;
        sg.y0 = iybeg + (int)(tile / tiles_x) * TY;
        sg.zs = izbeg + zbase + z0;
        pos += sg.len;
        return true;
    }
};

// ---------------------------------------------------------------------------
// Free-surface resolution of the buoyancy-scaled z-derivative queue.
// q[j] holds the derivative at position z-3+j.  The z-marching pipeline
// already zeroes positions outside the interior (the reference's derivative
// volumes are never written in the halo).  With a free surface, positions
// <= izbeg instead take the value at 2*izbeg+1-pos (kernel_type2_small.cu:
// 34-39), which is in the queue itself for the four outputs nearest the
// surface: j' = 7 - 2*(z-izbeg) - j.
template <typename T>
__device__ __forceinline__ void resolve_dz(T (&q)[8], int dtop)
{
    switch (dtop) {
    case 0:
        q[0] = q[7];
        q[1] = q[6];
        q[2] = q[5];
        q[3] = q[4];
        break;
    case 1:
        q[0] = q[5];
        q[1] = q[4];
        q[2] = q[3];
        break;
    case 2:
        q[0] = q[3];
        q[1] = q[2];
        break;
    case 3: q[0] = q[1]; break;
    default: break;
    }
}

// D- z-stage coefficient for a scatter from arrival plane L into queue slot j
// (position L-3+j): ir = 3-j  ->  +c1(ir+1) for ir>=0, -c1(-ir) for ir<0.
__device__ __forceinline__ float dminus_coef(int j) { return (j <= 3) ? c1(4 - j) : -c1(j - 3); }

struct FwdParams {
    float* pout;
    float* qout;
    float* f3;
    float* f4;
    const float *irho, *m1, *m2, *m3, *m4, *rx, *ry, *rz;
    const float2 *abx, *aby, *abz;
    void* snap;
    int snap_prec;
    const float* snap_scale;
    unsigned int* snap_amax;
    int64_t src_index;
    float src_term;
    Layout L;
    int bz;    // planes per CTA (of the bottoms when ztop > 0)
    int ztop;  // > 0: top/bottom split
    int fs;
    float dt, invdx, invdy, invdz, invdxdy, invdydz, invdzdx;
    int* err;
    int wave_prec;            // 0, or p/q rounded to FP16 (1) / BF16 (2) each step
    const float* wave_scale;  // 2 scales (p, q) of this step's output
    float* trace;             // receivers of this step (nullptr: not sampled here)
    RecMap rec;
};

// Offset of plane z's receiver table, or -1 when no receiver lies on it
// (uniform over a block working on plane z).
__device__ __forceinline__ int receiver_plane(const RecMap& m, int z)
{
    int off = -1;
    if (z < m.zlo || z > m.zhi) return off;
#pragma unroll
    for (int k = 0; k < kRecPlanesFolded; ++k)
        if (k < m.nz && m.z[k] == z) off = m.off[k];
    return off;
}

constexpr int FWD_NS = 11;  // ring: planes L-8 .. L+2
constexpr int FWD_PF = 2;   // prefetch distance
constexpr size_t FWD_SLOT_P = (size_t)2 * PH * PW * sizeof(float);  // p and q tiles
constexpr size_t FWD_SLOT_I = (size_t)IH * IW * sizeof(float);      // irho tile
constexpr size_t FWD_DX = (size_t)2 * TY * IW * sizeof(float);
constexpr size_t FWD_DY = (size_t)2 * IH * TX * sizeof(float);
constexpr size_t FWD_SMEM = FWD_NS * (FWD_SLOT_P + FWD_SLOT_I) + FWD_DX + FWD_DY + FWD_NS * sizeof(uint64_t);

template <bool TTI>
__global__ void __launch_bounds__(NT, 1)
    k_fused_forward(const __grid_constant__ CUtensorMap tm_p, const __grid_constant__ CUtensorMap tm_q,
                    const __grid_constant__ CUtensorMap tm_i, const FwdParams a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    float* ring = reinterpret_cast<float*>(smem);                                  // [NS][2][PH][PW]
    float* iring = reinterpret_cast<float*>(smem + FWD_NS * FWD_SLOT_P);           // [NS][IH][IW]
    // x/y derivative tiles, both fields of a cell side by side
    float2* dxs = reinterpret_cast<float2*>(smem + FWD_NS * (FWD_SLOT_P + FWD_SLOT_I));           // [TY][IW]
    float2* dys = reinterpret_cast<float2*>(smem + FWD_NS * (FWD_SLOT_P + FWD_SLOT_I) + FWD_DX);  // [IH][TX]
    uint64_t* bars =
        reinterpret_cast<uint64_t*>(smem + FWD_NS * (FWD_SLOT_P + FWD_SLOT_I) + FWD_DX + FWD_DY);

    const Layout& L = a.L;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    bool dead = false;
    bool stop = false;             // the CTA gave up (a bounded wait timed out)
    int g_issued = 0, g_wait = 0;  // planes issued (thread 0) / plane last waited on

    if (tid == 0) {
        for (int s = 0; s < FWD_NS; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    unsigned tmax[4] = {0u, 0u, 0u, 0u};  // max |stored value| seen by this thread
    int s = 0;                            // ring slot of the current plane
    uint32_t phase = 0;                   // mbarrier parity of slot s for this use
    int gbase = 0;                        // planes consumed by earlier segments
    // This CTA's share of the (tile, z) work in tile-major order: a.bz planes
    // from blockIdx.x * a.bz, as one or more segments of a tile column.
    WorkRange wr(L, a.bz, a.ztop);
    for (Segment sg; wr.next(sg); gbase += sg.len + 2 * LAG) {
    const int x0 = sg.x0, y0 = sg.y0, zs = sg.zs;
    const int ntot = sg.len + 2 * LAG;  // arrival planes zs-7 .. ze+7
    const int x = x0 + tx, y = y0 + ty;
    const bool owner = (x <= L.ixend) && (y <= L.iyend);
    if (__syncthreads_or(dead)) {  // barriers initialised; the previous segment is done with the ring
        stop = true;
        break;
    }

    auto issue = [&](int t) {
        ++g_issued;
        const int s = (gbase + t) % FWD_NS, z = zs - LAG + t;
        float* dst = ring + (size_t)s * 2 * PH * PW;
        mbar_expect_tx(&bars[s], (uint32_t)(FWD_SLOT_P + FWD_SLOT_I));
        tma_load_3d(dst, &tm_p, x0 - 8, y0 - 8, z, &bars[s]);
        tma_load_3d(dst + PH * PW, &tm_q, x0 - 8, y0 - 8, z, &bars[s]);
        tma_load_3d(iring + (size_t)s * IH * IW, &tm_i, x0 - 4, y0 - 4, z, &bars[s]);
    };
    if (tid == 0)
        for (int t = 0; t < FWD_PF && t < ntot; ++t) issue(t);

    float dzq1[8], dzq2[8];  // D- partial sums, positions L-3 .. L+4
    float dZ1[8], dZ2[8];    // buoyancy-scaled z derivatives, positions L-10 .. L-3
    float mq[3][4];          // zx1, zx2, yz1, yz2 for outputs L-7, L-6, L-5
#pragma unroll
    for (int j = 0; j < 8; ++j) dzq1[j] = dzq2[j] = dZ1[j] = dZ2[j] = 0.0f;
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int c = 0; c < 4; ++c) mq[j][c] = 0.0f;

    const int vc = (tx + 8), vr = (ty + 8);  // this column inside a p/q tile

    auto back = [&](int k) { const int v = s - k; return v < 0 ? v + FWD_NS : v; };
    for (int t = 0; t < ntot; ++t) {
        if (__syncthreads_or(dead)) {  // every thread is done with iteration t-1
            stop = true;
            break;
        }
        if (tid == 0 && t + FWD_PF < ntot) {
            fence_proxy_async();
            issue(t + FWD_PF);
        }
        g_wait = gbase + t;
        mbar_wait(&bars[s], phase, a.err, dead);
        const int Lz = zs - LAG + t;
        const float* P1 = ring + (size_t)s * 2 * PH * PW;
        const float* P2 = P1 + PH * PW;

        // (a) D- z stage: scatter plane L into positions L-3 .. L+4.
        {
            const float v1 = P1[vr * PW + vc], v2 = P2[vr * PW + vc];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float c = dminus_coef(j);
                dzq1[j] = dzq1[j] + c * v1;
                dzq2[j] = dzq2[j] + c * v2;
            }
        }
        // completed position L-3: scale by 1/dz and the buoyancy there
        {
            const int zp = Lz - 3;
            const bool valid = (zp >= L.izbeg + (a.fs ? 1 : 0)) && zp <= L.izend;
            const float* I3 = iring + (size_t)back(3) * IH * IW;
            const float ir3 = I3[(ty + 4) * IW + tx + 4];
            const float n1 = valid ? (dzq1[0] * a.invdz) * ir3 : 0.0f;
            const float n2 = valid ? (dzq2[0] * a.invdz) * ir3 : 0.0f;
#pragma unroll
            for (int j = 0; j < 7; ++j) {
                dZ1[j] = dZ1[j + 1];
                dZ2[j] = dZ2[j + 1];
                dzq1[j] = dzq1[j + 1];
                dzq2[j] = dzq2[j + 1];
            }
            dZ1[7] = n1;
            dZ2[7] = n2;
            dzq1[7] = 0.0f;
            dzq2[7] = 0.0f;
        }
        // (b) mixed zx/yz for output L-4 from planes L-8 .. L (ring), TTI only.
        float mz[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if constexpr (TTI) {
#pragma unroll
            for (int m = -4; m <= 4; ++m) {
                if (m == 0) continue;
                const float c = c2(m < 0 ? -m : m);
                const float* Q1 = ring + (size_t)back(4 - m) * 2 * PH * PW;
                const float* Q2 = Q1 + PH * PW;
                mz[0] += c * (Q1[vr * PW + vc + m] - Q1[vr * PW + vc - m]);
                mz[1] += c * (Q2[vr * PW + vc + m] - Q2[vr * PW + vc - m]);
                mz[2] += c * (Q1[(vr + m) * PW + vc] - Q1[(vr - m) * PW + vc]);
                mz[3] += c * (Q2[(vr + m) * PW + vc] - Q2[(vr - m) * PW + vc]);
            }
            mz[0] *= a.invdzdx;
            mz[1] *= a.invdzdx;
            mz[2] *= a.invdydz;
            mz[3] *= a.invdydz;
        }

        // (c) output plane L-7
        const int z = Lz - LAG;
        if (z >= zs) {  // block-uniform
            const int s7 = back(LAG);
            const float* O1 = ring + (size_t)s7 * 2 * PH * PW;
            const float* I7 = iring + (size_t)s7 * IH * IW;
            // issue the point-wise loads of this cell early
            const int64_t gi = L.idx(x, y, z);
            float a1 = 0, a2 = 0, a3 = 0, a4 = 0, vrx = 0, vry = 0, vrz = 1, o3 = 0, o4 = 0;
            float2 sx = make_float2(1, 1), sy = sx, sz = sx;
            if (owner) {
                a1 = __ldg(a.m1 + gi);
                a2 = __ldg(a.m2 + gi);
                a3 = __ldg(a.m3 + gi);
                a4 = __ldg(a.m4 + gi);
                if constexpr (TTI) {
                    vrx = __ldg(a.rx + gi);
                    vry = __ldg(a.ry + gi);
                    vrz = __ldg(a.rz + gi);
                }
                o3 = a.f3[gi];
                o4 = a.f4[gi];
                sx = __ldg(a.abx + x);
                sy = __ldg(a.aby + y);
                sz = __ldg(a.abz + z);
            }
            // buoyancy-scaled first derivatives of plane z on the halo'd tile
            // dxs[r][c]: x = x0-4+c, y = y0+r;  dys[r][c]: x = x0+c, y = y0-4+r
            auto dx_at = [&](int r, int c) {
                const bool in = (x0 - 4 + c >= L.ixbeg) && (x0 - 4 + c <= L.ixend);
                const float irv = I7[(r + 4) * IW + c];
                float acc[2];
#pragma unroll
                for (int f = 0; f < 2; ++f) {
                    const float* Pr = O1 + f * PH * PW + (r + 8) * PW + c + 4;
                    acc[f] = 0.0f;
#pragma unroll
                    for (int i = 1; i <= 4; ++i) acc[f] += c1(i) * (Pr[i - 1] - Pr[-i]);
                    acc[f] *= a.invdx;
                }
                dxs[r * IW + c] = in ? make_float2(acc[0] * irv, acc[1] * irv) : make_float2(0.0f, 0.0f);
            };
            auto dy_at = [&](int r, int c) {
                const bool in = (y0 - 4 + r >= L.iybeg) && (y0 - 4 + r <= L.iyend);
                const float irv = I7[r * IW + c + 4];
                float acc[2];
#pragma unroll
                for (int f = 0; f < 2; ++f) {
                    const float* Pc = O1 + f * PH * PW + (r + 4) * PW + c + 8;
                    acc[f] = 0.0f;
#pragma unroll
                    for (int i = 1; i <= 4; ++i) acc[f] += c1(i) * (Pc[(i - 1) * PW] - Pc[-i * PW]);
                    acc[f] *= a.invdy;
                }
                dys[r * TX + c] = in ? make_float2(acc[0] * irv, acc[1] * irv) : make_float2(0.0f, 0.0f);
            };
            dx_at(ty, tx);
            // the halos by whole warps, spread so that no warp does more than
            // three tile cells: the (IW-TX) x TY halo columns by warps 0..3,
            // the (IH-TY) halo rows by warps 4..11
            if (tid < (IW - TX) * TY) dx_at(tid / (IW - TX), TX + tid % (IW - TX));
            dy_at(ty, tx);
            if (ty >= 4 && ty < 4 + IH - TY) dy_at(ty - 4 + TY, tx);
            __syncthreads();
            float snapv[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (owner) {
                float xx1 = 0, xx2 = 0, yy1 = 0, yy2 = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float2 vx = dxs[ty * IW + tx + 1 + k];
                    const float2 vy = dys[(ty + 1 + k) * TX + tx];
                    xx1 += tap(k) * vx.x;
                    xx2 += tap(k) * vx.y;
                    yy1 += tap(k) * vy.x;
                    yy2 += tap(k) * vy.y;
                }
                xx1 *= a.invdx;
                xx2 *= a.invdx;
                yy1 *= a.invdy;
                yy2 *= a.invdy;
                float q1[8], q2[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    q1[j] = dZ1[j];
                    q2[j] = dZ2[j];
                }
                if (a.fs) {
                    resolve_dz(q1, z - L.izbeg);
                    resolve_dz(q2, z - L.izbeg);
                }
                float zz1 = 0, zz2 = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    zz1 = zz1 + tap(k) * q1[k];
                    zz2 = zz2 + tap(k) * q2[k];
                }
                zz1 *= a.invdz;
                zz2 *= a.invdz;
                const float ir = I7[(ty + 4) * IW + tx + 4];
                const float rho = __frcp_rn(ir);
                float r3, r4;
                const float* O2 = O1 + PH * PW;
                if constexpr (TTI) {
                    float xy1 = 0, xy2 = 0;
#pragma unroll
                    for (int k = -4; k <= 4; ++k) {
                        if (k == 0) continue;
                        const float c = c2(k < 0 ? -k : k);
                        xy1 += c * (O1[(vr + k) * PW + vc + k] - O1[(vr - k) * PW + vc + k]);
                        xy2 += c * (O2[(vr + k) * PW + vc + k] - O2[(vr - k) * PW + vc + k]);
                    }
                    xy1 *= a.invdxdy;
                    xy2 *= a.invdxdy;
                    const float zx1 = mq[0][0], zx2 = mq[0][1], yz1 = mq[0][2], yz2 = mq[0][3];
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
                    r3 = a1 * H1 + a4 * V1 + a2 * V2;
                    r4 = a2 * H1 + a3 * V2 + a4 * H2;
                } else {
                    // rx = ry = 0, rz = 1: V = zz exactly, H = xx + yy + zz - zz.
                    xx1 *= rho;
                    yy1 *= rho;
                    zz1 *= rho;
                    xx2 *= rho;
                    yy2 *= rho;
                    zz2 *= rho;
                    const float V1 = zz1, V2 = zz2;
                    const float H1 = xx1 + yy1 + zz1 - V1;
                    const float H2 = xx2 + yy2 + zz2 - V2;
                    r3 = a1 * H1 + a4 * V1 + a2 * V2;
                    r4 = a2 * H1 + a3 * V2 + a4 * H2;
                }
                float n3 = o3 + r3 * a.dt;
                float n4 = o4 + r4 * a.dt;
                if (gi == a.src_index) {
                    n3 += a.src_term;
                    n4 += a.src_term;
                }
                a.f3[gi] = n3;
                a.f4[gi] = n4;
                const float pc = O1[vr * PW + vc], qc = O2[vr * PW + vc];
                if (a.trace) {  // the pressure -(2p + q)/3 of the incoming state (simulator2SetUp.cu:31-42)
                    const int off = receiver_plane(a.rec, z);
                    if (off >= 0) {
                        const int r = __ldg(a.rec.xy + off + (y - L.iybeg) * L.nx() + (x - L.ixbeg));
                        if (r >= 0) a.trace[r] = -(2 * pc + qc) / 3;
                    }
                }
                if (a.snap) {
                    const int64_t nin = (int64_t)L.nx() * L.ny() * L.nz();
                    const int64_t d = ((int64_t)(z - L.izbeg) * L.ny() + (y - L.iybeg)) * L.nx() + (x - L.ixbeg);
                    snapv[0] = n3;
                    snapv[1] = n4;
                    snapv[2] = pc;
                    snapv[3] = qc;
                    bool sat = false;
#pragma unroll
                    for (int f = 0; f < 4; ++f) {
                        const float sc = (a.snap_prec == SNAP_F32) ? 1.0f : a.snap_scale[f];
                        sat |= snap_store(a.snap, f * nin + d, snapv[f] * sc, a.snap_prec);
                    }
                    if (sat) atomicOr(a.err, 2);
                }
                // next step's loop2 (kernel_base.cu:92-101) and free surface (:142-162)
                const float A = fminf(sx.x, fminf(sy.x, sz.x));
                const float B = fminf(sx.y, fminf(sy.y, sz.y));
                float np = A * pc + B * n3 * a.dt;
                float nq = A * qc + B * n4 * a.dt;
                if (a.fs && z == L.izbeg) {
                    np = 0.0f;
                    nq = 0.0f;
                }
                wave_apply(a.wave_prec, a.wave_scale, np, nq);
                a.pout[gi] = np;
                a.qout[gi] = nq;
                if (a.fs && z > L.izbeg && z <= L.izbeg + kRadius) {
                    const int64_t gm = L.idx(x, y, 2 * L.izbeg - z);
                    a.pout[gm] = -np;
                    a.qout[gm] = -nq;
                }
            }
            // running max |value| of each stored field (the bits of a
            // non-negative float order like the float)
#pragma unroll
            for (int f = 0; f < 4; ++f) tmax[f] = max(tmax[f], __float_as_uint(fabsf(snapv[f])));
        }
        if constexpr (TTI) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                mq[0][c] = mq[1][c];
                mq[1][c] = mq[2][c];
                mq[2][c] = mz[c];
            }
        }
        if (++s == FWD_NS) {
            s = 0;
            phase ^= 1u;
        }
    }
    if (stop) break;
    }  // segments
    if (stop && tid == 0) drain_loads(bars, FWD_NS, g_wait, g_issued);
    // one atomic per warp and field for all segments; the next
    // snapshot's scale is taken from this running max
    if (a.snap && a.snap_prec != SNAP_F32) {
#pragma unroll
        for (int f = 0; f < 4; ++f) {
            const unsigned m = __reduce_max_sync(0xffffffffu, tmax[f]);
            if ((tid & 31) == 0 && m) atomicMax(a.snap_amax + f, m);
        }
    }
}



// ---------------------------------------------------------------------------
// Fused adjoint step (one reference adjoint step: adj_drv, loop4_derivatives,
// update_adj_kernel_main_3, loop2, loop4).  The transposed model is applied
// before the derivatives (kernel_type2_grad_snap.cu:98-129), so every term of
// an output cell is a plain sum and the terms are accumulated in per-thread
// queues as the planes arrive: the x+y and xy parts when plane z arrives,
// the yz/zx part plane by plane from z-4 to z+4 (the reference's order), the
// z part when plane z+7 arrives.
//
// Each staged plane holds p and q, and the model as two interleaved float4
// volumes, (m1, m2, m3, m4) and (irho, rx, ry, rz) (VTI: irho alone), all
// with a halo of 8, so a staging position's nine model values are two
// 128-bit shared loads.  The transposed-model temporaries of a plane are
// formed once per staging position that needs them, in passes whose role
// (which temporaries a position feeds) is uniform per warp.
struct AdjParams {
    float* pout;
    float* qout;
    float* f3;
    float* f4;
    const float* pin;
    const float* qin;
    const float2 *abx, *aby, *abz;
    Layout L;
    int bz;
    int ztop;
    int fs;
    int sponge;
    float dt;
    int* err;
    int wave_prec;            // 0, or p/q rounded to FP16 (1) / BF16 (2) each step
    const float* wave_scale;  // 2 scales (p, q) of this step's output
    // stencil coefficients with the grid spacings folded in, as (c, c) pairs
    float2 kd[3][4];  // c1(i)/dx, /dy, /dz, i = 1..4 (staggered D- and D+)
    float2 kzm[8];    // D- z scatter into queue slot j: +c1(4-j)/dz (j <= 3), -c1(j-3)/dz
    float2 kyz[9];    // sign(i) c2(|i|)/(4 dy dz) for plane offset i = -4..4
    float2 kzx[9];    // sign(i) c2(|i|)/(4 dz dx)
    float2 kxy[4];    // c2(k)/(4 dx dy), k = 1..4
    // residual injection and source trace of this step (nullptr: not here)
    const float* res;
    const float* obs;
    RecMap rec;
    float* srctr;
    int64_t src_index;
    int src_z;  // plane of src_index (-1: no source trace)
};

// Staging per plane: p, q (float), MA = (m1, m2, m3, m4) and MB = (irho, rx,
// ry, rz) (float4; VTI: irho as float), each PW x PH (halo 8).
constexpr int ADJ_NSTAGE = 3;
constexpr int ADJ_PF = 2;
constexpr size_t ADJ_F1 = (size_t)PH * PW * sizeof(float);
constexpr size_t ADJ_F4 = (size_t)PH * PW * sizeof(float4);
__host__ __device__ constexpr size_t adj_stage(bool tti) { return 2 * ADJ_F1 + ADJ_F4 + (tti ? ADJ_F4 : ADJ_F1); }
constexpr size_t ADJ_TXX = (size_t)2 * TY * PW * sizeof(float);  // rows y0.., cols x0-8..
constexpr size_t ADJ_TYY = (size_t)2 * PH * TX * sizeof(float);  // rows y0-8.., cols x0..
constexpr size_t ADJ_TXY = (size_t)2 * IH * IW * sizeof(float);  // rows y0-4.., cols x0-4..
constexpr size_t ADJ_TYZ = (size_t)2 * IH * TX * sizeof(float);  // rows y0-4.., cols x0..
constexpr size_t ADJ_TZX = (size_t)2 * TY * IW * sizeof(float);  // rows y0.., cols x0-4..
constexpr size_t ADJ_DX = (size_t)2 * TY * IW * sizeof(float);   // rows y0.., cols x0-4..
constexpr size_t ADJ_DY = (size_t)2 * IH * TX * sizeof(float);   // rows y0-4.., cols x0..
__host__ __device__ constexpr size_t adj_smem(bool tti)
{
    return ADJ_NSTAGE * adj_stage(tti) + ADJ_TXX + ADJ_TYY + ADJ_TXY + ADJ_TYZ + ADJ_TZX + ADJ_DX + ADJ_DY +
           ADJ_NSTAGE * sizeof(uint64_t);
}
static_assert(adj_smem(true) <= 227 * 1024, "adjoint staging and tiles fit one CTA's shared memory");

struct AdjMaps {
    CUtensorMap p, q;  // box PW x PH
    CUtensorMap ma;    // 4D (4, x, y, z), box 4 x PW x PH
    CUtensorMap mb;    // TTI: 4D like ma; VTI: irho, box PW x PH
};

template <bool TTI>
__global__ void __launch_bounds__(NT, 1) k_fused_adjoint(const __grid_constant__ AdjMaps tm, const AdjParams a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr size_t STAGE = adj_stage(TTI);
    unsigned char* stage = smem;
    unsigned char* sp = smem + ADJ_NSTAGE * STAGE;
    // temporaries and derivative tiles: both fields of a cell side by side
    float2* txx = reinterpret_cast<float2*>(sp);  // [TY][PW]
    sp += ADJ_TXX;
    float2* tyy = reinterpret_cast<float2*>(sp);  // [PH][TX]
    sp += ADJ_TYY;
    float2* txy = reinterpret_cast<float2*>(sp);  // [IH][IW]
    sp += ADJ_TXY;
    float2* tyz = reinterpret_cast<float2*>(sp);  // [IH][TX]
    sp += ADJ_TYZ;
    float2* tzx = reinterpret_cast<float2*>(sp);  // [TY][IW]
    sp += ADJ_TZX;
    float2* dxs = reinterpret_cast<float2*>(sp);  // [TY][IW]
    sp += ADJ_DX;
    float2* dys = reinterpret_cast<float2*>(sp);  // [IH][TX]
    sp += ADJ_DY;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sp);

    const Layout& L = a.L;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int warp = tid >> 5, lane = tid & 31;
    bool dead = false;
    bool stop = false;             // the CTA gave up (a bounded wait timed out)
    int g_issued = 0, g_wait = 0;  // planes issued (thread 0) / plane last waited on

    if (tid == 0) {
        for (int s = 0; s < ADJ_NSTAGE; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    int s = 0;
    uint32_t phase = 0;
    int gbase = 0;  // planes consumed by earlier segments
    WorkRange wr(L, a.bz, a.ztop);
    for (Segment sg; wr.next(sg); gbase += sg.len + 2 * LAG) {
    const int x0 = sg.x0, y0 = sg.y0, zs = sg.zs;
    const int ntot = sg.len + 2 * LAG;
    const int x = x0 + tx, y = y0 + ty;
    const bool owner = (x <= L.ixend) && (y <= L.iyend);
    if (__syncthreads_or(dead)) {  // barriers initialised; the previous segment is done with the stages
        stop = true;
        break;
    }

    auto issue = [&](int t) {
        ++g_issued;
        const int sl = (gbase + t) % ADJ_NSTAGE, z = zs - LAG + t;
        unsigned char* dst = stage + (size_t)sl * STAGE;
        mbar_expect_tx(&bars[sl], (uint32_t)STAGE);
        tma_load_3d(dst, &tm.p, x0 - 8, y0 - 8, z, &bars[sl]);
        tma_load_3d(dst + ADJ_F1, &tm.q, x0 - 8, y0 - 8, z, &bars[sl]);
        tma_load_4d(dst + 2 * ADJ_F1, &tm.ma, 0, x0 - 8, y0 - 8, z, &bars[sl]);
        if constexpr (TTI)
            tma_load_4d(dst + 2 * ADJ_F1 + ADJ_F4, &tm.mb, 0, x0 - 8, y0 - 8, z, &bars[sl]);
        else
            tma_load_3d(dst + 2 * ADJ_F1 + ADJ_F4, &tm.mb, x0 - 8, y0 - 8, z, &bars[sl]);
    };
    if (tid == 0)
        for (int t = 0; t < ADJ_PF && t < ntot; ++t) issue(t);

    // register queues, both fields of a cell in one pair
    float2 dzq[8];  // D- partial sums, positions L-3 .. L+4
    float2 dZ[8];   // buoyancy-scaled z derivatives, positions L-10 .. L-3
    float2 mq[8];   // yz/zx parts of outputs L-4 .. L+3 (before plane L)
    float2 sxy[8];  // completed in-plane parts (x, y, xy, and yz/zx once complete), outputs L-7 .. L
    float irq[4];   // buoyancy of this column, planes L-3 .. L
    const float2 sx = owner ? __ldg(a.abx + x) : make_float2(1.0f, 1.0f);
    const float2 sy = owner ? __ldg(a.aby + y) : make_float2(1.0f, 1.0f);
#pragma unroll
    for (int j = 0; j < 8; ++j) dzq[j] = dZ[j] = mq[j] = sxy[j] = f2(0.0f);
#pragma unroll
    for (int j = 0; j < 4; ++j) irq[j] = 0.0f;

    for (int t = 0; t < ntot; ++t) {
        // Stage (t+2)%3 was last read in iteration t-1, before its second barrier.
        if (tid == 0 && t + ADJ_PF < ntot) {
            fence_proxy_async();
            issue(t + ADJ_PF);
        }
        const int Lz = zs - LAG + t;
        // point-wise values of the output plane L-7, loaded ahead of their use
        const int zo = Lz - LAG;
        const bool out_here = (zo >= zs) && owner;
        const int64_t go = L.idx(x, y, max(zo, 0));
        float2 o34 = f2(0.0f), opq = f2(0.0f);
        float2 osz = make_float2(1.0f, 1.0f);
        if (out_here) {
            o34 = make_float2(a.f3[go], a.f4[go]);
            opq = make_float2(__ldg(a.pin + go), __ldg(a.qin + go));
            osz = __ldg(a.abz + zo);
        }
        g_wait = gbase + t;
        mbar_wait(&bars[s], phase, a.err, dead);
        const unsigned char* st = stage + (size_t)s * STAGE;
        const float* SP = reinterpret_cast<const float*>(st);
        const float* SQ = SP + PH * PW;
        const float4* SMA = reinterpret_cast<const float4*>(st + 2 * ADJ_F1);
        const float4* SMB = reinterpret_cast<const float4*>(st + 2 * ADJ_F1 + ADJ_F4);  // TTI
        const float* SIR = reinterpret_cast<const float*>(st + 2 * ADJ_F1 + ADJ_F4);    // VTI
        // transposed model at staging offset k (kernel_type2_grad_snap.cu:98-129):
        // S = (m1 p + m2 q, m4 q), H = ((m4 - m1) p - m2 q, m2 p + (m3 - m4) q)
        auto base = [&](int k, float2& S, float2& H) {
            const float p = SP[k], q = SQ[k];
            const float4 m = SMA[k];
            S = fma2(make_float2(m.y, m.w), f2(q), make_float2(m.x * p, 0.0f));
            H = fma2(make_float2(m.w - m.x, m.z - m.w), make_float2(p, q), make_float2(-(m.y * q), m.y * p));
        };
        // (irho, rx, ry, rz) at staging offset k
        auto geo = [&](int k) {
            if constexpr (TTI) return SMB[k];
            else return make_float4(SIR[k], 0.0f, 0.0f, 1.0f);
        };

        // (1) temporaries of plane L.  Position (r, c) of the staging tile
        //     (y = y0-8+r, x = x0-8+c) feeds xx if 8<=r<24; yy if 8<=c<40;
        //     xy if 4<=r<28 and 4<=c<44; yz if 4<=r<28 and 8<=c<40; zx if
        //     8<=r<24 and 4<=c<44.
        // core (r, c) = (ty+8, tx+8): all of them, and this column's zz
        float2 tz;
        float irc;  // buoyancy of this column at plane L
        {
            const int k = (ty + 8) * PW + tx + 8;
            float2 S, H;
            base(k, S, H);
            const float4 g = geo(k);
            irc = g.x;
            const float2 rho = f2(rcp_approx(g.x));
            txx[ty * PW + tx + 8] = mul2(rho, fma2(f2(g.y * g.y), H, S));
            tyy[(ty + 8) * TX + tx] = mul2(rho, fma2(f2(g.z * g.z), H, S));
            tz = mul2(rho, fma2(f2(g.w * g.w), H, S));
            if constexpr (TTI) {
                txy[(ty + 4) * IW + tx + 4] = mul2(f2(2.0f * g.y * g.z), H);
                tyz[(ty + 4) * TX + tx] = mul2(f2(2.0f * g.z * g.w), H);
                tzx[ty * IW + tx + 4] = mul2(f2(2.0f * g.w * g.y), H);
            }
        }
        // rows above and below the core, columns 8..39: yy (rows 0..3, 28..31),
        // yy + xy + yz (rows 4..7, 24..27); one row per warp
        {
            const bool inner = warp >= 8;  // rows 4..7, 24..27
            const int w = warp & 7;
            const int r = inner ? (w < 4 ? 4 + w : 20 + w) : (w < 4 ? w : 24 + w);
            const int c = 8 + lane;
            const int k = r * PW + c;
            float2 S, H;
            base(k, S, H);
            const float4 g = geo(k);
            tyy[r * TX + lane] = mul2(f2(rcp_approx(g.x)), fma2(f2(g.z * g.z), H, S));
            if constexpr (TTI) {
                if (inner) {
                    txy[(r - 4) * IW + c - 4] = mul2(f2(2.0f * g.y * g.z), H);
                    tyz[(r - 4) * TX + lane] = mul2(f2(2.0f * g.z * g.w), H);
                }
            }
        }
        // columns left and right of the core, rows 8..23: xx (columns 0..3,
        // 44..47; warps 0..3), xx + xy + zx (columns 4..7, 40..43; warps
        // 4..7); the xy corners (rows 4..7, 24..27 x columns 4..7, 40..43;
        // warps 8, 9)
        if (warp < 8) {
            const bool inner = warp >= 4;
            const int r = 8 + 4 * (warp & 3) + (lane >> 3), cc = lane & 7;
            const int c = inner ? (cc < 4 ? 4 + cc : 36 + cc) : (cc < 4 ? cc : 40 + cc);
            const int k = r * PW + c;
            float2 S, H;
            base(k, S, H);
            const float4 g = geo(k);
            txx[(r - 8) * PW + c] = mul2(f2(rcp_approx(g.x)), fma2(f2(g.y * g.y), H, S));
            if constexpr (TTI) {
                if (inner) {
                    txy[(r - 4) * IW + c - 4] = mul2(f2(2.0f * g.y * g.z), H);
                    tzx[(r - 8) * IW + c - 4] = mul2(f2(2.0f * g.w * g.y), H);
                }
            }
        } else if (TTI && warp < 10) {
            const int i = (warp - 8) * 32 + lane, rr = i >> 3, cc = i & 7;
            const int r = rr < 4 ? 4 + rr : 20 + rr, c = cc < 4 ? 4 + cc : 36 + cc;
            const int k = r * PW + c;
            float2 S, H;
            base(k, S, H);
            const float4 g = geo(k);
            txy[(r - 4) * IW + c - 4] = mul2(f2(2.0f * g.y * g.z), H);
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) irq[j] = irq[j + 1];
        irq[3] = irc;
        if (__syncthreads_or(dead)) {  // temporaries of plane L are ready
            stop = true;
            break;
        }

        // (2) buoyancy-scaled x/y derivatives of plane L (compute_xy_contributions)
        // dxs[r][c]: x = x0-4+c, y = y0+r;  dys[r][c]: x = x0+c, y = y0-4+r
        auto dx_at = [&](int r, int c, float irv) {
            const bool in = (x0 - 4 + c >= L.ixbeg) && (x0 - 4 + c <= L.ixend);
            const float2* T = txx + r * PW + c + 4;
            float2 acc = f2(0.0f);
#pragma unroll
            for (int i = 1; i <= 4; ++i) acc = fma2(a.kd[0][i - 1], sub2(T[i - 1], T[-i]), acc);
            dxs[r * IW + c] = in ? mul2(acc, f2(irv)) : f2(0.0f);
        };
        auto dy_at = [&](int r, int c, float irv) {
            const bool in = (y0 - 4 + r >= L.iybeg) && (y0 - 4 + r <= L.iyend);
            const float2* T = tyy + (r + 4) * TX + c;
            float2 acc = f2(0.0f);
#pragma unroll
            for (int i = 1; i <= 4; ++i) acc = fma2(a.kd[1][i - 1], sub2(T[(i - 1) * TX], T[-i * TX]), acc);
            dys[r * TX + c] = in ? mul2(acc, f2(irv)) : f2(0.0f);
        };
        dx_at(ty, tx + 4, irc);
        dy_at(ty + 4, tx, irc);
        if (warp < 4) {  // x halo of dxs: columns 0..3, 36..39
            const int i = warp * 32 + lane, r = i >> 3, cc = i & 7;
            const int c = cc < 4 ? cc : 32 + cc;
            dx_at(r, c, geo((r + 8) * PW + c + 4).x);
        } else if (warp < 12) {  // y halo of dys: rows 0..3, 20..23
            const int w = warp - 4;
            const int r = w < 4 ? w : 16 + w;
            dy_at(r, lane, geo((r + 4) * PW + lane + 8).x);
        }
        // (3) D- z stage (compute_z_contributionsdtd), completes position L-3
#pragma unroll
        for (int j = 0; j < 8; ++j) dzq[j] = fma2(a.kzm[j], tz, dzq[j]);
        {
            const int zp = Lz - 3;
            const bool valid = (zp >= L.izbeg + (a.fs ? 1 : 0)) && zp <= L.izend;
            const float2 n = valid ? mul2(dzq[0], f2(irq[0])) : f2(0.0f);
#pragma unroll
            for (int j = 0; j < 7; ++j) {
                dZ[j] = dZ[j + 1];
                dzq[j] = dzq[j + 1];
            }
            dZ[7] = n;
            dzq[7] = f2(0.0f);
        }
        // (4) yz/zx rhs: scatter of plane L into outputs L-4 .. L+4; output
        //     L-4 is then complete and moves to the in-plane queue
        float2 xy34 = f2(0.0f);
        if constexpr (TTI) {
            // differences around this column, once per distance i: plane L
            // adds c2(i)*(T[+i] - T[-i]) to output L-i and its negative to L+i
            float2 dyz[4], dzx[4];
#pragma unroll
            for (int i = 1; i <= 4; ++i) {
                dyz[i - 1] = sub2(tyz[(ty + 4 + i) * TX + tx], tyz[(ty + 4 - i) * TX + tx]);
                dzx[i - 1] = sub2(tzx[ty * IW + tx + 4 + i], tzx[ty * IW + tx + 4 - i]);
            }
            float2 top = f2(0.0f);  // output L+4
#pragma unroll
            for (int ir = -4; ir <= 4; ++ir) {
                if (ir == 0) continue;
                const int i = ir < 0 ? -ir : ir;
                float2& o = (ir == -4) ? top : mq[4 - ir];  // output L - ir
                o = fma2(a.kyz[ir + 4], dyz[i - 1], o);
                o = fma2(a.kzx[ir + 4], dzx[i - 1], o);
            }
            sxy[3] = add2(sxy[3], mq[0]);  // output L-4 is complete
#pragma unroll
            for (int j = 0; j < 7; ++j) mq[j] = mq[j + 1];
            mq[7] = top;
            // xy of output L from plane L
            const int cc = tx + 4, rr = ty + 4;
#pragma unroll
            for (int k = 1; k <= 4; ++k) {
                const float2 pp = txy[(rr + k) * IW + cc + k], pm = txy[(rr + k) * IW + cc - k];
                const float2 mm = txy[(rr - k) * IW + cc - k], mp = txy[(rr - k) * IW + cc + k];
                xy34 = fma2(a.kxy[k - 1], sub2(add2(sub2(pp, pm), mm), mp), xy34);
            }
        }
        __syncthreads();  // dxs/dys of plane L are ready

        // (5) x+y parts of output L (dfdx_stg_right, kernel_type2_adj.cu:85-98)
        {
            float2 acc = xy34;
#pragma unroll
            for (int k = 1; k <= 4; ++k) {
                acc = fma2(a.kd[0][k - 1], sub2(dxs[ty * IW + tx + 4 + k], dxs[ty * IW + tx + 5 - k]), acc);
                acc = fma2(a.kd[1][k - 1], sub2(dys[(ty + 4 + k) * TX + tx], dys[(ty + 5 - k) * TX + tx]), acc);
            }
            sxy[7] = acc;
        }
        // (6) output plane L-7
        const int z = zo;
        if (out_here) {
            const int64_t gi = go;
            if (a.res) {  // residual injection, the transpose of the pressure receiver
                const int off = receiver_plane(a.rec, z);
                if (off >= 0) {
                    const int r = __ldg(a.rec.xy + off + (y - L.iybeg) * L.nx() + (x - L.ixbeg));
                    if (r >= 0) {
                        const float v = a.obs ? a.res[r] - a.obs[r] : a.res[r];
                        o34.x += (-2.0f / 3.0f) * v;
                        o34.y += (-1.0f / 3.0f) * v;
                    }
                }
            }
            if (z == a.src_z && gi == a.src_index) *a.srctr = opq.x + opq.y;
            float2 q[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) q[j] = dZ[j];
            if (a.fs) resolve_dz(q, z - L.izbeg);
            float2 r34 = sxy[0];
#pragma unroll
            for (int k = 1; k <= 4; ++k) r34 = fma2(a.kd[2][k - 1], sub2(q[3 + k], q[4 - k]), r34);
            const float2 sz = osz;
            float2 n34;
            if (a.sponge) {
                const float A = fminf(fminf(sx.x, sy.x), sz.x);
                const float B = fminf(fminf(sx.y, sy.y), sz.y) * a.dt;
                n34 = fma2(f2(B), r34, mul2(f2(A), o34));
            } else {
                n34 = fma2(r34, f2(a.dt), o34);
            }
            a.f3[gi] = n34.x;
            a.f4[gi] = n34.y;
            // loop2 (kernel_base.cu:92-101) and free surface (:142-162)
            const float A = fminf(sx.x, fminf(sy.x, sz.x));
            const float B = fminf(sx.y, fminf(sy.y, sz.y));
            float2 npq = fma2(mul2(f2(B), n34), f2(a.dt), mul2(f2(A), opq));
            if (a.fs && z == L.izbeg) npq = f2(0.0f);
            wave_apply(a.wave_prec, a.wave_scale, npq.x, npq.y);
            a.pout[gi] = npq.x;
            a.qout[gi] = npq.y;
            if (a.fs && z > L.izbeg && z <= L.izbeg + kRadius) {
                const int64_t gm = L.idx(x, y, 2 * L.izbeg - z);
                a.pout[gm] = -npq.x;
                a.qout[gm] = -npq.y;
            }
        }
        // (7) rotate the in-plane queue
#pragma unroll
        for (int j = 0; j < 7; ++j) sxy[j] = sxy[j + 1];
        if (++s == ADJ_NSTAGE) {
            s = 0;
            phase ^= 1u;
        }
    }
    if (stop) break;
    }  // segments
    if (stop && tid == 0) drain_loads(bars, ADJ_NSTAGE, g_wait, g_issued);
}

// ---------------------------------------------------------------------------
// Fused imaging at a snapshot step: the reference's update_grad_loop_1
// (Vp image, kernel_type2_small.cu:42-59), snaps_loop (forward derivatives of
// the stored p/q, kernel_type2.cu:295-303), kernel_loop4_derivative and
// update_grad_loop_2 (density gradient, kernel_type2_grad.cu:344-509) in one
// z-marching pass.  The stored p/q come from the device snapshot store (dense
// interior volumes, free-surface halo re-derived by mirroring); the adjoint
// temporaries adj_a = rho*(s1 + ra^2 h1) come from the current adjoint p/q.
struct ImgParams {
    const float* snap_scale;    // the 4 multipliers the slot was stored with
    float *gvp, *grho;           // dense images
    Layout L;
    int bz;
    int ztop;
    int fs;
    int slot;                    // snapshot index in the store
    float hx, hy, hz;
    int* err;
    // stg_d1 coefficients with the grid spacings folded in, as (c, c) pairs
    float2 kcx[4], kcy[4], kcz[4];  // cs(r)/dx, /dy, /dz
    float2 kcxn[4], kcyn[4];        // -cs(r)/dx, -cs(r)/dy
};

constexpr int IMG_NSTAGE = 3;
constexpr int IMG_PF = 2;
// Staging per plane: the stored p, q (storage type, halo 8), then the
// adjoint p, q (float) and the interleaved model (m1, m2, m3, m4) and
// (irho, rx, ry, rz) (float4; VTI: irho as float), halo 4.
__host__ __device__ constexpr size_t img_p(size_t elt) { return (size_t)PH * PW * elt; }
constexpr size_t IMG_A = (size_t)IH * IW * sizeof(float);
constexpr size_t IMG_A4 = (size_t)IH * IW * sizeof(float4);
// then the point-wise values of the plane's output columns (TX x TY, no
// halo): the stored pdot, qdot (storage type), the adjoint pdot, qdot and the
// Vp image at this plane, and the density gradient at plane L-7 (float)
__host__ __device__ constexpr size_t img_halo_part(size_t elt, bool tti)
{
    return 2 * img_p(elt) + 2 * IMG_A + IMG_A4 + (tti ? IMG_A4 : IMG_A);
}
__host__ __device__ constexpr size_t img_stage(size_t elt, bool tti)
{
    return img_halo_part(elt, tti) + (size_t)TX * TY * (2 * elt + 4 * sizeof(float));
}
constexpr size_t IMG_T1 = (size_t)2 * TY * IW * sizeof(float);  // x-type tiles: rows y0.., cols x0-4..
constexpr size_t IMG_T2 = (size_t)2 * IH * TX * sizeof(float);  // y-type tiles: rows y0-4.., cols x0..
__host__ __device__ constexpr size_t img_smem(size_t elt, bool tti)
{
    return IMG_NSTAGE * img_stage(elt, tti) + 2 * IMG_T1 + 2 * IMG_T2 + IMG_NSTAGE * sizeof(uint64_t);
}

struct ImgMaps {
    CUtensorMap snap;   // 4D over the store: (nx, ny, nz, 4*nsnap), box PW x PH
    CUtensorMap p, q;   // adjoint p, q: box IW x IH
    CUtensorMap ma;     // 4D (4, x, y, z), box 4 x IW x IH
    CUtensorMap mb;     // TTI: like ma; VTI: irho, box IW x IH
    CUtensorMap snapc;  // the store again, box TX x TY
    CUtensorMap f3, f4; // adjoint pdot, qdot: box TX x TY
    CUtensorMap gv, gr; // the dense images (nx, ny, nz, 1): box TX x TY
};


template <bool TTI, typename T>
__global__ void __launch_bounds__(NT, 1) k_fused_image(const __grid_constant__ ImgMaps tm, const ImgParams a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr size_t IMG_P = img_p(sizeof(T));
    constexpr size_t IMG_STAGE = img_stage(sizeof(T), TTI);
    constexpr size_t IMG_CT = (size_t)TX * TY * sizeof(T);  // one point-wise tile of the storage type
    unsigned char* stage = smem;
    unsigned char* sp = smem + IMG_NSTAGE * IMG_STAGE;
    // x-type and y-type tiles, one float4 per cell: forward derivative of
    // field 1 and 2, adjoint temporary of field 1 and 2
    static_assert((IMG_NSTAGE * IMG_STAGE) % 16 == 0 && IMG_T1 % 16 == 0, "float4 tiles");
    float4* xs = reinterpret_cast<float4*>(sp);  // [TY][IW]
    sp += 2 * IMG_T1;
    float4* ys = reinterpret_cast<float4*>(sp);  // [IH][TX]
    sp += 2 * IMG_T2;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sp);

    const Layout& L = a.L;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int nx = L.nx(), ny = L.ny();
    bool dead = false;
    bool stop = false;             // the CTA gave up (a bounded wait timed out)
    int g_issued = 0, g_wait = 0;  // planes issued (thread 0) / plane last waited on
    constexpr uint32_t TX_BYTES = (uint32_t)IMG_STAGE;
    // stored values are value*scale with a power-of-two scale: undo exactly
    float us1 = 1.0f, us2 = 1.0f, us3 = 1.0f, us4 = 1.0f;
    if (a.snap_scale) {
        us3 = 1.0f / a.snap_scale[0];
        us4 = 1.0f / a.snap_scale[1];
        us1 = 1.0f / a.snap_scale[2];
        us2 = 1.0f / a.snap_scale[3];
    }
    // unscaling of the stored p, q folded into the derivative scales (exact:
    // powers of two)
    const float2 ux = make_float2(us1 * a.hx, us2 * a.hx), uy = make_float2(us1 * a.hy, us2 * a.hy);
    const float2 uz = make_float2(us1 * a.hz, us2 * a.hz), u12 = make_float2(us1, us2);

    if (tid == 0) {
        for (int s = 0; s < IMG_NSTAGE; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    int s = 0;
    uint32_t phase = 0;
    int gbase = 0;  // planes consumed by earlier segments
    WorkRange wr(L, a.bz, a.ztop);
    for (Segment sg; wr.next(sg); gbase += sg.len + 2 * LAG) {
    const int x0 = sg.x0, y0 = sg.y0, zs = sg.zs;
    const int xd0 = x0 - L.ixbeg, yd0 = y0 - L.iybeg;  // dense (interior) origin
    const int ze = zs + sg.len - 1;
    const int ntot = sg.len + 2 * LAG;
    const int x = x0 + tx, y = y0 + ty;
    const bool owner = (x <= L.ixend) && (y <= L.iyend);
    if (__syncthreads_or(dead)) {  // barriers initialised; the previous segment is done with the stages
        stop = true;
        break;
    }

    // plane z of the stored p/q: dense z = z - izbeg; above the surface the
    // free surface mirrors it (2*izbeg - z), without one it is zero halo.
    auto issue = [&](int t) {
        ++g_issued;
        const int s = (gbase + t) % IMG_NSTAGE, z = zs - LAG + t;
        unsigned char* dst = stage + (size_t)s * IMG_STAGE;
        mbar_expect_tx(&bars[s], TX_BYTES);
        int zd = z - L.izbeg;
        if (a.fs && zd < 0) zd = -zd;
        tma_load_4d(dst, &tm.snap, xd0 - 8, yd0 - 8, zd, 4 * a.slot + 2, &bars[s]);
        tma_load_4d(dst + IMG_P, &tm.snap, xd0 - 8, yd0 - 8, zd, 4 * a.slot + 3, &bars[s]);
        unsigned char* adst = dst + 2 * IMG_P;
        tma_load_3d(adst, &tm.p, x0 - 4, y0 - 4, z, &bars[s]);
        tma_load_3d(adst + IMG_A, &tm.q, x0 - 4, y0 - 4, z, &bars[s]);
        tma_load_4d(adst + 2 * IMG_A, &tm.ma, 0, x0 - 4, y0 - 4, z, &bars[s]);
        if constexpr (TTI)
            tma_load_4d(adst + 2 * IMG_A + IMG_A4, &tm.mb, 0, x0 - 4, y0 - 4, z, &bars[s]);
        else
            tma_load_3d(adst + 2 * IMG_A + IMG_A4, &tm.mb, x0 - 4, y0 - 4, z, &bars[s]);
        // point-wise values (zero-filled where z or z-LAG is outside the grid)
        unsigned char* cdst = dst + img_halo_part(sizeof(T), TTI);
        const int zc = z - L.izbeg;
        tma_load_4d(cdst, &tm.snapc, xd0, yd0, zc, 4 * a.slot, &bars[s]);
        tma_load_4d(cdst + IMG_CT, &tm.snapc, xd0, yd0, zc, 4 * a.slot + 1, &bars[s]);
        float* cf = reinterpret_cast<float*>(cdst + 2 * IMG_CT);
        tma_load_3d(cf, &tm.f3, x0, y0, z, &bars[s]);
        tma_load_3d(cf + TX * TY, &tm.f4, x0, y0, z, &bars[s]);
        tma_load_4d(cf + 2 * TX * TY, &tm.gv, xd0, yd0, zc, 0, &bars[s]);
        tma_load_4d(cf + 3 * TX * TY, &tm.gr, xd0, yd0, zc - LAG, 0, &bars[s]);
    };
    if (tid == 0)
        for (int t = 0; t < IMG_PF && t < ntot; ++t) issue(t);

    // register queues, both fields of a cell in one pair
    float2 dzq[8];   // D- partial sums of the stored p/q, positions L-3 .. L+4
    float2 fz[8];    // forward z derivatives, positions L-10 .. L-3
    float2 azq[12];  // adjoint z temporaries, planes L-11 .. L
    float rxy[8];    // x+y part of the gradient rhs, outputs L-7 .. L
    float irq[8];    // buoyancy of this column, planes L-7 .. L
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        dzq[j] = fz[j] = f2(0.0f);
        rxy[j] = irq[j] = 0.0f;
    }
#pragma unroll
    for (int j = 0; j < 12; ++j) azq[j] = f2(0.0f);

    for (int t = 0; t < ntot; ++t) {
        if (__syncthreads_or(dead)) {  // the x/y tiles of plane L-1 have been read by every thread
            stop = true;
            break;
        }
        if (tid == 0 && t + IMG_PF < ntot) {
            fence_proxy_async();
            issue(t + IMG_PF);
        }
        const int Lz = zs - LAG + t;
        const bool vp_here = owner && Lz >= zs && Lz <= ze;
        const bool rho_here = owner && (Lz - LAG) >= zs;
        const int64_t dvp = ((int64_t)(Lz - L.izbeg) * ny + (y - L.iybeg)) * nx + (x - L.ixbeg);
        const int64_t drho = dvp - (int64_t)LAG * nx * ny;
        g_wait = gbase + t;
        mbar_wait(&bars[s], phase, a.err, dead);
        unsigned char* st = stage + (size_t)s * IMG_STAGE;
        // point-wise values of this column, staged with the plane
        float ps3, ps4, pa3, pa4, pgv, pgr;
        {
            const unsigned char* cst = st + img_halo_part(sizeof(T), TTI);
            const T* S3 = reinterpret_cast<const T*>(cst);
            const float* CF = reinterpret_cast<const float*>(cst + 2 * IMG_CT);
            const int kc0 = ty * TX + tx;
            ps3 = to_f32(S3[kc0]) * us3;
            ps4 = to_f32(S3[TX * TY + kc0]) * us4;
            pa3 = CF[kc0];
            pa4 = CF[TX * TY + kc0];
            pgv = CF[2 * TX * TY + kc0];
            pgr = CF[3 * TX * TY + kc0];
        }
        const bool mirrored = a.fs && Lz < L.izbeg;
        if (mirrored) {  // block-uniform
            T* pt = reinterpret_cast<T*>(st);
            for (int e = tid; e < 2 * PH * PW; e += NT) pt[e] = T(-to_f32(pt[e]));
            __syncthreads();
        }
        const T* P1 = reinterpret_cast<const T*>(st);
        const T* P2 = P1 + PH * PW;
        const float* AP = reinterpret_cast<const float*>(st + 2 * IMG_P);
        const float* AQ = AP + IH * IW;
        const float4* AMA = reinterpret_cast<const float4*>(st + 2 * IMG_P + 2 * IMG_A);
        const float4* AMB = AMA + IH * IW;                                // TTI
        const float* AIR = reinterpret_cast<const float*>(AMA + IH * IW);  // VTI
        // (irho, rx, ry, rz) at offset k of the halo-4 tiles
        auto geo = [&](int k) {
            if constexpr (TTI) return AMB[k];
            else return make_float4(AIR[k], 0.0f, 0.0f, 1.0f);
        };
        // adjoint temporary rho*(S + r^2 H) at offset k (kernel_type2_grad.cu:
        // 435-439), S = (m1 p + m2 q, m4 q), H = ((m4 - m1) p - m2 q, m2 p + (m3 - m4) q)
        auto adj_t = [&](int k, float irho, float ra) {
            const float p = AP[k], q = AQ[k];
            const float4 m = AMA[k];
            const float2 S = fma2(make_float2(m.y, m.w), f2(q), make_float2(m.x * p, 0.0f));
            const float2 H = fma2(make_float2(m.w - m.x, m.z - m.w), make_float2(p, q), make_float2(-(m.y * q), m.y * p));
            return mul2(f2(rcp_approx(irho)), fma2(f2(ra * ra), H, S));
        };
        const int kc = (ty + 4) * IW + tx + 4;  // this column in a halo-4 tile
        // the stored (p, q) pair at offset k of the halo-8 tiles
        auto spq = [&](int k) { return make_float2(to_f32(P1[k]), to_f32(P2[k])); };

        // (1) forward x/y derivatives of the stored p/q (fwd_drv) and the
        //     adjoint x/y temporaries of plane L.
        //     x-type tiles [r][c]: x = x0-4+c, y = y0+r; y-type: x = x0+c, y = y0-4+r
        auto xt_at = [&](int r, int c) {
            const bool in = (x0 - 4 + c >= L.ixbeg) && (x0 - 4 + c <= L.ixend);
            const int k = (r + 4) * IW + c;
            const float4 g = geo(k);
            const int k0 = (r + 8) * PW + c + 4;
            float2 acc = f2(0.0f);
#pragma unroll
            for (int i = 1; i <= 4; ++i) acc = fma2(f2(c1(i)), sub2(spq(k0 + i - 1), spq(k0 - i)), acc);
            acc = in ? mul2(mul2(acc, ux), f2(g.x)) : f2(0.0f);
            const float2 t2 = adj_t(k, g.x, g.y);
            xs[r * IW + c] = make_float4(acc.x, acc.y, t2.x, t2.y);
        };
        auto yt_at = [&](int r, int c) {
            const bool in = (y0 - 4 + r >= L.iybeg) && (y0 - 4 + r <= L.iyend);
            const int k = r * IW + c + 4;
            const float4 g = geo(k);
            const int k0 = (r + 4) * PW + c + 8;
            float2 acc = f2(0.0f);
#pragma unroll
            for (int i = 1; i <= 4; ++i) acc = fma2(f2(c1(i)), sub2(spq(k0 + (i - 1) * PW), spq(k0 - i * PW)), acc);
            acc = in ? mul2(mul2(acc, uy), f2(g.x)) : f2(0.0f);
            const float2 t2 = adj_t(k, g.x, g.z);
            ys[r * TX + c] = make_float4(acc.x, acc.y, t2.x, t2.y);
        };
        xt_at(ty, tx);
        // halos spread over warps 0..3 (x) and 4..11 (y): at most three
        // tile cells per warp
        if (tid < (IW - TX) * TY) xt_at(tid / (IW - TX), TX + tid % (IW - TX));
        yt_at(ty, tx);
        if (ty >= 4 && ty < 4 + IH - TY) yt_at(ty - 4 + TY, tx);
        // (2) column values: z temporaries, buoyancy, D- z stage of the stored p/q
        {
            const float4 g = geo(kc);
            const float2 t2 = adj_t(kc, g.x, g.w);
#pragma unroll
            for (int j = 0; j < 11; ++j) azq[j] = azq[j + 1];
            azq[11] = t2;
#pragma unroll
            for (int j = 0; j < 7; ++j) irq[j] = irq[j + 1];
            irq[7] = g.x;
            const float2 v = spq((ty + 8) * PW + tx + 8);
#pragma unroll
            for (int j = 0; j < 8; ++j) dzq[j] = fma2(f2(dminus_coef(j)), v, dzq[j]);
            const int zp = Lz - 3;
            const bool valid = (zp >= L.izbeg + (a.fs ? 1 : 0)) && zp <= L.izend;
            const float ir3 = irq[4];  // plane L-3
            const float2 n = valid ? mul2(mul2(dzq[0], uz), f2(ir3)) : f2(0.0f);
#pragma unroll
            for (int j = 0; j < 7; ++j) {
                fz[j] = fz[j + 1];
                dzq[j] = dzq[j + 1];
            }
            fz[7] = n;
            dzq[7] = f2(0.0f);
        }
        if (__syncthreads_or(dead)) {  // x/y tiles of plane L ready; staging slot s fully consumed
            stop = true;
            break;
        }

        // (3) x+y part of the gradient rhs at plane L (compute_xy_contributions
        //     of kernel_type2_grad.cu:314-342 and :435-439) and the Vp image
        {
            const int cx = ty * IW + tx + 4;    // x in the x-type tiles
            const int cy = (ty + 4) * TX + tx;  // y in the y-type tiles
            // positions -4 .. +4 around the cell, one 128-bit load each, folded
            // into the staggered sums as they arrive (D+ of the forward
            // derivatives uses -3..+4, D- of the adjoint temporaries -4..+3)
            float2 dfx = f2(0.0f), dfy = f2(0.0f), dax = f2(0.0f), day = f2(0.0f);
            float4 xc, yc;
#pragma unroll
            for (int j = 0; j < 9; ++j) {
                const float4 u = xs[cx - 4 + j], w = ys[cy + (j - 4) * TX];
                const float2 uf = make_float2(u.x, u.y), ua = make_float2(u.z, u.w);
                const float2 wf = make_float2(w.x, w.y), wa = make_float2(w.z, w.w);
                if (j >= 5) {
                    dfx = fma2(a.kcx[j - 5], uf, dfx);
                    dfy = fma2(a.kcy[j - 5], wf, dfy);
                }
                if (j >= 1 && j <= 4) {
                    dfx = fma2(a.kcxn[4 - j], uf, dfx);
                    dfy = fma2(a.kcyn[4 - j], wf, dfy);
                }
                if (j >= 4 && j <= 7) {
                    dax = fma2(a.kcx[j - 4], ua, dax);
                    day = fma2(a.kcy[j - 4], wa, day);
                }
                if (j <= 3) {
                    dax = fma2(a.kcxn[3 - j], ua, dax);
                    day = fma2(a.kcyn[3 - j], wa, day);
                }
                if (j == 4) {
                    xc = u;
                    yc = w;
                }
            }
            float2 v2 = mul2(make_float2(xc.z, xc.w), dfx);
            v2 = fma2(make_float2(yc.z, yc.w), dfy, v2);
            v2 = fma2(dax, make_float2(xc.x, xc.y), v2);
            v2 = fma2(day, make_float2(yc.x, yc.y), v2);
#pragma unroll
            for (int j = 0; j < 7; ++j) rxy[j] = rxy[j + 1];
            rxy[7] = v2.x + v2.y;
            if (vp_here) a.gvp[dvp] = pgv + (pa3 * ps3 + pa4 * ps4);
        }
        // (4) output plane L-7: z terms and the density gradient
        const int z = Lz - LAG;
        if (rho_here) {
            float2 q[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) q[j] = fz[j];
            if (a.fs) resolve_dz(q, z - L.izbeg);
            // q[j] is position z-3+j; azq[j] is plane z-4+j
            float2 dfz = f2(0.0f), daz = f2(0.0f);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                dfz = fma2(a.kcz[r], sub2(q[4 + r], q[3 - r]), dfz);
                daz = fma2(a.kcz[r], sub2(azq[4 + r], azq[3 - r]), daz);
            }
            float2 r2 = mul2(azq[4], dfz);
            r2 = fma2(daz, q[3], r2);
            const float rhs = rxy[0] + (r2.x + r2.y);
            a.grho[drho] = pgr + -irq[0] * rhs;
        }
        if (++s == IMG_NSTAGE) {
            s = 0;
            phase ^= 1u;
        }
    }
    if (stop) break;
    }  // segments
    if (stop && tid == 0) drain_loads(bars, IMG_NSTAGE, g_wait, g_issued);
}

// ---------------------------------------------------------------------------
// Type1 fused step kernels (constant density, centred second derivatives,
// kernels/kernel_type1_gpu_*.cu).  No first-derivative stage, so every
// stencil reaches only 4 cells: tiles carry a halo of 4 and the output plane
// lags the arriving plane by 4.
constexpr int T1_LAG = 4;
constexpr int T1_NS = 11;  // ring: planes L-8 .. L+2
constexpr int T1_PF = 2;
constexpr size_t T1_SLOT = (size_t)2 * IH * IW * sizeof(float);  // p and q, halo 4
constexpr size_t T1F_SMEM = T1_NS * T1_SLOT + T1_NS * sizeof(uint64_t);

struct T1Fd {
    float xx, yy, zz, xy, yz, zx;  // 1/d^2 and 1/(4 d d') of compute_fd_const
};

struct T1FwdParams {
    float *pout, *qout, *f3, *f4;
    const float *m1, *m2, *m3, *m4, *rx, *ry, *rz;
    const float2 *abx, *aby, *abz;
    void* snap;
    int snap_prec;
    const float* snap_scale;
    unsigned int* snap_amax;
    int64_t src_index;
    float src_term;
    Layout L;
    int bz;
    int ztop;
    int fs;
    int sponge;  // 1: pdot = A pdot + B dt rhs (the launcher's use_sponge)
    float dt;
    T1Fd k;
    int* err;
    int wave_prec;            // 0, or p/q rounded to FP16 (1) / BF16 (2) each step
    const float* wave_scale;  // 2 scales (p, q) of this step's output
};

// Centred second derivatives of one field at one point, scaled by the
// finite-difference constants; sums in the order of compute_z_contributions /
// compute_xy_contributions (kernel_type1_gpu_fwd.cu:150-232).
struct T1Drv {
    float xx, yy, zz, xy, yz, zx;
};

// One fused type1 forward step: the launcher's operator and pdot/qdot update
// (with the sponge form when a.sponge), the point source, the snapshot, then
// the next step's loop2 and free surface, as k_fused_forward does for type2.
// Each thread computes two x-neighbouring outputs (x0+2tx, x0+2tx+1) from
// an 11-plane ring of p,q tiles (halo 4; plane z+ir in slot back(4-ir)),
// reading it with 64-bit loads: an even column pair is one aligned float2, a
// pair that starts on an odd column takes the halves of two.
constexpr int T1X2_TX = TX / 2;  // 16 x 16 threads
constexpr int T1X2_NT = T1X2_TX * TY;

template <int OFF>
__device__ __forceinline__ float2 t1_pair(const float* row, int vc)
{
    // (row[vc+OFF], row[vc+OFF+1]) with vc even
    if constexpr ((OFF & 1) == 0) {
        return *reinterpret_cast<const float2*>(row + vc + OFF);
    } else {
        const float2 lo = *reinterpret_cast<const float2*>(row + vc + OFF - 1);
        const float2 hi = *reinterpret_cast<const float2*>(row + vc + OFF + 1);
        return make_float2(lo.y, hi.x);
    }
}

template <int IR, bool TTI, typename Back>
__device__ __forceinline__ void t1x2_zterm(const float* ring, int field, Back back, int vr, int vc, float2& zz,
                                           float2& zx, float2& yz)
{
    const float c = c2(IR < 0 ? -IR : IR);
    const float* P = ring + (size_t)back(4 - IR) * 2 * IH * IW + field * IH * IW;
    const float2 v = t1_pair<0>(P + vr * IW, vc);
    zz.x = zz.x + c * v.x;
    zz.y = zz.y + c * v.y;
    if constexpr (TTI && IR != 0) {
        const float2 xp = t1_pair<IR>(P + vr * IW, vc), xm = t1_pair<-IR>(P + vr * IW, vc);
        zx.x = zx.x + c * (xp.x - xm.x);
        zx.y = zx.y + c * (xp.y - xm.y);
        const float2 yp = t1_pair<0>(P + (vr + IR) * IW, vc), ym = t1_pair<0>(P + (vr - IR) * IW, vc);
        yz.x = yz.x + c * (yp.x - ym.x);
        yz.y = yz.y + c * (yp.y - ym.y);
    }
}

template <int Q, bool TTI>
__device__ __forceinline__ void t1x2_xyterm(const float* P, int vr, int vc, const float (&w)[10], float2& xx,
                                            float2& yy, float2& xy)
{
    const float c = c2(Q);
    xx.x += c * (w[4 + Q] + w[4 - Q]);
    xx.y += c * (w[5 + Q] + w[5 - Q]);
    const float2 yp = t1_pair<0>(P + (vr + Q) * IW, vc), ym = t1_pair<0>(P + (vr - Q) * IW, vc);
    yy.x += c * (yp.x + ym.x);
    yy.y += c * (yp.y + ym.y);
    if constexpr (TTI) {
        const float2 pp = t1_pair<Q>(P + (vr + Q) * IW, vc), pm = t1_pair<-Q>(P + (vr + Q) * IW, vc);
        const float2 mm = t1_pair<-Q>(P + (vr - Q) * IW, vc), mp = t1_pair<Q>(P + (vr - Q) * IW, vc);
        xy.x += c * (pp.x - pm.x + mm.x - mp.x);
        xy.y += c * (pp.y - pm.y + mm.y - mp.y);
    }
}

struct T1Drv2 {
    T1Drv a, b;
};

template <bool TTI, typename Back>
__device__ __forceinline__ T1Drv2 t1x2_derivs(const float* ring, int field, Back back, int vr, int vc, const T1Fd& k)
{
    float2 zz = make_float2(0.0f, 0.0f), zx = zz, yz = zz;
    t1x2_zterm<-4, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<-3, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<-2, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<-1, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<0, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<1, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<2, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<3, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    t1x2_zterm<4, TTI>(ring, field, back, vr, vc, zz, zx, yz);
    const float* P = ring + (size_t)back(4) * 2 * IH * IW + field * IH * IW;
    float w[10];  // row vr, columns vc-4 .. vc+5
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        const float2 v = *reinterpret_cast<const float2*>(P + vr * IW + vc - 4 + 2 * j);
        w[2 * j] = v.x;
        w[2 * j + 1] = v.y;
    }
    float2 xx = make_float2(c2(0) * w[4], c2(0) * w[5]), yy = xx, xy = make_float2(0.0f, 0.0f);
    t1x2_xyterm<1, TTI>(P, vr, vc, w, xx, yy, xy);
    t1x2_xyterm<2, TTI>(P, vr, vc, w, xx, yy, xy);
    t1x2_xyterm<3, TTI>(P, vr, vc, w, xx, yy, xy);
    t1x2_xyterm<4, TTI>(P, vr, vc, w, xx, yy, xy);
    T1Drv2 d;
    d.a = T1Drv{xx.x * k.xx, yy.x * k.yy, zz.x * k.zz, xy.x * k.xy, yz.x * k.yz, zx.x * k.zx};
    d.b = T1Drv{xx.y * k.xx, yy.y * k.yy, zz.y * k.zz, xy.y * k.xy, yz.y * k.yz, zx.y * k.zx};
    return d;
}

// Operator of one point (compute_result, kernel_type1_gpu_fwd.cu:122-146).
template <bool TTI>
__device__ __forceinline__ void t1_rhs(const T1Drv& d1, const T1Drv& d2, float a1, float a2, float a3, float a4,
                                       float vrx, float vry, float vrz, float& r3, float& r4)
{
    if constexpr (TTI) {
        const float rxx = vrx * vrx, ryy = vry * vry, rzz = vrz * vrz;
        const float rxy = 2.0f * vrx * vry, ryz = 2.0f * vry * vrz, rzx = 2.0f * vrz * vrx;
        const float V1 = rxx * d1.xx + ryy * d1.yy + rzz * d1.zz + rxy * d1.xy + rzx * d1.zx + ryz * d1.yz;
        const float H1 = d1.xx + d1.yy + d1.zz - V1;
        const float V2 = rxx * d2.xx + ryy * d2.yy + rzz * d2.zz + rxy * d2.xy + rzx * d2.zx + ryz * d2.yz;
        const float H2 = d2.xx + d2.yy + d2.zz - V2;
        r3 = a1 * H1 + a4 * V1 + a2 * V2;
        r4 = a2 * H1 + a3 * V2 + a4 * H2;
    } else {
        const float V1 = d1.zz, H1 = d1.xx + d1.yy + d1.zz - V1;
        const float V2 = d2.zz, H2 = d2.xx + d2.yy + d2.zz - V2;
        r3 = a1 * H1 + a4 * V1 + a2 * V2;
        r4 = a2 * H1 + a3 * V2 + a4 * H2;
    }
}

template <bool TTI>
__global__ void __launch_bounds__(T1X2_NT, 2)
    k_t1_fused_forward_x2(const __grid_constant__ CUtensorMap tm_p, const __grid_constant__ CUtensorMap tm_q,
                          const T1FwdParams a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    float* ring = reinterpret_cast<float*>(smem);  // [NS][2][IH][IW]
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + T1_NS * T1_SLOT);
    const Layout& L = a.L;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * T1X2_TX + tx;
    bool dead = false;
    bool stop = false;                   // the CTA gave up (a bounded wait timed out)
    int g_issued = 0, g_wait = 0;  // planes issued (thread 0) / plane last waited on
    if (tid == 0) {
        for (int s = 0; s < T1_NS; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    unsigned tmax[2] = {0u, 0u};
    int s = 0;
    uint32_t phase = 0;
    int gbase = 0;
    WorkRange wr(L, a.bz, a.ztop);
    for (Segment sg; wr.next(sg); gbase += sg.len + 2 * T1_LAG) {
        const int x0 = sg.x0, y0 = sg.y0, zs = sg.zs;
        const int ntot = sg.len + 2 * T1_LAG;  // arrival planes zs-4 .. ze+4
        const int xa = x0 + 2 * tx, y = y0 + ty;
        const bool own_a = (xa <= L.ixend) && (y <= L.iyend);
        const bool own_b = own_a && (xa + 1 <= L.ixend);
        if (__syncthreads_or(dead)) {
            stop = true;
            break;
        }
        auto issue = [&](int t) {
            ++g_issued;
            const int sl = (gbase + t) % T1_NS, z = zs - T1_LAG + t;
            float* dst = ring + (size_t)sl * 2 * IH * IW;
            mbar_expect_tx(&bars[sl], (uint32_t)T1_SLOT);
            tma_load_3d(dst, &tm_p, x0 - 4, y0 - 4, z, &bars[sl]);
            tma_load_3d(dst + IH * IW, &tm_q, x0 - 4, y0 - 4, z, &bars[sl]);
        };
        if (tid == 0)
            for (int t = 0; t < T1_PF && t < ntot; ++t) issue(t);
        const int vc = 2 * tx + 4, vr = ty + 4;
        auto back = [&](int kk) { const int v = s - kk; return v < 0 ? v + T1_NS : v; };
        for (int t = 0; t < ntot; ++t) {
            if (__syncthreads_or(dead)) {  // every thread is done with iteration t-1
                stop = true;
                break;
            }
            if (tid == 0 && t + T1_PF < ntot) {
                fence_proxy_async();
                issue(t + T1_PF);
            }
            g_wait = gbase + t;
            mbar_wait(&bars[s], phase, a.err, dead);
            const int z = zs - T1_LAG + t - T1_LAG;  // output plane
            float snapv[2][2] = {{0.0f, 0.0f}, {0.0f, 0.0f}};
            if (z >= zs && own_a) {
                // the pair's point-wise values (x even, so every pair is 8-byte aligned)
                const int64_t gi = L.idx(xa, y, z);
                const float2 a1 = __ldg(reinterpret_cast<const float2*>(a.m1 + gi));
                const float2 a2 = __ldg(reinterpret_cast<const float2*>(a.m2 + gi));
                const float2 a3 = __ldg(reinterpret_cast<const float2*>(a.m3 + gi));
                const float2 a4 = __ldg(reinterpret_cast<const float2*>(a.m4 + gi));
                float2 vrx = make_float2(0.0f, 0.0f), vry = vrx, vrz = make_float2(1.0f, 1.0f);
                if constexpr (TTI) {
                    vrx = __ldg(reinterpret_cast<const float2*>(a.rx + gi));
                    vry = __ldg(reinterpret_cast<const float2*>(a.ry + gi));
                    vrz = __ldg(reinterpret_cast<const float2*>(a.rz + gi));
                }
                const float2 o3 = *reinterpret_cast<const float2*>(a.f3 + gi);
                const float2 o4 = *reinterpret_cast<const float2*>(a.f4 + gi);
                const float4 sx = __ldg(reinterpret_cast<const float4*>(a.abx + xa));
                const float2 sy = __ldg(a.aby + y), sz = __ldg(a.abz + z);
                const T1Drv2 d1 = t1x2_derivs<TTI>(ring, 0, back, vr, vc, a.k);
                const T1Drv2 d2 = t1x2_derivs<TTI>(ring, 1, back, vr, vc, a.k);
                float r3a, r4a, r3b, r4b;
                t1_rhs<TTI>(d1.a, d2.a, a1.x, a2.x, a3.x, a4.x, vrx.x, vry.x, vrz.x, r3a, r4a);
                t1_rhs<TTI>(d1.b, d2.b, a1.y, a2.y, a3.y, a4.y, vrx.y, vry.y, vrz.y, r3b, r4b);
                const float Aa = fminf(sx.x, fminf(sy.x, sz.x)), Ba = fminf(sx.y, fminf(sy.y, sz.y));
                const float Ab = fminf(sx.z, fminf(sy.x, sz.x)), Bb = fminf(sx.w, fminf(sy.y, sz.y));
                float n3a = a.sponge ? Aa * o3.x + Ba * r3a * a.dt : o3.x + r3a * a.dt;
                float n4a = a.sponge ? Aa * o4.x + Ba * r4a * a.dt : o4.x + r4a * a.dt;
                float n3b = a.sponge ? Ab * o3.y + Bb * r3b * a.dt : o3.y + r3b * a.dt;
                float n4b = a.sponge ? Ab * o4.y + Bb * r4b * a.dt : o4.y + r4b * a.dt;
                if (gi == a.src_index) {
                    n3a += a.src_term;
                    n4a += a.src_term;
                }
                if (gi + 1 == a.src_index) {
                    n3b += a.src_term;
                    n4b += a.src_term;
                }
                const float* C = ring + (size_t)back(T1_LAG) * 2 * IH * IW;
                const float2 pc = *reinterpret_cast<const float2*>(C + vr * IW + vc);
                const float2 qc = *reinterpret_cast<const float2*>(C + IH * IW + vr * IW + vc);
                // next step's loop2 (kernel_base.cu:92-101) and free surface (:142-162)
                float2 np = make_float2(Aa * pc.x + Ba * n3a * a.dt, Ab * pc.y + Bb * n3b * a.dt);
                float2 nq = make_float2(Aa * qc.x + Ba * n4a * a.dt, Ab * qc.y + Bb * n4b * a.dt);
                if (a.fs && z == L.izbeg) {
                    np = make_float2(0.0f, 0.0f);
                    nq = np;
                }
                wave_apply(a.wave_prec, a.wave_scale, np.x, nq.x);
                if (own_b) wave_apply(a.wave_prec, a.wave_scale, np.y, nq.y);
                const bool mirror = a.fs && z > L.izbeg && z <= L.izbeg + kRadius;
                const int64_t gm = L.idx(xa, y, 2 * L.izbeg - z);
                if (own_b) {
                    *reinterpret_cast<float2*>(a.f3 + gi) = make_float2(n3a, n3b);
                    *reinterpret_cast<float2*>(a.f4 + gi) = make_float2(n4a, n4b);
                    *reinterpret_cast<float2*>(a.pout + gi) = np;
                    *reinterpret_cast<float2*>(a.qout + gi) = nq;
                    if (mirror) {
                        *reinterpret_cast<float2*>(a.pout + gm) = make_float2(-np.x, -np.y);
                        *reinterpret_cast<float2*>(a.qout + gm) = make_float2(-nq.x, -nq.y);
                    }
                } else {
                    a.f3[gi] = n3a;
                    a.f4[gi] = n4a;
                    a.pout[gi] = np.x;
                    a.qout[gi] = nq.x;
                    if (mirror) {
                        a.pout[gm] = -np.x;
                        a.qout[gm] = -nq.x;
                    }
                }
                if (a.snap) {  // two-field slot: pdot, qdot (all the type1 image reads)
                    const int64_t nin = (int64_t)L.nx() * L.ny() * L.nz();
                    const int64_t dd = ((int64_t)(z - L.izbeg) * L.ny() + (y - L.iybeg)) * L.nx() + (xa - L.ixbeg);
                    snapv[0][0] = n3a;
                    snapv[1][0] = n4a;
                    if (own_b) {
                        snapv[0][1] = n3b;
                        snapv[1][1] = n4b;
                    }
                    bool sat = false;
#pragma unroll
                    for (int f = 0; f < 2; ++f) {
                        const float sc = (a.snap_prec == SNAP_F32) ? 1.0f : a.snap_scale[f];
                        sat |= snap_store(a.snap, f * nin + dd, snapv[f][0] * sc, a.snap_prec);
                        if (own_b) sat |= snap_store(a.snap, f * nin + dd + 1, snapv[f][1] * sc, a.snap_prec);
                    }
                    if (sat) atomicOr(a.err, 2);
                }
            }
#pragma unroll
            for (int f = 0; f < 2; ++f)
                tmax[f] = max(tmax[f], max(__float_as_uint(fabsf(snapv[f][0])), __float_as_uint(fabsf(snapv[f][1]))));
            if (++s == T1_NS) {
                s = 0;
                phase ^= 1u;
            }
        }
    if (stop) break;
    }  // segments
    if (stop && tid == 0) drain_loads(bars, T1_NS, g_wait, g_issued);
    if (a.snap && a.snap_prec != SNAP_F32) {
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            const unsigned m = __reduce_max_sync(0xffffffffu, tmax[f]);
            if ((tid & 31) == 0 && m) atomicMax(a.snap_amax + f, m);
        }
    }
}

// Type1 adjoint step: pdot += dt * D(M^T (p, q)) (or the sponge form), then
// loop2 and the free surface.  The transposed-model temporaries of each
// arriving plane (lap/hz of both fields weighted per derivative,
// compute_temp_arrays, kernel_type1_gpu_adj.cu:103-153) go to shared tiles;
// their z terms are scattered into a queue of the outputs L-4 .. L+4 and
// their x/y terms into output L.
constexpr int T1A_NSTAGE = 3;
constexpr int T1A_PF = 2;
constexpr int T1A_NARR = 9;  // p, q, m1, m2, m3, m4, rx, ry, rz (halo 4)
constexpr size_t T1A_STAGE = (size_t)T1A_NARR * IH * IW * sizeof(float);
constexpr size_t T1A_TXX = (size_t)TY * IW * sizeof(float2);  // rows y0.., cols x0-4..
constexpr size_t T1A_TYY = (size_t)IH * TX * sizeof(float2);  // rows y0-4.., cols x0..
constexpr size_t T1A_TXY = (size_t)IH * IW * sizeof(float2);
constexpr size_t T1A_TZZ = (size_t)TY * TX * sizeof(float2);
constexpr size_t T1A_SMEM = T1A_NSTAGE * T1A_STAGE + 2 * T1A_TXX + 2 * T1A_TYY + T1A_TXY + T1A_TZZ +
                            T1A_NSTAGE * sizeof(uint64_t);
enum { U_P = 0, U_Q, U_M1, U_M2, U_M3, U_M4, U_RX, U_RY, U_RZ };

struct T1AdjMaps {
    CUtensorMap m[T1A_NARR];
};

struct T1AdjParams {
    float *pout, *qout, *f3, *f4;
    const float *pin, *qin;
    const float2 *abx, *aby, *abz;
    Layout L;
    int bz;
    int ztop;
    int fs;
    int sponge;
    float dt;
    T1Fd k;
    int* err;
    int wave_prec;            // 0, or p/q rounded to FP16 (1) / BF16 (2) each step
    const float* wave_scale;  // 2 scales (p, q) of this step's output
};

template <bool TTI>
__global__ void __launch_bounds__(NT, 1) k_t1_fused_adjoint(const __grid_constant__ T1AdjMaps tm, const T1AdjParams a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    float* stage = reinterpret_cast<float*>(smem);
    unsigned char* sp = smem + T1A_NSTAGE * T1A_STAGE;
    float2* txx = reinterpret_cast<float2*>(sp);  // lap + rx^2 hz      [TY][IW]
    sp += T1A_TXX;
    float2* tzx = reinterpret_cast<float2*>(sp);  // 2 rz rx hz         [TY][IW]
    sp += T1A_TXX;
    float2* tyy = reinterpret_cast<float2*>(sp);  // lap + ry^2 hz      [IH][TX]
    sp += T1A_TYY;
    float2* tyz = reinterpret_cast<float2*>(sp);  // 2 ry rz hz         [IH][TX]
    sp += T1A_TYY;
    float2* txy = reinterpret_cast<float2*>(sp);  // 2 rx ry hz         [IH][IW]
    sp += T1A_TXY;
    float2* tzz = reinterpret_cast<float2*>(sp);  // lap + rz^2 hz      [TY][TX]
    sp += T1A_TZZ;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sp);

    const Layout& L = a.L;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    bool dead = false;
    bool stop = false;                   // the CTA gave up (a bounded wait timed out)
    int g_issued = 0, g_wait = 0;  // planes issued (thread 0) / plane last waited on
    constexpr int NLOAD = TTI ? T1A_NARR : U_RX;
    constexpr uint32_t TX_BYTES = (uint32_t)(NLOAD * IH * IW * sizeof(float));
    if (tid == 0) {
        for (int s = 0; s < T1A_NSTAGE; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    int s = 0;
    uint32_t phase = 0;
    int gbase = 0;
    WorkRange wr(L, a.bz, a.ztop);
    for (Segment sg; wr.next(sg); gbase += sg.len + 2 * T1_LAG) {
        const int x0 = sg.x0, y0 = sg.y0, zs = sg.zs;
        const int ntot = sg.len + 2 * T1_LAG;
        const int x = x0 + tx, y = y0 + ty;
        const bool owner = (x <= L.ixend) && (y <= L.iyend);
        if (__syncthreads_or(dead)) {
            stop = true;
            break;
        }
        auto issue = [&](int t) {
            ++g_issued;
            const int sl = (gbase + t) % T1A_NSTAGE, z = zs - T1_LAG + t;
            float* dst = stage + (size_t)sl * (T1A_STAGE / sizeof(float));
            mbar_expect_tx(&bars[sl], TX_BYTES);
#pragma unroll
            for (int kk = 0; kk < NLOAD; ++kk) tma_load_3d(dst + kk * IH * IW, &tm.m[kk], x0 - 4, y0 - 4, z, &bars[sl]);
        };
        if (tid == 0)
            for (int t = 0; t < T1A_PF && t < ntot; ++t) issue(t);
        float q3[9], q4[9];  // rhs of outputs L-4 .. L+4
#pragma unroll
        for (int j = 0; j < 9; ++j) q3[j] = q4[j] = 0.0f;
        for (int t = 0; t < ntot; ++t) {
            if (__syncthreads_or(dead)) {  // the tiles of plane L-1 have been read; stage (t+2)%3 is free
                stop = true;
                break;
            }
            if (tid == 0 && t + T1A_PF < ntot) {
                fence_proxy_async();
                issue(t + T1A_PF);
            }
            const int Lz = zs - T1_LAG + t;
            const int zo = Lz - T1_LAG;
            const bool out_here = (zo >= zs) && owner;
            const int64_t go = L.idx(x, y, max(zo, 0));
            float o3 = 0.0f, o4 = 0.0f, opc = 0.0f, oqc = 0.0f;
            float2 osz = make_float2(1.0f, 1.0f), osx = osz, osy = osz;
            if (out_here) {
                o3 = a.f3[go];
                o4 = a.f4[go];
                opc = __ldg(a.pin + go);
                oqc = __ldg(a.qin + go);
                osx = __ldg(a.abx + x);
                osy = __ldg(a.aby + y);
                osz = __ldg(a.abz + zo);
            }
            g_wait = gbase + t;
            mbar_wait(&bars[s], phase, a.err, dead);
            const float* st = stage + (size_t)s * (T1A_STAGE / sizeof(float));
            // (1) temporaries of plane L on the halo-4 box, 960 positions
            for (int e = tid; e < IH * IW; e += NT) {
                const int r = e / IW, c = e % IW;
                const float p = st[U_P * IH * IW + e], q = st[U_Q * IH * IW + e];
                const float m1 = st[U_M1 * IH * IW + e], m2 = st[U_M2 * IH * IW + e], m3 = st[U_M3 * IH * IW + e],
                            m4 = st[U_M4 * IH * IW + e];
                const float lx = m1 * p + m2 * q, hx = (-m1 + m4) * p - m2 * q;
                const float lz = m4 * q, hz = m2 * p + (-m4 + m3) * q;
                const float rx = TTI ? st[U_RX * IH * IW + e] : 0.0f, ry = TTI ? st[U_RY * IH * IW + e] : 0.0f,
                            rz = TTI ? st[U_RZ * IH * IW + e] : 1.0f;
                const bool rowb = r >= 4 && r < 4 + TY, colb = c >= 4 && c < 4 + TX;
                if (TTI) txy[e] = make_float2(2.0f * rx * ry * hx, 2.0f * rx * ry * hz);
                if (rowb) {
                    txx[(r - 4) * IW + c] = make_float2(lx + rx * rx * hx, lz + rx * rx * hz);
                    if (TTI) tzx[(r - 4) * IW + c] = make_float2(2.0f * rz * rx * hx, 2.0f * rz * rx * hz);
                }
                if (colb) {
                    tyy[r * TX + c - 4] = make_float2(lx + ry * ry * hx, lz + ry * ry * hz);
                    if (TTI) tyz[r * TX + c - 4] = make_float2(2.0f * ry * rz * hx, 2.0f * ry * rz * hz);
                }
                if (rowb && colb) tzz[(r - 4) * TX + c - 4] = make_float2(lx + rz * rz * hx, lz + rz * rz * hz);
            }
            __syncthreads();  // tiles of plane L ready
            // (2) z terms of plane L into outputs L-4 .. L+4 (compute_z_contributions, :162-186)
            {
                const float2 cz = tzz[ty * TX + tx];
#pragma unroll
                for (int ir = -4; ir <= 4; ++ir) {
                    const float c = c2(ir < 0 ? -ir : ir);
                    const int j = 4 - ir;  // output L - ir
                    float a3 = a.k.zz * c * cz.x, a4 = a.k.zz * c * cz.y;
                    if (TTI && ir != 0) {
                        const float2 yp = tyz[(ty + 4 + ir) * TX + tx], ym = tyz[(ty + 4 - ir) * TX + tx];
                        const float2 xp = tzx[ty * IW + tx + 4 + ir], xm = tzx[ty * IW + tx + 4 - ir];
                        a3 = a3 + a.k.yz * c * (yp.x - ym.x);
                        a4 = a4 + a.k.yz * c * (yp.y - ym.y);
                        a3 = a3 + a.k.zx * c * (xp.x - xm.x);
                        a4 = a4 + a.k.zx * c * (xp.y - xm.y);
                    }
                    q3[j] = q3[j] + a3;
                    q4[j] = q4[j] + a4;
                }
            }
            // (3) x/y terms of output L (compute_xy_contributions, :191-217)
            {
                const float2 x0v = txx[ty * IW + tx + 4], y0v = tyy[(ty + 4) * TX + tx];
                float xx3 = c2(0) * x0v.x, xx4 = c2(0) * x0v.y, yy3 = c2(0) * y0v.x, yy4 = c2(0) * y0v.y;
                float xy3 = 0.0f, xy4 = 0.0f;
#pragma unroll
                for (int i = 1; i <= 4; ++i) {
                    const float c = c2(i);
                    const float2 xp = txx[ty * IW + tx + 4 + i], xm = txx[ty * IW + tx + 4 - i];
                    const float2 yp = tyy[(ty + 4 + i) * TX + tx], ym = tyy[(ty + 4 - i) * TX + tx];
                    xx3 += c * (xp.x + xm.x);
                    xx4 += c * (xp.y + xm.y);
                    yy3 += c * (yp.x + ym.x);
                    yy4 += c * (yp.y + ym.y);
                    if (TTI) {
                        const int rr = ty + 4, cc = tx + 4;
                        const float2 pp = txy[(rr + i) * IW + cc + i], pm = txy[(rr + i) * IW + cc - i];
                        const float2 mm = txy[(rr - i) * IW + cc - i], mp = txy[(rr - i) * IW + cc + i];
                        xy3 += c * (pp.x - pm.x + mm.x - mp.x);
                        xy4 += c * (pp.y - pm.y + mm.y - mp.y);
                    }
                }
                q3[4] += a.k.xx * xx3 + a.k.yy * yy3 + a.k.xy * xy3;
                q4[4] += a.k.xx * xx4 + a.k.yy * yy4 + a.k.xy * xy4;
            }
            // (4) output L-4: update, then loop2 and the free surface
            if (out_here) {
                const float A = fminf(osx.x, fminf(osy.x, osz.x));
                const float B = fminf(osx.y, fminf(osy.y, osz.y));
                const float n3 = a.sponge ? A * o3 + B * q3[0] * a.dt : o3 + q3[0] * a.dt;
                const float n4 = a.sponge ? A * o4 + B * q4[0] * a.dt : o4 + q4[0] * a.dt;
                a.f3[go] = n3;
                a.f4[go] = n4;
                float np = A * opc + B * n3 * a.dt;
                float nq = A * oqc + B * n4 * a.dt;
                if (a.fs && zo == L.izbeg) {
                    np = 0.0f;
                    nq = 0.0f;
                }
                wave_apply(a.wave_prec, a.wave_scale, np, nq);
                a.pout[go] = np;
                a.qout[go] = nq;
                if (a.fs && zo > L.izbeg && zo <= L.izbeg + kRadius) {
                    const int64_t gm = L.idx(x, y, 2 * L.izbeg - zo);
                    a.pout[gm] = -np;
                    a.qout[gm] = -nq;
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                q3[j] = q3[j + 1];
                q4[j] = q4[j + 1];
            }
            q3[8] = 0.0f;
            q4[8] = 0.0f;
            if (++s == T1A_NSTAGE) {
                s = 0;
                phase ^= 1u;
            }
        }
    if (stop) break;
    }  // segments
    if (stop && tid == 0) drain_loads(bars, T1A_NSTAGE, g_wait, g_issued);
}

// Type1 imaging (kernel_type1_gpu_grad.cu:4-21) on the snapshot store:
// grad += adj_pdot * pdot_snap + adj_qdot * qdot_snap, stored values unscaled.
template <typename T>
__global__ void __launch_bounds__(256)
    k_t1_image(const T* __restrict__ s3, const T* __restrict__ s4, const float* __restrict__ scale,
               const float* __restrict__ adj3, const float* __restrict__ adj4, float* __restrict__ grad, Layout L)
{
    const int64_t n = (int64_t)L.nx() * L.ny() * L.nz();
    const float u3 = scale ? 1.0f / scale[0] : 1.0f, u4 = scale ? 1.0f / scale[1] : 1.0f;
    for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < n; d += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(d % L.nx()), iy = (int)((d / L.nx()) % L.ny()), iz = (int)(d / ((int64_t)L.nx() * L.ny()));
        const int64_t i = L.idx(ix + L.ixbeg, iy + L.iybeg, iz + L.izbeg);
        grad[d] += adj3[i] * (to_f32(s3[d]) * u3) + adj4[i] * (to_f32(s4[d]) * u4);
    }
}

// ---------------------------------------------------------------------------
// Host side: tensor maps and launchers.
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// 3D FP32 tensor map over a halo'd volume with a (bx, by, 1) box; reads
// outside the volume are zero-filled.
bool make_map(CUtensorMap* m, const float* base, const Layout& L, int bx, int by)
{
    auto fn = encode_fn();
    if (!fn || !base) return false;
    cuuint64_t dims[3] = {(cuuint64_t)L.ldimx, (cuuint64_t)L.ldimy, (cuuint64_t)L.ldimz};
    cuuint64_t strides[2] = {(cuuint64_t)L.ldimx * sizeof(float), (cuuint64_t)L.ldimx * L.ldimy * sizeof(float)};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Maps are keyed by (address, box, layout) and cached for the process.
struct MapKey {
    const float* p;
    int bx, by, lx, ly, lz;
    bool operator<(const MapKey& o) const
    {
        return std::tie(p, bx, by, lx, ly, lz) < std::tie(o.p, o.bx, o.by, o.lx, o.ly, o.lz);
    }
};
std::mutex g_map_mu;
std::map<MapKey, CUtensorMap> g_maps;

// Map of a volume of float4 cells (the interleaved model), as a 4D tensor
// (4, ldimx, ldimy, ldimz) with box (4, bx, by, 1): a tile lands in shared
// memory as float4 [by][bx].
bool make_map4(CUtensorMap* m, const float4* base, const Layout& L, int bx, int by)
{
    auto fn = encode_fn();
    if (!fn || !base) return false;
    cuuint64_t dims[4] = {4, (cuuint64_t)L.ldimx, (cuuint64_t)L.ldimy, (cuuint64_t)L.ldimz};
    cuuint64_t strides[3] = {(cuuint64_t)sizeof(float4), (cuuint64_t)L.ldimx * sizeof(float4),
                             (cuuint64_t)L.ldimx * L.ldimy * sizeof(float4)};
    cuuint32_t box[4] = {4, (cuuint32_t)bx, (cuuint32_t)by, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float4*>(base), dims, strides, box, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool get_map4(CUtensorMap* out, const float4* p, const Layout& L, int bx, int by)
{
    MapKey k{reinterpret_cast<const float*>(p), -bx, by, L.ldimx, L.ldimy, L.ldimz};  // negative width: float4 cells
    std::lock_guard<std::mutex> lk(g_map_mu);
    auto it = g_maps.find(k);
    if (it != g_maps.end()) {
        *out = it->second;
        return true;
    }
    CUtensorMap m;
    if (!make_map4(&m, p, L, bx, by)) return false;
    if (g_maps.size() > 4096) g_maps.clear();
    g_maps[k] = m;
    *out = m;
    return true;
}

bool get_map(CUtensorMap* out, const float* p, const Layout& L, int bx, int by)
{
    MapKey k{p, bx, by, L.ldimx, L.ldimy, L.ldimz};
    std::lock_guard<std::mutex> lk(g_map_mu);
    auto it = g_maps.find(k);
    if (it != g_maps.end()) {
        *out = it->second;
        return true;
    }
    CUtensorMap m;
    if (!make_map(&m, p, L, bx, by)) return false;
    if (g_maps.size() > 4096) g_maps.clear();
    g_maps[k] = m;
    *out = m;
    return true;
}

// Per-device error word for the bounded waits.
int* err_word()
{
    static std::mutex mu;
    static std::map<int, int*> words;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    auto it = words.find(dev);
    if (it != words.end()) return it->second;
    int* p = nullptr;
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemset(p, 0, sizeof(int));
    words[dev] = p;
    return p;
}

// Kernel attributes (dynamic shared memory above 48 KB) and the error word are
// set up once per device, outside any stream capture.
template <typename K>
bool set_smem(K kernel, size_t bytes)
{
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess;
}

bool prepare_device()
{
    bool ok = err_word() != nullptr;
    ok = ok && set_smem(k_fused_forward<false>, FWD_SMEM) && set_smem(k_fused_forward<true>, FWD_SMEM);
    ok = ok && set_smem(k_fused_adjoint<false>, adj_smem(false)) && set_smem(k_fused_adjoint<true>, adj_smem(true));
    ok = ok && set_smem(k_fused_image<false, float>, img_smem(4, false)) &&
         set_smem(k_fused_image<true, float>, img_smem(4, true));
    ok = ok && set_smem(k_fused_image<false, __half>, img_smem(2, false)) &&
         set_smem(k_fused_image<true, __half>, img_smem(2, true));
    ok = ok && set_smem(k_fused_image<false, __nv_bfloat16>, img_smem(2, false)) &&
         set_smem(k_fused_image<true, __nv_bfloat16>, img_smem(2, true));
    ok = ok && set_smem(k_t1_fused_forward_x2<false>, T1F_SMEM) && set_smem(k_t1_fused_forward_x2<true>, T1F_SMEM);
    ok = ok && set_smem(k_t1_fused_adjoint<false>, T1A_SMEM) && set_smem(k_t1_fused_adjoint<true>, T1A_SMEM);
    if (!ok) cudaGetLastError();
    return ok;
}

constexpr int kMaxDevices = 64;
std::atomic<int> g_prepared[kMaxDevices];  // 0 no, 1 yes, -1 failed
std::mutex g_prepare_mu;

bool kernels_prepared()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return false;
    }
    int v = g_prepared[dev].load(std::memory_order_acquire);
    if (v) return v > 0;
    std::lock_guard<std::mutex> lk(g_prepare_mu);
    v = g_prepared[dev].load(std::memory_order_relaxed);
    if (!v) {
        v = prepare_device() ? 1 : -1;
        g_prepared[dev].store(v, std::memory_order_release);
    }
    return v > 0;
}

bool layout_supported(const Layout& L)
{
    // TMA box origins x0-8 and x0-4 must be multiples of 4 floats (16 bytes):
    // ixbeg = 4 and a 32-wide tile guarantee it.
    return L.ixbeg == kRadius && L.iybeg == kRadius && L.izbeg == kRadius && L.ldimx % 32 == 0 &&
           L.ldimx >= L.ixend + 1 + kRadius && L.ldimy == L.iyend + 1 + kRadius &&
           L.ldimz == L.izend + 1 + kRadius;
}

int device_sms()
{
    int sms = 148;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    return sms;
}

long long work_planes(const Layout& L)
{
    return (long long)((L.nx() + TX - 1) / TX) * ((L.ny() + TY - 1) / TY) * L.nz();
}

long long tile_count(const Layout& L) { return (long long)((L.nx() + TX - 1) / TX) * ((L.ny() + TY - 1) / TY); }

// CTAs of a launch with the given split.
unsigned cta_count(const Layout& L, Split sp)
{
    if (sp.ztop <= 0) return (unsigned)((work_planes(L) + sp.bz - 1) / sp.bz);
    const long long T = tile_count(L);
    return (unsigned)(T + (T * (L.nz() - sp.ztop) + sp.bz - 1) / sp.bz);
}

// Planes per CTA worth trying: whole-column chunks ceil(nz/n), and shares
// that give every SM one, two, ... equal parts of the work; at least 8.
std::vector<int> plane_candidates(const Layout& L)
{
    std::vector<int> c;
    const int nz = L.nz();
    for (int nch = 1; nch <= nz; ++nch) {
        const int bz = (nz + nch - 1) / nch;
        if (bz < 8 && nch > 1) break;
        c.push_back(bz);
        if (nz % nch == 0) c.push_back(nz / nch);
    }
    const long long W = work_planes(L);
    const int sms = device_sms();
    for (int k = 1; k <= 8; ++k) {
        const long long b = (W + (long long)sms * k - 1) / ((long long)sms * k);
        if (b >= 8 && b <= (1LL << 30)) c.push_back((int)b);
    }
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    return c;
}

// CTAs of a kind resident per SM: shared memory (and registers) allow two
// of the type1 forward kernel's 256-thread CTAs, one of the others.
int kind_ctas_per_sm(int kind) { return kind == KIND_T1F ? 2 : 1; }

// Modelled time of a step, in plane-iterations of the slowest CTA: per_sm
// resident CTAs per SM, each segment pays the 2*LAG-plane pipeline fill, a
// range of bz planes covers at most ceil((bz-1)/nz)+1 columns (one when
// whole columns divide evenly).
double plane_cost(const Layout& L, int bz, int lag, int per_sm)
{
    const int nz = L.nz();
    const long long ctas = cta_count(L, Split{bz, 0});
    const long long slots = (long long)device_sms() * per_sm;
    const double waves = (double)((ctas + slots - 1) / slots);
    int segs;
    if (bz <= nz && nz % bz == 0)
        segs = 1;
    else if (bz % nz == 0)
        segs = bz / nz;
    else
        segs = (bz - 1) / nz + 2;
    return waves * (bz + 2.0 * lag * segs);
}

// Column-aligned shares (bz divides nz): every CTA works down whole chunks
// of one column, and all CTAs stay at about the same z, so the halo planes
// that neighbouring tiles share are still in L2 when the neighbour reads
// them.  Unaligned shares balance the SMs better but spread the CTAs over
// all of z; a kernel that stages many halo'd arrays then re-reads its halos
// from HBM (the adjoint stages nine, the imaging kernel eleven; the forward
// kernel three).
bool column_aligned(const Layout& L, int bz) { return bz <= L.nz() && L.nz() % bz == 0; }

// Modelled cost of a top/bottom split in one wave: the tops (one segment
// each) against the bottom CTAs, whose bz planes cross at most
// ceil((bz-1)/span)+1 column bottoms.
double split_cost(const Layout& L, Split sp, int lag, int per_sm)
{
    const int span = L.nz() - sp.ztop;
    const int segs = (sp.bz - 1) / span + 2;
    const long long slots = (long long)device_sms() * per_sm;
    const double waves = (double)((cta_count(L, sp) + slots - 1) / slots);
    return waves * std::max(sp.ztop + 2.0 * lag, sp.bz + 2.0 * lag * segs);
}

int kind_lag(int kind) { return (kind == KIND_T1F || kind == KIND_T1A) ? T1_LAG : LAG; }

// Top/bottom splits for grids with fewer columns than SMs: the balance point
// ztop = T (nz + 2 lag) / S of the tops against S - T bottom CTAs, and
// neighbours 8 and 16 planes either side.
std::vector<Split> topbottom_candidates(const Layout& L, int kind)
{
    std::vector<Split> c;
    const long long T = tile_count(L);
    const int nz = L.nz();
    const int lag = kind_lag(kind);
    // S: CTAs resident at once (one or two per SM)
    for (int S : {device_sms(), 2 * device_sms()}) {
        if (T >= S || nz < 16) continue;
        const int z0 = (int)(T * (nz + 2LL * lag) / S);
        for (int dz : {0, -8, 8, -16, 16}) {
            const int zt = z0 + dz;
            if (zt < 8 || zt > nz - 4) continue;
            const long long bottoms = T * (long long)(nz - zt);
            const int bz = (int)((bottoms + (S - T) - 1) / (S - T));
            if (bz < 1) continue;
            const Split sp{bz, zt};
            if (std::find(c.begin(), c.end(), sp) == c.end()) c.push_back(sp);
        }
    }
    return c;
}

// The model's split: the cheapest tile-major candidate (column-aligned only
// for the kernels that stage many halo'd arrays) or top/bottom split.
Split pick_split(const Layout& L, int kind)
{
    Split best{L.nz(), 0};
    double best_cost = 1e300;
    const bool any_split = kind == KIND_FWD || kind == KIND_T1F;  // few staged arrays
    const int lag = kind_lag(kind), per_sm = kind_ctas_per_sm(kind);
    for (int bz : plane_candidates(L)) {
        if (!any_split && !column_aligned(L, bz)) continue;
        const double cost = plane_cost(L, bz, lag, per_sm);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = Split{bz, 0};
        }
    }
    for (const Split& sp : topbottom_candidates(L, kind)) {
        const double cost = split_cost(L, sp, lag, per_sm);
        if (cost < best_cost - 1e-9) {
            best_cost = cost;
            best = sp;
        }
    }
    return best;
}

} // namespace

inline float2 pair(float c) { return make_float2(c, c); }

int launch_fused_forward(const Layout& L, const FwdStepArgs& s, cudaStream_t st)
{
    if (!layout_supported(L)) return TTI_EINVAL;
    CUtensorMap mp, mq, mi;
    if (!get_map(&mp, s.pin, L, PW, PH) || !get_map(&mq, s.qin, L, PW, PH) || !get_map(&mi, s.m.irho, L, IW, IH))
        return TTI_ELAUNCH;
    FwdParams a{};
    a.pout = s.pout;
    a.qout = s.qout;
    a.f3 = s.f3;
    a.f4 = s.f4;
    a.irho = s.m.irho;
    a.m1 = s.m.m1;
    a.m2 = s.m.m2;
    a.m3 = s.m.m3;
    a.m4 = s.m.m4;
    a.rx = s.m.rx;
    a.ry = s.m.ry;
    a.rz = s.m.rz;
    a.abx = s.abx;
    a.aby = s.aby;
    a.abz = s.abz;
    a.snap = s.snap;
    a.snap_prec = s.snap_prec;
    a.snap_scale = s.snap_scale;
    a.snap_amax = s.snap_amax;
    if (s.snap && s.snap_prec != SNAP_F32 && (!s.snap_scale || !s.snap_amax)) return TTI_EINVAL;
    a.src_index = s.src_index;
    a.src_term = s.src_term;
    a.trace = s.trace;
    a.rec = s.rec;
    if (a.trace && !a.rec.xy) return TTI_EINVAL;
    a.L = L;
    const Split sp = s.bz > 0 ? Split{s.bz, s.ztop} : choose_split(L, KIND_FWD);
    if (!split_valid(L, sp)) return TTI_EINVAL;
    a.bz = sp.bz;
    a.ztop = sp.ztop;
    a.fs = s.free_surface;
    a.dt = s.dt;
    a.invdx = 1.0 / s.dx;
    a.invdy = 1.0 / s.dy;
    a.invdz = 1.0 / s.dz;
    a.invdxdy = 1.0 / (4 * s.dx * s.dy);
    a.invdydz = 1.0 / (4 * s.dy * s.dz);
    a.invdzdx = 1.0 / (4 * s.dx * s.dz);
    a.err = s.err ? s.err : err_word();
    a.wave_prec = s.wave_prec;
    a.wave_scale = s.wave_scale;
    if (a.wave_prec && !a.wave_scale) return TTI_EINVAL;
    if (!a.err) return TTI_ENOMEM;
    dim3 grid(cta_count(L, sp));
    if (!kernels_prepared()) return TTI_ELAUNCH;
    if (s.vti)
        k_fused_forward<false><<<grid, dim3(TX, TY), FWD_SMEM, st>>>(mp, mq, mi, a);
    else
        k_fused_forward<true><<<grid, dim3(TX, TY), FWD_SMEM, st>>>(mp, mq, mi, a);
    return launch_status();
}

int launch_fused_adjoint(const Layout& L, const AdjStepArgs& s, cudaStream_t st)
{
    if (!layout_supported(L)) return TTI_EINVAL;
    const bool tti = !s.vti;
    if (!s.m.ma || (tti && !s.m.mb)) return TTI_EINVAL;
    AdjMaps tm;
    if (!get_map(&tm.p, s.pin, L, PW, PH) || !get_map(&tm.q, s.qin, L, PW, PH) ||
        !get_map4(&tm.ma, s.m.ma, L, PW, PH))
        return TTI_ELAUNCH;
    if (tti ? !get_map4(&tm.mb, s.m.mb, L, PW, PH) : !get_map(&tm.mb, s.m.irho, L, PW, PH)) return TTI_ELAUNCH;
    AdjParams a{};
    a.pout = s.pout;
    a.qout = s.qout;
    a.f3 = s.f3;
    a.f4 = s.f4;
    a.pin = s.pin;
    a.qin = s.qin;
    a.abx = s.abx;
    a.aby = s.aby;
    a.abz = s.abz;
    a.L = L;
    const Split sp = s.bz > 0 ? Split{s.bz, s.ztop} : choose_split(L, KIND_ADJ);
    if (!split_valid(L, sp)) return TTI_EINVAL;
    a.bz = sp.bz;
    a.ztop = sp.ztop;
    a.fs = s.free_surface;
    a.sponge = s.sponge_active;
    a.dt = s.dt;
    a.res = s.res;
    a.obs = s.obs;
    a.rec = s.rec;
    a.srctr = s.srctr;
    a.src_index = s.src_index;
    a.src_z = (s.srctr && s.src_index >= 0) ? (int)(s.src_index / L.zstride()) : -1;
    if (a.res && !a.rec.xy) return TTI_EINVAL;
    const float invd[3] = {(float)(1.0 / s.dx), (float)(1.0 / s.dy), (float)(1.0 / s.dz)};
    const float invdxy = 1.0 / (4 * s.dx * s.dy), invdyz = 1.0 / (4 * s.dy * s.dz), invdzx = 1.0 / (4 * s.dx * s.dz);
    for (int d = 0; d < 3; ++d)
        for (int i = 1; i <= 4; ++i) a.kd[d][i - 1] = pair(invd[d] * c1(i));
    for (int j = 0; j < 8; ++j) a.kzm[j] = pair((j <= 3) ? invd[2] * c1(4 - j) : -invd[2] * c1(j - 3));
    for (int i = -4; i <= 4; ++i) {
        const float c = i == 0 ? 0.0f : c2(i < 0 ? -i : i) * (i < 0 ? -1.0f : 1.0f);
        a.kyz[i + 4] = pair(invdyz * c);
        a.kzx[i + 4] = pair(invdzx * c);
    }
    for (int k = 1; k <= 4; ++k) a.kxy[k - 1] = pair(invdxy * c2(k));
    a.err = s.err ? s.err : err_word();
    a.wave_prec = s.wave_prec;
    a.wave_scale = s.wave_scale;
    if (a.wave_prec && !a.wave_scale) return TTI_EINVAL;
    if (!a.err) return TTI_ENOMEM;
    dim3 grid(cta_count(L, sp));
    if (!kernels_prepared()) return TTI_ELAUNCH;
    if (!tti)
        k_fused_adjoint<false><<<grid, dim3(TX, TY), adj_smem(false), st>>>(tm, a);
    else
        k_fused_adjoint<true><<<grid, dim3(TX, TY), adj_smem(true), st>>>(tm, a);
    return launch_status();
}

namespace {
// 4D tensor map over the dense snapshot store (nx, ny, nz, 4*nsnap), element
// type per storage precision.
bool make_store_map(CUtensorMap* m, const void* base, int prec, int nx, int ny, int nz, int nvol, int bx, int by)
{
    auto fn = encode_fn();
    if (!fn || !base) return false;
    const size_t elt = snap_elt_bytes(prec);
    const CUtensorMapDataType dt = prec == SNAP_F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : prec == SNAP_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                      : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nvol};
    cuuint64_t strides[3] = {(cuuint64_t)nx * elt, (cuuint64_t)nx * ny * elt, (cuuint64_t)nx * ny * nz * elt};
    cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, 1};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, dt, 4, const_cast<void*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool TTI, typename T>
int launch_image_t(const ImgMaps& tm, const ImgParams& a, dim3 grid, cudaStream_t st)
{
    const size_t smem = img_smem(sizeof(T), TTI);
    k_fused_image<TTI, T><<<grid, dim3(TX, TY), smem, st>>>(tm, a);
    return launch_status();
}
} // namespace

bool fused_image_supported(const Layout& L) { return layout_supported(L) && L.nx() % 8 == 0; }

int launch_fused_image(const Layout& L, const ImageArgs& s, cudaStream_t st)
{
    if (!fused_image_supported(L) || !s.store || s.slot < 0 || s.slot >= s.nsnap) return TTI_EINVAL;
    if (s.snap_prec != SNAP_F32 && !s.snap_scale) return TTI_EINVAL;
    ImgMaps tm;
    {
        // store maps keyed by (store address, grid, slots, precision)
        static std::mutex mu;
        static std::map<std::tuple<const void*, int, int, int, int, int>, CUtensorMap> cache;
        std::lock_guard<std::mutex> lk(mu);
        const auto key = std::make_tuple(s.store, L.nx(), L.ny(), L.nz(), 4 * s.nsnap, s.snap_prec);
        auto it = cache.find(key);
        if (it == cache.end()) {
            CUtensorMap m;
            if (!make_store_map(&m, s.store, s.snap_prec, L.nx(), L.ny(), L.nz(), 4 * s.nsnap, PW, PH))
                return TTI_ELAUNCH;
            if (cache.size() > 1024) cache.clear();
            it = cache.emplace(key, m).first;
        }
        tm.snap = it->second;
    }
    const bool tti = !s.vti;
    if (!s.m.ma || (tti && !s.m.mb)) return TTI_EINVAL;
    if (!get_map(&tm.p, s.adj1, L, IW, IH) || !get_map(&tm.q, s.adj2, L, IW, IH) ||
        !get_map4(&tm.ma, s.m.ma, L, IW, IH))
        return TTI_ELAUNCH;
    if (tti ? !get_map4(&tm.mb, s.m.mb, L, IW, IH) : !get_map(&tm.mb, s.m.irho, L, IW, IH)) return TTI_ELAUNCH;
    if (!get_map(&tm.f3, s.adj3, L, TX, TY) || !get_map(&tm.f4, s.adj4, L, TX, TY)) return TTI_ELAUNCH;
    if (!make_store_map(&tm.snapc, s.store, s.snap_prec, L.nx(), L.ny(), L.nz(), 4 * s.nsnap, TX, TY) ||
        !make_store_map(&tm.gv, s.grad_vp, SNAP_F32, L.nx(), L.ny(), L.nz(), 1, TX, TY) ||
        !make_store_map(&tm.gr, s.grad_rho, SNAP_F32, L.nx(), L.ny(), L.nz(), 1, TX, TY))
        return TTI_ELAUNCH;
    ImgParams a{};
    a.snap_scale = s.snap_prec == SNAP_F32 ? nullptr : s.snap_scale;
    a.gvp = s.grad_vp;
    a.grho = s.grad_rho;
    a.L = L;
    const Split sp = s.bz > 0 ? Split{s.bz, s.ztop} : choose_split(L, KIND_IMG);
    if (!split_valid(L, sp)) return TTI_EINVAL;
    a.bz = sp.bz;
    a.ztop = sp.ztop;
    a.fs = s.free_surface;
    a.slot = s.slot;
    a.hx = 1.0 / s.dx;
    a.hy = 1.0 / s.dy;
    a.hz = 1.0 / s.dz;
    for (int r = 0; r < 4; ++r) {
        a.kcx[r] = pair(cs(r) * a.hx);
        a.kcy[r] = pair(cs(r) * a.hy);
        a.kcz[r] = pair(cs(r) * a.hz);
        a.kcxn[r] = pair(-cs(r) * a.hx);
        a.kcyn[r] = pair(-cs(r) * a.hy);
    }
    a.err = s.err ? s.err : err_word();
    if (!a.err) return TTI_ENOMEM;
    dim3 grid(cta_count(L, sp));
    if (!kernels_prepared()) return TTI_ELAUNCH;
    switch (s.snap_prec) {
    case SNAP_F32: return tti ? launch_image_t<true, float>(tm, a, grid, st) : launch_image_t<false, float>(tm, a, grid, st);
    case SNAP_F16: return tti ? launch_image_t<true, __half>(tm, a, grid, st) : launch_image_t<false, __half>(tm, a, grid, st);
    case SNAP_BF16:
        return tti ? launch_image_t<true, __nv_bfloat16>(tm, a, grid, st)
                   : launch_image_t<false, __nv_bfloat16>(tm, a, grid, st);
    default: return TTI_EINVAL;
    }
}

namespace {
T1Fd t1_fd(double dx, double dy, double dz)
{
    return T1Fd{(float)(1.0 / (dx * dx)), (float)(1.0 / (dy * dy)), (float)(1.0 / (dz * dz)),
                (float)(1.0 / (4 * dx * dy)), (float)(1.0 / (4 * dy * dz)), (float)(1.0 / (4 * dx * dz))};
}
} // namespace

int launch_t1_fused_forward(const Layout& L, const FwdStepArgs& s, int sponge, cudaStream_t st)
{
    if (!layout_supported(L)) return TTI_EINVAL;
    CUtensorMap mp, mq;
    if (!get_map(&mp, s.pin, L, IW, IH) || !get_map(&mq, s.qin, L, IW, IH)) return TTI_ELAUNCH;
    if (s.snap && s.snap_prec != SNAP_F32 && (!s.snap_scale || !s.snap_amax)) return TTI_EINVAL;
    T1FwdParams a{};
    a.pout = s.pout;
    a.qout = s.qout;
    a.f3 = s.f3;
    a.f4 = s.f4;
    a.m1 = s.m.m1;
    a.m2 = s.m.m2;
    a.m3 = s.m.m3;
    a.m4 = s.m.m4;
    a.rx = s.m.rx;
    a.ry = s.m.ry;
    a.rz = s.m.rz;
    a.abx = s.abx;
    a.aby = s.aby;
    a.abz = s.abz;
    a.snap = s.snap;
    a.snap_prec = s.snap_prec;
    a.snap_scale = s.snap_scale;
    a.snap_amax = s.snap_amax;
    a.src_index = s.src_index;
    a.src_term = s.src_term;
    a.L = L;
    const Split sp = s.bz > 0 ? Split{s.bz, s.ztop} : choose_split(L, KIND_T1F);
    if (!split_valid(L, sp)) return TTI_EINVAL;
    a.bz = sp.bz;
    a.ztop = sp.ztop;
    a.fs = s.free_surface;
    a.sponge = sponge;
    a.dt = s.dt;
    a.k = t1_fd(s.dx, s.dy, s.dz);
    a.err = s.err ? s.err : err_word();
    a.wave_prec = s.wave_prec;
    a.wave_scale = s.wave_scale;
    if (a.wave_prec && !a.wave_scale) return TTI_EINVAL;
    if (!a.err) return TTI_ENOMEM;
    if (!kernels_prepared()) return TTI_ELAUNCH;
    const dim3 grid(cta_count(L, sp));
    if (s.vti)
        k_t1_fused_forward_x2<false><<<grid, dim3(T1X2_TX, TY), T1F_SMEM, st>>>(mp, mq, a);
    else
        k_t1_fused_forward_x2<true><<<grid, dim3(T1X2_TX, TY), T1F_SMEM, st>>>(mp, mq, a);
    return launch_status();
}

int launch_t1_fused_adjoint(const Layout& L, const AdjStepArgs& s, cudaStream_t st)
{
    if (!layout_supported(L)) return TTI_EINVAL;
    T1AdjMaps tm;
    const float* arr[T1A_NARR] = {s.pin, s.qin, s.m.m1, s.m.m2, s.m.m3, s.m.m4, s.m.rx, s.m.ry, s.m.rz};
    for (int kk = 0; kk < T1A_NARR; ++kk)
        if (!get_map(&tm.m[kk], arr[kk], L, IW, IH)) return TTI_ELAUNCH;
    T1AdjParams a{};
    a.pout = s.pout;
    a.qout = s.qout;
    a.f3 = s.f3;
    a.f4 = s.f4;
    a.pin = s.pin;
    a.qin = s.qin;
    a.abx = s.abx;
    a.aby = s.aby;
    a.abz = s.abz;
    a.L = L;
    const Split sp = s.bz > 0 ? Split{s.bz, s.ztop} : choose_split(L, KIND_T1A);
    if (!split_valid(L, sp)) return TTI_EINVAL;
    a.bz = sp.bz;
    a.ztop = sp.ztop;
    a.fs = s.free_surface;
    a.sponge = s.sponge_active;
    a.dt = s.dt;
    a.k = t1_fd(s.dx, s.dy, s.dz);
    a.err = s.err ? s.err : err_word();
    a.wave_prec = s.wave_prec;
    a.wave_scale = s.wave_scale;
    if (a.wave_prec && !a.wave_scale) return TTI_EINVAL;
    if (!a.err) return TTI_ENOMEM;
    if (!kernels_prepared()) return TTI_ELAUNCH;
    const dim3 grid(cta_count(L, sp));
    if (s.vti)
        k_t1_fused_adjoint<false><<<grid, dim3(TX, TY), T1A_SMEM, st>>>(tm, a);
    else
        k_t1_fused_adjoint<true><<<grid, dim3(TX, TY), T1A_SMEM, st>>>(tm, a);
    return launch_status();
}

int launch_t1_image(const Layout& L, const ImageArgs& s, cudaStream_t st)
{
    if (!s.store || s.slot < 0 || s.slot >= s.nsnap) return TTI_EINVAL;
    if (s.snap_prec != SNAP_F32 && !s.snap_scale) return TTI_EINVAL;
    const int64_t nin = (int64_t)L.nx() * L.ny() * L.nz();
    const size_t elt = snap_elt_bytes(s.snap_prec);
    const unsigned char* s3 = static_cast<const unsigned char*>(s.store) + (size_t)s.slot * 2 * nin * elt;
    const unsigned char* s4 = s3 + (size_t)nin * elt;
    const float* sc = s.snap_prec == SNAP_F32 ? nullptr : s.snap_scale;
    const int blocks = (int)std::min<int64_t>((nin + 255) / 256, 148LL * 16);
    switch (s.snap_prec) {
    case SNAP_F32:
        k_t1_image<float><<<blocks, 256, 0, st>>>(reinterpret_cast<const float*>(s3), reinterpret_cast<const float*>(s4),
                                                   sc, s.adj3, s.adj4, s.grad_vp, L);
        break;
    case SNAP_F16:
        k_t1_image<__half><<<blocks, 256, 0, st>>>(reinterpret_cast<const __half*>(s3), reinterpret_cast<const __half*>(s4),
                                                    sc, s.adj3, s.adj4, s.grad_vp, L);
        break;
    case SNAP_BF16:
        k_t1_image<__nv_bfloat16><<<blocks, 256, 0, st>>>(reinterpret_cast<const __nv_bfloat16*>(s3),
                                                           reinterpret_cast<const __nv_bfloat16*>(s4), sc, s.adj3,
                                                           s.adj4, s.grad_vp, L);
        break;
    default: return TTI_EINVAL;
    }
    return launch_status();
}

int prepare_fused_kernels() { return kernels_prepared() ? TTI_OK : TTI_ELAUNCH; }

namespace {
// One CTA waits on a shared-memory mbarrier that expects bytes no copy will
// deliver: the bounded wait of the fused kernels gives up after its clock
// limit, records the timeout in the error word and the kernel returns.
// Nothing is in flight when it does.
__global__ void k_wait_selfcheck(int* err, unsigned long long limit)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_expect_tx(&bar, 16u);
    __syncthreads();
    if (mbar_try_wait(&bar, 0)) return;  // cannot complete: no copy was issued
    const long long t0 = clock64();
    while (!mbar_try_wait(&bar, 0))
        if ((unsigned long long)(clock64() - t0) > limit) {
            if (threadIdx.x == 0) atomicExch(err, 1);
            return;
        }
}
} // namespace

int wait_selfcheck(cudaStream_t st, long long limit_cycles)
{
    int* w = nullptr;
    if (cudaMallocAsync(&w, sizeof(int), st) != cudaSuccess) {
        cudaGetLastError();
        return TTI_ENOMEM;
    }
    cudaMemsetAsync(w, 0, sizeof(int), st);
    k_wait_selfcheck<<<1, 32, 0, st>>>(w, (unsigned long long)limit_cycles);
    int rc = launch_status();
    if (!rc) rc = fused_wait_status(st, w);
    cudaFreeAsync(w, st);
    cudaStreamSynchronize(st);
    cudaGetLastError();
    return rc;
}



namespace {
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, Split> g_tuned;  // (device, nx, ny, nz, kind) -> split
int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
    return dev;
}
} // namespace

bool split_valid(const Layout& L, Split sp)
{
    if (sp.bz < 1 || sp.ztop < 0 || sp.ztop >= L.nz()) return false;
    return sp.ztop == 0 || tile_count(L) < (long long)cta_count(L, sp);
}

void record_tuned_split(const Layout& L, int kind, Split sp)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const auto key = std::make_tuple(current_device(), L.nx(), L.ny(), L.nz(), kind);
    if (sp.bz > 0)
        g_tuned[key] = sp;
    else
        g_tuned.erase(key);
}

Split tuned_split(const Layout& L, int kind)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(std::make_tuple(current_device(), L.nx(), L.ny(), L.nz(), kind));
    return it == g_tuned.end() ? Split{} : it->second;
}

Split model_split(const Layout& L, int kind) { return pick_split(L, kind); }

Split choose_split(const Layout& L, int kind)
{
    const Split t = tuned_split(L, kind);
    return t.bz > 0 ? t : model_split(L, kind);
}

std::vector<Split> split_candidates(const Layout& L, int kind)
{
    std::vector<Split> c;
    for (int bz : plane_candidates(L)) c.push_back(Split{bz, 0});
    for (const Split& sp : topbottom_candidates(L, kind)) c.push_back(sp);
    return c;
}

// Bounded-wait status of the fused kernels on the current device: 0 if no
// wait gave up since the last call; the word is cleared.
int fused_wait_status(cudaStream_t st, int* word)
{
    int* w = word ? word : err_word();
    if (!w) return TTI_ENOMEM;
    int h = 0;
    if (cudaMemcpyAsync(&h, w, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return TTI_ELAUNCH;
    }
    if (h) {
        cudaMemsetAsync(w, 0, sizeof(int), st);
        cudaStreamSynchronize(st);
        return (h & 1) ? TTI_ETIMEOUT : TTI_ERANGE;
    }
    return TTI_OK;
}

} // namespace tti
