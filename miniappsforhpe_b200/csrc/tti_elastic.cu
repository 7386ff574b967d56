// Elastic step kernels of the reference's simulator3 (its eTTI proxy):
// velocity gradients, the z-mixed interpolations, the stress update with 21
// Cij, the velocity update, the free-surface mirrors and the pressure, with
// the reference's constants and arithmetic (simulator3/simulator3SetUp.cu).
//
// The reference's proxy is a stand-in: its first-derivative and
// interpolation tables are {1.01, 2.01, 3.01, 4.01}, its inverse spacings
// are hard-coded (1.01, 2.01 or 2.02, and zprime[iz] in z), and its model
// is cos/sin of the cell indices.  These kernels reproduce it as it is, so
// that its step can be dropped in.  They are short single-pass stencils
// over many volumes: blocks of 32x8 threads walk z through a column tile,
// every operand of a plane staged in double-buffered shared tiles by
// asynchronous copies while the previous plane is used, and z taps kept in
// per-thread register windows (the reference's shared planes and register
// queues, with the copies in flight a plane ahead).
//
// Volumes: FP32, x fastest, radius-4 halo on every axis, interior cells
// [4, 4+n-1] per axis, idx = (iz*ldimy + iy)*ldimx + ix.
#include <cuda_runtime.h>

#include <cstdint>
#include <initializer_list>

#include <cuda_pipeline.h>

#include "tti_common.cuh"

namespace tti {
namespace {

constexpr int E3X = 32, E3Y = 8;  // threads per block: one warp row per y
constexpr int E3Z = 16;           // planes per thread (point-wise kernels)
constexpr int E3ZC = 64;          // planes per thread (z-windowed velocity kernels)

__device__ __forceinline__ float e3_df(int i)
{
    constexpr float c[4] = {1.01f, 2.01f, 3.01f, 4.01f};  // DF_order8 (simulator3SetUp.cu:31)
    return c[i];
}
__device__ __forceinline__ float e3_int(int i)
{
    constexpr float c[4] = {1.01f, 2.01f, 3.01f, 4.01f};  // INT_S_O8 (simulator3SetUp.cu:32)
    return c[i];
}

struct E3Grid {
    int nx, ny, nz, ldimx, ldimy;
    __device__ int64_t idx(int ix, int iy, int iz) const { return ((int64_t)iz * ldimy + iy) * ldimx + ix; }
};

dim3 e3_blocks(const E3Grid& g, int zper) { return dim3((g.nx + E3X - 1) / E3X, (g.ny + E3Y - 1) / E3Y, (g.nz + zper - 1) / zper); }

// z-window derivatives on a 9-plane register window w[k] = plane iz+k-4, with
// drv1_8's tap order (simulator3SetUp.cu:37-45): unshifted reaches -3..+4,
// shifted -4..+3.
__device__ __forceinline__ float zdrv(const float (&w)[9], bool shift)
{
    const int b = shift ? 3 : 4;  // plane of the first difference's lower tap
    float d = e3_df(0) * (w[b + 1] - w[b]);
#pragma unroll
    for (int i = 1; i < 4; ++i) d += e3_df(i) * (w[b + 1 + i] - w[b - i]);
    return d;
}

// Shift a 9-plane window one plane down and append the new plane's value.
__device__ __forceinline__ void zpush(float (&w)[9], float v)
{
#pragma unroll
    for (int k = 0; k < 8; ++k) w[k] = w[k + 1];
    w[8] = v;
}

// drv1_8<SHIFT, STRIDE> (simulator3SetUp.cu:37-45) on a shared-memory tile
// (stride s between taps).
template <bool SHIFT>
__device__ __forceinline__ float drv8s(const float* p, int s)
{
    constexpr int is = SHIFT ? -1 : 0;
    float d = e3_df(0) * (p[(is + 1) * s] - p[is * s]);
#pragma unroll
    for (int i = 1; i < 4; ++i) d += e3_df(i) * (p[(is + i + 1) * s] - p[(is - i) * s]);
    return d;
}

// Stage rows ys .. ys+R-1, columns xs .. xs+C-1 of one plane into t by
// asynchronous copies (LDGSTS) of V floats (1, or 4 when ldimx is a
// multiple of 4 and the volumes are 16-byte aligned: then, xs being a
// multiple of 4, a chunk lies wholly inside or wholly past a row's end);
// the caller commits and waits.  Cells past the allocation's row or plane
// end are zeroed directly (no interior output reads them).
template <int V, int R, int C>
__device__ __forceinline__ void stage_tile_async(float (&t)[R][C], const float* __restrict__ plane, int xs, int ys,
                                                 const E3Grid& g, int tid)
{
    static_assert(C % V == 0, "rows of whole chunks");
    constexpr int CC = C / V;
    for (int e = tid; e < R * CC; e += E3X * E3Y) {
        const int r = e / CC, c = V * (e - r * CC), x = xs + c, y = ys + r;
        if (x < g.ldimx && y < g.ldimy) {
            __pipeline_memcpy_async(&t[r][c], plane + (int64_t)y * g.ldimx + x, V * sizeof(float));
        } else {
#pragma unroll
            for (int k = 0; k < V; ++k) t[r][c + k] = 0.0f;
        }
    }
}

// vgPlainKernel (simulator3SetUp.cu:1218-1362): the six strain volumes.  A
// block walks E3ZC planes of a 32x8 column tile: the x/y taps of each plane
// come from shared-memory tiles of f1, f2, f3 with a halo of 4, the z taps
// from per-thread register windows (one load per plane and field), as the
// reference's shared planes and queues do.
template <int V>
__global__ void __launch_bounds__(E3X* E3Y) k_e3_vgplain(const float* __restrict__ f1, const float* __restrict__ f2,
                                                        const float* __restrict__ f3, float* __restrict__ d4,
                                                        float* __restrict__ d5, float* __restrict__ d6,
                                                        float* __restrict__ d7, float* __restrict__ d8,
                                                        float* __restrict__ d9, const float* __restrict__ zprime,
                                                        E3Grid g)
{
    __shared__ __align__(16) float t1[2][E3Y + 8][E3X + 8], t2[2][E3Y + 8][E3X + 8], t3[2][E3Y + 8][E3X + 8];
    __shared__ __align__(16) float tw[2][3][E3Y][E3X];  // f1, f2, f3 of plane iz+4 (the windows' new plane)
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * E3X + tx;
    const int x0 = 4 + blockIdx.x * E3X, y0 = 4 + blockIdx.y * E3Y;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool act = ix < 4 + g.nx && iy < 4 + g.ny;
    const float invd1 = 1.01f, invd2 = 2.02f;
    const int64_t sz = (int64_t)g.ldimx * g.ldimy;
    const int z0 = 4 + blockIdx.z * E3ZC, z1 = min(z0 + E3ZC, 4 + g.nz);
    float w1[9] = {}, w2[9] = {}, w3[9] = {};  // planes iz-4 .. iz+4
    if (act) {
        const int64_t i0 = g.idx(ix, iy, z0 - 4);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            w1[k + 1] = __ldg(f1 + i0 + k * sz);
            w2[k + 1] = __ldg(f2 + i0 + k * sz);
            w3[k + 1] = __ldg(f3 + i0 + k * sz);
        }
    }
    // planes double-buffered: plane iz+1 is copied in while plane iz is used
    auto stage = [&](int b, int iz) {
        const int64_t pb = (int64_t)iz * sz;
        stage_tile_async<V>(t1[b], f1 + pb, x0 - 4, y0 - 4, g, tid);
        stage_tile_async<V>(t2[b], f2 + pb, x0 - 4, y0 - 4, g, tid);
        stage_tile_async<V>(t3[b], f3 + pb, x0 - 4, y0 - 4, g, tid);
        const int64_t pw = pb + 4 * sz;
        stage_tile_async<V>(tw[b][0], f1 + pw, x0, y0, g, tid);
        stage_tile_async<V>(tw[b][1], f2 + pw, x0, y0, g, tid);
        stage_tile_async<V>(tw[b][2], f3 + pw, x0, y0, g, tid);
        __pipeline_commit();
    };
    if (z0 < z1) stage(0, z0);
    for (int iz = z0, b = 0; iz < z1; ++iz, b ^= 1) {
        const int64_t i = g.idx(ix, iy, iz);
        if (iz + 1 < z1) stage(b ^ 1, iz + 1);
        __pipeline_wait_prior(iz + 1 < z1 ? 1 : 0);
        __syncthreads();
        if (act) {
            zpush(w1, tw[b][0][ty][tx]);
            zpush(w2, tw[b][1][ty][tx]);
            zpush(w3, tw[b][2][ty][tx]);
            constexpr int S = E3X + 8;
            const float* c1 = &t1[b][ty + 4][tx + 4];
            const float* c2 = &t2[b][ty + 4][tx + 4];
            const float* c3 = &t3[b][ty + 4][tx + 4];
            const float d19 = drv8s<false>(c1, 1), d20 = drv8s<false>(c2, S), d21 = zdrv(w3, false);
            const float d22 = drv8s<true>(c1, S), d23 = drv8s<true>(c2, 1), d24 = zdrv(w1, true);
            const float d25 = drv8s<true>(c3, 1), d26 = zdrv(w2, true), d27 = drv8s<true>(c3, S);
            const float zpr = __ldg(zprime + iz);
            d4[i] = invd1 * d19;
            d5[i] = invd2 * d22 + invd1 * d23;
            d6[i] = zpr * d24 + invd1 * d25;
            d7[i] = invd2 * d20;
            d8[i] = zpr * d26 + invd2 * d27;
            d9[i] = zpr * d21;
        }
        __syncthreads();
    }
}

// precompute_xz_yz<XS, YS, ZS> (simulator3SetUp.cu:47-187), in the
// reference's own form: a thread walks one 64-plane z block of its column
// (the reference launch's blocks) and keeps the partial sums of the eight
// outputs a plane feeds in a register queue.  Plane s of the block (the
// block's planes start at P0 = 64 b + 1 - ZS) adds, to queue slot i (the
// output m = s - 7 + i), the pair at x offsets X1 + i and X2 - i (X1 = -3 -
// XS, X2 = 4 - XS; likewise in y) weighted by INT_S_O8[max(3 - i, i - 4)]
// -- except that planes s <= 6, which the reference adds while priming its
// queues, weigh by INT_S_O8[max(3 - s, s - 4)] (its loop at :120-129 uses
// the arriving plane's index): the blocking shows in its result, and it is
// kept.  Slot 0 is complete once its eighth plane has arrived.  The planes
// come through double-buffered shared tiles with a halo of 4.
template <int XS, int YS, int ZS, int V>
__global__ void __launch_bounds__(E3X* E3Y) k_e3_precompute(const float* __restrict__ in, float* __restrict__ xz,
                                                           float* __restrict__ yz, E3Grid g)
{
    // planes staged in triple-buffered shared tiles (halo 4) by async copies,
    // two planes in flight while one is used
    __shared__ __align__(16) float t[3][E3Y + 8][E3X + 8];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * E3X + tx;
    const int x0 = 4 + blockIdx.x * E3X, y0 = 4 + blockIdx.y * E3Y;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool act = ix < 4 + g.nx && iy < 4 + g.ny;
    constexpr int X1 = -3 - XS, X2 = 4 - XS, Y1 = -3 - YS, Y2 = 4 - YS;
    const int b = blockIdx.z;
    const int mend = min(64, g.nz - 64 * b), p0 = 64 * b + 1 - ZS;
    const int64_t sz = (int64_t)g.ldimx * g.ldimy;
    float* oxz = xz + g.idx(ix, iy, 4 + 64 * b);
    float* oyz = yz + g.idx(ix, iy, 4 + 64 * b);
    float qxz[8], qyz[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) qxz[i] = qyz[i] = 0.0f;
    const int ns = mend + 7;
    auto stage = [&](int bb, int s) {
        stage_tile_async<V>(t[bb], in + (int64_t)(p0 + s) * sz, x0 - 4, y0 - 4, g, tid);
        __pipeline_commit();
    };
    stage(0, 0);
    if (ns > 1) stage(1, 1);
    for (int s = 0, bb = 0; s < ns; ++s, bb = bb == 2 ? 0 : bb + 1) {
        if (s + 2 < ns) stage(bb == 0 ? 2 : bb - 1, s + 2);  // the buffer plane s-1 used
        __pipeline_wait_prior(s + 2 < ns ? 2 : s + 1 < ns ? 1 : 0);
        __syncthreads();
        const float* pl = &t[bb][ty + 4][tx + 4];
        constexpr int S = E3X + 8;
        if (s <= 6) {  // priming: one weight for the whole plane
            const int ic = max(3 - s, s - 4);
            const float c = ic == 0 ? e3_int(0) : ic == 1 ? e3_int(1) : ic == 2 ? e3_int(2) : e3_int(3);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                qxz[i] += c * (pl[X1 + i] + pl[X2 - i]);
                qyz[i] += c * (pl[(Y1 + i) * S] + pl[(Y2 - i) * S]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float c = e3_int(max(3 - i, i - 4));
                qxz[i] += c * (pl[X1 + i] + pl[X2 - i]);
                qyz[i] += c * (pl[(Y1 + i) * S] + pl[(Y2 - i) * S]);
            }
        }
        const int m = s - 7;  // the output slot 0 holds
        if (act && m >= 0) {
            oxz[m * sz] = 0.5f * qxz[0];
            oyz[m * sz] = 0.5f * qyz[0];
        }
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            qxz[i] = qxz[i + 1];
            qyz[i] = qyz[i + 1];
        }
        qxz[7] = qyz[7] = 0.0f;
        __syncthreads();  // every thread is done with buffer bb before it is refilled
    }
}

struct E3Stress {
    float *f4, *f5, *f6, *f7, *f8, *f9;
    const float* M[21];
    const float *e11, *e12, *e13, *e22, *e23, *e33;  // f1_1, f1_2, f1_3, f2_2, f2_3, f3_3
    const float* p[12];                             // f10 .. f21
};

// mixed_XY<XS, YS> (simulator3SetUp.cu:214-227) on a shared-memory tile
// (row stride sy).
template <bool XS, bool YS>
__device__ __forceinline__ float mixed8s(const float* p, int sy)
{
    constexpr int xs = XS ? -1 : 0, ys = YS ? -1 : 0;
    float d = 0.0f;
#pragma unroll
    for (int i = 0; i < 4; ++i)
        d += e3_int(i) * (p[(ys + i + 1) * sy + xs + i + 1] + p[(ys + i + 1) * sy + xs - i] +
                          p[(ys - i) * sy + xs + i + 1] + p[(ys - i) * sy + xs - i]);
    return 0.5f * d;
}

// sPlainKernel (simulator3SetUp.cu:980-1103): the stress update.  A block
// walks E3ZS planes of a 32x8 column tile; every array it reads comes
// through shared memory, double-buffered and filled by asynchronous copies
// while the previous plane is used: the 21 Cij, the 12 z-mixed volumes and
// the 6 stresses it updates as 32x8 tiles, the 6 strains as tiles with a
// halo of 4 for their mixed x/y taps.
constexpr int E3ZS = 16;                         // planes per block
constexpr int E3C = E3X * E3Y;                   // a center tile
constexpr int E3H = (E3Y + 8) * (E3X + 8);       // a tile with a halo of 4
constexpr int E3SBUF = 39 * E3C + 6 * E3H;       // floats per buffer
constexpr size_t E3S_SMEM = 2 * E3SBUF * sizeof(float);

template <int V>
__global__ void __launch_bounds__(E3X* E3Y, 2) k_e3_splain(E3Stress a, E3Grid g)
{
    extern __shared__ __align__(16) float e3s[];
    using Ctile = float[E3Y][E3X];
    using Htile = float[E3Y + 8][E3X + 8];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * E3X + tx;
    const int x0 = 4 + blockIdx.x * E3X, y0 = 4 + blockIdx.y * E3Y;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool act = ix < 4 + g.nx && iy < 4 + g.ny;
    const int64_t sz = (int64_t)g.ldimx * g.ldimy;
    const int z0 = 4 + blockIdx.z * E3ZS, z1 = min(z0 + E3ZS, 4 + g.nz);
    const float* const ein[6] = {a.e11, a.e12, a.e13, a.e22, a.e23, a.e33};
    float* const fout[6] = {a.f4, a.f5, a.f6, a.f7, a.f8, a.f9};
    auto ctile = [&](int b, int k) -> Ctile& { return *reinterpret_cast<Ctile*>(e3s + b * E3SBUF + k * E3C); };
    auto htile = [&](int b, int k) -> Htile& {
        return *reinterpret_cast<Htile*>(e3s + b * E3SBUF + 39 * E3C + k * E3H);
    };
    // tiles 0..20: M1..M21, 21..32: f10..f21, 33..38: f4..f9; halo tiles: e11, e12, e13, e22, e23, e33
    auto stage = [&](int b, int iz) {
        const int64_t pb = (int64_t)iz * sz;
        for (int k = 0; k < 21; ++k) stage_tile_async<V>(ctile(b, k), a.M[k] + pb, x0, y0, g, tid);
        for (int k = 0; k < 12; ++k) stage_tile_async<V>(ctile(b, 21 + k), a.p[k] + pb, x0, y0, g, tid);
        for (int k = 0; k < 6; ++k) stage_tile_async<V>(ctile(b, 33 + k), fout[k] + pb, x0, y0, g, tid);
        for (int k = 0; k < 6; ++k) stage_tile_async<V>(htile(b, k), ein[k] + pb, x0 - 4, y0 - 4, g, tid);
        __pipeline_commit();
    };
    if (z0 < z1) stage(0, z0);
    for (int iz = z0, b = 0; iz < z1; ++iz, b ^= 1) {
        if (iz + 1 < z1) stage(b ^ 1, iz + 1);
        __pipeline_wait_prior(iz + 1 < z1 ? 1 : 0);
        __syncthreads();
        if (act) {
            const int64_t i = g.idx(ix, iy, iz);
            constexpr int S = E3X + 8;
            auto m = [&](int k) { return ctile(b, k - 1)[ty][tx]; };
            auto p = [&](int k) { return ctile(b, 21 + k - 10)[ty][tx]; };  // f10 .. f21
            auto f = [&](int k) { return ctile(b, 33 + k)[ty][tx]; };       // f4 .. f9
            const float* c11 = &htile(b, 0)[ty + 4][tx + 4];
            const float* c12 = &htile(b, 1)[ty + 4][tx + 4];
            const float* c13 = &htile(b, 2)[ty + 4][tx + 4];
            const float* c22 = &htile(b, 3)[ty + 4][tx + 4];
            const float* c23 = &htile(b, 4)[ty + 4][tx + 4];
            const float* c33 = &htile(b, 5)[ty + 4][tx + 4];
            const float d19 = *c11, d20 = *c22, d21 = *c33, d22 = *c12, d24 = *c13, d26 = *c23;
            const float xx12 = mixed8s<false, false>(c12, S), xx13 = p(14), xx23 = p(19);
            a.f4[i] = f(0) + (m(1) * d19 + m(2) * d20 + m(3) * d21 + m(6) * xx12 + m(5) * xx13 + m(4) * xx23);
            a.f5[i] = f(1) + (m(2) * d19 + m(7) * d20 + m(8) * d21 + m(11) * xx12 + m(10) * xx13 + m(9) * xx23);
            a.f6[i] = f(2) + (m(3) * d19 + m(8) * d20 + m(12) * d21 + m(15) * xx12 + m(14) * xx13 + m(13) * xx23);
            const float xy11 = mixed8s<true, true>(c11, S), xy22 = mixed8s<true, true>(c22, S);
            const float xy33 = mixed8s<true, true>(c33, S), xy13 = p(15), xy23 = p(18);
            a.f7[i] = f(3) + (m(6) * xy11 + m(11) * xy22 + m(15) * xy33 + m(20) * xy13 + m(18) * xy23 + m(21) * d22);
            const float xz11 = p(10), xz22 = p(16), xz33 = p(20), xz12 = p(13);
            const float xz23 = mixed8s<true, false>(c23, S);
            a.f8[i] = f(4) + (m(5) * xz11 + m(10) * xz22 + m(14) * xz33 + m(20) * xz12 + m(17) * xz23 + m(19) * d24);
            const float yz11 = p(11), yz22 = p(17), yz33 = p(21), yz12 = p(12);
            const float yz13 = mixed8s<false, true>(c13, S);
            a.f9[i] = f(5) + (m(4) * yz11 + m(9) * yz22 + m(13) * yz33 + m(18) * yz12 + m(17) * yz13 + m(16) * d26);
        }
        __syncthreads();  // buffer b is refilled next iteration
    }
}

// vPlainKernel (simulator3SetUp.cu:820-979): the velocity update.  As for
// the strains: x/y taps of f4, f5, f7, f8, f9 from shared-memory tiles of
// each plane, z taps of f6, f8, f9 from register windows, and M22 of the
// plane below kept from the previous plane; M22 (with the row above and
// the columns left of the tile) and the three velocities it updates come
// through shared tiles of the plane too.
template <int V>
__global__ void __launch_bounds__(E3X* E3Y) k_e3_vplain(float* __restrict__ f1, float* __restrict__ f2,
                                                       float* __restrict__ f3, const float* __restrict__ f4,
                                                       const float* __restrict__ f5, const float* __restrict__ f6,
                                                       const float* __restrict__ f7, const float* __restrict__ f8,
                                                       const float* __restrict__ f9, const float* __restrict__ M22,
                                                       const float* __restrict__ zprime, E3Grid g)
{
    __shared__ __align__(16) float t4[2][E3Y][E3X + 8], t8[2][E3Y][E3X + 8];  // x taps
    __shared__ __align__(16) float t5[2][E3Y + 8][E3X], t9[2][E3Y + 8][E3X];  // y taps
    __shared__ __align__(16) float t7[2][E3Y + 8][E3X + 8];                   // x and y taps
    __shared__ __align__(16) float tm[2][E3Y + 1][E3X + 4];                   // M22: rows y0-1.., cols x0-4..
    __shared__ __align__(16) float tv[2][3][E3Y][E3X];                        // f1, f2, f3
    __shared__ __align__(16) float tw[2][3][E3Y][E3X];  // f6, f8, f9 of plane iz+4 (the windows' new plane)
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * E3X + tx;
    const int x0 = 4 + blockIdx.x * E3X, y0 = 4 + blockIdx.y * E3Y;
    const int ix = x0 + tx, iy = y0 + ty;
    const bool act = ix < 4 + g.nx && iy < 4 + g.ny;
    const float invd1 = 1.01f, invd2 = 2.01f;
    const int64_t sz = (int64_t)g.ldimx * g.ldimy;
    const int z0 = 4 + blockIdx.z * E3ZC, z1 = min(z0 + E3ZC, 4 + g.nz);
    float w6[9] = {}, w8[9] = {}, w9[9] = {};  // planes iz-4 .. iz+4
    float m22z = 0.0f;
    if (act) {
        const int64_t i0 = g.idx(ix, iy, z0 - 4);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            w6[k + 1] = __ldg(f6 + i0 + k * sz);
            w8[k + 1] = __ldg(f8 + i0 + k * sz);
            w9[k + 1] = __ldg(f9 + i0 + k * sz);
        }
        m22z = __ldg(M22 + g.idx(ix, iy, z0 - 1));
    }
    // planes double-buffered: plane iz+1 is copied in while plane iz is used
    auto stage = [&](int b, int iz) {
        const int64_t pb = (int64_t)iz * sz;
        stage_tile_async<V>(t4[b], f4 + pb, x0 - 4, y0, g, tid);
        stage_tile_async<V>(t8[b], f8 + pb, x0 - 4, y0, g, tid);
        stage_tile_async<V>(t5[b], f5 + pb, x0, y0 - 4, g, tid);
        stage_tile_async<V>(t9[b], f9 + pb, x0, y0 - 4, g, tid);
        stage_tile_async<V>(t7[b], f7 + pb, x0 - 4, y0 - 4, g, tid);
        stage_tile_async<V>(tm[b], M22 + pb, x0 - 4, y0 - 1, g, tid);
        stage_tile_async<V>(tv[b][0], f1 + pb, x0, y0, g, tid);
        stage_tile_async<V>(tv[b][1], f2 + pb, x0, y0, g, tid);
        stage_tile_async<V>(tv[b][2], f3 + pb, x0, y0, g, tid);
        const int64_t pw = pb + 4 * sz;
        stage_tile_async<V>(tw[b][0], f6 + pw, x0, y0, g, tid);
        stage_tile_async<V>(tw[b][1], f8 + pw, x0, y0, g, tid);
        stage_tile_async<V>(tw[b][2], f9 + pw, x0, y0, g, tid);
        __pipeline_commit();
    };
    if (z0 < z1) stage(0, z0);
    for (int iz = z0, b = 0; iz < z1; ++iz, b ^= 1) {
        const int64_t i = g.idx(ix, iy, iz);
        if (iz + 1 < z1) stage(b ^ 1, iz + 1);
        __pipeline_wait_prior(iz + 1 < z1 ? 1 : 0);
        __syncthreads();
        if (act) {
            zpush(w6, tw[b][0][ty][tx]);
            zpush(w8, tw[b][1][ty][tx]);
            zpush(w9, tw[b][2][ty][tx]);
            const float m22c = tm[b][ty + 1][tx + 4], mx = tm[b][ty + 1][tx + 3], my = tm[b][ty][tx + 4];
            const float d10 = drv8s<true>(&t4[b][ty][tx + 4], 1), d11 = drv8s<true>(&t5[b][ty + 4][tx], E3X);
            const float d12 = zdrv(w6, true);
            const float d13 = drv8s<false>(&t7[b][ty + 4][tx + 4], 1);
            const float d14 = drv8s<false>(&t7[b][ty + 4][tx + 4], E3X + 8);
            const float d15 = zdrv(w8, false);
            const float d16 = drv8s<false>(&t8[b][ty][tx + 4], 1), d17 = drv8s<false>(&t9[b][ty + 4][tx], E3X);
            const float d18 = zdrv(w9, false);
            const float zpr = __ldg(zprime + iz);
            f1[i] = tv[b][0][ty][tx] + (2.0f * mx) * (d10 * invd1 + d14 * invd2 + d15 * zpr);
            f2[i] = tv[b][1][ty][tx] + (2.0f * my) * (d13 * invd1 + d11 * invd2 + d18 * zpr);
            f3[i] = tv[b][2][ty][tx] + (2.0f * m22z) * (d16 * invd1 + d17 * invd2 + d12 * zpr);
            m22z = m22c;
        }
        __syncthreads();
    }
}

// mirror_s_kernel / mirror_v_kernel (simulator3SetUp.cu:1387-1492): zero at
// the surface izbeg, the negated mirror 2*izbeg - iz above it.
struct E3Fields {
    float* f[6];
};
__global__ void k_e3_mirror(E3Fields a, int nf, int64_t plane, int izbeg)
{
    const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int iz = blockIdx.z;
    if (j >= plane) return;
    const int64_t i = iz * plane + j;
    for (int k = 0; k < nf; ++k) a.f[k][i] = iz == izbeg ? 0.0f : -a.f[k][(2 * izbeg - iz) * plane + j];
}

// update_gv (simulator3SetUp.cu:1494-1511): the velocity image
// g += a_v1 * snap_v1 + a_v3 * snap_v3, with g and the snapshots in the
// halo-free layout (leading dimensions gx, gy) and the adjoint velocities in
// the halo'd one.
__global__ void __launch_bounds__(E3X* E3Y) k_e3_update_gv(float* __restrict__ g, const float* __restrict__ s1,
                                                          const float* __restrict__ s3,
                                                          const float* __restrict__ a1,
                                                          const float* __restrict__ a3, E3Grid grid, int gx, int gy)
{
    const int x = blockIdx.x * E3X + threadIdx.x, y = blockIdx.y * E3Y + threadIdx.y;
    if (x >= grid.nx || y >= grid.ny) return;
    const int z0 = blockIdx.z * E3Z, z1 = min(z0 + E3Z, grid.nz);
    for (int z = z0; z < z1; ++z) {
        const int64_t gi = ((int64_t)z * gy + y) * gx + x, ai = grid.idx(x + 4, y + 4, z + 4);
        g[gi] += __ldg(a1 + ai) * __ldg(s1 + gi) + __ldg(a3 + ai) * __ldg(s3 + gi);
    }
}

// compute_p_kernel (simulator3SetUp.cu:275-289)
__global__ void k_e3_pressure(float* __restrict__ p, const float* __restrict__ f4, const float* __restrict__ f5,
                              const float* __restrict__ f6, const float* __restrict__ f7,
                              const float* __restrict__ f8, const float* __restrict__ f9, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    p[i] = -(2.0f * f4[i] + 3.0f * f5[i] + 4.0f * f6[i] + 5.0f * f7[i] + 6.0f * f8[i] + 7.0f * f9[i]) / 27.0f;
}

// init_cijs_kernel (simulator3SetUp.cu:229-273): the stand-in model, over
// the interior x range and every y and z of the allocation.
struct E3Model {
    float* M[22];
    float* d[6];
    float* zprime;
};
__global__ void k_e3_init_model(E3Model a, int nx, int ldimx, int ldimy, int ldimz)
{
    const int ix = 4 + blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y, iz = blockIdx.z;
    if (ix >= 4 + nx) return;
    if (ix == 4 && iy == 0) a.zprime[iz] = cosf(6.0f * iz);
    const int64_t i = ((int64_t)iz * ldimy + iy) * ldimx + ix;
    const float t[11] = {2.0f * iz + iy + ix, iz + 2.0f * iy + ix, iz + iy + 2.0f * ix, 3.0f * iz + iy + ix,
                         iz + 3.0f * iy + ix, iz + iy + 3.0f * ix, 4.0f * iz + iy + ix, iz + 4.0f * iy + ix,
                         iz + iy + 4.0f * ix, 5.0f * iz + iy + ix, iz + 5.0f * iy + ix};
#pragma unroll
    for (int k = 0; k < 11; ++k) {
        a.M[2 * k][i] = cosf(t[k]);
        a.M[2 * k + 1][i] = sinf(t[k]);
    }
    a.d[0][i] = cosf(iz + iy + 5.0f * ix);
    a.d[1][i] = sinf(iz + iy + 5.0f * ix);
    a.d[2][i] = cosf(6.0f * iz + iy + ix);
    a.d[3][i] = sinf(6.0f * iz + iy + ix);
    a.d[4][i] = cosf(iz + 6.0f * iy + ix);
    a.d[5][i] = sinf(iz + 6.0f * iy + ix);
}

inline cudaStream_t S(tti_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// 16-byte staging copies need rows of whole 4-float chunks and aligned volumes.
bool vec4_ok(int ldimx, std::initializer_list<const float*> vols)
{
    if (ldimx % 4) return false;
    for (const float* v : vols)
        if (reinterpret_cast<uintptr_t>(v) % 16) return false;
    return true;
}

bool e3_grid_ok(int nx, int ny, int nz, int ldimx, int ldimy)
{
    return nx > 0 && ny > 0 && nz > 0 && ldimx >= nx + 8 && ldimy >= ny + 8;
}

} // namespace
} // namespace tti

using namespace tti;

extern "C" {

int tti_e3_launch_vgplain(const float* f1, const float* f2, const float* f3, float* d4, float* d5, float* d6,
                          float* d7, float* d8, float* d9, const float* zprime, int nx, int ny, int nz, int ldimx,
                          int ldimy, tti_stream_t stream)
{
    if (!e3_grid_ok(nx, ny, nz, ldimx, ldimy) || !f1 || !f2 || !f3 || !d4 || !d5 || !d6 || !d7 || !d8 || !d9 ||
        !zprime)
        return TTI_EINVAL;
    const E3Grid g{nx, ny, nz, ldimx, ldimy};
    if (vec4_ok(ldimx, {f1, f2, f3}))
        k_e3_vgplain<4><<<e3_blocks(g, E3ZC), dim3(E3X, E3Y), 0, S(stream)>>>(f1, f2, f3, d4, d5, d6, d7, d8, d9,
                                                                              zprime, g);
    else
        k_e3_vgplain<1><<<e3_blocks(g, E3ZC), dim3(E3X, E3Y), 0, S(stream)>>>(f1, f2, f3, d4, d5, d6, d7, d8, d9,
                                                                              zprime, g);
    return launch_status();
}

int tti_e3_launch_splain(float* f4, float* f5, float* f6, float* f7, float* f8, float* f9, const float* const* M,
                         const float* f1_1, const float* f1_2, const float* f1_3, const float* f2_2,
                         const float* f2_3, const float* f3_3, float* const* f10_21, int nx, int ny, int nz,
                         int ldimx, int ldimy, tti_stream_t stream)
{
    if (!e3_grid_ok(nx, ny, nz, ldimx, ldimy) || !f4 || !f5 || !f6 || !f7 || !f8 || !f9 || !M || !f10_21 || !f1_1 ||
        !f1_2 || !f1_3 || !f2_2 || !f2_3 || !f3_3)
        return TTI_EINVAL;
    for (int k = 0; k < 21; ++k)
        if (!M[k]) return TTI_EINVAL;
    for (int k = 0; k < 12; ++k)
        if (!f10_21[k]) return TTI_EINVAL;
    const E3Grid g{nx, ny, nz, ldimx, ldimy};
    cudaStream_t st = S(stream);
    // the six z-mixed precomputes of sPlainLoop (simulator3SetUp.cu:1177-1186)
    const dim3 pb((nx + E3X - 1) / E3X, (ny + E3Y - 1) / E3Y, (nz - 1) / 64 + 1), t(E3X, E3Y);
    float* const* p = f10_21;
    if (vec4_ok(ldimx, {f1_1, f2_2, f3_3, f1_2, f1_3, f2_3})) {
        k_e3_precompute<1, 1, 1, 4><<<pb, t, 0, st>>>(f1_1, p[0], p[1], g);
        k_e3_precompute<1, 1, 1, 4><<<pb, t, 0, st>>>(f2_2, p[6], p[7], g);
        k_e3_precompute<1, 1, 1, 4><<<pb, t, 0, st>>>(f3_3, p[10], p[11], g);
        k_e3_precompute<0, 0, 1, 4><<<pb, t, 0, st>>>(f1_2, p[2], p[3], g);
        k_e3_precompute<0, 1, 0, 4><<<pb, t, 0, st>>>(f1_3, p[4], p[5], g);
        k_e3_precompute<1, 0, 0, 4><<<pb, t, 0, st>>>(f2_3, p[8], p[9], g);
    } else {
        k_e3_precompute<1, 1, 1, 1><<<pb, t, 0, st>>>(f1_1, p[0], p[1], g);
        k_e3_precompute<1, 1, 1, 1><<<pb, t, 0, st>>>(f2_2, p[6], p[7], g);
        k_e3_precompute<1, 1, 1, 1><<<pb, t, 0, st>>>(f3_3, p[10], p[11], g);
        k_e3_precompute<0, 0, 1, 1><<<pb, t, 0, st>>>(f1_2, p[2], p[3], g);
        k_e3_precompute<0, 1, 0, 1><<<pb, t, 0, st>>>(f1_3, p[4], p[5], g);
        k_e3_precompute<1, 0, 0, 1><<<pb, t, 0, st>>>(f2_3, p[8], p[9], g);
    }
    E3Stress a{};
    float* out[6] = {f4, f5, f6, f7, f8, f9};
    a.f4 = out[0];
    a.f5 = out[1];
    a.f6 = out[2];
    a.f7 = out[3];
    a.f8 = out[4];
    a.f9 = out[5];
    for (int k = 0; k < 21; ++k) a.M[k] = M[k];
    a.e11 = f1_1;
    a.e12 = f1_2;
    a.e13 = f1_3;
    a.e22 = f2_2;
    a.e23 = f2_3;
    a.e33 = f3_3;
    for (int k = 0; k < 12; ++k) a.p[k] = p[k];
    const dim3 sb = e3_blocks(g, E3ZS);
    if (cudaFuncSetAttribute(k_e3_splain<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)E3S_SMEM) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_e3_splain<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)E3S_SMEM) !=
            cudaSuccess)
        return TTI_ELAUNCH;
    if (vec4_ok(ldimx, {f4, f5, f6, f7, f8, f9, f1_1, f1_2, f1_3, f2_2, f2_3, f3_3}) &&
        vec4_ok(ldimx, {M[0], M[1], M[2], M[3], M[4], M[5], M[6], M[7], M[8], M[9], M[10], M[11], M[12], M[13],
                        M[14], M[15], M[16], M[17], M[18], M[19], M[20]}) &&
        vec4_ok(ldimx, {p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], p[11]}))
        k_e3_splain<4><<<sb, t, E3S_SMEM, st>>>(a, g);
    else
        k_e3_splain<1><<<sb, t, E3S_SMEM, st>>>(a, g);
    return launch_status();
}

int tti_e3_launch_vplain(float* f1, float* f2, float* f3, const float* f4, const float* f5, const float* f6,
                         const float* f7, const float* f8, const float* f9, const float* M22, const float* zprime,
                         int nx, int ny, int nz, int ldimx, int ldimy, tti_stream_t stream)
{
    if (!e3_grid_ok(nx, ny, nz, ldimx, ldimy) || !f1 || !f2 || !f3 || !f4 || !f5 || !f6 || !f7 || !f8 || !f9 ||
        !M22 || !zprime)
        return TTI_EINVAL;
    const E3Grid g{nx, ny, nz, ldimx, ldimy};
    if (vec4_ok(ldimx, {f1, f2, f3, f4, f5, f6, f7, f8, f9, M22}))
        k_e3_vplain<4><<<e3_blocks(g, E3ZC), dim3(E3X, E3Y), 0, S(stream)>>>(f1, f2, f3, f4, f5, f6, f7, f8, f9, M22,
                                                                             zprime, g);
    else
        k_e3_vplain<1><<<e3_blocks(g, E3ZC), dim3(E3X, E3Y), 0, S(stream)>>>(f1, f2, f3, f4, f5, f6, f7, f8, f9, M22,
                                                                             zprime, g);
    return launch_status();
}

int tti_e3_launch_mirror(float* const* fields, int nfields, int ldimx, int ldimy, int ldimz, int izbeg,
                         tti_stream_t stream)
{
    if (!fields || nfields < 1 || nfields > 6 || ldimx < 1 || ldimy < 1 || izbeg < 0 || 2 * izbeg >= ldimz)
        return TTI_EINVAL;
    E3Fields a{};
    for (int k = 0; k < nfields; ++k) {
        if (!fields[k]) return TTI_EINVAL;
        a.f[k] = fields[k];
    }
    const int64_t plane = (int64_t)ldimx * ldimy;
    k_e3_mirror<<<dim3((unsigned)((plane + 1023) / 1024), 1, izbeg + 1), 1024, 0, S(stream)>>>(a, nfields, plane,
                                                                                               izbeg);
    return launch_status();
}

int tti_e3_launch_update_gv(float* g1, const float* snap_v1, const float* snap_v3, const float* a_v1,
                            const float* a_v3, int nx, int ny, int nz, int ldimx, int ldimy, int g_ldimx, int g_ldimy,
                            tti_stream_t stream)
{
    if (!e3_grid_ok(nx, ny, nz, ldimx, ldimy) || g_ldimx < nx || g_ldimy < ny || !g1 || !snap_v1 || !snap_v3 ||
        !a_v1 || !a_v3)
        return TTI_EINVAL;
    const E3Grid g{nx, ny, nz, ldimx, ldimy};
    k_e3_update_gv<<<e3_blocks(g, E3Z), dim3(E3X, E3Y), 0, S(stream)>>>(g1, snap_v1, snap_v3, a_v1, a_v3, g, g_ldimx,
                                                                         g_ldimy);
    return launch_status();
}

int tti_e3_launch_compute_p(float* p, const float* f4, const float* f5, const float* f6, const float* f7,
                            const float* f8, const float* f9, int64_t n, tti_stream_t stream)
{
    if (n < 0 || !p || !f4 || !f5 || !f6 || !f7 || !f8 || !f9) return TTI_EINVAL;
    if (n == 0) return TTI_OK;
    k_e3_pressure<<<(unsigned)((n + 255) / 256), 256, 0, S(stream)>>>(p, f4, f5, f6, f7, f8, f9, n);
    return launch_status();
}

int tti_e3_launch_init_model(float* const* M22, float* const* d4_9, float* zprime, int nx, int ldimx, int ldimy,
                             int ldimz, tti_stream_t stream)
{
    if (!M22 || !d4_9 || !zprime || nx < 1 || ldimx < nx + 8 || ldimy < 1 || ldimz < 1) return TTI_EINVAL;
    E3Model a{};
    for (int k = 0; k < 22; ++k) {
        if (!M22[k]) return TTI_EINVAL;
        a.M[k] = M22[k];
    }
    for (int k = 0; k < 6; ++k) {
        if (!d4_9[k]) return TTI_EINVAL;
        a.d[k] = d4_9[k];
    }
    a.zprime = zprime;
    k_e3_init_model<<<dim3((nx + 127) / 128, ldimy, ldimz), 128, 0, S(stream)>>>(a, nx, ldimx, ldimy, ldimz);
    return launch_status();
}

} // extern "C"
