/* CPU oracle for the elastic (eTTI proxy) step kernels of the reference's
 * simulator3 -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement, per cell, of the reference's simulator3 kernels,
 * with the reference's own constants (its stand-in coefficients
 * DF_order8 = INT_S_O8 = {1.01, 2.01, 3.01, 4.01} and the hard-coded inverse
 * spacings) and its accumulation order:
 *   vgPlainKernel      simulator3/simulator3SetUp.cu:1218-1362  (velocity gradients)
 *   precompute_xz_yz   simulator3/simulator3SetUp.cu:47-187     (z-mixed interpolations)
 *   sPlainKernel       simulator3/simulator3SetUp.cu:980-1103   (stress update, 21 Cij)
 *   sPlainLoop         simulator3/simulator3SetUp.cu:1127-1216  (the 6 precomputes, then s)
 *   vPlainKernel       simulator3/simulator3SetUp.cu:820-979    (velocity update)
 *   mirror_s/mirror_v  simulator3/simulator3SetUp.cu:1387-1492  (free surface)
 *   update_gv          simulator3/simulator3SetUp.cu:1494-1511  (velocity image)
 *   compute_p_kernel   simulator3/simulator3SetUp.cu:275-289    (pressure)
 *   init_cijs_kernel   simulator3/simulator3SetUp.cu:229-273    (stand-in model)
 * The reference's translation unit needs MPI and zfp headers, so its kernels
 * cannot be built here to pin this restatement: parity of this path is
 * unpinned (the restatement follows the source as read).
 *
 * Volumes: FP32, x fastest, radius-4 halo on every axis, interior
 * [4, 4+n-1] per axis, idx = (iz*ldimy + iy)*ldimx + ix.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef int64_t i64;

static const float E3_DF[4] = {1.01f, 2.01f, 3.01f, 4.01f};  /* DF_order8 (simulator3SetUp.cu:31) */
static const float E3_INT[4] = {1.01f, 2.01f, 3.01f, 4.01f}; /* INT_S_O8 (simulator3SetUp.cu:32) */

/* drv1_8<SHIFT, STRIDE> (simulator3SetUp.cu:37-45): staggered first
 * derivative, shifted half a cell back (SHIFT) or forward. */
static float drv1_8(const float* p, int shift, i64 s)
{
    const i64 is = shift ? -1 : 0;
    float d = E3_DF[0] * (p[(is + 1) * s] - p[is * s]);
    for (int i = 1; i < 4; ++i) d += E3_DF[i] * (p[(is + i + 1) * s] - p[(is - i) * s]);
    return d;
}

/* mixed_XY<XS, YS> (simulator3SetUp.cu:214-227): 4-point averages along the
 * xy diagonals, halved. */
static float mixed_xy(const float* p, int xsh, int ysh, i64 sy)
{
    const i64 xs = xsh ? -1 : 0, ys = ysh ? -1 : 0;
    float d = 0.0f;
    for (int i = 0; i < 4; ++i)
        d += E3_INT[i] * (p[(ys + i + 1) * sy + xs + i + 1] + p[(ys + i + 1) * sy + xs - i] +
                          p[(ys - i) * sy + xs + i + 1] + p[(ys - i) * sy + xs - i]);
    return 0.5f * d;
}

#define IDX(ix, iy, iz) (((i64)(iz) * ldimy + (iy)) * ldimx + (ix))

/* vgPlainKernel: d4 = dv1/dx, d5 = dv1/dy + dv2/dx, d6 = dv1/dz + dv3/dx,
 * d7 = dv2/dy, d8 = dv2/dz + dv3/dy, d9 = dv3/dz with the reference's
 * stand-in spacings 1/dx = 1.01, 1/dy = 2.02 and 1/dz = zprime[iz]. */
void orc_e3_vgplain(const float* f1, const float* f2, const float* f3, float* d4, float* d5, float* d6, float* d7,
                    float* d8, float* d9, const float* zprime, int nx, int ny, int nz, int ldimx, int ldimy)
{
    const float invd1 = 1.01f, invd2 = 2.02f;
    const i64 sy = ldimx, sz = (i64)ldimx * ldimy;
#pragma omp parallel for collapse(2)
    for (int iz = 4; iz < 4 + nz; ++iz)
        for (int iy = 4; iy < 4 + ny; ++iy)
            for (int ix = 4; ix < 4 + nx; ++ix) {
                const i64 i = IDX(ix, iy, iz);
                const float d19 = drv1_8(f1 + i, 0, 1), d20 = drv1_8(f2 + i, 0, sy), d21 = drv1_8(f3 + i, 0, sz);
                const float d22 = drv1_8(f1 + i, 1, sy), d23 = drv1_8(f2 + i, 1, 1), d24 = drv1_8(f1 + i, 1, sz);
                const float d25 = drv1_8(f3 + i, 1, 1), d26 = drv1_8(f2 + i, 1, sz), d27 = drv1_8(f3 + i, 1, sy);
                const float zpr = zprime[iz];
                d4[i] = invd1 * d19;
                d5[i] = invd2 * d22 + invd1 * d23;
                d6[i] = zpr * d24 + invd1 * d25;
                d7[i] = invd2 * d20;
                d8[i] = zpr * d26 + invd2 * d27;
                d9[i] = zpr * d21;
            }
}

/* precompute_xz_yz<XS, YS, ZS> with the reference launch's z blocks of 64
 * planes.  Output plane o = 4 + 64 b + m of block b sums, over the planes
 * P0 + s (P0 = 64 b + 1 - ZS, s = m .. m+7), the pair of values at x offsets
 * X1 + 7 - d and X2 - 7 + d (d = s - m; X1 = -3 - XS, X2 = 4 - XS), weighted
 * by INT_S_O8[max(3 - i, i - 4)], i = 7 - d, and halves the sum; likewise in
 * y.  The reference primes its register queues with the weight of the
 * arriving plane (simulator3SetUp.cu:128: index max(3 - s, s - 4)) where the
 * steady state uses the output offset (:167), so the contributions of planes
 * s <= 6 to the block's outputs m = 1..6 take that weight: the result depends
 * on the blocking, and this restatement keeps it. */
void orc_e3_precompute(const float* in, float* drvxz, float* drvyz, int xs, int ys, int zs, int nx, int ny, int nz,
                       int ldimx, int ldimy)
{
    const int X1 = -3 - xs, X2 = 4 - xs, Y1 = -3 - ys, Y2 = 4 - ys;
    const int nb = (nz - 1) / 64 + 1;
#pragma omp parallel for collapse(2)
    for (int b = 0; b < nb; ++b)
        for (int iy = 4; iy < 4 + ny; ++iy) {
            const int mend = (nz - 64 * b) < 64 ? nz - 64 * b : 64;
            const int p0 = 64 * b + 1 - zs;
            for (int m = 0; m < mend; ++m) {
                const int o = 4 + 64 * b + m;
                for (int ix = 4; ix < 4 + nx; ++ix) {
                    float rxz = 0.0f, ryz = 0.0f;
                    for (int s = m; s <= m + 7; ++s) {
                        const int d = s - m, i = 7 - d;
                        const int ic = s <= 6 ? (3 - s > s - 4 ? 3 - s : s - 4) : (3 - i > i - 4 ? 3 - i : i - 4);
                        const float* pl = in + (i64)(p0 + s) * ldimx * ldimy;
                        rxz += E3_INT[ic] * (pl[(i64)iy * ldimx + ix + X1 + i] + pl[(i64)iy * ldimx + ix + X2 - i]);
                        ryz += E3_INT[ic] * (pl[(i64)(iy + Y1 + i) * ldimx + ix] + pl[(i64)(iy + Y2 - i) * ldimx + ix]);
                    }
                    drvxz[IDX(ix, iy, o)] = 0.5f * rxz;
                    drvyz[IDX(ix, iy, o)] = 0.5f * ryz;
                }
            }
        }
}

/* sPlainKernel after the six precomputes of sPlainLoop: the stress update
 * with the 21 Cij M1..M21.  e11..e33 are the strain volumes (the simulator
 * passes d4, d5, d6, d7, d8, d9 as f1_1, f1_2, f1_3, f2_2, f2_3, f3_3);
 * p10..p21 receive the precomputed z-mixed terms (as the reference's f10..f21). */
void orc_e3_splain(float* f4, float* f5, float* f6, float* f7, float* f8, float* f9, const float* const* M,
                   const float* e11, const float* e12, const float* e13, const float* e22, const float* e23,
                   const float* e33, float* const* p, int nx, int ny, int nz, int ldimx, int ldimy)
{
    /* p[0..11] = f10 .. f21 */
    orc_e3_precompute(e11, p[0], p[1], 1, 1, 1, nx, ny, nz, ldimx, ldimy);
    orc_e3_precompute(e22, p[6], p[7], 1, 1, 1, nx, ny, nz, ldimx, ldimy);
    orc_e3_precompute(e33, p[10], p[11], 1, 1, 1, nx, ny, nz, ldimx, ldimy);
    orc_e3_precompute(e12, p[2], p[3], 0, 0, 1, nx, ny, nz, ldimx, ldimy);
    orc_e3_precompute(e13, p[4], p[5], 0, 1, 0, nx, ny, nz, ldimx, ldimy);
    orc_e3_precompute(e23, p[8], p[9], 1, 0, 0, nx, ny, nz, ldimx, ldimy);
    const i64 sy = ldimx;
#pragma omp parallel for collapse(2)
    for (int iz = 4; iz < 4 + nz; ++iz)
        for (int iy = 4; iy < 4 + ny; ++iy)
            for (int ix = 4; ix < 4 + nx; ++ix) {
                const i64 i = IDX(ix, iy, iz);
#define m(k) M[(k) - 1][i]
                const float d19 = e11[i], d20 = e22[i], d21 = e33[i], d22 = e12[i], d24 = e13[i], d26 = e23[i];
                const float xx12 = mixed_xy(e12 + i, 0, 0, sy), xx13 = p[4][i], xx23 = p[9][i];
                f4[i] += m(1) * d19 + m(2) * d20 + m(3) * d21 + m(6) * xx12 + m(5) * xx13 + m(4) * xx23;
                f5[i] += m(2) * d19 + m(7) * d20 + m(8) * d21 + m(11) * xx12 + m(10) * xx13 + m(9) * xx23;
                f6[i] += m(3) * d19 + m(8) * d20 + m(12) * d21 + m(15) * xx12 + m(14) * xx13 + m(13) * xx23;
                const float xy11 = mixed_xy(e11 + i, 1, 1, sy), xy22 = mixed_xy(e22 + i, 1, 1, sy);
                const float xy33 = mixed_xy(e33 + i, 1, 1, sy), xy13 = p[5][i], xy23 = p[8][i];
                f7[i] += m(6) * xy11 + m(11) * xy22 + m(15) * xy33 + m(20) * xy13 + m(18) * xy23 + m(21) * d22;
                const float xz11 = p[0][i], xz22 = p[6][i], xz33 = p[10][i], xz12 = p[3][i];
                const float xz23 = mixed_xy(e23 + i, 1, 0, sy);
                f8[i] += m(5) * xz11 + m(10) * xz22 + m(14) * xz33 + m(20) * xz12 + m(17) * xz23 + m(19) * d24;
                const float yz11 = p[1][i], yz22 = p[7][i], yz33 = p[11][i], yz12 = p[2][i];
                const float yz13 = mixed_xy(e13 + i, 0, 1, sy);
                f9[i] += m(4) * yz11 + m(9) * yz22 + m(13) * yz33 + m(18) * yz12 + m(17) * yz13 + m(16) * d26;
#undef m
            }
}

/* vPlainKernel: velocity update from the stress divergence, each component
 * scaled by 2*M22 at the staggered position below it (x-1, y-1, z-1); the
 * reference's stand-in 1/dx = 1.01, 1/dy = 2.01, 1/dz = zprime[iz]. */
void orc_e3_vplain(float* f1, float* f2, float* f3, const float* f4, const float* f5, const float* f6,
                   const float* f7, const float* f8, const float* f9, const float* M22, const float* zprime, int nx,
                   int ny, int nz, int ldimx, int ldimy)
{
    const float invd1 = 1.01f, invd2 = 2.01f;
    const i64 sy = ldimx, sz = (i64)ldimx * ldimy;
#pragma omp parallel for collapse(2)
    for (int iz = 4; iz < 4 + nz; ++iz)
        for (int iy = 4; iy < 4 + ny; ++iy)
            for (int ix = 4; ix < 4 + nx; ++ix) {
                const i64 i = IDX(ix, iy, iz);
                const float d10 = drv1_8(f4 + i, 1, 1), d11 = drv1_8(f5 + i, 1, sy), d12 = drv1_8(f6 + i, 1, sz);
                const float d13 = drv1_8(f7 + i, 0, 1), d14 = drv1_8(f7 + i, 0, sy), d15 = drv1_8(f8 + i, 0, sz);
                const float d16 = drv1_8(f8 + i, 0, 1), d17 = drv1_8(f9 + i, 0, sy), d18 = drv1_8(f9 + i, 0, sz);
                const float zpr = zprime[iz];
                f1[i] += (2.0f * M22[i - 1]) * (d10 * invd1 + d14 * invd2 + d15 * zpr);
                f2[i] += (2.0f * M22[i - sy]) * (d13 * invd1 + d11 * invd2 + d18 * zpr);
                f3[i] += (2.0f * M22[i - sz]) * (d16 * invd1 + d17 * invd2 + d12 * zpr);
            }
}

/* mirror_s_kernel / mirror_v_kernel: at the free surface izbeg the fields
 * are zero, above it they are the negated mirror 2*izbeg - iz (whole planes,
 * halos included). */
void orc_e3_mirror(float* const* f, int nf, int ldimx, int ldimy, int izbeg)
{
    const i64 plane = (i64)ldimx * ldimy;
    for (int k = 0; k < nf; ++k)
        for (int iz = 0; iz <= izbeg; ++iz)
            for (i64 j = 0; j < plane; ++j) {
                const i64 i = iz * plane + j;
                f[k][i] = iz == izbeg ? 0.0f : -f[k][(2 * izbeg - iz) * plane + j];
            }
}

/* update_gv (simulator3SetUp.cu:1494-1511): g += a1 * s1 + a3 * s3 with g
 * and the snapshots halo-free (leading dimensions gx, gy) and the adjoint
 * velocities a1, a3 halo'd. */
void orc_e3_update_gv(float* g, const float* s1, const float* s3, const float* a1, const float* a3, int nx, int ny,
                      int nz, int ldimx, int ldimy, int gx, int gy)
{
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                const i64 gi = ((i64)z * gy + y) * gx + x, ai = IDX(x + 4, y + 4, z + 4);
                g[gi] += a1[ai] * s1[gi] + a3[ai] * s3[gi];
            }
}

/* compute_p_kernel: P = -(2 f4 + 3 f5 + 4 f6 + 5 f7 + 6 f8 + 7 f9) / 27 over
 * the x range [0, xtot) of every (y, z) of the grid given. */
void orc_e3_pressure(float* p, const float* f4, const float* f5, const float* f6, const float* f7, const float* f8,
                     const float* f9, i64 n)
{
    for (i64 i = 0; i < n; ++i)
        p[i] = -(2.0f * f4[i] + 3.0f * f5[i] + 4.0f * f6[i] + 5.0f * f7[i] + 6.0f * f8[i] + 7.0f * f9[i]) / 27.0f;
}

/* init_cijs_kernel: the stand-in model M1..M22, the six strain stand-ins
 * d4..d9 and zprime, from cos/sin of the halo'd cell indices, over the
 * interior x range and every y and z of the allocation (the reference's
 * launch covers ntot in y and z and checks x only). */
void orc_e3_init_model(float* const* M, float* const* d, float* zprime, int nx, int ldimx, int ldimy, int ldimz)
{
    for (int iz = 0; iz < ldimz; ++iz) {
        zprime[iz] = cosf(6.0f * iz);
        for (int iy = 0; iy < ldimy; ++iy)
            for (int ix = 4; ix < 4 + nx; ++ix) {
                const i64 i = IDX(ix, iy, iz);
                const float a[6] = {2.0f * iz + iy + ix, iz + 2.0f * iy + ix, iz + iy + 2.0f * ix,
                                    3.0f * iz + iy + ix, iz + 3.0f * iy + ix, iz + iy + 3.0f * ix};
                for (int k = 0; k < 6; ++k) {
                    M[2 * k][i] = cosf(a[k]);
                    M[2 * k + 1][i] = sinf(a[k]);
                }
                const float b[5] = {4.0f * iz + iy + ix, iz + 4.0f * iy + ix, iz + iy + 4.0f * ix,
                                    5.0f * iz + iy + ix, iz + 5.0f * iy + ix};
                for (int k = 0; k < 5; ++k) {
                    M[12 + 2 * k][i] = cosf(b[k]);
                    M[13 + 2 * k][i] = sinf(b[k]);
                }
                d[0][i] = cosf(iz + iy + 5.0f * ix);
                d[1][i] = sinf(iz + iy + 5.0f * ix);
                d[2][i] = cosf(6.0f * iz + iy + ix);
                d[3][i] = sinf(6.0f * iz + iy + ix);
                d[4][i] = cosf(iz + 6.0f * iy + ix);
                d[5][i] = sinf(iz + 6.0f * iy + ix);
            }
    }
}
