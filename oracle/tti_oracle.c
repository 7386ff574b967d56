/*
 * CPU oracle for the TTI/VTI pseudo-acoustic RTM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * is compared against; it is never linked into the product library and the
 * product never calls it.  Only tests/, the smoke check and the CPU-baseline
 * leg of the benchmark load it.
 *
 * It is a plain-C restatement of the reference's GPU kernels for this path
 * (MiniAppsForHPE, simulatorsForNvidia/).  Every function below cites the
 * reference kernel it restates and follows that kernel's accumulation order
 * (tap order, where the 1/h factor and the buoyancy factor are applied), so
 * that in FP32 it agrees with the reference to rounding.  The same source is
 * compiled twice: REAL=float (reference-order FP32) and REAL=double (the FP64
 * oracle used for mixed-precision error reports and dot-product tests).
 *
 * Layout (reference contract, utils/volume_index.h:20-23): x fastest,
 * idx = (iz*ldimy + iy)*ldimx + ix, every axis carries a radius-4 halo,
 * interior = [ibeg, iend] with ibeg = 4.
 *
 * Parity of this oracle is pinned against the reference's own kernels
 * (compiled from the reference sources for sm_100a by oracle/Makefile and
 * run on a B200) through the fixtures in tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL float
#endif
#ifndef SFX
#define SFX _f32
#endif
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

typedef REAL real;
typedef int64_t i64;

#define IDX(ix, iy, iz) ((((i64)(iz)) * ldimy + (iy)) * (i64)ldimx + (ix))

/* ------------------------------------------------------------------------
 * FD coefficients.  Least-squares 8th-order sets used by every launcher of
 * the path (kernels/fd_coef.h:464-470 DF_order8 staggered first derivative,
 * kernels/fd_coef.h:516-521 DF2_order8 centred second derivative used for the
 * rotated mixed derivatives; kernels/fd_coefficients.h:16-97 stg_d1<8>,
 * identical in float).  Values are kept in float so that the double build
 * uses the same stencil as the float build.
 * ---------------------------------------------------------------------- */
static const float C1[5] = {0.0f, 1.19628906250000e+00f, -7.97526041666667e-02f,
                            9.57031250000000e-03f, -6.97544642857143e-04f};
static const float C2[5] = {-0.2903117E+1f, 0.1645351E+1f, -0.2236606E+0f,
                            0.3265851E-1f, -0.2790073E-2f};
/* stg_d1<8> (kernels/fd_coefficients.h:28-31) rounds to the same floats. */
static const float CS[4] = {1.1962891e+0f, -7.9752604e-2f, 9.5703125e-3f, -6.9754464e-4f};

/* Coefficient of tap k (0..7) of the 8-point staggered operator written as a
 * sum over consecutive points starting 3 (D+) or 4 (D-) below the output:
 * -c4,-c3,-c2,-c1,+c1,+c2,+c3,+c4  (kernel_type2_fwd.cu:104-115). */
static inline real tapc(int k) { return (k < 4) ? -(real)C1[4 - k] : (real)C1[k - 3]; }

void FN(orc_coefficients)(float* c1, float* c2, float* cs)
{
    for (int i = 0; i < 5; ++i) { c1[i] = C1[i]; c2[i] = C2[i]; }
    for (int i = 0; i < 4; ++i) cs[i] = CS[i];
}

/* ------------------------------------------------------------------------
 * a1: p = A*p + B*dt*pdot, q likewise; A,B = min over the three axis
 * profiles.  kernel_base.cu:82-104 (kernel_loop2_inner_kernel).
 * ab_* are interleaved (A,B) pairs indexed by the global axis index.
 * ---------------------------------------------------------------------- */
void FN(orc_loop2)(real* f1, real* f2, const real* f3, const real* f4, int ldimx, int ldimy,
                   int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                   const float* abx, const float* aby, const float* abz, float dt)
{
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy) {
            real Ayz = fminf(aby[2 * iy], abz[2 * iz]);
            real Byz = fminf(aby[2 * iy + 1], abz[2 * iz + 1]);
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                real A = fminf(abx[2 * ix], Ayz);
                real B = fminf(abx[2 * ix + 1], Byz);
                i64 i = IDX(ix, iy, iz);
                real r1 = A * f1[i] + B * f3[i] * (real)dt;
                real r2 = A * f2[i] + B * f4[i] * (real)dt;
                f1[i] = r1;
                f2[i] = r2;
            }
        }
}

/* ------------------------------------------------------------------------
 * a2: free surface at izbeg: p=q=0 on the surface plane, odd mirror above.
 * kernel_base.cu:142-162 (kernel_loop4_kernel).  Whole XY planes.
 * ---------------------------------------------------------------------- */
void FN(orc_loop4)(real* f1, real* f2, int ldimx, int ldimy, int izbeg)
{
    i64 plane = (i64)ldimx * ldimy;
    for (int iz = 0; iz <= izbeg; ++iz) {
        for (i64 j = 0; j < plane; ++j) {
            i64 i = iz * plane + j;
            if (iz == izbeg) {
                f1[i] = 0;
                f2[i] = 0;
            } else {
                i64 m = (i64)(2 * izbeg - iz) * plane + j;
                f1[i] = -f1[m];
                f2[i] = -f2[m];
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * a3: six staggered first derivatives (shift -1/2) times buoyancy.
 * kernel_type2_fwd_drv.cu:36-116,134-348: per axis
 *   d = ( sum_{taps low..high} c * f ) * invd ; out = d * Model11.
 * z taps accumulate from plane z-4 to z+3 (compute_dz_negative_shift),
 * x/y taps as pairs c_i*(f[x+i-1]-f[x-i]) for i=1..4.
 * Writes the interior only.
 * ---------------------------------------------------------------------- */
void FN(orc_fwd_drv)(const real* f1, const real* f2, const real* irho, real* d1x, real* d1y, real* d1z,
                     real* d2x, real* d2y, real* d2z, int ixbeg, int ixend, int iybeg, int iyend,
                     int izbeg, int izend, float invdx, float invdy, float invdz, int ldimx, int ldimy)
{
    i64 zs = (i64)ldimx * ldimy, ys = ldimx;
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                real az1 = 0, az2 = 0;
                for (int ir = -4; ir <= 3; ++ir) {
                    if (ir >= 0) {
                        real c = C1[ir + 1];
                        az1 = az1 + c * f1[i + ir * zs];
                        az2 = az2 + c * f2[i + ir * zs];
                    } else {
                        real c = C1[-ir];
                        az1 = az1 - c * f1[i + ir * zs];
                        az2 = az2 - c * f2[i + ir * zs];
                    }
                }
                az1 *= (real)invdz;
                az2 *= (real)invdz;
                real ax1 = 0, ay1 = 0, ax2 = 0, ay2 = 0;
                for (int k = 1; k <= 4; ++k) {
                    real c = C1[k];
                    ax1 += c * (f1[i + (k - 1)] - f1[i - k]);
                    ay1 += c * (f1[i + (k - 1) * ys] - f1[i - k * ys]);
                    ax2 += c * (f2[i + (k - 1)] - f2[i - k]);
                    ay2 += c * (f2[i + (k - 1) * ys] - f2[i - k * ys]);
                }
                ax1 *= (real)invdx;
                ay1 *= (real)invdy;
                ax2 *= (real)invdx;
                ay2 *= (real)invdy;
                real rho = irho[i];
                d1x[i] = ax1 * rho;
                d1y[i] = ay1 * rho;
                d1z[i] = az1 * rho;
                d2x[i] = ax2 * rho;
                d2y[i] = ay2 * rho;
                d2z[i] = az2 * rho;
            }
}

/* ------------------------------------------------------------------------
 * a4: free-surface mirror of the derivative volumes.
 * kernel_type2_small.cu:5-40: for iz<=izbeg over whole XY planes, d/dx and
 * d/dy odd about izbeg (zero on it), d/dz even about izbeg+1/2.
 * ---------------------------------------------------------------------- */
void FN(orc_loop4_derivatives)(real* d1x, real* d1y, real* d1z, real* d2x, real* d2y, real* d2z,
                               int ldimx, int ldimy, int izbeg)
{
    i64 plane = (i64)ldimx * ldimy;
    for (int iz = 0; iz <= izbeg; ++iz) {
        for (i64 j = 0; j < plane; ++j) {
            i64 i = iz * plane + j;
            if (iz == izbeg) {
                d1x[i] = 0; d1y[i] = 0; d2x[i] = 0; d2y[i] = 0;
            } else {
                i64 m = (i64)(2 * izbeg - iz) * plane + j;
                d1x[i] = -d1x[m]; d1y[i] = -d1y[m]; d2x[i] = -d2x[m]; d2y[i] = -d2y[m];
            }
            i64 mz = (i64)(2 * izbeg + 1 - iz) * plane + j;
            d1z[i] = d1z[mz];
            d2z[i] = d2z[mz];
        }
    }
}

/* ------------------------------------------------------------------------
 * a5: forward TTI update.  kernel_type2_fwd.cu:98-235 (helpers) and
 * :360-539 (accumulation order).  Normal second derivatives are D+ of the
 * buoyancy-scaled first derivatives, taps summed one at a time from the
 * lowest point (compute_d2x_d2y, update_d2z), times 1/h, times rho.  Mixed
 * derivatives use the centred LS coefficients along the diagonals:
 * xy in the plane (compute_dxy), zx/yz accumulated plane by plane from z-4 to
 * z+4 (update_z_mixed).  Then V/H split and the p/q right-hand sides
 * (calculate_result_interior), and field3/4 += rhs*dt.
 * ---------------------------------------------------------------------- */
static inline void fwd_point(const real* d1x, const real* d2x, const real* d1y, const real* d2y,
                             const real* d1z, const real* d2z, const real* f1, const real* f2,
                             const real* irho, const real* m1, const real* m2, const real* m3,
                             const real* m4, const real* rx, const real* ry, const real* rz, i64 i,
                             i64 ys, i64 zs, real invdx, real invdy, real invdz, real invdxdy,
                             real invdydz, real invdzdx, real* out3, real* out4)
{
    real xx1 = 0, xx2 = 0, yy1 = 0, yy2 = 0, zz1 = 0, zz2 = 0;
    for (int k = 0; k < 8; ++k) {
        real c = tapc(k);
        xx1 += c * d1x[i + (k - 3)];
        xx2 += c * d2x[i + (k - 3)];
        yy1 += c * d1y[i + (k - 3) * ys];
        yy2 += c * d2y[i + (k - 3) * ys];
    }
    xx1 *= invdx; xx2 *= invdx; yy1 *= invdy; yy2 *= invdy;
    for (int k = 0; k < 8; ++k) {
        real c = tapc(k);
        zz1 = zz1 + c * d1z[i + (k - 3) * zs];
        zz2 = zz2 + c * d2z[i + (k - 3) * zs];
    }
    zz1 *= invdz; zz2 *= invdz;
    real zx1 = 0, zx2 = 0, yz1 = 0, yz2 = 0;
    for (int m = -4; m <= 4; ++m) {
        if (m == 0) continue;
        real c = C2[abs(m)];
        i64 p = i + m * zs;
        zx1 += c * (f1[p + m] - f1[p - m]);
        yz1 += c * (f1[p + m * ys] - f1[p - m * ys]);
        zx2 += c * (f2[p + m] - f2[p - m]);
        yz2 += c * (f2[p + m * ys] - f2[p - m * ys]);
    }
    yz1 *= invdydz; zx1 *= invdzdx; yz2 *= invdydz; zx2 *= invdzdx;
    real xy1 = 0, xy2 = 0;
    for (int k = -4; k <= 4; ++k) {
        if (k == 0) continue;
        real c = C2[abs(k)];
        xy1 += c * (f1[i + k * ys + k] - f1[i - k * ys + k]);
        xy2 += c * (f2[i + k * ys + k] - f2[i - k * ys + k]);
    }
    xy1 *= invdxdy; xy2 *= invdxdy;

    real rho = (real)1 / irho[i];
    real vrx = rx[i], vry = ry[i], vrz = rz[i];
    real rx2 = vrx * vrx, ry2 = vry * vry, rz2 = vrz * vrz;
    real rxy = (real)2 * vrx * vry, ryz = (real)2 * vry * vrz, rzx = (real)2 * vrz * vrx;
    xx1 *= rho; yy1 *= rho; zz1 *= rho;
    xx2 *= rho; yy2 *= rho; zz2 *= rho;
    real V1 = rx2 * xx1 + ry2 * yy1 + rz2 * zz1 + rxy * xy1 + rzx * zx1 + ryz * yz1;
    real H1 = xx1 + yy1 + zz1 - V1;
    real V2 = rx2 * xx2 + ry2 * yy2 + rz2 * zz2 + rxy * xy2 + rzx * zx2 + ryz * yz2;
    real H2 = xx2 + yy2 + zz2 - V2;
    *out3 = m1[i] * H1 + m4[i] * V1 + m2[i] * V2;
    *out4 = m2[i] * H1 + m3[i] * V2 + m4[i] * H2;
}

void FN(orc_fwd_update)(real* f3, real* f4, const real* d1x, const real* d2x, const real* d1y,
                        const real* d2y, const real* d1z, const real* d2z, const real* f1,
                        const real* f2, const real* irho, const real* m1, const real* m2,
                        const real* m3, const real* m4, const real* rx, const real* ry,
                        const real* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                        int izend, int ldimx, int ldimy, float dt, double dx, double dy, double dz)
{
    i64 zs = (i64)ldimx * ldimy, ys = ldimx;
    /* kernel_utils.h:89-101 compute_fd_const: reciprocals formed in double. */
    real invdx = (float)(1.0 / dx), invdy = (float)(1.0 / dy), invdz = (float)(1.0 / dz);
    real invdxdy = (float)(1.0 / (4 * dx * dy)), invdydz = (float)(1.0 / (4 * dy * dz));
    real invdzdx = (float)(1.0 / (4 * dx * dz));
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                real r3, r4;
                fwd_point(d1x, d2x, d1y, d2y, d1z, d2z, f1, f2, irho, m1, m2, m3, m4, rx, ry, rz, i,
                          ys, zs, invdx, invdy, invdz, invdxdy, invdydz, invdzdx, &r3, &r4);
                f3[i] += r3 * (real)dt;
                f4[i] += r4 * (real)dt;
            }
}

/* ------------------------------------------------------------------------
 * a6: adjoint derivatives.  kernel_type2_grad_snap.cu:66-240,242-427.
 * Point-wise transposed model (compute_temp_arrays) on the halo'd tile,
 * then staggered D- (shift -1/2) with the buoyancy inside each x/y term and
 * applied after the z sum; the rotated mixed terms are scattered into the
 * field3/field4 rhs volumes in the order z-4..z-1, xy, z+1..z+4.
 * Temporaries are formed at any point of the volume including halos, so
 * Model11 must be non-zero in the halo.
 * ---------------------------------------------------------------------- */
typedef struct {
    real t1xx, t2xx, t1yy, t2yy, t1zz, t2zz, t1xy, t2xy, t1yz, t2yz, t1zx, t2zx;
} adj_temps;

static inline adj_temps adj_temp(const real* f1, const real* f2, const real* irho, const real* m1,
                                 const real* m2, const real* m3, const real* m4, const real* rx,
                                 const real* ry, const real* rz, i64 i)
{
    adj_temps t;
    real vrx = rx[i], vry = ry[i], vrz = rz[i];
    real rho = (real)1 / irho[i];
    real rxx = vrx * vrx, ryy = vry * vry, rzz = vrz * vrz;
    real rxy = (real)2 * vrx * vry, ryz = (real)2 * vry * vrz, rzx = (real)2 * vrz * vrx;
    real a1 = m1[i], a2 = m2[i], a3 = m3[i], a4 = m4[i], p = f1[i], q = f2[i];
    real lap_x = a1 * p + a2 * q;
    real hz_x = (-a1 + a4) * p - a2 * q;
    real lap_z = a4 * q;
    real hz_z = a2 * p + (-a4 + a3) * q;
    t.t1xy = rxy * hz_x; t.t2xy = rxy * hz_z;
    t.t1xx = rho * (lap_x + rxx * hz_x); t.t2xx = rho * (lap_z + rxx * hz_z);
    t.t1zx = rzx * hz_x; t.t2zx = rzx * hz_z;
    t.t1yy = rho * (lap_x + ryy * hz_x); t.t2yy = rho * (lap_z + ryy * hz_z);
    t.t1yz = ryz * hz_x; t.t2yz = ryz * hz_z;
    t.t1zz = rho * (lap_x + rzz * hz_x); t.t2zz = rho * (lap_z + rzz * hz_z);
    return t;
}

void FN(orc_adj_drv)(real* d1x, real* d2x, real* d1y, real* d2y, real* d1z, real* d2z, real* rhs3,
                     real* rhs4, const real* f1, const real* f2, const real* irho, const real* m1,
                     const real* m2, const real* m3, const real* m4, const real* rx, const real* ry,
                     const real* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend,
                     float invdxy, float invdyz, float invdzx, int ldimx, int ldimy, float invdx,
                     float invdy, float invdz)
{
    i64 zs = (i64)ldimx * ldimy, ys = ldimx, nvol = zs * (i64)(izend + 5);
    /* Temporaries over the whole allocation (halos included), as the
     * reference forms them on its halo'd tiles. */
    adj_temps* T = (adj_temps*)malloc(sizeof(adj_temps) * (size_t)nvol);
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < nvol; ++i) T[i] = adj_temp(f1, f2, irho, m1, m2, m3, m4, rx, ry, rz, i);
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                real ir_ = irho[i];
                /* z taps (compute_z_contributionsdtd) */
                real z1 = 0, z2 = 0;
                for (int ir = -4; ir <= 3; ++ir) {
                    real alpha = (ir < 0) ? -(real)invdz * (real)C1[-ir] : (real)invdz * (real)C1[ir + 1];
                    z1 = z1 + alpha * T[i + ir * zs].t1zz;
                    z2 = z2 + alpha * T[i + ir * zs].t2zz;
                }
                /* x/y taps with buoyancy inside each term (compute_xy_contributions) */
                real x1 = 0, x2 = 0, y1 = 0, y2 = 0, s3 = 0, s4 = 0;
                /* mixed z terms below the plane */
                for (int ir = -4; ir <= -1; ++ir) {
                    real c = C2[-ir];
                    i64 p = i + ir * zs;
                    s3 = s3 + ((real)invdyz * c * (T[p + ir * ys].t1yz - T[p - ir * ys].t1yz)) +
                         ((real)invdzx * c * (T[p + ir].t1zx - T[p - ir].t1zx));
                    s4 = s4 + ((real)invdyz * c * (T[p + ir * ys].t2yz - T[p - ir * ys].t2yz)) +
                         ((real)invdzx * c * (T[p + ir].t2zx - T[p - ir].t2zx));
                }
                for (int k = 1; k <= 4; ++k) {
                    real ax = (real)invdx * (real)C1[k];
                    x1 += ax * (T[i + (k - 1)].t1xx - T[i - k].t1xx) * ir_;
                    x2 += ax * (T[i + (k - 1)].t2xx - T[i - k].t2xx) * ir_;
                    real ay = (real)invdy * (real)C1[k];
                    y1 += ay * (T[i + (k - 1) * ys].t1yy - T[i - k * ys].t1yy) * ir_;
                    y2 += ay * (T[i + (k - 1) * ys].t2yy - T[i - k * ys].t2yy) * ir_;
                    real axy = (real)invdxy * (real)C2[k];
                    s3 += axy * (T[i + k * ys + k].t1xy - T[i + k * ys - k].t1xy + T[i - k * ys - k].t1xy -
                                 T[i - k * ys + k].t1xy);
                    s4 += axy * (T[i + k * ys + k].t2xy - T[i + k * ys - k].t2xy + T[i - k * ys - k].t2xy -
                                 T[i - k * ys + k].t2xy);
                }
                for (int ir = 1; ir <= 4; ++ir) {
                    real c = C2[ir];
                    i64 p = i + ir * zs;
                    s3 = s3 + ((real)invdyz * c * (T[p + ir * ys].t1yz - T[p - ir * ys].t1yz)) +
                         ((real)invdzx * c * (T[p + ir].t1zx - T[p - ir].t1zx));
                    s4 = s4 + ((real)invdyz * c * (T[p + ir * ys].t2yz - T[p - ir * ys].t2yz)) +
                         ((real)invdzx * c * (T[p + ir].t2zx - T[p - ir].t2zx));
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
    free(T);
}

/* ------------------------------------------------------------------------
 * a7: adjoint update.  kernel_type2_adj.cu:85-98,196-239:
 *   rhs = D+x(d_x)*invdx + D+y(d_y)*invdy + D+z(d_z)*invdz + rhs_mixed
 * with D+ summed as pairs c_i*(f[i]-f[1-i]) (dfdx_stg_right);
 *   sponge off: field3 += rhs*dt;  on: field3 = A*field3 + (B*dt)*rhs,
 * A,B = min over the three axis profiles.
 * ---------------------------------------------------------------------- */
static inline real stg_right(const real* f, i64 i, i64 s, real h)
{
    real out = 0;
    for (int k = 1; k <= 4; ++k) out += (real)C1[k] * (f[i + k * s] - f[i + (1 - k) * s]);
    return out * h;
}

void FN(orc_adj_update)(real* f3, real* f4, const real* d1x, const real* d2x, const real* d1y,
                        const real* d2y, const real* d1z, const real* d2z, const real* rhs3,
                        const real* rhs4, const float* abx, const float* aby, const float* abz,
                        int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int ldimx,
                        int ldimy, float dt, double dx, double dy, double dz, int sponge_active)
{
    i64 zs = (i64)ldimx * ldimy, ys = ldimx;
    real invdx = (float)(1.0 / dx), invdy = (float)(1.0 / dy), invdz = (float)(1.0 / dz);
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                real r3 = stg_right(d1x, i, 1, invdx) + stg_right(d1y, i, ys, invdy) +
                          stg_right(d1z, i, zs, invdz);
                real r4 = stg_right(d2x, i, 1, invdx) + stg_right(d2y, i, ys, invdy) +
                          stg_right(d2z, i, zs, invdz);
                r3 += rhs3[i];
                r4 += rhs4[i];
                if (!sponge_active) {
                    f3[i] += r3 * (real)dt;
                    f4[i] += r4 * (real)dt;
                } else {
                    real A = fminf(fminf(abx[2 * ix], aby[2 * iy]), abz[2 * iz]);
                    real B = fminf(fminf(abx[2 * ix + 1], aby[2 * iy + 1]), abz[2 * iz + 1]) * (real)dt;
                    f3[i] = A * f3[i] + B * r3;
                    f4[i] = A * f4[i] + B * r4;
                }
            }
}

/* ------------------------------------------------------------------------
 * a8: imaging condition g += adj3*snap3 + adj4*snap4.
 * kernel_type2_small.cu:42-59.  snap/grad volumes carry no halo and have
 * their own leading dimensions (snx, sny); the adjoint fields are halo'd.
 * ---------------------------------------------------------------------- */
void FN(orc_update_vp_gradient)(const real* snap3, const real* snap4, real* grad, const real* adj3,
                                const real* adj4, int ixbeg, int ixend, int iybeg, int iyend,
                                int izbeg, int izend, int snx, int sny, int ldimx, int ldimy)
{
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 g = ((i64)(iz - izbeg) * sny + (iy - iybeg)) * snx + (ix - ixbeg);
                i64 i = IDX(ix, iy, iz);
                real s3 = snap3[g], s4 = snap4[g];
                grad[g] += adj3[i] * s3 + adj4[i] * s4;
            }
}

/* a11: g *= -2*dt_xcorr/vp, vp = sqrt(model3).  kernel_type2_small.cu:61-74. */
void FN(orc_finalize_vp_gradient)(const real* model3, real* grad, int ixbeg, int ixend, int iybeg,
                                  int iyend, int izbeg, int izend, int snx, int sny, int ldimx,
                                  int ldimy, float dt_xcorr)
{
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 g = ((i64)(iz - izbeg) * sny + (iy - iybeg)) * snx + (ix - ixbeg);
                real vp = (real)sqrt((double)model3[IDX(ix, iy, iz)]);
                grad[g] = (real)((double)grad[g] * (-(double)dt_xcorr * 2.0 / (double)vp));
            }
}

/* ------------------------------------------------------------------------
 * a10: density gradient.  kernel_type2_grad.cu:188-260 (adj(), stg()) and
 * :344-509 (compute_grad_model10 accumulation):
 *   rhs_xy = ax1*D+(fx1) + ax2*D+(fx2) + ay1*D+(fy1) + ay2*D+(fy2)
 *          + D-(ax1)*fx1 + D-(ax2)*fx2 + D-(ay1)*fy1 + D-(ay2)*fy2
 *   rhs    = rhs_xy + az1*D+(fz1) + az2*D+(fz2) + D-(az1)*fz1 + D-(az2)*fz2
 *   grad  -= irho*rhs   (grad indexed from 0 at the first interior point,
 *                        with its own strides, as in the reference launcher)
 * ---------------------------------------------------------------------- */
static inline void rho_temp(const real* f1, const real* f2, const real* irho, const real* m1,
                            const real* m2, const real* m3, const real* m4, const real* ra, i64 i,
                            real* o1, real* o2)
{
    real p = f1[i], q = f2[i];
    real rho = (real)1 / irho[i];
    real a1 = m1[i], a2 = m2[i], a3 = m3[i], a4 = m4[i];
    real rr = ra[i] * ra[i];
    real lx = (a4 - a1) * p - a2 * q;
    real lz = a2 * p + (a3 - a4) * q;
    *o1 = rho * (a1 * p + a2 * q + rr * lx);
    *o2 = rho * (a4 * q + rr * lz);
}

static inline real stg_plus(const real* t, i64 i, i64 s, real h)
{
    real d = 0;
    for (int r = 0; r < 4; ++r) d += (real)CS[r] * (t[i + (r + 1) * s] - t[i - r * s]);
    return d * h;
}

void FN(orc_rho_gradient)(real* grad, const real* fd1x, const real* fd2x, const real* fd1y,
                          const real* fd2y, const real* fd1z, const real* fd2z, const real* f1,
                          const real* f2, const real* irho, const real* m1, const real* m2,
                          const real* m3, const real* m4, const real* rx, const real* ry,
                          const real* rz, int ixbeg, int ixend, int iybeg, int iyend, int izbeg,
                          int izend, int ldimx, int ldimy, int grad_ldimx, int grad_ldimy, double dx,
                          double dy, double dz)
{
    i64 zs = (i64)ldimx * ldimy, ys = ldimx;
    real hx = (float)(1.0 / dx), hy = (float)(1.0 / dy), hz = (float)(1.0 / dz);
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                real ax1, ax2, ay1, ay2, az1, az2;
                rho_temp(f1, f2, irho, m1, m2, m3, m4, rx, i, &ax1, &ax2);
                rho_temp(f1, f2, irho, m1, m2, m3, m4, ry, i, &ay1, &ay2);
                rho_temp(f1, f2, irho, m1, m2, m3, m4, rz, i, &az1, &az2);
                /* D- of the adjoint temporaries (stg<ORD,false> on the temps) */
                real dax1 = 0, dax2 = 0, day1 = 0, day2 = 0, daz1 = 0, daz2 = 0;
                for (int r = 0; r < 4; ++r) {
                    real c = CS[r], p1, p2, m1_, m2_;
                    rho_temp(f1, f2, irho, m1, m2, m3, m4, rx, i + r, &p1, &p2);
                    rho_temp(f1, f2, irho, m1, m2, m3, m4, rx, i - (r + 1), &m1_, &m2_);
                    dax1 += c * (p1 - m1_);
                    dax2 += c * (p2 - m2_);
                    rho_temp(f1, f2, irho, m1, m2, m3, m4, ry, i + r * ys, &p1, &p2);
                    rho_temp(f1, f2, irho, m1, m2, m3, m4, ry, i - (r + 1) * ys, &m1_, &m2_);
                    day1 += c * (p1 - m1_);
                    day2 += c * (p2 - m2_);
                    rho_temp(f1, f2, irho, m1, m2, m3, m4, rz, i + r * zs, &p1, &p2);
                    rho_temp(f1, f2, irho, m1, m2, m3, m4, rz, i - (r + 1) * zs, &m1_, &m2_);
                    daz1 += c * (p1 - m1_);
                    daz2 += c * (p2 - m2_);
                }
                dax1 *= hx; dax2 *= hx; day1 *= hy; day2 *= hy; daz1 *= hz; daz2 *= hz;
                real dfx1 = stg_plus(fd1x, i, 1, hx), dfx2 = stg_plus(fd2x, i, 1, hx);
                real dfy1 = stg_plus(fd1y, i, ys, hy), dfy2 = stg_plus(fd2y, i, ys, hy);
                real dfz1 = stg_plus(fd1z, i, zs, hz), dfz2 = stg_plus(fd2z, i, zs, hz);
                real rxy = ax1 * dfx1 + ax2 * dfx2 + ay1 * dfy1 + ay2 * dfy2 + dax1 * fd1x[i] +
                           dax2 * fd2x[i] + day1 * fd1y[i] + day2 * fd2y[i];
                real rhs = rxy + az1 * dfz1 + az2 * dfz2 + daz1 * fd1z[i] + daz2 * fd2z[i];
                i64 g = ((i64)(iz - izbeg) * grad_ldimy + (iy - iybeg)) * grad_ldimx + (ix - ixbeg);
                grad[g] += -irho[i] * rhs;
            }
}

/* ------------------------------------------------------------------------
 * a12: model parameters from (vp, eps, delta, vs, theta, phi), per point.
 * simulator2SetUp.cu:10-29 (init_cijs_kernel) restated per cell.
 * ---------------------------------------------------------------------- */
void FN(orc_init_cijs)(const float* vp, const float* eps, const float* delta, const float* vs,
                       const float* theta, const float* phi, real* m1, real* m2, real* m3, real* m4,
                       real* m5, real* m6, real* m7, i64 n)
{
    for (i64 i = 0; i < n; ++i) {
        float v = vp[i], s = vs[i];
        m1[i] = v * v * (1 + 2 * eps[i]);
        m2[i] = sqrtf((v * v - s * s) * (v * v * (1 + 2 * delta[i]) - s * s));
        m3[i] = v * v;
        m4[i] = s * s;
        m5[i] = sinf(theta[i]) * cosf(phi[i]);
        m6[i] = sinf(theta[i]) * sinf(phi[i]);
        m7[i] = cosf(theta[i]);
    }
}

/* a16: pressure P = -(2p+q)/3.  simulator2SetUp.cu:31-42. */
void FN(orc_pressure)(real* out, const real* f1, const real* f2, i64 n)
{
    for (i64 i = 0; i < n; ++i) out[i] = -(2 * f1[i] + f2[i]) / 3;
}

/* ------------------------------------------------------------------------
 * Step drivers in the reference schedule (simulator2SetUp.cu:517-651 forward,
 * :654-782 adjoint), with nsub = 1 and the build's source injection and
 * receiver sampling:
 *   forward step n: loop2, loop4 (free surface), fwd_drv, loop4_derivatives,
 *     fwd_update, f3/f4[src] += w*dt, traces[r] = -(2p+q)/3 at receivers.
 *   adjoint step n: f3/f4[rec] += (-2/3, -1/3)*res, adj_drv,
 *     loop4_derivatives, adj_update (sponge form when active), loop2, loop4.
 * ---------------------------------------------------------------------- */
typedef struct {
    int ldimx, ldimy, ldimz, ixbeg, ixend, iybeg, iyend, izbeg, izend;
    int free_surface, sponge_active;
    float dt;
    double dx, dy, dz;
} orc_grid;

void FN(orc_fwd_step)(const orc_grid* g, real* f1, real* f2, real* f3, real* f4, real* d1x, real* d1y,
                      real* d1z, real* d2x, real* d2y, real* d2z, const real* irho, const real* m1,
                      const real* m2, const real* m3, const real* m4, const real* rx, const real* ry,
                      const real* rz, const float* abx, const float* aby, const float* abz,
                      i64 src_index, float src_amp, int nrec, const i64* rec_index, real* traces)
{
    int ldimx = g->ldimx, ldimy = g->ldimy;
    FN(orc_loop2)(f1, f2, f3, f4, ldimx, ldimy, g->ixbeg, g->ixend, g->iybeg, g->iyend, g->izbeg, g->izend,
                  abx, aby, abz, g->dt);
    if (g->free_surface) FN(orc_loop4)(f1, f2, ldimx, ldimy, g->izbeg);
    FN(orc_fwd_drv)(f1, f2, irho, d1x, d1y, d1z, d2x, d2y, d2z, g->ixbeg, g->ixend, g->iybeg, g->iyend,
                    g->izbeg, g->izend, (float)(1.0 / g->dx), (float)(1.0 / g->dy), (float)(1.0 / g->dz),
                    ldimx, ldimy);
    if (g->free_surface) FN(orc_loop4_derivatives)(d1x, d1y, d1z, d2x, d2y, d2z, ldimx, ldimy, g->izbeg);
    FN(orc_fwd_update)(f3, f4, d1x, d2x, d1y, d2y, d1z, d2z, f1, f2, irho, m1, m2, m3, m4, rx, ry, rz,
                       g->ixbeg, g->ixend, g->iybeg, g->iyend, g->izbeg, g->izend, ldimx, ldimy, g->dt,
                       g->dx, g->dy, g->dz);
    if (src_index >= 0) {
        f3[src_index] += (real)src_amp * (real)g->dt;
        f4[src_index] += (real)src_amp * (real)g->dt;
    }
    for (int r = 0; r < nrec; ++r) {
        i64 i = rec_index[r];
        traces[r] = -(2 * f1[i] + f2[i]) / 3;
    }
}

void FN(orc_adj_step)(const orc_grid* g, real* f1, real* f2, real* f3, real* f4, real* d1x, real* d1y,
                      real* d1z, real* d2x, real* d2y, real* d2z, real* rhs3, real* rhs4,
                      const real* irho, const real* m1, const real* m2, const real* m3, const real* m4,
                      const real* rx, const real* ry, const real* rz, const float* abx,
                      const float* aby, const float* abz, int nrec, const i64* rec_index,
                      const real* residual)
{
    int ldimx = g->ldimx, ldimy = g->ldimy;
    for (int r = 0; r < nrec; ++r) {
        i64 i = rec_index[r];
        f3[i] += (real)(-2.0f / 3.0f) * residual[r];
        f4[i] += (real)(-1.0f / 3.0f) * residual[r];
    }
    double dx = g->dx, dy = g->dy, dz = g->dz;
    FN(orc_adj_drv)(d1x, d2x, d1y, d2y, d1z, d2z, rhs3, rhs4, f1, f2, irho, m1, m2, m3, m4, rx, ry, rz,
                    g->ixbeg, g->ixend, g->iybeg, g->iyend, g->izbeg, g->izend, (float)(1.0 / (4 * dx * dy)),
                    (float)(1.0 / (4 * dy * dz)), (float)(1.0 / (4 * dx * dz)), ldimx, ldimy,
                    (float)(1.0 / dx), (float)(1.0 / dy), (float)(1.0 / dz));
    if (g->free_surface) FN(orc_loop4_derivatives)(d1x, d1y, d1z, d2x, d2y, d2z, ldimx, ldimy, g->izbeg);
    FN(orc_adj_update)(f3, f4, d1x, d2x, d1y, d2y, d1z, d2z, rhs3, rhs4, abx, aby, abz, g->ixbeg, g->ixend,
                       g->iybeg, g->iyend, g->izbeg, g->izend, ldimx, ldimy, g->dt, dx, dy, dz,
                       g->sponge_active);
    FN(orc_loop2)(f1, f2, f3, f4, ldimx, ldimy, g->ixbeg, g->ixend, g->iybeg, g->iyend, g->izbeg, g->izend,
                  abx, aby, abz, g->dt);
    if (g->free_surface) FN(orc_loop4)(f1, f2, ldimx, ldimy, g->izbeg);
}

/* ------------------------------------------------------------------------
 * Type1 discretisation (kernels/kernel_type1_gpu_{fwd,adj,grad}.cu): the
 * constant-density TTI operator with centred second derivatives (DF2
 * coefficients on the normal directions, the same diagonal form for the
 * mixed ones) and no separate first-derivative stage.  The restatement
 * follows the launchers' default (optimised) kernels:
 * fwd_main_loop_2_1 (kernel_type1_gpu_fwd.cu:150-232 for the derivative
 * sums, :122-146 for V/H and the right-hand sides) and adj_main_loop_2
 * (kernel_type1_gpu_adj.cu:103-235).  Finite-difference constants as
 * kernel_utils::compute_fd_const: invdxx = 1/dx^2, invdxy = 1/(4 dx dy), ...
 * ---------------------------------------------------------------------- */
typedef struct {
    real xx, yy, zz, xy, yz, zx;
} t1_drv;

/* Centred second derivatives of f at i (strides sx = 1, sy = ldimx, sz). */
static inline t1_drv t1_derivs(const real* f, i64 i, i64 sy, i64 sz, real ixx, real iyy, real izz,
                               real ixy, real iyz, real izx)
{
    t1_drv d;
    /* z terms in plane order iz-4 .. iz+4 (compute_z_contributions, :150-185) */
    real zz = 0, zx = 0, yz = 0;
    for (int ir = -4; ir <= 4; ++ir) {
        real c = (real)C2[ir < 0 ? -ir : ir];
        i64 j = i + ir * sz;
        zz = zz + c * f[j];
        if (ir != 0) {
            zx = zx + c * (f[j + ir] - f[j - ir]);
            yz = yz + c * (f[j + ir * sy] - f[j - ir * sy]);
        }
    }
    d.zz = zz * izz;
    d.zx = zx * izx;
    d.yz = yz * iyz;
    /* x and y terms (compute_xy_contributions, :190-232) */
    real xx = (real)C2[0] * f[i], yy = (real)C2[0] * f[i], xy = 0;
    for (int k = 1; k <= 4; ++k) {
        real c = (real)C2[k];
        xx += c * (f[i + k] + f[i - k]);
        yy += c * (f[i + k * sy] + f[i - k * sy]);
        xy += c * (f[i + k * sy + k] - f[i + k * sy - k] + f[i - k * sy - k] - f[i - k * sy + k]);
    }
    d.xx = xx * ixx;
    d.yy = yy * iyy;
    d.xy = xy * ixy;
    return d;
}

/* mode 0: f3 += dt*rhs, f4 += dt*rhs (no sponge);  mode 1: f = A f + B rhs dt
 * (sponge, A,B = min over the axis profiles);  mode 2 (calc_snap): the
 * right-hand sides themselves into halo-free outputs with ldimx_out/ldimy_out.
 * In modes 0 and 1 outputs use the input strides (the reference offsets the
 * output base with the input dimensions, kernel_type1_gpu_fwd.cu:488-492). */
void FN(orc_t1_fwd)(real* f3, real* f4, const real* f1, const real* f2, const real* m1, const real* m2,
                    const real* m3, const real* m4, const real* m5, const real* m6, const real* m7,
                    const float* abx, const float* aby, const float* abz, int ixbeg, int ixend, int iybeg,
                    int iyend, int izbeg, int izend, int ldimx, int ldimy, int ldimx_out, int ldimy_out,
                    float dt, double dx, double dy, double dz, int mode)
{
    const real ixx = (real)(float)(1.0 / (dx * dx)), iyy = (real)(float)(1.0 / (dy * dy)),
               izz = (real)(float)(1.0 / (dz * dz));
    const real ixy = (real)(float)(1.0 / (4 * dx * dy)), iyz = (real)(float)(1.0 / (4 * dy * dz)),
               izx = (real)(float)(1.0 / (4 * dx * dz));
    const i64 sy = ldimx, sz = (i64)ldimx * ldimy;
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                t1_drv a = t1_derivs(f1, i, sy, sz, ixx, iyy, izz, ixy, iyz, izx);
                t1_drv b = t1_derivs(f2, i, sy, sz, ixx, iyy, izz, ixy, iyz, izx);
                real rx = m5[i], ry = m6[i], rz = m7[i];
                real rxx = rx * rx, ryy = ry * ry, rzz = rz * rz;
                real rxy = (real)2 * rx * ry, ryz = (real)2 * ry * rz, rzx = (real)2 * rz * rx;
                real V1 = rxx * a.xx + ryy * a.yy + rzz * a.zz + rxy * a.xy + rzx * a.zx + ryz * a.yz;
                real H1 = a.xx + a.yy + a.zz - V1;
                real V2 = rxx * b.xx + ryy * b.yy + rzz * b.zz + rxy * b.xy + rzx * b.zx + ryz * b.yz;
                real H2 = b.xx + b.yy + b.zz - V2;
                real r3 = m1[i] * H1 + m4[i] * V1 + m2[i] * V2;
                real r4 = m2[i] * H1 + m3[i] * V2 + m4[i] * H2;
                if (mode == 2) {
                    i64 o = ((i64)(iz - izbeg) * ldimy_out + (iy - iybeg)) * ldimx_out + (ix - ixbeg);
                    f3[o] = r3;
                    f4[o] = r4;
                } else if (mode == 1) {
                    real A = fminf(abx[2 * ix], fminf(aby[2 * iy], abz[2 * iz]));
                    real B = fminf(abx[2 * ix + 1], fminf(aby[2 * iy + 1], abz[2 * iz + 1]));
                    f3[i] = A * f3[i] + B * r3 * (real)dt;
                    f4[i] = A * f4[i] + B * r4 * (real)dt;
                } else {
                    f3[i] += r3 * (real)dt;
                    f4[i] += r4 * (real)dt;
                }
            }
}

/* Adjoint temporaries at j (compute_temp_arrays, kernel_type1_gpu_adj.cu:103-153):
 * lap/hz of both fields, weighted per derivative by r_a r_b. */
typedef struct {
    real lx, hx, lz, hz;
} t1_base;
static inline t1_base t1_base_at(const real* f1, const real* f2, const real* m1, const real* m2,
                                 const real* m3, const real* m4, i64 j)
{
    t1_base b;
    b.lx = m1[j] * f1[j] + m2[j] * f2[j];
    b.hx = (-m1[j] + m4[j]) * f1[j] - m2[j] * f2[j];
    b.lz = m4[j] * f2[j];
    b.hz = m2[j] * f1[j] + (-m4[j] + m3[j]) * f2[j];
    return b;
}

void FN(orc_t1_adj)(real* f3, real* f4, const real* f1, const real* f2, const real* m1, const real* m2,
                    const real* m3, const real* m4, const real* m5, const real* m6, const real* m7,
                    const float* abx, const float* aby, const float* abz, int ixbeg, int ixend, int iybeg,
                    int iyend, int izbeg, int izend, int ldimx, int ldimy, float dt, double dx, double dy,
                    double dz, int use_sponge)
{
    const real ixx = (real)(float)(1.0 / (dx * dx)), iyy = (real)(float)(1.0 / (dy * dy)),
               izz = (real)(float)(1.0 / (dz * dz));
    const real ixy = (real)(float)(1.0 / (4 * dx * dy)), iyz = (real)(float)(1.0 / (4 * dy * dz)),
               izx = (real)(float)(1.0 / (4 * dx * dz));
    const i64 sy = ldimx, sz = (i64)ldimx * ldimy;
#define T1_W(j, w1, w2, lap, o3, o4)                                                                 \
    do {                                                                                             \
        t1_base b_ = t1_base_at(f1, f2, m1, m2, m3, m4, (j));                                        \
        real w_ = (w1) * (w2);                                                                       \
        o3 = ((lap) ? b_.lx : (real)0) + w_ * b_.hx;                                                 \
        o4 = ((lap) ? b_.lz : (real)0) + w_ * b_.hz;                                                 \
    } while (0)
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 i = IDX(ix, iy, iz);
                real s3 = 0, s4 = 0, t3, t4, u3, u4;
                /* z terms, planes iz-4 .. iz+4 (compute_z_contributions, :162-186) */
                for (int ir = -4; ir <= 4; ++ir) {
                    real c = (real)C2[ir < 0 ? -ir : ir];
                    i64 j = i + ir * sz;
                    T1_W(j, m7[j], m7[j], 1, t3, t4);
                    real a3 = izz * c * t3, a4 = izz * c * t4;
                    if (ir != 0) {
                        i64 jp = j + ir * sy, jm = j - ir * sy;
                        T1_W(jp, (real)2 * m6[jp], m7[jp], 0, t3, t4);
                        T1_W(jm, (real)2 * m6[jm], m7[jm], 0, u3, u4);
                        a3 = a3 + iyz * c * (t3 - u3);
                        a4 = a4 + iyz * c * (t4 - u4);
                        jp = j + ir;
                        jm = j - ir;
                        T1_W(jp, (real)2 * m7[jp], m5[jp], 0, t3, t4);
                        T1_W(jm, (real)2 * m7[jm], m5[jm], 0, u3, u4);
                        a3 = a3 + izx * c * (t3 - u3);
                        a4 = a4 + izx * c * (t4 - u4);
                    }
                    s3 = s3 + a3;
                    s4 = s4 + a4;
                }
                /* x and y terms (compute_xy_contributions, :191-217) */
                real xx3, xx4, yy3, yy4, xy3 = 0, xy4 = 0;
                T1_W(i, m5[i], m5[i], 1, t3, t4);
                xx3 = (real)C2[0] * t3;
                xx4 = (real)C2[0] * t4;
                T1_W(i, m6[i], m6[i], 1, t3, t4);
                yy3 = (real)C2[0] * t3;
                yy4 = (real)C2[0] * t4;
                for (int k = 1; k <= 4; ++k) {
                    real c = (real)C2[k];
                    i64 jp = i + k, jm = i - k;
                    T1_W(jp, m5[jp], m5[jp], 1, t3, t4);
                    T1_W(jm, m5[jm], m5[jm], 1, u3, u4);
                    xx3 += c * (t3 + u3);
                    xx4 += c * (t4 + u4);
                    jp = i + k * sy;
                    jm = i - k * sy;
                    T1_W(jp, m6[jp], m6[jp], 1, t3, t4);
                    T1_W(jm, m6[jm], m6[jm], 1, u3, u4);
                    yy3 += c * (t3 + u3);
                    yy4 += c * (t4 + u4);
                    real p3, p4, q3, q4, r3, r4, w3, w4;
                    i64 jpp = i + k * sy + k, jpm = i + k * sy - k, jmm = i - k * sy - k, jmp = i - k * sy + k;
                    T1_W(jpp, (real)2 * m5[jpp], m6[jpp], 0, p3, p4);
                    T1_W(jpm, (real)2 * m5[jpm], m6[jpm], 0, q3, q4);
                    T1_W(jmm, (real)2 * m5[jmm], m6[jmm], 0, r3, r4);
                    T1_W(jmp, (real)2 * m5[jmp], m6[jmp], 0, w3, w4);
                    xy3 += c * (p3 - q3 + r3 - w3);
                    xy4 += c * (p4 - q4 + r4 - w4);
                }
                s3 += ixx * xx3 + iyy * yy3 + ixy * xy3;
                s4 += ixx * xx4 + iyy * yy4 + ixy * xy4;
                if (use_sponge) {
                    real A = fminf(abx[2 * ix], fminf(aby[2 * iy], abz[2 * iz]));
                    real B = fminf(abx[2 * ix + 1], fminf(aby[2 * iy + 1], abz[2 * iz + 1]));
                    f3[i] = A * f3[i] + B * s3 * (real)dt;
                    f4[i] = A * f4[i] + B * s4 * (real)dt;
                } else {
                    f3[i] += s3 * (real)dt;
                    f4[i] += s4 * (real)dt;
                }
            }
#undef T1_W
}

/* Type1 imaging: grad += adj_x*snap_x + adj_z*snap_z over the interior
 * (kernel_type1_gpu_grad.cu:4-21); snapshots and gradient are halo-free. */
void FN(orc_t1_grad)(const real* snap_x, const real* snap_z, real* grad, const real* adj_x, const real* adj_z,
                     int ixbeg, int ixend, int iybeg, int iyend, int izbeg, int izend, int sldx, int sldy,
                     int ldimx, int ldimy)
{
#pragma omp parallel for schedule(static)
    for (int iz = izbeg; iz <= izend; ++iz)
        for (int iy = iybeg; iy <= iyend; ++iy)
            for (int ix = ixbeg; ix <= ixend; ++ix) {
                i64 d = ((i64)(iz - izbeg) * sldy + (iy - iybeg)) * sldx + (ix - ixbeg);
                i64 i = IDX(ix, iy, iz);
                grad[d] += adj_x[i] * snap_x[d] + adj_z[i] * snap_z[d];
            }
}

int FN(orc_num_threads)(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
