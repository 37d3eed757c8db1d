/*
 * Oracle: Okada (1992) rectangular dislocation in a half-space.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates, statement by statement,
 *   fortran/3d/src/dc3d.f:1-198    DC3D   (finite source, real + image parts)
 *   fortran/3d/src/dc3d.f:200-282  UA     (part A of Okada's Table 6)
 *   fortran/3d/src/dc3d.f:284-400  UB     (part B)
 *   fortran/3d/src/dc3d.f:402-507  UC     (part C)
 *   fortran/3d/src/dc3d.f:509-544  DCCON0
 *   fortran/3d/src/dc3d.f:596-665  DCCON2
 *   fortran/3d/src/okada92.f90:59-87    computeReferenceSystemOkada92
 *   fortran/3d/src/okada92.f90:109-207  computeStressOkada92
 *
 * Two modes:
 *   ORC_OKADA_REF32IO  reproduces the reference's REAL*4 interface: every input
 *       of DC3D is rounded to binary32 (SNGL), the two REAL*4 differences
 *       XI=X-AL and D=DEPTH+/-Z are taken in binary32, the REAL*4 EPS=1e-6 of
 *       DC3D is the binary32 value, and the 12 outputs are rounded to binary32
 *       (REAL(U,4)) before the FP64 rotation to stress.
 *   ORC_OKADA_FP64     the same statements with every value kept in binary64.
 *
 * Compiled with -ffp-contract=off so that each statement rounds exactly as the
 * gfortran/gcc build of the reference does on x86-64 (no FMA contraction).
 */
#include <math.h>
#include <string.h>
#include "oracle.h"

#define PI2 6.283185307179586

typedef struct {
    double alp1, alp2, alp3, alp4, alp5, sd, cd, sdsd, cdcd, sdcd, s2d, c2d;
} c0_t;

typedef struct {
    double xi2, et2, q2, r, r2, r3, r5, y, d, tt, alx, ale, x11, y11, x32, y32;
    double ey, ez, fy, fz, gy, gz, hy, hz;
} c2_t;

static double f32(double v) { return (double)(float)v; }

/* dc3d.f:509-544 */
static void dccon0(double alpha, double dip, c0_t *c)
{
    const double eps = 1.0e-6;
    c->alp1 = (1.0 - alpha) / 2.0;
    c->alp2 = alpha / 2.0;
    c->alp3 = (1.0 - alpha) / alpha;
    c->alp4 = 1.0 - alpha;
    c->alp5 = alpha;
    double p18 = PI2 / 360.0;
    c->sd = sin(dip * p18);
    c->cd = cos(dip * p18);
    if (fabs(c->cd) < eps) {
        c->cd = 0.0;
        if (c->sd > 0.0) c->sd = 1.0;
        if (c->sd < 0.0) c->sd = -1.0;
    }
    c->sdsd = c->sd * c->sd;
    c->cdcd = c->cd * c->cd;
    c->sdcd = c->sd * c->cd;
    c->s2d = 2.0 * c->sdcd;
    c->c2d = c->cdcd - c->sdsd;
}

/* dc3d.f:596-665.  XI, ET, Q are snapped in place (Fortran pass by reference). */
static void dccon2(double *xi, double *et, double *q, double sd, double cd,
                   int kxi, int ket, c2_t *c)
{
    const double eps = 1.0e-6;
    if (fabs(*xi) < eps) *xi = 0.0;
    if (fabs(*et) < eps) *et = 0.0;
    if (fabs(*q) < eps) *q = 0.0;
    double XI = *xi, ET = *et, Q = *q;
    c->xi2 = XI * XI;
    c->et2 = ET * ET;
    c->q2 = Q * Q;
    c->r2 = c->xi2 + c->et2 + c->q2;
    c->r = sqrt(c->r2);
    if (c->r == 0.0) return;
    c->r3 = c->r * c->r2;
    c->r5 = c->r3 * c->r2;
    c->y = ET * cd + Q * sd;
    c->d = ET * sd - Q * cd;
    if (Q == 0.0) c->tt = 0.0;
    else c->tt = atan(XI * ET / (Q * c->r));
    if (kxi == 1) {
        c->alx = -log(c->r - XI);
        c->x11 = 0.0;
        c->x32 = 0.0;
    } else {
        double rxi = c->r + XI;
        c->alx = log(rxi);
        c->x11 = 1.0 / (c->r * rxi);
        c->x32 = (c->r + rxi) * c->x11 * c->x11 / c->r;
    }
    if (ket == 1) {
        c->ale = -log(c->r - ET);
        c->y11 = 0.0;
        c->y32 = 0.0;
    } else {
        double ret = c->r + ET;
        c->ale = log(ret);
        c->y11 = 1.0 / (c->r * ret);
        c->y32 = (c->r + ret) * c->y11 * c->y11 / c->r;
    }
    c->ey = sd / c->r - c->y * Q / c->r3;
    c->ez = cd / c->r + c->d * Q / c->r3;
    c->fy = c->d / c->r3 + c->xi2 * c->y32 * sd;
    c->fz = c->y / c->r3 + c->xi2 * c->y32 * cd;
    c->gy = 2.0 * c->x11 * sd - c->y * Q * c->x32;
    c->gz = 2.0 * c->x11 * cd + c->d * Q * c->x32;
    c->hy = c->d * Q * c->x32 + XI * Q * c->y32 * sd;
    c->hz = c->y * Q * c->x32 + XI * Q * c->y32 * cd;
}

static void acc(double u[12], double disl, const double du[12])
{
    for (int i = 0; i < 12; i++) u[i] = u[i] + disl / PI2 * du[i];
}

/* dc3d.f:200-282 */
static void ua(double XI, double ET, double Q, double d1, double d2, double d3,
               const c0_t *a, const c2_t *c, double u[12])
{
    double du[12];
    for (int i = 0; i < 12; i++) u[i] = 0.0;
    double xy = XI * c->y11, qx = Q * c->x11, qy = Q * c->y11;
    double R = c->r, R3 = c->r3, Y = c->y, D = c->d;
    if (d1 != 0.0) {
        du[0] = c->tt / 2.0 + a->alp2 * XI * qy;
        du[1] = a->alp2 * Q / R;
        du[2] = a->alp1 * c->ale - a->alp2 * Q * qy;
        du[3] = -a->alp1 * qy - a->alp2 * c->xi2 * Q * c->y32;
        du[4] = -a->alp2 * XI * Q / R3;
        du[5] = a->alp1 * xy + a->alp2 * XI * c->q2 * c->y32;
        du[6] = a->alp1 * xy * a->sd + a->alp2 * XI * c->fy + D / 2.0 * c->x11;
        du[7] = a->alp2 * c->ey;
        du[8] = a->alp1 * (a->cd / R + qy * a->sd) - a->alp2 * Q * c->fy;
        du[9] = a->alp1 * xy * a->cd + a->alp2 * XI * c->fz + Y / 2.0 * c->x11;
        du[10] = a->alp2 * c->ez;
        du[11] = -a->alp1 * (a->sd / R - qy * a->cd) - a->alp2 * Q * c->fz;
        acc(u, d1, du);
    }
    if (d2 != 0.0) {
        du[0] = a->alp2 * Q / R;
        du[1] = c->tt / 2.0 + a->alp2 * ET * qx;
        du[2] = a->alp1 * c->alx - a->alp2 * Q * qx;
        du[3] = -a->alp2 * XI * Q / R3;
        du[4] = -qy / 2.0 - a->alp2 * ET * Q / R3;
        du[5] = a->alp1 / R + a->alp2 * c->q2 / R3;
        du[6] = a->alp2 * c->ey;
        du[7] = a->alp1 * D * c->x11 + xy / 2.0 * a->sd + a->alp2 * ET * c->gy;
        du[8] = a->alp1 * Y * c->x11 - a->alp2 * Q * c->gy;
        du[9] = a->alp2 * c->ez;
        du[10] = a->alp1 * Y * c->x11 + xy / 2.0 * a->cd + a->alp2 * ET * c->gz;
        du[11] = -a->alp1 * D * c->x11 - a->alp2 * Q * c->gz;
        acc(u, d2, du);
    }
    if (d3 != 0.0) {
        du[0] = -a->alp1 * c->ale - a->alp2 * Q * qy;
        du[1] = -a->alp1 * c->alx - a->alp2 * Q * qx;
        du[2] = c->tt / 2.0 - a->alp2 * (ET * qx + XI * qy);
        du[3] = -a->alp1 * xy + a->alp2 * XI * c->q2 * c->y32;
        du[4] = -a->alp1 / R + a->alp2 * c->q2 / R3;
        du[5] = -a->alp1 * qy - a->alp2 * Q * c->q2 * c->y32;
        du[6] = -a->alp1 * (a->cd / R + qy * a->sd) - a->alp2 * Q * c->fy;
        du[7] = -a->alp1 * Y * c->x11 - a->alp2 * Q * c->gy;
        du[8] = a->alp1 * (D * c->x11 + xy * a->sd) + a->alp2 * Q * c->hy;
        du[9] = a->alp1 * (a->sd / R - qy * a->cd) - a->alp2 * Q * c->fz;
        du[10] = a->alp1 * D * c->x11 - a->alp2 * Q * c->gz;
        du[11] = a->alp1 * (Y * c->x11 + xy * a->cd) + a->alp2 * Q * c->hz;
        acc(u, d3, du);
    }
}

/* dc3d.f:284-400 */
static void ub(double XI, double ET, double Q, double d1, double d2, double d3,
               const c0_t *a, const c2_t *c, double u[12])
{
    double du[12];
    double R = c->r, Y = c->y, D = c->d;
    double rd = R + D;
    double d11 = 1.0 / (R * rd);
    double aj2 = XI * Y / rd * d11;
    double aj5 = -(D + Y * Y / rd) * d11;
    double ai1, ai2, ai3, ai4, ak1, ak2, ak3, ak4, aj1, aj3, aj4, aj6;
    if (a->cd != 0.0) {
        if (XI == 0.0) {
            ai4 = 0.0;
        } else {
            double x = sqrt(c->xi2 + c->q2);
            ai4 = 1.0 / a->cdcd * (XI / rd * a->sdcd +
                  2.0 * atan((ET * (x + Q * a->cd) + x * (R + x) * a->sd) /
                             (XI * (R + x) * a->cd)));
        }
        ai3 = (Y * a->cd / rd - c->ale + a->sd * log(rd)) / a->cdcd;
        ak1 = XI * (d11 - c->y11 * a->sd) / a->cd;
        ak3 = (Q * c->y11 - Y * d11) / a->cd;
        aj3 = (ak1 - aj2 * a->sd) / a->cd;
        aj6 = (ak3 - aj5 * a->sd) / a->cd;
    } else {
        double rd2 = rd * rd;
        ai3 = (ET / rd + Y * Q / rd2 - c->ale) / 2.0;
        ai4 = XI * Y / rd2 / 2.0;
        ak1 = XI * Q / rd * d11;
        ak3 = a->sd / rd * (c->xi2 * d11 - 1.0);
        aj3 = -XI / rd2 * (c->q2 * d11 - 1.0 / 2.0);
        aj6 = -Y / rd2 * (c->xi2 * d11 - 1.0 / 2.0);
    }
    double xy = XI * c->y11;
    ai1 = -XI / rd * a->cd - ai4 * a->sd;
    ai2 = log(rd) + ai3 * a->sd;
    ak2 = 1.0 / R + ak3 * a->sd;
    ak4 = xy * a->cd - ak1 * a->sd;
    aj1 = aj5 * a->cd - aj6 * a->sd;
    aj4 = -xy - aj2 * a->cd + aj3 * a->sd;
    for (int i = 0; i < 12; i++) u[i] = 0.0;
    double qx = Q * c->x11, qy = Q * c->y11;
    double R3 = c->r3;
    if (d1 != 0.0) {
        du[0] = -XI * qy - c->tt - a->alp3 * ai1 * a->sd;
        du[1] = -Q / R + a->alp3 * Y / rd * a->sd;
        du[2] = Q * qy - a->alp3 * ai2 * a->sd;
        du[3] = c->xi2 * Q * c->y32 - a->alp3 * aj1 * a->sd;
        du[4] = XI * Q / R3 - a->alp3 * aj2 * a->sd;
        du[5] = -XI * c->q2 * c->y32 - a->alp3 * aj3 * a->sd;
        du[6] = -XI * c->fy - D * c->x11 + a->alp3 * (xy + aj4) * a->sd;
        du[7] = -c->ey + a->alp3 * (1.0 / R + aj5) * a->sd;
        du[8] = Q * c->fy - a->alp3 * (qy - aj6) * a->sd;
        du[9] = -XI * c->fz - Y * c->x11 + a->alp3 * ak1 * a->sd;
        du[10] = -c->ez + a->alp3 * Y * d11 * a->sd;
        du[11] = Q * c->fz + a->alp3 * ak2 * a->sd;
        acc(u, d1, du);
    }
    if (d2 != 0.0) {
        du[0] = -Q / R + a->alp3 * ai3 * a->sdcd;
        du[1] = -ET * qx - c->tt - a->alp3 * XI / rd * a->sdcd;
        du[2] = Q * qx + a->alp3 * ai4 * a->sdcd;
        du[3] = XI * Q / R3 + a->alp3 * aj4 * a->sdcd;
        du[4] = ET * Q / R3 + qy + a->alp3 * aj5 * a->sdcd;
        du[5] = -c->q2 / R3 + a->alp3 * aj6 * a->sdcd;
        du[6] = -c->ey + a->alp3 * aj1 * a->sdcd;
        du[7] = -ET * c->gy - xy * a->sd + a->alp3 * aj2 * a->sdcd;
        du[8] = Q * c->gy + a->alp3 * aj3 * a->sdcd;
        du[9] = -c->ez - a->alp3 * ak3 * a->sdcd;
        du[10] = -ET * c->gz - xy * a->cd - a->alp3 * XI * d11 * a->sdcd;
        du[11] = Q * c->gz - a->alp3 * ak4 * a->sdcd;
        acc(u, d2, du);
    }
    if (d3 != 0.0) {
        du[0] = Q * qy - a->alp3 * ai3 * a->sdsd;
        du[1] = Q * qx + a->alp3 * XI / rd * a->sdsd;
        du[2] = ET * qx + XI * qy - c->tt - a->alp3 * ai4 * a->sdsd;
        du[3] = -XI * c->q2 * c->y32 - a->alp3 * aj4 * a->sdsd;
        du[4] = -c->q2 / R3 - a->alp3 * aj5 * a->sdsd;
        du[5] = Q * c->q2 * c->y32 - a->alp3 * aj6 * a->sdsd;
        du[6] = Q * c->fy - a->alp3 * aj1 * a->sdsd;
        du[7] = Q * c->gy - a->alp3 * aj2 * a->sdsd;
        du[8] = -Q * c->hy - a->alp3 * aj3 * a->sdsd;
        du[9] = Q * c->fz + a->alp3 * ak3 * a->sdsd;
        du[10] = Q * c->gz + a->alp3 * XI * d11 * a->sdsd;
        du[11] = -Q * c->hz + a->alp3 * ak4 * a->sdsd;
        acc(u, d3, du);
    }
}

/* dc3d.f:402-507 */
static void uc(double XI, double ET, double Q, double Z, double d1, double d2,
               double d3, const c0_t *a, const c2_t *c, double u[12])
{
    double du[12];
    double R = c->r, R2 = c->r2, R3 = c->r3, R5 = c->r5, Y = c->y, D = c->d;
    double sd = a->sd, cd = a->cd, sdsd = a->sdsd, cdcd = a->cdcd, sdcd = a->sdcd;
    double alp4 = a->alp4, alp5 = a->alp5;
    double C = D + Z;
    double x53 = (8.0 * R2 + 9.0 * R * XI + 3.0 * c->xi2) * c->x11 * c->x11 * c->x11 / R2;
    double y53 = (8.0 * R2 + 9.0 * R * ET + 3.0 * c->et2) * c->y11 * c->y11 * c->y11 / R2;
    double h = Q * cd - Z;
    double z32 = sd / R3 - h * c->y32;
    double z53 = 3.0 * sd / R5 - h * y53;
    double y0 = c->y11 - c->xi2 * c->y32;
    double z0 = z32 - c->xi2 * z53;
    double ppy = cd / R3 + Q * c->y32 * sd;
    double ppz = sd / R3 - Q * c->y32 * cd;
    double qq = Z * c->y32 + z32 + z0;
    double qqy = 3.0 * C * D / R5 - qq * sd;
    double qqz = 3.0 * C * Y / R5 - qq * cd + Q * c->y32;
    double xy = XI * c->y11;
    double qx = Q * c->x11;
    double qy = Q * c->y11;
    double qr = 3.0 * Q / R5;
    double cqx = C * Q * x53;
    double cdr = (C + D) / R3;
    double yy0 = Y / R3 - y0 * cd;
    (void)qx; (void)cqx;
    double X11 = c->x11, X32 = c->x32, Y11 = c->y11, Y32 = c->y32, Q2 = c->q2;
    for (int i = 0; i < 12; i++) u[i] = 0.0;
    if (d1 != 0.0) {
        du[0] = alp4 * xy * cd - alp5 * XI * Q * z32;
        du[1] = alp4 * (cd / R + 2.0 * qy * sd) - alp5 * C * Q / R3;
        du[2] = alp4 * qy * cd - alp5 * (C * ET / R3 - Z * Y11 + c->xi2 * z32);
        du[3] = alp4 * y0 * cd - alp5 * Q * z0;
        du[4] = -alp4 * XI * (cd / R3 + 2.0 * Q * Y32 * sd) + alp5 * C * XI * qr;
        du[5] = -alp4 * XI * Q * Y32 * cd + alp5 * XI * (3.0 * C * ET / R5 - qq);
        du[6] = -alp4 * XI * ppy * cd - alp5 * XI * qqy;
        du[7] = alp4 * 2.0 * (D / R3 - y0 * sd) * sd - Y / R3 * cd
                - alp5 * (cdr * sd - ET / R3 - C * Y * qr);
        du[8] = -alp4 * Q / R3 + yy0 * sd + alp5 * (cdr * cd + C * D * qr - (y0 * cd + Q * z0) * sd);
        du[9] = alp4 * XI * ppz * cd - alp5 * XI * qqz;
        du[10] = alp4 * 2.0 * (Y / R3 - y0 * cd) * sd + D / R3 * cd - alp5 * (cdr * cd + C * D * qr);
        du[11] = yy0 * cd - alp5 * (cdr * sd - C * Y * qr - y0 * sdsd + Q * z0 * cd);
        acc(u, d1, du);
    }
    if (d2 != 0.0) {
        du[0] = alp4 * cd / R - qy * sd - alp5 * C * Q / R3;
        du[1] = alp4 * Y * X11 - alp5 * C * ET * Q * X32;
        du[2] = -D * X11 - xy * sd - alp5 * C * (X11 - Q2 * X32);
        du[3] = -alp4 * XI / R3 * cd + alp5 * C * XI * qr + XI * Q * Y32 * sd;
        du[4] = -alp4 * Y / R3 + alp5 * C * ET * qr;
        du[5] = D / R3 - y0 * sd + alp5 * C / R3 * (1.0 - 3.0 * Q2 / R2);
        du[6] = -alp4 * ET / R3 + y0 * sdsd - alp5 * (cdr * sd - C * Y * qr);
        du[7] = alp4 * (X11 - Y * Y * X32) - alp5 * C * ((D + 2.0 * Q * cd) * X32 - Y * ET * Q * x53);
        du[8] = XI * ppy * sd + Y * D * X32 + alp5 * C * ((Y + 2.0 * Q * sd) * X32 - Y * Q2 * x53);
        du[9] = -Q / R3 + y0 * sdcd - alp5 * (cdr * cd + C * D * qr);
        du[10] = alp4 * Y * D * X32 - alp5 * C * ((Y - 2.0 * Q * sd) * X32 + D * ET * Q * x53);
        du[11] = -XI * ppz * sd + X11 - D * D * X32 - alp5 * C * ((D - 2.0 * Q * cd) * X32 - D * Q2 * x53);
        acc(u, d2, du);
    }
    if (d3 != 0.0) {
        du[0] = -alp4 * (sd / R + qy * cd) - alp5 * (Z * Y11 - Q2 * z32);
        du[1] = alp4 * 2.0 * xy * sd + D * X11 - alp5 * C * (X11 - Q2 * X32);
        du[2] = alp4 * (Y * X11 + xy * cd) + alp5 * Q * (C * ET * X32 + XI * z32);
        du[3] = alp4 * XI / R3 * sd + XI * Q * Y32 * cd + alp5 * XI * (3.0 * C * ET / R5 - 2.0 * z32 - z0);
        du[4] = alp4 * 2.0 * y0 * sd - D / R3 + alp5 * C / R3 * (1.0 - 3.0 * Q2 / R2);
        du[5] = -alp4 * yy0 - alp5 * (C * ET * qr - Q * z0);
        du[6] = alp4 * (Q / R3 + y0 * sdcd) + alp5 * (Z / R3 * cd + C * D * qr - Q * z0 * sd);
        du[7] = -alp4 * 2.0 * XI * ppy * sd - Y * D * X32
                + alp5 * C * ((Y + 2.0 * Q * sd) * X32 - Y * Q2 * x53);
        du[8] = -alp4 * (XI * ppy * cd - X11 + Y * Y * X32)
                + alp5 * (C * ((D + 2.0 * Q * cd) * X32 - Y * ET * Q * x53) + XI * qqy);
        du[9] = -ET / R3 + y0 * cdcd - alp5 * (Z / R3 * sd - C * Y * qr - y0 * sdsd + Q * z0 * cd);
        du[10] = alp4 * 2.0 * XI * ppz * sd - X11 + D * D * X32
                 - alp5 * C * ((D - 2.0 * Q * cd) * X32 - D * Q2 * x53);
        du[11] = alp4 * (XI * ppz * cd + Y * D * X32)
                 + alp5 * (C * ((Y - 2.0 * Q * sd) * X32 + D * ET * Q * x53) + XI * qqz);
        acc(u, d3, du);
    }
}

/* Singular-edge test and negative-extension flags, dc3d.f:70-87 / 122-139. */
static int edge_setup(double xi[2], double et[2], double q, double eps, int kxi[2], int ket[2])
{
    if (q == 0.0 && ((xi[0] * xi[1] <= 0.0 && et[0] * et[1] == 0.0) ||
                     (et[0] * et[1] <= 0.0 && xi[0] * xi[1] == 0.0)))
        return 1;
    kxi[0] = kxi[1] = ket[0] = ket[1] = 0;
    double r12 = sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q);
    double r21 = sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q);
    double r22 = sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q);
    if (xi[0] < 0.0 && r21 + xi[1] < eps) kxi[0] = 1;
    if (xi[0] < 0.0 && r22 + xi[1] < eps) kxi[1] = 1;
    if (et[0] < 0.0 && r12 + et[1] < eps) ket[0] = 1;
    if (et[0] < 0.0 && r22 + et[1] < eps) ket[1] = 1;
    return 0;
}

/*
 * DC3D, dc3d.f:1-198.  In REF32IO mode the caller passes binary32-representable
 * inputs (the REAL*4 dummies); the result u[] holds the REAL*4 outputs widened to
 * double.  Returns IRET (0 normal, 1 singular -> u = 0).
 */
int orc_dc3d(int mode, double alpha, double x, double y, double z, double depth,
             double dip, double al1, double al2, double aw1, double aw2,
             double disl1, double disl2, double disl3, double out[12])
{
    const int r32 = (mode == ORC_OKADA_REF32IO);
    const double eps = r32 ? (double)1.0e-6f : 1.0e-6;   /* REAL*4 EPS */
    double u[12], du[12], dua[12], dub[12], duc[12];
    double xi[2], et[2];
    int kxi[2], ket[2];
    c0_t c0;
    c2_t c2;
    memset(&c2, 0, sizeof c2);
    for (int i = 0; i < 12; i++) { u[i] = 0.0; dua[i] = dub[i] = duc[i] = 0.0; }
    dccon0(alpha, dip, &c0);
    double zz = z, dd1 = disl1, dd2 = disl2, dd3 = disl3;
    if (r32) {
        xi[0] = (double)((float)x - (float)al1);
        xi[1] = (double)((float)x - (float)al2);
    } else {
        xi[0] = x - al1;
        xi[1] = x - al2;
    }
    if (fabs(xi[0]) < eps) xi[0] = 0.0;
    if (fabs(xi[1]) < eps) xi[1] = 0.0;

    /* real-source contribution, dc3d.f:59-111 */
    double d = r32 ? (double)((float)depth + (float)z) : depth + z;
    double p = y * c0.cd + d * c0.sd;
    double q = y * c0.sd - d * c0.cd;
    et[0] = p - aw1;
    et[1] = p - aw2;
    if (fabs(q) < eps) q = 0.0;
    if (fabs(et[0]) < eps) et[0] = 0.0;
    if (fabs(et[1]) < eps) et[1] = 0.0;
    if (edge_setup(xi, et, q, eps, kxi, ket)) goto singular;
    for (int k = 0; k < 2; k++) {
        for (int j = 0; j < 2; j++) {
            dccon2(&xi[j], &et[k], &q, c0.sd, c0.cd, kxi[k], ket[j], &c2);
            ua(xi[j], et[k], q, dd1, dd2, dd3, &c0, &c2, dua);
            for (int i = 0; i < 12; i += 3) {
                du[i] = -dua[i];
                du[i + 1] = -dua[i + 1] * c0.cd + dua[i + 2] * c0.sd;
                du[i + 2] = -dua[i + 1] * c0.sd - dua[i + 2] * c0.cd;
                if (i < 9) continue;
                du[i] = -du[i];
                du[i + 1] = -du[i + 1];
                du[i + 2] = -du[i + 2];
            }
            for (int i = 0; i < 12; i++) {
                if (j + k != 1) u[i] = u[i] + du[i];
                else u[i] = u[i] - du[i];
            }
        }
    }

    /* image-source contribution, dc3d.f:112-165 */
    d = r32 ? (double)((float)depth - (float)z) : depth - z;
    p = y * c0.cd + d * c0.sd;
    q = y * c0.sd - d * c0.cd;
    et[0] = p - aw1;
    et[1] = p - aw2;
    if (fabs(q) < eps) q = 0.0;
    if (fabs(et[0]) < eps) et[0] = 0.0;
    if (fabs(et[1]) < eps) et[1] = 0.0;
    if (edge_setup(xi, et, q, eps, kxi, ket)) goto singular;
    for (int k = 0; k < 2; k++) {
        for (int j = 0; j < 2; j++) {
            dccon2(&xi[j], &et[k], &q, c0.sd, c0.cd, kxi[k], ket[j], &c2);
            ua(xi[j], et[k], q, dd1, dd2, dd3, &c0, &c2, dua);
            ub(xi[j], et[k], q, dd1, dd2, dd3, &c0, &c2, dub);
            uc(xi[j], et[k], q, zz, dd1, dd2, dd3, &c0, &c2, duc);
            for (int i = 0; i < 12; i += 3) {
                du[i] = dua[i] + dub[i] + z * duc[i];
                du[i + 1] = (dua[i + 1] + dub[i + 1] + z * duc[i + 1]) * c0.cd
                          - (dua[i + 2] + dub[i + 2] + z * duc[i + 2]) * c0.sd;
                du[i + 2] = (dua[i + 1] + dub[i + 1] - z * duc[i + 1]) * c0.sd
                          + (dua[i + 2] + dub[i + 2] - z * duc[i + 2]) * c0.cd;
                if (i < 9) continue;
                du[9] = du[9] + duc[0];
                du[10] = du[10] + duc[1] * c0.cd - duc[2] * c0.sd;
                du[11] = du[11] - duc[1] * c0.sd - duc[2] * c0.cd;
            }
            for (int i = 0; i < 12; i++) {
                if (j + k != 1) u[i] = u[i] + du[i];
                else u[i] = u[i] - du[i];
            }
        }
    }
    for (int i = 0; i < 12; i++) out[i] = r32 ? f32(u[i]) : u[i];
    return 0;
singular:
    for (int i = 0; i < 12; i++) out[i] = 0.0;
    return 1;
}

/* okada92.f90:59-87 */
void orc_okada_frames(int ns, const double *x, const double *L, const double *W,
                      const double *strike, const double *dip,
                      double *sv, double *dv, double *nv, double *xc)
{
    for (int i = 0; i < ns; i++) {
        sv[3 * i + 0] = cos(strike[i]);
        sv[3 * i + 1] = sin(strike[i]);
        sv[3 * i + 2] = 0.0;
        dv[3 * i + 0] = +sin(strike[i]) * cos(dip[i]);
        dv[3 * i + 1] = -cos(strike[i]) * cos(dip[i]);
        dv[3 * i + 2] = -sin(dip[i]);
        nv[3 * i + 0] = -sin(strike[i]) * sin(dip[i]);
        nv[3 * i + 1] = +cos(strike[i]) * sin(dip[i]);
        nv[3 * i + 2] = -cos(dip[i]);
        for (int k = 0; k < 3; k++)
            xc[3 * i + k] = x[3 * i + k] + L[i] / 2 * sv[3 * i + k] - W[i] / 2 * dv[3 * i + k];
    }
}

/* okada92.f90:109-207 (computeStressOkada92).  sig = s11,s12,s13,s22,s23,s33. */
void orc_okada_stress(int mode, double x1, double x2, double x3,
                      double q1, double q2, double q3, double L, double W,
                      double strike, double dipd, double s, double d, double t,
                      double G, double lambda, double sig[6])
{
    const double RAD2DEG = 57.29577951308232;
    const int r32 = (mode == ORC_OKADA_REF32IO);
#define CV(v) (r32 ? f32(v) : (v))
    double alpha = CV((lambda + G) / (lambda + 2.0 * G));
    double z = CV(-x3);
    double csst = cos(strike), ssst = sin(strike);
    double x = CV((x1 - q1) * csst + (x2 - q2) * ssst);
    double y = CV((x1 - q1) * ssst - (x2 - q2) * csst);
    double depth = CV(q3);
    double dip = CV(dipd * RAD2DEG);
    double al1 = 0.0, al2 = CV(L), aw1 = -CV(W), aw2 = 0.0;
    double disl1 = CV(s), disl2 = CV(d), disl3 = CV(t);
#undef CV
    double u[12];
    orc_dc3d(mode, alpha, x, y, z, depth, dip, al1, al2, aw1, aw2, disl1, disl2, disl3, u);
    double uxx = u[3], uyx = u[4], uzx = u[5], uxy = u[6], uyy = u[7], uzy = u[8];
    double uxz = u[9], uyz = u[10], uzz = u[11];
    double uxxr = (csst * uxx + ssst * uyx) * csst - (-csst * uxy - ssst * uyy) * ssst;
    double uxyr = (csst * uxx + ssst * uyx) * ssst + (-csst * uxy - ssst * uyy) * csst;
    double uxzr = -csst * uxz + ssst * uyz;
    double uyxr = (ssst * uxx - csst * uyx) * csst - (-ssst * uxy + csst * uyy) * ssst;
    double uyyr = (ssst * uxx - csst * uyx) * ssst + (-ssst * uxy + csst * uyy) * csst;
    double uyzr = -ssst * uxz + csst * uyz;
    double uzxr = -csst * uzx - ssst * uzy;
    double uzyr = -ssst * uzx + csst * uzy;
    double e11 = uxxr, e12 = (uxyr + uyxr) / 2.0, e13 = (uxzr + uzxr) / 2.0;
    double e22 = uyyr, e23 = (uyzr + uzyr) / 2.0, e33 = uzz;
    double ekk = e11 + e22 + e33;
    sig[0] = lambda * ekk + 2.0 * G * e11;
    sig[1] = 2.0 * G * e12;
    sig[2] = 2.0 * G * e13;
    sig[3] = lambda * ekk + 2.0 * G * e22;
    sig[4] = 2.0 * G * e23;
    sig[5] = lambda * ekk + 2.0 * G * e33;
}

/* computeDisplacementOkada92, okada92.f90:230-298: displacement (north, east,
   down) at x from slip (s, d, t) on a rectangle; zero where DC3D reports a
   singular edge */
void orc_okada_disp(int mode, double x1, double x2, double x3, double q1, double q2, double q3,
                    double L, double W, double strike, double dipd, double s, double d, double t,
                    double G, double lambda, double u[3])
{
    const double RAD2DEG = 57.29577951308232;
    const int r32 = (mode == ORC_OKADA_REF32IO);
#define CV(v) (r32 ? f32(v) : (v))
    double alpha = CV((lambda + G) / (lambda + 2.0 * G));
    double z = CV(-x3);
    double csst = cos(strike), ssst = sin(strike);
    double x = CV((x1 - q1) * csst + (x2 - q2) * ssst);
    double y = CV((x1 - q1) * ssst - (x2 - q2) * csst);
    double depth = CV(q3);
    double dip = CV(dipd * RAD2DEG);
    double al2 = CV(L), aw1 = -CV(W);
    double disl1 = CV(s), disl2 = CV(d), disl3 = CV(t);
#undef CV
    double o[12];
    if (orc_dc3d(mode, alpha, x, y, z, depth, dip, 0.0, al2, aw1, 0.0, disl1, disl2, disl3, o) != 0) {
        u[0] = u[1] = u[2] = 0.0;
        return;
    }
    u[0] = o[0] * csst + o[1] * ssst;
    u[1] = o[0] * ssst - o[1] * csst;
    u[2] = -o[2];
}
