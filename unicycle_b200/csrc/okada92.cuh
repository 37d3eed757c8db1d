// Okada (1992) displacement gradient of a rectangular dislocation in an elastic
// half-space, evaluated on the device for unit strike slip and unit dip slip at
// once.  Follows Okada's finite-source solution as coded in DC3D
// (fortran/3d/src/dc3d.f:1-198, parts A/B/C at dc3d.f:200-507, the geometry
// constants at dc3d.f:509-544 and 596-665):
//   - real source: part A; image source: parts A + B + z*C;
//   - the 2x2 corner sum with the sign rule of dc3d.f:103-106;
//   - the EPS = 1e-6 snapping of xi, eta, q and the singular-edge rejection
//     (result zero) of dc3d.f:65-87;
//   - the DCCON2 call keeps the reference's index pairing (KXI(K), KET(J)).
// Only the nine derivative outputs are formed (the displacement itself is not
// needed for stress), and the corner geometry, logs and arctangents are shared
// by the two slip components instead of being recomputed per DC3D call.
//
// R32 = true reproduces the reference's REAL*4 interface (okada92.f90:121-160):
// the caller rounds the inputs to binary32, the two REAL*4 differences are taken
// in binary32, the REAL*4 EPS is used in DC3D, and the outputs are rounded to
// binary32.
#pragma once
#include <cuda_runtime.h>

namespace ucg {

struct OkDip {           // DCCON0 (dc3d.f:509-544)
    double sd, cd, sdsd, cdcd, sdcd;
};

struct OkMed {           // medium constants alp1..alp5
    double alp1, alp2, alp3, alp4, alp5;
};

struct OkCorner {        // DCCON2 outputs (dc3d.f:596-665)
    double xi, et, q;
    double xi2, et2, q2, r, r2, r3, r5, y, d, x11, y11, x32, y32;
    double ey, ez, fy, fz, gy, gz, hy, hz;
};

__host__ __device__ inline OkDip ok_dip(double dip_deg)
{
    const double p18 = 6.283185307179586 / 360.0;
    OkDip c;
    c.sd = sin(dip_deg * p18);
    c.cd = cos(dip_deg * p18);
    if (fabs(c.cd) < 1.0e-6) {
        c.cd = 0.0;
        if (c.sd > 0.0) c.sd = 1.0;
        if (c.sd < 0.0) c.sd = -1.0;
    }
    c.sdsd = c.sd * c.sd;
    c.cdcd = c.cd * c.cd;
    c.sdcd = c.sd * c.cd;
    return c;
}

__host__ __device__ inline OkMed ok_med(double alpha)
{
    OkMed m;
    m.alp1 = (1.0 - alpha) / 2.0;
    m.alp2 = alpha / 2.0;
    m.alp3 = (1.0 - alpha) / alpha;
    m.alp4 = 1.0 - alpha;
    m.alp5 = alpha;
    return m;
}

// Corner geometry.  xi, et, q are snapped in place (the reference passes them
// by reference).  Returns false when r == 0 (unreachable after edge rejection).
__device__ inline bool ok_corner(double &xi, double &et, double &q, const OkDip &dp, int kxi,
                                 int ket, OkCorner &c)
{
    const double eps = 1.0e-6;
    if (fabs(xi) < eps) xi = 0.0;
    if (fabs(et) < eps) et = 0.0;
    if (fabs(q) < eps) q = 0.0;
    c.xi = xi; c.et = et; c.q = q;
    c.xi2 = xi * xi;
    c.et2 = et * et;
    c.q2 = q * q;
    c.r2 = c.xi2 + c.et2 + c.q2;
    c.r = sqrt(c.r2);
    if (c.r == 0.0) return false;
    c.r3 = c.r * c.r2;
    c.r5 = c.r3 * c.r2;
    c.y = et * dp.cd + q * dp.sd;
    c.d = et * dp.sd - q * dp.cd;
    // tt, alx and ale enter only the displacement entries of parts A/B/C, which the
    // gradient does not use; the flags still select the x11/x32, y11/y32 forms.
    if (kxi == 1) {
        c.x11 = 0.0;
        c.x32 = 0.0;
    } else {
        double rxi = c.r + xi;
        c.x11 = 1.0 / (c.r * rxi);
        c.x32 = (c.r + rxi) * c.x11 * c.x11 / c.r;
    }
    if (ket == 1) {
        c.y11 = 0.0;
        c.y32 = 0.0;
    } else {
        double ret = c.r + et;
        c.y11 = 1.0 / (c.r * ret);
        c.y32 = (c.r + ret) * c.y11 * c.y11 / c.r;
    }
    c.ey = dp.sd / c.r - c.y * q / c.r3;
    c.ez = dp.cd / c.r + c.d * q / c.r3;
    c.fy = c.d / c.r3 + c.xi2 * c.y32 * dp.sd;
    c.fz = c.y / c.r3 + c.xi2 * c.y32 * dp.cd;
    c.gy = 2.0 * c.x11 * dp.sd - c.y * q * c.x32;
    c.gz = 2.0 * c.x11 * dp.cd + c.d * q * c.x32;
    c.hy = c.d * q * c.x32 + xi * q * c.y32 * dp.sd;
    c.hz = c.y * q * c.x32 + xi * q * c.y32 * dp.cd;
    return true;
}

// Gradient entries g[0..8] correspond to DC3D's U(4..12):
// uxx, uyx, uzx, uxy, uyy, uzy, uxz, uyz, uzz.
#define OK_K (1.0 / 6.283185307179586)

// Part A (dc3d.f:200-282), strike (s) and dip (d) slip, gradient entries only.
__device__ inline void ok_part_a(const OkCorner &c, const OkDip &dp, const OkMed &m, double s[9],
                                 double d[9])
{
    const double xi = c.xi, et = c.et, q = c.q, R = c.r, R3 = c.r3;
    const double xy = xi * c.y11, qx = q * c.x11, qy = q * c.y11;
    (void)qx;
    s[0] = OK_K * (-m.alp1 * qy - m.alp2 * c.xi2 * q * c.y32);
    s[1] = OK_K * (-m.alp2 * xi * q / R3);
    s[2] = OK_K * (m.alp1 * xy + m.alp2 * xi * c.q2 * c.y32);
    s[3] = OK_K * (m.alp1 * xy * dp.sd + m.alp2 * xi * c.fy + c.d / 2.0 * c.x11);
    s[4] = OK_K * (m.alp2 * c.ey);
    s[5] = OK_K * (m.alp1 * (dp.cd / R + qy * dp.sd) - m.alp2 * q * c.fy);
    s[6] = OK_K * (m.alp1 * xy * dp.cd + m.alp2 * xi * c.fz + c.y / 2.0 * c.x11);
    s[7] = OK_K * (m.alp2 * c.ez);
    s[8] = OK_K * (-m.alp1 * (dp.sd / R - qy * dp.cd) - m.alp2 * q * c.fz);

    d[0] = OK_K * (-m.alp2 * xi * q / R3);
    d[1] = OK_K * (-qy / 2.0 - m.alp2 * et * q / R3);
    d[2] = OK_K * (m.alp1 / R + m.alp2 * c.q2 / R3);
    d[3] = OK_K * (m.alp2 * c.ey);
    d[4] = OK_K * (m.alp1 * c.d * c.x11 + xy / 2.0 * dp.sd + m.alp2 * et * c.gy);
    d[5] = OK_K * (m.alp1 * c.y * c.x11 - m.alp2 * q * c.gy);
    d[6] = OK_K * (m.alp2 * c.ez);
    d[7] = OK_K * (m.alp1 * c.y * c.x11 + xy / 2.0 * dp.cd + m.alp2 * et * c.gz);
    d[8] = OK_K * (-m.alp1 * c.d * c.x11 - m.alp2 * q * c.gz);
}

// Part B (dc3d.f:284-400).
__device__ inline void ok_part_b(const OkCorner &c, const OkDip &dp, const OkMed &m, double s[9],
                                 double d[9])
{
    const double xi = c.xi, et = c.et, q = c.q, R = c.r, R3 = c.r3, Y = c.y, D = c.d;
    const double rd = R + D;
    const double d11 = 1.0 / (R * rd);
    const double aj2 = xi * Y / rd * d11;
    const double aj5 = -(D + Y * Y / rd) * d11;
    // ai1..ai4 enter only the displacement entries and are not formed.
    double ak1, ak3, aj3, aj6;
    if (dp.cd != 0.0) {
        ak1 = xi * (d11 - c.y11 * dp.sd) / dp.cd;
        ak3 = (q * c.y11 - Y * d11) / dp.cd;
        aj3 = (ak1 - aj2 * dp.sd) / dp.cd;
        aj6 = (ak3 - aj5 * dp.sd) / dp.cd;
    } else {
        double rd2 = rd * rd;
        ak1 = xi * q / rd * d11;
        ak3 = dp.sd / rd * (c.xi2 * d11 - 1.0);
        aj3 = -xi / rd2 * (c.q2 * d11 - 1.0 / 2.0);
        aj6 = -Y / rd2 * (c.xi2 * d11 - 1.0 / 2.0);
    }
    const double xy = xi * c.y11;
    const double ak2 = 1.0 / R + ak3 * dp.sd;
    const double ak4 = xy * dp.cd - ak1 * dp.sd;
    const double aj1 = aj5 * dp.cd - aj6 * dp.sd;
    const double aj4 = -xy - aj2 * dp.cd + aj3 * dp.sd;
    const double qy = q * c.y11;
    const double a3 = m.alp3;

    s[0] = OK_K * (c.xi2 * q * c.y32 - a3 * aj1 * dp.sd);
    s[1] = OK_K * (xi * q / R3 - a3 * aj2 * dp.sd);
    s[2] = OK_K * (-xi * c.q2 * c.y32 - a3 * aj3 * dp.sd);
    s[3] = OK_K * (-xi * c.fy - D * c.x11 + a3 * (xy + aj4) * dp.sd);
    s[4] = OK_K * (-c.ey + a3 * (1.0 / R + aj5) * dp.sd);
    s[5] = OK_K * (q * c.fy - a3 * (qy - aj6) * dp.sd);
    s[6] = OK_K * (-xi * c.fz - Y * c.x11 + a3 * ak1 * dp.sd);
    s[7] = OK_K * (-c.ez + a3 * Y * d11 * dp.sd);
    s[8] = OK_K * (q * c.fz + a3 * ak2 * dp.sd);

    d[0] = OK_K * (xi * q / R3 + a3 * aj4 * dp.sdcd);
    d[1] = OK_K * (et * q / R3 + qy + a3 * aj5 * dp.sdcd);
    d[2] = OK_K * (-c.q2 / R3 + a3 * aj6 * dp.sdcd);
    d[3] = OK_K * (-c.ey + a3 * aj1 * dp.sdcd);
    d[4] = OK_K * (-et * c.gy - xy * dp.sd + a3 * aj2 * dp.sdcd);
    d[5] = OK_K * (q * c.gy + a3 * aj3 * dp.sdcd);
    d[6] = OK_K * (-c.ez - a3 * ak3 * dp.sdcd);
    d[7] = OK_K * (-et * c.gz - xy * dp.cd - a3 * xi * d11 * dp.sdcd);
    d[8] = OK_K * (q * c.gz - a3 * ak4 * dp.sdcd);
}

// Part C (dc3d.f:402-507).  Also returns the displacement entries 1..3 of part C
// (c0 for strike, e0 for dip), which the image sum adds to the z-derivatives.
__device__ inline void ok_part_c(const OkCorner &c, const OkDip &dp, const OkMed &m, double Z,
                                 double s[9], double d[9], double cs[3], double cdp[3])
{
    const double xi = c.xi, et = c.et, q = c.q, R = c.r, R2 = c.r2, R3 = c.r3, R5 = c.r5;
    const double Y = c.y, D = c.d, sd = dp.sd, cd = dp.cd;
    const double a4 = m.alp4, a5 = m.alp5;
    const double C = D + Z;
    const double x53 = (8.0 * R2 + 9.0 * R * xi + 3.0 * c.xi2) * c.x11 * c.x11 * c.x11 / R2;
    const double y53 = (8.0 * R2 + 9.0 * R * et + 3.0 * c.et2) * c.y11 * c.y11 * c.y11 / R2;
    const double h = q * cd - Z;
    const double z32 = sd / R3 - h * c.y32;
    const double z53 = 3.0 * sd / R5 - h * y53;
    const double y0 = c.y11 - c.xi2 * c.y32;
    const double z0 = z32 - c.xi2 * z53;
    const double ppy = cd / R3 + q * c.y32 * sd;
    const double ppz = sd / R3 - q * c.y32 * cd;
    const double qq = Z * c.y32 + z32 + z0;
    const double qqy = 3.0 * C * D / R5 - qq * sd;
    const double qqz = 3.0 * C * Y / R5 - qq * cd + q * c.y32;
    const double xy = xi * c.y11;
    const double qy = q * c.y11;
    const double qr = 3.0 * q / R5;
    const double cdr = (C + D) / R3;
    const double yy0 = Y / R3 - y0 * cd;
    const double X11 = c.x11, X32 = c.x32, Y11 = c.y11, Y32 = c.y32, Q2 = c.q2;

    cs[0] = OK_K * (a4 * xy * cd - a5 * xi * q * z32);
    cs[1] = OK_K * (a4 * (cd / R + 2.0 * qy * sd) - a5 * C * q / R3);
    cs[2] = OK_K * (a4 * qy * cd - a5 * (C * et / R3 - Z * Y11 + c.xi2 * z32));
    s[0] = OK_K * (a4 * y0 * cd - a5 * q * z0);
    s[1] = OK_K * (-a4 * xi * (cd / R3 + 2.0 * q * Y32 * sd) + a5 * C * xi * qr);
    s[2] = OK_K * (-a4 * xi * q * Y32 * cd + a5 * xi * (3.0 * C * et / R5 - qq));
    s[3] = OK_K * (-a4 * xi * ppy * cd - a5 * xi * qqy);
    s[4] = OK_K * (a4 * 2.0 * (D / R3 - y0 * sd) * sd - Y / R3 * cd
                   - a5 * (cdr * sd - et / R3 - C * Y * qr));
    s[5] = OK_K * (-a4 * q / R3 + yy0 * sd + a5 * (cdr * cd + C * D * qr - (y0 * cd + q * z0) * sd));
    s[6] = OK_K * (a4 * xi * ppz * cd - a5 * xi * qqz);
    s[7] = OK_K * (a4 * 2.0 * (Y / R3 - y0 * cd) * sd + D / R3 * cd - a5 * (cdr * cd + C * D * qr));
    s[8] = OK_K * (yy0 * cd - a5 * (cdr * sd - C * Y * qr - y0 * dp.sdsd + q * z0 * cd));

    cdp[0] = OK_K * (a4 * cd / R - qy * sd - a5 * C * q / R3);
    cdp[1] = OK_K * (a4 * Y * X11 - a5 * C * et * q * X32);
    cdp[2] = OK_K * (-D * X11 - xy * sd - a5 * C * (X11 - Q2 * X32));
    d[0] = OK_K * (-a4 * xi / R3 * cd + a5 * C * xi * qr + xi * q * Y32 * sd);
    d[1] = OK_K * (-a4 * Y / R3 + a5 * C * et * qr);
    d[2] = OK_K * (D / R3 - y0 * sd + a5 * C / R3 * (1.0 - 3.0 * Q2 / R2));
    d[3] = OK_K * (-a4 * et / R3 + y0 * dp.sdsd - a5 * (cdr * sd - C * Y * qr));
    d[4] = OK_K * (a4 * (X11 - Y * Y * X32) - a5 * C * ((D + 2.0 * q * cd) * X32 - Y * et * q * x53));
    d[5] = OK_K * (xi * ppy * sd + Y * D * X32 + a5 * C * ((Y + 2.0 * q * sd) * X32 - Y * Q2 * x53));
    d[6] = OK_K * (-q / R3 + y0 * dp.sdcd - a5 * (cdr * cd + C * D * qr));
    d[7] = OK_K * (a4 * Y * D * X32 - a5 * C * ((Y - 2.0 * q * sd) * X32 + D * et * q * x53));
    d[8] = OK_K * (-xi * ppz * sd + X11 - D * D * X32 - a5 * C * ((D - 2.0 * q * cd) * X32 - D * Q2 * x53));
}

// Part C's displacement entries are the same statements as DU(1..3) of UC.

// Singular-edge rejection and negative-extension flags (dc3d.f:70-87).
__device__ inline bool ok_edges(const double xi[2], const double et[2], double q, double eps,
                                int kxi[2], int ket[2])
{
    if (q == 0.0 && ((xi[0] * xi[1] <= 0.0 && et[0] * et[1] == 0.0) ||
                     (et[0] * et[1] <= 0.0 && xi[0] * xi[1] == 0.0)))
        return true;
    double r12 = sqrt(xi[0] * xi[0] + et[1] * et[1] + q * q);
    double r21 = sqrt(xi[1] * xi[1] + et[0] * et[0] + q * q);
    double r22 = sqrt(xi[1] * xi[1] + et[1] * et[1] + q * q);
    kxi[0] = (xi[0] < 0.0 && r21 + xi[1] < eps);
    kxi[1] = (xi[0] < 0.0 && r22 + xi[1] < eps);
    ket[0] = (et[0] < 0.0 && r12 + et[1] < eps);
    ket[1] = (et[0] < 0.0 && r22 + et[1] < eps);
    return false;
}

// Displacement gradient for unit strike slip (gs) and unit dip slip (gd) of a
// source at (depth, dip) spanning x in [0, al2] and eta in [aw1, 0], observed at
// (x, y, z) in the DC3D frame (x along strike, z up).  Returns false on the
// singular edge (gradients zero).
template <bool R32>
__device__ inline bool ok_dc3d_grad(const OkMed &m, const OkDip &dp, double x, double y, double z,
                                    double depth, double al2, double aw1, double gs[9],
                                    double gd[9])
{
    const double eps = R32 ? (double)1.0e-6f : 1.0e-6;
#pragma unroll
    for (int i = 0; i < 9; i++) { gs[i] = 0.0; gd[i] = 0.0; }
    double xi[2], et[2];
    if (R32) {
        xi[0] = (double)((float)x - 0.0f);
        xi[1] = (double)((float)x - (float)al2);
    } else {
        xi[0] = x;
        xi[1] = x - al2;
    }
    if (fabs(xi[0]) < eps) xi[0] = 0.0;
    if (fabs(xi[1]) < eps) xi[1] = 0.0;
    int kxi[2], ket[2];
    OkCorner c;
    double as[9], ad[9];

    // real source
    {
        double D = R32 ? (double)((float)depth + (float)z) : depth + z;
        double p = y * dp.cd + D * dp.sd;
        double q = y * dp.sd - D * dp.cd;
        et[0] = p - aw1;
        et[1] = p;
        if (fabs(q) < eps) q = 0.0;
        if (fabs(et[0]) < eps) et[0] = 0.0;
        if (fabs(et[1]) < eps) et[1] = 0.0;
        if (ok_edges(xi, et, q, eps, kxi, ket)) goto singular;
#pragma unroll 1
        for (int kk = 0; kk < 4; kk++) {
            const int k = kk >> 1, j = kk & 1;
            ok_corner(xi[j], et[k], q, dp, kxi[k], ket[j], c);
            ok_part_a(c, dp, m, as, ad);
            const double sg = (j + k != 1) ? 1.0 : -1.0;
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const double *a = t ? ad : as;
                double *g = t ? gd : gs;
                double du[9];
                // rows 1..3 of DC3D's 4x3 block rotation; the z-derivative row is negated
                du[0] = -a[0];
                du[1] = -a[1] * dp.cd + a[2] * dp.sd;
                du[2] = -a[1] * dp.sd - a[2] * dp.cd;
                du[3] = -a[3];
                du[4] = -a[4] * dp.cd + a[5] * dp.sd;
                du[5] = -a[4] * dp.sd - a[5] * dp.cd;
                du[6] = -(-a[6]);
                du[7] = -(-a[7] * dp.cd + a[8] * dp.sd);
                du[8] = -(-a[7] * dp.sd - a[8] * dp.cd);
#pragma unroll
                for (int i = 0; i < 9; i++) g[i] = (sg > 0.0) ? g[i] + du[i] : g[i] - du[i];
            }
        }
    }
    // image source
    {
        double D = R32 ? (double)((float)depth - (float)z) : depth - z;
        double p = y * dp.cd + D * dp.sd;
        double q = y * dp.sd - D * dp.cd;
        et[0] = p - aw1;
        et[1] = p;
        if (fabs(q) < eps) q = 0.0;
        if (fabs(et[0]) < eps) et[0] = 0.0;
        if (fabs(et[1]) < eps) et[1] = 0.0;
        if (ok_edges(xi, et, q, eps, kxi, ket)) goto singular;
#pragma unroll 1
        for (int kk = 0; kk < 4; kk++) {
            const int k = kk >> 1, j = kk & 1;
            ok_corner(xi[j], et[k], q, dp, kxi[k], ket[j], c);
            double bs[9], bd[9], cs9[9], cd9[9], c0s[3], c0d[3];
            ok_part_a(c, dp, m, as, ad);
            ok_part_b(c, dp, m, bs, bd);
            ok_part_c(c, dp, m, z, cs9, cd9, c0s, c0d);
            const double sg = (j + k != 1) ? 1.0 : -1.0;
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const double *a = t ? ad : as;
                const double *b = t ? bd : bs;
                const double *cc = t ? cd9 : cs9;
                const double *c0 = t ? c0d : c0s;
                double *g = t ? gd : gs;
                double du[9];
#pragma unroll
                for (int r = 0; r < 3; r++) {
                    const int i = 3 * r;
                    du[i] = a[i] + b[i] + z * cc[i];
                    du[i + 1] = (a[i + 1] + b[i + 1] + z * cc[i + 1]) * dp.cd
                              - (a[i + 2] + b[i + 2] + z * cc[i + 2]) * dp.sd;
                    du[i + 2] = (a[i + 1] + b[i + 1] - z * cc[i + 1]) * dp.sd
                              + (a[i + 2] + b[i + 2] - z * cc[i + 2]) * dp.cd;
                }
                du[6] = du[6] + c0[0];
                du[7] = du[7] + c0[1] * dp.cd - c0[2] * dp.sd;
                du[8] = du[8] - c0[1] * dp.sd - c0[2] * dp.cd;
#pragma unroll
                for (int i = 0; i < 9; i++) g[i] = (sg > 0.0) ? g[i] + du[i] : g[i] - du[i];
            }
        }
    }
    if (R32) {
#pragma unroll
        for (int i = 0; i < 9; i++) {
            gs[i] = (double)__double2float_rn(gs[i]);
            gd[i] = (double)__double2float_rn(gd[i]);
        }
    }
    return true;
singular:
#pragma unroll
    for (int i = 0; i < 9; i++) { gs[i] = 0.0; gd[i] = 0.0; }
    return false;
}

// ---- displacement (observation points) ------------------------------------------

// The displacement entries DU(1..3) of parts A/B/C need three more corner
// quantities of DCCON2 (dc3d.f:596-665): TT, ALX, ALE.
struct OkLogs {
    double tt, alx, ale;
};

__device__ inline OkLogs ok_logs(const OkCorner &c, int kxi, int ket)
{
    OkLogs l;
    l.tt = (c.q == 0.0) ? 0.0 : atan(c.xi * c.et / (c.q * c.r));
    l.alx = (kxi == 1) ? -log(c.r - c.xi) : log(c.r + c.xi);
    l.ale = (ket == 1) ? -log(c.r - c.et) : log(c.r + c.et);
    return l;
}

// Part A (dc3d.f:200-282) DU(1..3), strike (s) and dip (d) slip.
__device__ inline void ok_part_a_disp(const OkCorner &c, const OkLogs &l, const OkMed &m, double s[3],
                                      double d[3])
{
    const double qx = c.q * c.x11, qy = c.q * c.y11;
    s[0] = OK_K * (l.tt / 2.0 + m.alp2 * c.xi * qy);
    s[1] = OK_K * (m.alp2 * c.q / c.r);
    s[2] = OK_K * (m.alp1 * l.ale - m.alp2 * c.q * qy);
    d[0] = OK_K * (m.alp2 * c.q / c.r);
    d[1] = OK_K * (l.tt / 2.0 + m.alp2 * c.et * qx);
    d[2] = OK_K * (m.alp1 * l.alx - m.alp2 * c.q * qx);
}

// Part B (dc3d.f:284-400) DU(1..3), with the I1..I4 terms the gradient does not use.
__device__ inline void ok_part_b_disp(const OkCorner &c, const OkLogs &l, const OkDip &dp, const OkMed &m,
                                      double s[3], double d[3])
{
    const double xi = c.xi, et = c.et, q = c.q, R = c.r, Y = c.y;
    const double rd = R + c.d;
    double ai3, ai4;
    if (dp.cd != 0.0) {
        if (xi == 0.0) {
            ai4 = 0.0;
        } else {
            const double x = sqrt(c.xi2 + c.q2);
            ai4 = 1.0 / dp.cdcd * (xi / rd * dp.sdcd +
                  2.0 * atan((et * (x + q * dp.cd) + x * (R + x) * dp.sd) / (xi * (R + x) * dp.cd)));
        }
        ai3 = (Y * dp.cd / rd - l.ale + dp.sd * log(rd)) / dp.cdcd;
    } else {
        const double rd2 = rd * rd;
        ai3 = (et / rd + Y * q / rd2 - l.ale) / 2.0;
        ai4 = xi * Y / rd2 / 2.0;
    }
    const double ai1 = -xi / rd * dp.cd - ai4 * dp.sd;
    const double ai2 = log(rd) + ai3 * dp.sd;
    const double qx = q * c.x11, qy = q * c.y11, a3 = m.alp3;
    s[0] = OK_K * (-xi * qy - l.tt - a3 * ai1 * dp.sd);
    s[1] = OK_K * (-q / R + a3 * Y / rd * dp.sd);
    s[2] = OK_K * (q * qy - a3 * ai2 * dp.sd);
    d[0] = OK_K * (-q / R + a3 * ai3 * dp.sdcd);
    d[1] = OK_K * (-et * qx - l.tt - a3 * xi / rd * dp.sdcd);
    d[2] = OK_K * (q * qx + a3 * ai4 * dp.sdcd);
}

// Displacement (ux, uy, uz in the DC3D frame) for unit strike slip (us) and
// unit dip slip (ud): DC3D's U(1..3) (dc3d.f:1-198) with the same corner
// loop, snapping, edge rejection and REAL*4 handling as ok_dc3d_grad.
template <bool R32>
__device__ inline bool ok_dc3d_disp(const OkMed &m, const OkDip &dp, double x, double y, double z,
                                    double depth, double al2, double aw1, double us[3], double ud[3])
{
    const double eps = R32 ? (double)1.0e-6f : 1.0e-6;
    for (int i = 0; i < 3; i++) { us[i] = 0.0; ud[i] = 0.0; }
    double xi[2], et[2];
    if (R32) {
        xi[0] = (double)((float)x - 0.0f);
        xi[1] = (double)((float)x - (float)al2);
    } else {
        xi[0] = x;
        xi[1] = x - al2;
    }
    if (fabs(xi[0]) < eps) xi[0] = 0.0;
    if (fabs(xi[1]) < eps) xi[1] = 0.0;
    int kxi[2], ket[2];
    OkCorner c;
#pragma unroll 1
    for (int img = 0; img < 2; img++) {
        const double D = R32 ? (double)(img ? (float)depth - (float)z : (float)depth + (float)z)
                             : (img ? depth - z : depth + z);
        const double p = y * dp.cd + D * dp.sd;
        double q = y * dp.sd - D * dp.cd;
        et[0] = p - aw1;
        et[1] = p;
        if (fabs(q) < eps) q = 0.0;
        if (fabs(et[0]) < eps) et[0] = 0.0;
        if (fabs(et[1]) < eps) et[1] = 0.0;
        if (ok_edges(xi, et, q, eps, kxi, ket)) {
            for (int i = 0; i < 3; i++) { us[i] = 0.0; ud[i] = 0.0; }
            return false;
        }
#pragma unroll 1
        for (int kk = 0; kk < 4; kk++) {
            const int k = kk >> 1, j = kk & 1;
            ok_corner(xi[j], et[k], q, dp, kxi[k], ket[j], c);
            const OkLogs l = ok_logs(c, kxi[k], ket[j]);
            double as[3], ad[3];
            ok_part_a_disp(c, l, m, as, ad);
            const double sg = (j + k != 1) ? 1.0 : -1.0;
            if (!img) {
#pragma unroll
                for (int t = 0; t < 2; t++) {
                    const double *a = t ? ad : as;
                    double *u = t ? ud : us;
                    const double du0 = -a[0];
                    const double du1 = -a[1] * dp.cd + a[2] * dp.sd;
                    const double du2 = -a[1] * dp.sd - a[2] * dp.cd;
                    u[0] = (sg > 0.0) ? u[0] + du0 : u[0] - du0;
                    u[1] = (sg > 0.0) ? u[1] + du1 : u[1] - du1;
                    u[2] = (sg > 0.0) ? u[2] + du2 : u[2] - du2;
                }
            } else {
                double bs[3], bd[3], cs9[9], cd9[9], c0s[3], c0d[3];
                ok_part_b_disp(c, l, dp, m, bs, bd);
                ok_part_c(c, dp, m, z, cs9, cd9, c0s, c0d);
#pragma unroll
                for (int t = 0; t < 2; t++) {
                    const double *a = t ? ad : as;
                    const double *b = t ? bd : bs;
                    const double *cc = t ? c0d : c0s;
                    double *u = t ? ud : us;
                    const double du0 = a[0] + b[0] + z * cc[0];
                    const double du1 = (a[1] + b[1] + z * cc[1]) * dp.cd - (a[2] + b[2] + z * cc[2]) * dp.sd;
                    const double du2 = (a[1] + b[1] - z * cc[1]) * dp.sd + (a[2] + b[2] - z * cc[2]) * dp.cd;
                    u[0] = (sg > 0.0) ? u[0] + du0 : u[0] - du0;
                    u[1] = (sg > 0.0) ? u[1] + du1 : u[1] - du1;
                    u[2] = (sg > 0.0) ? u[2] + du2 : u[2] - du2;
                }
            }
        }
    }
    if (R32) {
        for (int i = 0; i < 3; i++) {
            us[i] = (double)__double2float_rn(us[i]);
            ud[i] = (double)__double2float_rn(ud[i]);
        }
    }
    return true;
}

#undef OK_K

}  // namespace ucg
