// Nikkhoo & Walter (2015) triangular dislocation (TD) in an elastic half-space,
// device side.  Stress at a receiver due to unit strike slip and unit dip slip
// of one TD, both at once.
//
// The reference evaluates TD strain with straininhalfspace_
// (fortran/3d/src/StrainInHalfSpace.c:42-177), whose expressions are the
// analytic derivatives of the TD displacement field of the same paper
// (fortran/3d/src/DispInHalfSpace.c:153-617).  Here the displacement field is
// evaluated on dual numbers seeded with the observation point, which gives the
// exact displacement gradient, and the three parts are assembled as
// straininhalfspace_ does: main TD + image TD (vertices mirrored in z) +
// harmonic free-surface correction; the image's yz and zz stresses change sign
// when all vertices lie at z = 0 (StrainInHalfSpace.c:162-165); configuration I
// of the free-surface angular-dislocation pairs is taken in the mirrored frame
// (StrainInHalfSpace.c:644-652).  Because only the gradient is formed, the
// logarithms and arctangents of the displacement field contribute through their
// derivatives alone and are never evaluated.
//
// Per-source geometry (frames, vertex coordinates in the TD frame, angular-
// dislocation angles, free-surface side frames, slip vectors) is computed once
// per triangle by nw_prepare and read by every pair thread.
#pragma once
#include <cuda_runtime.h>
#include "dual.cuh"

namespace ucg {

// layout of the per-triangle record (doubles)
enum : int {
    // one TD (main or image), 28 doubles
    TD_P2 = 0,          // 3: origin of the TD frame
    TD_N = 3,           // 3: normal row of the frame
    TD_S = 6,           // 3: strike row
    TD_D = 9,           // 3: dip row
    TD_P1 = 12,         // 2: (y, z) of vertex 1 in the TD frame
    TD_P3 = 14,         // 2: (y, z) of vertex 3
    TD_E13 = 16,        // 2: (y, z) of unit side vectors
    TD_E12 = 18,
    TD_E23 = 20,
    TD_CS = 22,         // 6: cos, sin of (-pi + angle) for the three corners
    TD_SIZE = 28,
    // one free-surface side, 27 doubles
    FS_PA = 0,          // 3
    FS_E1 = 3,          // 2: ey1 (x, y)
    FS_E2 = 5,          // 2: ey2 (x, y)
    FS_SA = 7,          // 3: side vector in the angular-dislocation frame
    FS_I = 10,          // 4: sin, cos, cot, cot(half) for configuration I (pi - beta)
    FS_II = 14,         // 4: same for configuration II (beta)
    FS_AA = 18,         // 1: -PA[2]
    FS_AB = 19,         // 1: -PB[2]
    FS_DEG = 20,        // 1: 1 when the side is vertical (pair contributes zero)
    FS_B = 21,          // 6: slip (b1, b2, b3) in the side frame for strike, dip modes
    FS_SIZE = 27,
    // record
    NW_MAIN = 0,
    NW_IMG = TD_SIZE,
    NW_FS = 2 * TD_SIZE,
    NW_SURF = 2 * TD_SIZE + 3 * FS_SIZE,   // 1 when all vertices at z = 0
    NW_SIZE = 2 * TD_SIZE + 3 * FS_SIZE + 1
};

struct NwConst {
    double nu, mu, lambda;
};

// ---- per-triangle preparation ------------------------------------------------

__host__ __device__ inline void nw_frame(const double P1[3], const double P2[3], const double P3[3],
                                         bool image_fix, double vn[3], double vs[3], double vd[3])
{
    double t1[3] = {P2[0] - P1[0], P2[1] - P1[1], P2[2] - P1[2]};
    double t2[3] = {P3[0] - P1[0], P3[1] - P1[1], P3[2] - P1[2]};
    vn[0] = t1[1] * t2[2] - t1[2] * t2[1];
    vn[1] = t1[2] * t2[0] - t1[0] * t2[2];
    vn[2] = t1[0] * t2[1] - t1[1] * t2[0];
    double nn = sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
    for (int k = 0; k < 3; k++) vn[k] /= nn;
    vs[0] = -vn[1];
    vs[1] = vn[0];
    vs[2] = 0.0;
    double ns = sqrt(vs[0] * vs[0] + vs[1] * vs[1]);
    if (ns == 0.0) {   // horizontal TD
        vs[0] = 0.0;
        vs[1] = vn[2];
        if (image_fix && P1[2] > 0.0) vs[1] = -vs[1];
        ns = fabs(vs[1]);
    }
    for (int k = 0; k < 3; k++) vs[k] /= ns;
    vd[0] = vn[1] * vs[2] - vn[2] * vs[1];
    vd[1] = vn[2] * vs[0] - vn[0] * vs[2];
    vd[2] = vn[0] * vs[1] - vn[1] * vs[0];
    double nd = sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
    for (int k = 0; k < 3; k++) vd[k] /= nd;
}

__host__ __device__ inline void nw_prep_td(const double P1[3], const double P2[3], const double P3[3],
                                           double *r)
{
    double vn[3], vs[3], vd[3];
    nw_frame(P1, P2, P3, true, vn, vs, vd);
    double q1[3] = {P1[0] - P2[0], P1[1] - P2[1], P1[2] - P2[2]};
    double q3[3] = {P3[0] - P2[0], P3[1] - P2[1], P3[2] - P2[2]};
    double p1[3], p3[3];
    const double *rows[3] = {vn, vs, vd};
    for (int k = 0; k < 3; k++) {
        p1[k] = rows[k][0] * q1[0] + rows[k][1] * q1[1] + rows[k][2] * q1[2];
        p3[k] = rows[k][0] * q3[0] + rows[k][1] * q3[1] + rows[k][2] * q3[2];
    }
    double e12[3], e13[3], e23[3], n;
    n = sqrt(p1[0] * p1[0] + p1[1] * p1[1] + p1[2] * p1[2]);
    for (int k = 0; k < 3; k++) e12[k] = (0.0 - p1[k]) / n;
    n = sqrt((p3[0] - p1[0]) * (p3[0] - p1[0]) + (p3[1] - p1[1]) * (p3[1] - p1[1]) + (p3[2] - p1[2]) * (p3[2] - p1[2]));
    for (int k = 0; k < 3; k++) e13[k] = (p3[k] - p1[k]) / n;
    n = sqrt(p3[0] * p3[0] + p3[1] * p3[1] + p3[2] * p3[2]);
    for (int k = 0; k < 3; k++) e23[k] = (p3[k] - 0.0) / n;
    double A = acos(e12[0] * e13[0] + e12[1] * e13[1] + e12[2] * e13[2]);
    double B = acos(-e12[0] * e23[0] - e12[1] * e23[1] - e12[2] * e23[2]);
    double C = acos(e23[0] * e13[0] + e23[1] * e13[1] + e23[2] * e13[2]);
    for (int k = 0; k < 3; k++) {
        r[TD_P2 + k] = P2[k];
        r[TD_N + k] = vn[k];
        r[TD_S + k] = vs[k];
        r[TD_D + k] = vd[k];
    }
    r[TD_P1] = p1[1]; r[TD_P1 + 1] = p1[2];
    r[TD_P3] = p3[1]; r[TD_P3 + 1] = p3[2];
    r[TD_E13] = e13[1]; r[TD_E13 + 1] = e13[2];
    r[TD_E12] = e12[1]; r[TD_E12 + 1] = e12[2];
    r[TD_E23] = e23[1]; r[TD_E23 + 1] = e23[2];
    const double PI = 3.141592653589793;
    r[TD_CS + 0] = cos(-PI + A); r[TD_CS + 1] = sin(-PI + A);
    r[TD_CS + 2] = cos(-PI + B); r[TD_CS + 3] = sin(-PI + B);
    r[TD_CS + 4] = cos(-PI + C); r[TD_CS + 5] = sin(-PI + C);
}

// free-surface side PA -> PB; bS, bD: EFCS slip vectors of the two modes
__host__ __device__ inline void nw_prep_fs(const double PA[3], const double PB[3], const double bS[3],
                                           const double bD[3], double *r)
{
    const double PI = 3.141592653589793;
    const double EPS = 2.220446049250313e-16;
    double sv[3] = {PB[0] - PA[0], PB[1] - PA[1], PB[2] - PA[2]};
    double l = sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    double beta = acos(-sv[2] / l);
    for (int k = 0; k < FS_SIZE; k++) r[k] = 0.0;
    r[FS_AA] = -PA[2];
    r[FS_AB] = -PB[2];
    for (int k = 0; k < 3; k++) r[FS_PA + k] = PA[k];
    if (fabs(beta) < EPS || fabs(PI - beta) < EPS) {
        r[FS_DEG] = 1.0;
        return;
    }
    double n1 = sqrt(sv[0] * sv[0] + sv[1] * sv[1]);
    double e1x = sv[0] / n1, e1y = sv[1] / n1;
    // ey3 = (0,0,-1), ey2 = ey3 x ey1 = (e1y, -e1x, 0), normalized
    double e2x = e1y, e2y = -e1x;
    double n2 = sqrt(e2x * e2x + e2y * e2y);
    e2x /= n2; e2y /= n2;
    r[FS_E1] = e1x; r[FS_E1 + 1] = e1y;
    r[FS_E2] = e2x; r[FS_E2 + 1] = e2y;
    // A = [[e1x, e2x, 0], [e1y, e2y, 0], [0, 0, -1]] (symmetric)
    r[FS_SA + 0] = e1x * sv[0] + e2x * sv[1];
    r[FS_SA + 1] = e1y * sv[0] + e2y * sv[1];
    r[FS_SA + 2] = -sv[2];
    double bI = PI - beta;
    r[FS_I + 0] = sin(bI); r[FS_I + 1] = cos(bI);
    r[FS_I + 2] = cos(bI) / sin(bI);
    r[FS_I + 3] = cos(bI / 2.0) / sin(bI / 2.0);
    r[FS_II + 0] = sin(beta); r[FS_II + 1] = cos(beta);
    r[FS_II + 2] = cos(beta) / sin(beta);
    r[FS_II + 3] = cos(beta / 2.0) / sin(beta / 2.0);
    const double *bb[2] = {bS, bD};
    for (int m = 0; m < 2; m++) {
        r[FS_B + 3 * m + 0] = e1x * bb[m][0] + e2x * bb[m][1];
        r[FS_B + 3 * m + 1] = e1y * bb[m][0] + e2y * bb[m][1];
        r[FS_B + 3 * m + 2] = -bb[m][2];
    }
}

// P1..P3 in ENU.  Modes: strike (Ss=1) and dip (Ds=-1, the NED->ENU sign of
// nikkhoo15.f90:140).  r: NW_SIZE doubles.
__host__ __device__ inline void nw_prepare(const double P1[3], const double P2[3], const double P3[3],
                                           double *r)
{
    nw_prep_td(P1, P2, P3, r + NW_MAIN);
    double M1[3] = {P1[0], P1[1], -P1[2]}, M2[3] = {P2[0], P2[1], -P2[2]}, M3[3] = {P3[0], P3[1], -P3[2]};
    nw_prep_td(M1, M2, M3, r + NW_IMG);
    // harmonic term: slip (bx=Ts, by=Ss, bz=Ds) of the real TD frame -> EFCS
    double vn[3], vs[3], vd[3];
    nw_frame(P1, P2, P3, false, vn, vs, vd);
    double bS[3], bD[3];
    for (int k = 0; k < 3; k++) {
        bS[k] = vs[k] * 1.0;
        bD[k] = vd[k] * -1.0;
    }
    nw_prep_fs(P1, P2, bS, bD, r + NW_FS + 0 * FS_SIZE);
    nw_prep_fs(P2, P3, bS, bD, r + NW_FS + 1 * FS_SIZE);
    nw_prep_fs(P3, P1, bS, bD, r + NW_FS + 2 * FS_SIZE);
    r[NW_SURF] = (M1[2] == 0.0 && M2[2] == 0.0 && M3[2] == 0.0) ? 1.0 : 0.0;
}

// ---- per-pair evaluation -----------------------------------------------------

// record accessor: field f of source j in a field-major (SoA) table of ns records
struct NwRec {
    const double *__restrict__ base;
    long stride;
    __device__ __forceinline__ double operator[](int f) const { return __ldg(base + (long)f * stride); }
};

__device__ inline int nw_trimode(double x, double y, double z, double p1a, double p1b,
                                 double p3a, double p3b)
{
    // TriModeFind with p2 = (0, 0) (DispInHalfSpace.c:389-417)
    const double p2a = 0.0, p2b = 0.0;
    double den = (p2b - p3b) * (p1a - p3a) + (p3a - p2a) * (p1b - p3b);
    double a = ((p2b - p3b) * (x - p3a) + (p3a - p2a) * (y - p3b)) / den;
    double b = ((p3b - p1b) * (x - p3a) + (p1a - p3a) * (y - p3b)) / den;
    double c = 1.0 - a - b;
    int m = 1;
    if ((a <= 0.0) && (b > c) && (c > a)) m = -1;
    else if ((b <= 0.0) && (c > a) && (a > b)) m = -1;
    else if ((c <= 0.0) && (a > b) && (b > c)) m = -1;
    else if ((a == 0.0) && (b >= 0.0) && (c >= 0.0)) m = 0;
    else if ((a >= 0.0) && (b == 0.0) && (c >= 0.0)) m = 0;
    else if ((a >= 0.0) && (b >= 0.0) && (c == 0.0)) m = 0;
    if (m == 0 && z != 0.0) m = 1;
    return m;
}

// Angular dislocation (AngDisDisp without tensile term, DispInHalfSpace.c:541-575)
// plus the TDSetupD rotation (DispInHalfSpace.c:419-460).  Adds the TD-frame
// displacement of both modes into dS, dD.
template <class T>
__device__ inline void nw_angdis(T x, T y, T z, double cosA, double sinA, double nu,
                                 double tvy, double tvz, double svy, double svz, double bS_y,
                                 double bS_z, double bD_y, double bD_z, T dS[3], T dD[3])
{
    const double a00 = svz, a01 = -svy, a10 = svy, a11 = svz;
    T ty = y - tvy, tz = z - tvz;
    T y1 = a00 * ty + a01 * tz;
    T z1 = a10 * ty + a11 * tz;
    T eta = y1 * cosA - z1 * sinA;
    T zeta = y1 * sinA + z1 * cosA;
    T r, ir;
    dsqrt_inv(x * x + y1 * y1 + z1 * z1, r, ir);
    T rmz = r - z1, rmzeta = r - zeta;
    T irz = rcp(rmz), irze = rcp(rmzeta);
    T lz = dlog_gi(rmz, irz), lzeta = dlog_gi(rmzeta, irze);
    const double k = 1.0 / 8.0 / 3.141592653589793 / (1.0 - nu);
    const double n12 = 1.0 - 2.0 * nu;
    T x2 = x * x;
    // basis for by (F_y) and bz (F_z), ADCS components (u, v, w)
    T uy = k * (x2 * cosA * ir * irze - x2 * ir * irz - n12 * (cosA * lzeta - lz));
    T vy = k * x * (y1 * cosA * ir * irze - sinA * cosA * irze - y1 * ir * irz);
    T wy = k * x * (z1 * cosA * ir * irze - cosA * cosA * irze + ir);
    T uz = sinA * k * (n12 * lzeta - x2 * ir * irze);
    T vz = sinA * k * x * (sinA * irze - y1 * ir * irze);
    T wz = sinA * k * x * (cosA * irze - z1 * ir * irze);
    // modes: (by1, bz1) = A2 (by, bz)
    const double byS = a00 * bS_y + a01 * bS_z, bzS = a10 * bS_y + a11 * bS_z;
    const double byD = a00 * bD_y + a01 * bD_z, bzD = a10 * bD_y + a11 * bD_z;
    T u0S = byS * uy + bzS * uz, u1S = byS * vy + bzS * vz, u2S = byS * wy + bzS * wz;
    T u0D = byD * uy + bzD * uz, u1D = byD * vy + bzD * vz, u2D = byD * wy + bzD * wz;
    // back to the TD frame with the transpose of A2
    dS[0] = dS[0] + u0S;
    dS[1] = dS[1] + (a00 * u1S + a10 * u2S);
    dS[2] = dS[2] + (a01 * u1S + a11 * u2S);
    dD[0] = dD[0] + u0D;
    dD[1] = dD[1] + (a00 * u1D + a10 * u2D);
    dD[2] = dD[2] + (a01 * u1D + a11 * u2D);
}

// TDdispFS (DispInHalfSpace.c:153-302), EFCS displacements of both modes: their
// gradients for the dual types, their values for Dv.
// Returns false when the point lies on a TD side (reference result: NaN).
template <class T>
__device__ inline bool nw_td_fs(const T X[3], const NwRec &R, int o, double nu, T uS[3], T uD[3])
{
    T dX0 = X[0] - R[o + TD_P2], dX1 = X[1] - R[o + TD_P2 + 1], dX2 = X[2] - R[o + TD_P2 + 2];
    T x = R[o + TD_N] * dX0 + R[o + TD_N + 1] * dX1 + R[o + TD_N + 2] * dX2;
    T y = R[o + TD_S] * dX0 + R[o + TD_S + 1] * dX1 + R[o + TD_S + 2] * dX2;
    T z = R[o + TD_D] * dX0 + R[o + TD_D + 1] * dX1 + R[o + TD_D + 2] * dX2;
    const double p1y = R[o + TD_P1], p1z = R[o + TD_P1 + 1];
    const double p3y = R[o + TD_P3], p3z = R[o + TD_P3 + 1];
    const int mode = nw_trimode(y.v, z.v, x.v, p1y, p1z, p3y, p3z);
    if (mode == 0) return false;
    const double sg1 = (mode == 1) ? -1.0 : 1.0;   // sign on e13 (corner 1)
    const double sg2 = (mode == 1) ? 1.0 : -1.0;   // sign on e12, e23 (corners 2, 3)
    T dS[3] = {T(0.0), T(0.0), T(0.0)}, dD[3] = {T(0.0), T(0.0), T(0.0)};
    // modes in the TD frame: strike (by=1, bz=0), dip (by=0, bz=-1)
    nw_angdis(x, y, z, R[o + TD_CS + 0], R[o + TD_CS + 1], nu, p1y, p1z, sg1 * R[o + TD_E13],
              sg1 * R[o + TD_E13 + 1], 1.0, 0.0, 0.0, -1.0, dS, dD);
    nw_angdis(x, y, z, R[o + TD_CS + 2], R[o + TD_CS + 3], nu, 0.0, 0.0, sg2 * R[o + TD_E12],
              sg2 * R[o + TD_E12 + 1], 1.0, 0.0, 0.0, -1.0, dS, dD);
    nw_angdis(x, y, z, R[o + TD_CS + 4], R[o + TD_CS + 5], nu, p3y, p3z, sg2 * R[o + TD_E23],
              sg2 * R[o + TD_E23 + 1], 1.0, 0.0, 0.0, -1.0, dS, dD);
    // Burgers function of the TD (solid angle)
    T ax = -x, ay = p1y - y, az = p1z - z;
    T bx = -x, by = -y, bz = -z;
    T cx = -x, cy = p3y - y, cz = p3z - z;
    T na = dsqrt(ax * ax + ay * ay + az * az);
    T nb = dsqrt(bx * bx + by * by + bz * bz);
    T nc = dsqrt(cx * cx + cy * cy + cz * cz);
    T num = ax * (by * cz - bz * cy) - ay * (bx * cz - bz * cx) + az * (bx * cy - by * cx);
    T den = na * nb * nc + (ax * bx + ay * by + az * bz) * nc + (ax * cx + ay * cy + az * cz) * nb
           + (bx * cx + by * cy + bz * cz) * na;
    T Fi = datan2_g(num, den) * (-2.0 / 4.0 / 3.141592653589793);
    dS[1] = dS[1] + Fi;          // by = 1
    dD[2] = dD[2] - Fi;          // bz = -1
    for (int k = 0; k < 3; k++) {
        const double n = R[o + TD_N + k], s = R[o + TD_S + k], d = R[o + TD_D + k];
        uS[k] = n * dS[0] + s * dS[1] + d * dS[2];
        uD[k] = n * dD[0] + s * dD[1] + d * dD[2];
    }
    return true;
}

// AngDisDispFSC (DispInHalfSpace.c:577-617) for the two slip modes.
// sc: sinB, cosB, cotB, cot(B/2); b: (b1,b2,b3) per mode (6).
template <class Dd>
__device__ inline void nw_fsc(Dd y1, Dd y2, Dd y3, double sinB, double cosB, double cotB,
                              double coth, const double b[6], double nu, double a, Dd oS[3],
                              Dd oD[3])
{
    Dd y3b = y3 + 2.0 * a;
    Dd z1b = y1 * cosB + y3b * sinB;
    Dd z3b = -y1 * sinB + y3b * cosB;
    // divisions are the costliest FP64 operations here: rb and 1 / rb come from
    // one square root and one division, the logarithms' gradients reuse the
    // reciprocals, and the quotients by cos(beta) multiply by its reciprocal
    Dd rb, irb;
    dsqrt_inv(y1 * y1 + y2 * y2 + y3b * y3b, rb, irb);
    Dd Fib = 2.0 * datan_q_g(-y2, -(rb + y3b) * coth + y1);
    const double n12 = 1.0 - 2.0 * nu, n1 = 1.0 - nu, cot2 = cotB * cotB;
    const double k = 1.0 / 4.0 / 3.141592653589793 / n1;
    const double icB = 1.0 / cosB;
    Dd ry = rb + y3b, rz = rb + z3b, w = rb * cosB + y3b, ya = y3b - a;
    Dd iry = rcp(ry), irz = rcp(rz);
    Dd lry = dlog_gi(ry, iry), lrz = dlog_gi(rz, irz);
    Dd irb2 = irb * irb, irb3 = irb2 * irb;
    Dd cpa = cosB + a * irb;
    Dd rsy = rb * sinB - y1;
    Dd y2s = y2 * y2;

    // fold each basis term into the two modes as soon as it is formed, so
    // that only the outputs and the shared sub-terms stay live
    oS[0] = Dd(0.0); oS[1] = Dd(0.0); oS[2] = Dd(0.0); oD[0] = Dd(0.0); oD[1] = Dd(0.0); oD[2] = Dd(0.0);
    {
        const Dd e11 = -2.0 * n1 * n12 * Fib * cot2 + n12 * y2 * iry * ((n12 - a * irb) * cotB - y1 * iry * (nu + a * irb))
           + n12 * y2 * cosB * cotB * irz * cpa + a * y2 * ya * cotB * irb3
           + y2 * ya * irb * iry * (-n12 * cotB + y1 * iry * (2.0 * nu + a * irb) + a * y1 * irb2)
           + y2 * ya * irb * irz * (cosB * irz * (w * (n12 * cosB - a * irb) * cotB + 2.0 * n1 * rsy * cosB)
                                    - a * y3b * cosB * cotB * irb2);
        oS[0] = oS[0] + b[0] * e11;
        oD[0] = oD[0] + b[3] * e11;
    }
    {
        const Dd e12 = n12 * ((2.0 * n1 * cot2 - nu) * lry - (2.0 * n1 * cot2 + n12) * cosB * lrz)
           - n12 * iry * (y1 * cotB * (n12 - a * irb) + nu * y3b - a + y2s * iry * (nu + a * irb))
           - n12 * z1b * cotB * irz * cpa - a * y1 * ya * cotB * irb3
           + ya * iry * (-2.0 * nu + irb * (n12 * y1 * cotB - a) + y2s * irb * iry * (2.0 * nu + a * irb) + a * y2s * irb3)
           + ya * irz * (cosB * cosB - irb * (n12 * z1b * cotB + a * cosB) + a * y3b * z1b * cotB * irb3
                         - irb * irz * (y2s * cosB * cosB - a * z1b * cotB * irb * w));
        oS[1] = oS[1] + b[0] * e12;
        oD[1] = oD[1] + b[3] * e12;
    }
    {
        const Dd e13 = 2.0 * n1 * ((n12 * Fib * cotB) + (y2 * iry * (2.0 * nu + a * irb)) - (y2 * cosB * irz * cpa))
           + y2 * ya * irb * (2.0 * nu * iry + a * irb2)
           + y2 * ya * cosB * irb * irz * (n12 - w * irz * cpa - a * y3b * irb2);
        oS[2] = oS[2] + b[0] * e13;
        oD[2] = oD[2] + b[3] * e13;
    }
    {
        const Dd e21 = n12 * ((2.0 * n1 * cot2 + nu) * lry - (2.0 * n1 * cot2 + 1.0) * cosB * lrz)
           + n12 * iry * (-n12 * y1 * cotB + nu * y3b - a + a * y1 * cotB * irb + y1 * y1 * iry * (nu + a * irb))
           - n12 * cotB * irz * (z1b * cosB - a * rsy * irb * icB) - a * y1 * ya * cotB * irb3
           + ya * iry * (2.0 * nu + irb * (n12 * y1 * cotB + a) - y1 * y1 * irb * iry * (2.0 * nu + a * irb) - a * y1 * y1 * irb3)
           + ya * cotB * irz * (-cosB * sinB + a * y1 * y3b * irb3 * icB
                                + rsy * irb * (2.0 * n1 * cosB - w * irz * (1.0 + a * irb * icB)));
        oS[0] = oS[0] + b[1] * e21;
        oD[0] = oD[0] + b[4] * e21;
    }
    {
        const Dd e22 = 2.0 * n1 * n12 * Fib * cot2 + n12 * y2 * iry * (-(n12 - a * irb) * cotB + y1 * iry * (nu + a * irb))
           - n12 * y2 * cotB * irz * (1.0 + a * irb * icB) - a * y2 * ya * cotB * irb3
           + y2 * ya * irb * iry * (n12 * cotB - 2.0 * nu * y1 * iry - a * y1 * irb * (irb + iry))
           + y2 * ya * cotB * irb * irz * (-2.0 * n1 * cosB + w * irz * (1.0 + a * irb * icB) + a * y3b * irb2 * icB);
        oS[1] = oS[1] + b[1] * e22;
        oD[1] = oD[1] + b[4] * e22;
    }
    {
        const Dd e23 = -2.0 * n1 * n12 * cotB * (lry - cosB * lrz) - 2.0 * n1 * y1 * iry * (2.0 * nu + a * irb)
           + 2.0 * n1 * z1b * irz * cpa + ya * irb * (n12 * cotB - 2.0 * nu * y1 * iry - a * y1 * irb2)
           - ya * irz * (cosB * sinB + w * cotB * irb * (2.0 * n1 * cosB - w * irz)
                         + a * irb * (sinB - y3b * z1b * irb2 - z1b * w * irb * irz));
        oS[2] = oS[2] + b[1] * e23;
        oD[2] = oD[2] + b[4] * e23;
    }
    {
        const Dd e31 = n12 * (y2 * iry * (1.0 + a * irb) - y2 * cosB * irz * cpa) - y2 * ya * irb * (a * irb2 + iry)
           + y2 * ya * cosB * irb * irz * (w * irz * cpa + a * y3b * irb2);
        oS[0] = oS[0] + b[2] * e31;
        oD[0] = oD[0] + b[5] * e31;
    }
    {
        const Dd e32 = n12 * (-sinB * lrz - y1 * iry * (1.0 + a * irb) + z1b * irz * cpa)
           + y1 * ya * irb * (a * irb2 + iry)
           - ya * irz * (sinB * (cosB - a * irb) + z1b * irb * (1.0 + a * y3b * irb2)
                         - irb * irz * (y2s * cosB * sinB - a * z1b * irb * w));
        oS[1] = oS[1] + b[2] * e32;
        oD[1] = oD[1] + b[5] * e32;
    }
    {
        const Dd e33 = 2.0 * n1 * Fib + 2.0 * n1 * (y2 * sinB * irz * cpa)
           + y2 * ya * sinB * irb * irz * (1.0 + w * irz * cpa + a * y3b * irb2);
        oS[2] = oS[2] + b[2] * e33;
        oD[2] = oD[2] + b[5] * e33;
    }
    for (int c = 0; c < 3; c++) {
        oS[c] = k * oS[c];
        oD[c] = k * oD[c];
    }
}

// harmonic function of one side (AngSetupFSC), added into uS, uD (EFCS).
template <class Dd>
__device__ inline void nw_side(const Dd X[3], const NwRec &R, int o, double nu, Dd uS[3], Dd uD[3])
{
    if (R[o + FS_DEG] != 0.0) return;
    const double e1x = R[o + FS_E1], e1y = R[o + FS_E1 + 1];
    const double e2x = R[o + FS_E2], e2y = R[o + FS_E2 + 1];
    Dd d0 = X[0] - R[o + FS_PA], d1 = X[1] - R[o + FS_PA + 1], d2 = X[2] - R[o + FS_PA + 2];
    Dd yA0 = e1x * d0 + e2x * d1;
    Dd yA1 = e1y * d0 + e2y * d1;
    Dd yA2 = -d2;
    Dd yB0 = yA0 - R[o + FS_SA], yB1 = yA1 - R[o + FS_SA + 1], yB2 = yA2 - R[o + FS_SA + 2];
    double b[6];
    for (int k = 0; k < 6; k++) b[k] = R[o + FS_B + k];
    const double aA = R[o + FS_AA], aB = R[o + FS_AB];
    Dd aS[3], aD[3], cS[3], cD[3];
    if (yA0.v >= 0.0) {   // configuration I: mirrored frame, angle pi - beta
        double bm[6] = {-b[0], -b[1], b[2], -b[3], -b[4], b[5]};
        const double sB = R[o + FS_I], cB = R[o + FS_I + 1], ct = R[o + FS_I + 2], ch = R[o + FS_I + 3];
        nw_fsc(-yA0, -yA1, yA2, sB, cB, ct, ch, bm, nu, aA, aS, aD);
        nw_fsc(-yB0, -yB1, yB2, sB, cB, ct, ch, bm, nu, aB, cS, cD);
        aS[0] = -aS[0]; aS[1] = -aS[1]; aD[0] = -aD[0]; aD[1] = -aD[1];
        cS[0] = -cS[0]; cS[1] = -cS[1]; cD[0] = -cD[0]; cD[1] = -cD[1];
    } else {              // configuration II
        const double sB = R[o + FS_II], cB = R[o + FS_II + 1], ct = R[o + FS_II + 2], ch = R[o + FS_II + 3];
        nw_fsc(yA0, yA1, yA2, sB, cB, ct, ch, b, nu, aA, aS, aD);
        nw_fsc(yB0, yB1, yB2, sB, cB, ct, ch, b, nu, aB, cS, cD);
    }
    // v = vB - vA in the side frame, back to EFCS with the transposed frame
    // (rows ey1, ey2, ey3), as the strain routine's TensTrans(.., A_t) does
    Dd vS0 = cS[0] - aS[0], vS1 = cS[1] - aS[1], vS2 = cS[2] - aS[2];
    Dd vD0 = cD[0] - aD[0], vD1 = cD[1] - aD[1], vD2 = cD[2] - aD[2];
    uS[0] = uS[0] + (e1x * vS0 + e1y * vS1);
    uS[1] = uS[1] + (e2x * vS0 + e2y * vS1);
    uS[2] = uS[2] - vS2;
    uD[0] = uD[0] + (e1x * vD0 + e1y * vD1);
    uD[1] = uD[1] + (e2x * vD0 + e2y * vD1);
    uD[2] = uD[2] - vD2;
}

// gradient -> stress, C order xx, xy, xz, yy, yz, zz (ENU)
__device__ __forceinline__ void nw_stress(const Dd u[3], double mu, double lambda, double s[6])
{
    const double exx = u[0].x, eyy = u[1].y, ezz = u[2].z;
    const double exy = 0.5 * (u[0].y + u[1].x);
    const double exz = 0.5 * (u[0].z + u[2].x);
    const double eyz = 0.5 * (u[1].z + u[2].y);
    const double kk = exx + eyy + ezz;
    s[0] = 2.0 * mu * exx + lambda * kk;
    s[1] = 2.0 * mu * exy;
    s[2] = 2.0 * mu * exz;
    s[3] = 2.0 * mu * eyy + lambda * kk;
    s[4] = 2.0 * mu * eyz;
    s[5] = 2.0 * mu * ezz + lambda * kk;
}

// ENU stress (C order) -> NED s11,s12,s13,s22,s23,s33 (nikkhoo15.f90:156-161)
__device__ __forceinline__ void nw_to_ned(const double e[6], double s[6])
{
    s[0] = e[3]; s[1] = e[1]; s[2] = -e[4]; s[3] = e[0]; s[4] = -e[2]; s[5] = e[5];
}

// One part of the TD stress at receiver xr (NED) for unit strike slip (sS) and
// unit dip slip (sD): PART 0 main TD, 1 image TD (with the surface sign flip),
// 2 harmonic free-surface term.  The three parts sum to straininhalfspace_'s
// stress; evaluating them in separate passes keeps the live state of each pass
// small enough for the register file.
template <int PART>
__device__ inline void nw_part_stress(const double xr[3], const NwRec &R, const NwConst &c, double sS[6],
                                      double sD[6])
{
    Dd X[3] = {Dd{xr[1], 1.0, 0.0, 0.0}, Dd{xr[0], 0.0, 1.0, 0.0}, Dd{-xr[2], 0.0, 0.0, 1.0}};
    Dd uS[3] = {dd(0), dd(0), dd(0)}, uD[3] = {dd(0), dd(0), dd(0)};
    if (PART == 2) {
        // one pass per derivative direction with single-direction duals
        double gS[3][3], gD[3][3];
#pragma unroll 1
        for (int dir = 0; dir < 3; dir++) {
            Dd1 X1[3] = {Dd1{xr[1], dir == 0 ? 1.0 : 0.0}, Dd1{xr[0], dir == 1 ? 1.0 : 0.0},
                         Dd1{-xr[2], dir == 2 ? 1.0 : 0.0}};
            Dd1 vS[3] = {Dd1(0.0), Dd1(0.0), Dd1(0.0)}, vD[3] = {Dd1(0.0), Dd1(0.0), Dd1(0.0)};
#pragma unroll 1
            for (int side = 0; side < 3; side++) nw_side<Dd1>(X1, R, NW_FS + side * FS_SIZE, c.nu, vS, vD);
            for (int k = 0; k < 3; k++) { gS[k][dir] = vS[k].d; gD[k][dir] = vD[k].d; }
        }
        for (int k = 0; k < 3; k++) {
            uS[k] = Dd{0.0, gS[k][0], gS[k][1], gS[k][2]};
            uD[k] = Dd{0.0, gD[k][0], gD[k][1], gD[k][2]};
        }
    } else {
        if (!nw_td_fs(X, R, PART == 0 ? NW_MAIN : NW_IMG, c.nu, uS, uD)) {
            for (int k = 0; k < 6; k++) { sS[k] = nan(""); sD[k] = nan(""); }
            return;
        }
    }
    double eS[6], eD[6];
    nw_stress(uS, c.mu, c.lambda, eS);
    nw_stress(uD, c.mu, c.lambda, eD);
    if (PART == 1 && R[NW_SURF] != 0.0) { eS[4] = -eS[4]; eS[5] = -eS[5]; eD[4] = -eD[4]; eD[5] = -eD[5]; }
    nw_to_ned(eS, sS);
    nw_to_ned(eD, sD);
}

// Displacement (north, east, down) at xr (NED) for unit strike slip (uS) and
// unit dip slip (uD) of one TD, as dispinhalfspace_ called by
// computeDisplacementNikkhoo15 (nikkhoo15.f90:324-367; DispInHalfSpace.c:
// 64-151): main TD + image TD (vertical component negated when all vertices
// lie at z = 0) + the three free-surface sides, the whole sum negated for such
// surface TDs, then ENU -> NED.  A point on a TD side gives NaN, as in the
// reference.
__device__ inline void nw_pair_disp(const double xr[3], const NwRec &R, double nu, double uS[3], double uD[3])
{
    const Dv X[3] = {Dv(xr[1]), Dv(xr[0]), Dv(-xr[2])};
    Dv mS[3] = {Dv(0.0), Dv(0.0), Dv(0.0)}, mD[3] = {Dv(0.0), Dv(0.0), Dv(0.0)};
    Dv iS[3] = {Dv(0.0), Dv(0.0), Dv(0.0)}, iD[3] = {Dv(0.0), Dv(0.0), Dv(0.0)};
    Dv hS[3] = {Dv(0.0), Dv(0.0), Dv(0.0)}, hD[3] = {Dv(0.0), Dv(0.0), Dv(0.0)};
    if (!nw_td_fs(X, R, NW_MAIN, nu, mS, mD) || !nw_td_fs(X, R, NW_IMG, nu, iS, iD)) {
        for (int k = 0; k < 3; k++) { uS[k] = nan(""); uD[k] = nan(""); }
        return;
    }
    const bool surf = R[NW_SURF] != 0.0;
    if (surf) { iS[2] = -iS[2]; iD[2] = -iD[2]; }
#pragma unroll 1
    for (int side = 0; side < 3; side++) nw_side<Dv>(X, R, NW_FS + side * FS_SIZE, nu, hS, hD);
    double eS[3], eD[3];
    for (int k = 0; k < 3; k++) {
        eS[k] = (mS[k] + iS[k] + hS[k]).v;
        eD[k] = (mD[k] + iD[k] + hD[k]).v;
        if (surf) { eS[k] = -eS[k]; eD[k] = -eD[k]; }
    }
    uS[0] = eS[1]; uS[1] = eS[0]; uS[2] = -eS[2];
    uD[0] = eD[1]; uD[1] = eD[0]; uD[2] = -eD[2];
}

}  // namespace ucg
