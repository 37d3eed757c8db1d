/*
 * Oracle: Nikkhoo & Walter (2015) triangular dislocation (TD) in a half-space.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference computes TD stress with straininhalfspace_
 * (fortran/3d/src/StrainInHalfSpace.c:42-177), whose strain expressions are the
 * analytic derivatives of the TD displacement field published in the same paper
 * and coded in fortran/3d/src/DispInHalfSpace.c.  This restatement evaluates that
 * displacement field (DispInHalfSpace.c:153-617: TDdispFS, TDdisp_HarFunc,
 * TDSetupD, AngSetupFSC, AngDisDisp, AngDisDispFSC) on dual numbers seeded with
 * the observation point, which yields the exact displacement gradient, and then
 * follows straininhalfspace_ for the assembly of the three parts:
 *   - main TD, image TD (vertices mirrored in z), harmonic free-surface term;
 *   - the image's [4] and [5] components (yz and zz in the C routine's
 *     xx,xy,xz,yy,yz,zz order) change sign when all three vertices lie at z=0
 *     (StrainInHalfSpace.c:162-165);
 *   - the configuration-I free-surface angular dislocations are evaluated in the
 *     mirrored frame (-y1,-y2,y3), angle pi-beta, slip (-b1,-b2,b3)
 *     (StrainInHalfSpace.c:644-652), which is what the strain routine
 *     differentiates;
 *   - the angular-dislocation displacement clamps of AngDisDisp (zeta<=r, z<=r)
 *     are not applied: AngDisStrain has none.
 * computeStressNikkhoo15 (fortran/3d/src/nikkhoo15.f90:120-163) supplies the
 * NED<->ENU mapping: x=x2, y=x1, z=-x3, dip slip negated, and
 * s11=s(4), s12=s(2), s13=-s(5), s22=s(1), s23=-s(3), s33=s(6).
 *
 * Pinned against the reference C routine itself (built from the reference
 * sources into oracle/_ref) and against tests/golden fixtures made from it.
 */
#include <cmath>
#include <cfloat>
#include "dual3.h"
#include "oracle.h"

namespace {

const double PI = M_PI;

struct V3 { D3 c[3]; };

/* TD frame: normal, strike, dip (TDdispFS, DispInHalfSpace.c:178-208) */
void td_frame(const double P1[3], const double P2[3], const double P3[3], bool image_fix,
              double vn[3], double vs[3], double vd[3])
{
    double t1[3] = {P2[0] - P1[0], P2[1] - P1[1], P2[2] - P1[2]};
    double t2[3] = {P3[0] - P1[0], P3[1] - P1[1], P3[2] - P1[2]};
    vn[0] = t1[1] * t2[2] - t1[2] * t2[1];
    vn[1] = t1[2] * t2[0] - t1[0] * t2[2];
    vn[2] = t1[0] * t2[1] - t1[1] * t2[0];
    double nn = std::sqrt(vn[0] * vn[0] + vn[1] * vn[1] + vn[2] * vn[2]);
    for (int k = 0; k < 3; k++) vn[k] /= nn;
    /* strike = eZ x n */
    vs[0] = -vn[1];
    vs[1] = vn[0];
    vs[2] = 0.0;
    double ns = std::sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
    if (ns == 0.0) {
        vs[0] = 0.0; vs[1] = vn[2]; vs[2] = 0.0;
        if (image_fix && P1[2] > 0.0) { vs[1] = -vs[1]; }
        ns = std::sqrt(vs[0] * vs[0] + vs[1] * vs[1] + vs[2] * vs[2]);
    }
    for (int k = 0; k < 3; k++) vs[k] /= ns;
    vd[0] = vn[1] * vs[2] - vn[2] * vs[1];
    vd[1] = vn[2] * vs[0] - vn[0] * vs[2];
    vd[2] = vn[0] * vs[1] - vn[1] * vs[0];
    double nd = std::sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
    for (int k = 0; k < 3; k++) vd[k] /= nd;
}

/* TriModeFind, DispInHalfSpace.c:389-417 */
int tri_mode(double x, double y, double z, double p1a, double p1b, double p2a, double p2b,
             double p3a, double p3b)
{
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

/* AngDisDisp without the Burgers function (DispInHalfSpace.c:541-575) */
V3 ang_dis_disp(const D3 &x, const D3 &y, const D3 &z, double alpha, double bx, double by,
                double bz, double nu)
{
    double cosA = std::cos(alpha), sinA = std::sin(alpha);
    D3 eta = y * cosA - z * sinA;
    D3 zeta = y * sinA + z * cosA;
    D3 r = sqrt(x * x + y * y + z * z);
    double k = 1.0 / 8.0 / PI / (1.0 - nu);
    D3 rmz = r - z, rmzeta = r - zeta;
    D3 lz = log(rmz), lzeta = log(rmzeta);
    double n12 = 1.0 - 2.0 * nu;
    D3 ux = bx * k * (x * y / r / rmz - x * eta / r / rmzeta);
    D3 vx = bx * k * (eta * sinA / rmzeta - y * eta / r / rmzeta + y * y / r / rmz + n12 * (cosA * lzeta - lz));
    D3 wx = bx * k * (eta * cosA / rmzeta - y / r - eta * z / r / rmzeta - n12 * sinA * lzeta);
    D3 uy = by * k * (x * x * cosA / r / rmzeta - x * x / r / rmz - n12 * (cosA * lzeta - lz));
    D3 vy = by * k * x * (y * cosA / r / rmzeta - sinA * cosA / rmzeta - y / r / rmz);
    D3 wy = by * k * x * (z * cosA / r / rmzeta - cosA * cosA / rmzeta + 1.0 / r);
    D3 uz = bz * sinA * k * (n12 * lzeta - x * x / r / rmzeta);
    D3 vz = bz * sinA * k * x * (sinA / rmzeta - y / r / rmzeta);
    D3 wz = bz * sinA * k * x * (cosA / rmzeta - z / r / rmzeta);
    V3 o;
    o.c[0] = ux + uy + uz;
    o.c[1] = vx + vy + vz;
    o.c[2] = wx + wy + wz;
    return o;
}

/* TDSetupD, DispInHalfSpace.c:419-460 */
V3 td_setup(const D3 &x, const D3 &y, const D3 &z, double alpha, double bx, double by,
            double bz, double nu, const double tv[3], const double sv[3])
{
    double a00 = sv[2], a01 = -sv[1], a10 = sv[1], a11 = sv[2];
    D3 ty = y - tv[1], tz = z - tv[2];
    D3 y1 = a00 * ty + a01 * tz;
    D3 z1 = a10 * ty + a11 * tz;
    double by1 = a00 * by + a01 * bz;
    double bz1 = a10 * by + a11 * bz;
    V3 d = ang_dis_disp(x, y1, z1, -PI + alpha, bx, by1, bz1, nu);
    V3 o;
    o.c[0] = d.c[0];
    o.c[1] = a00 * d.c[1] + a10 * d.c[2];
    o.c[2] = a01 * d.c[1] + a11 * d.c[2];
    return o;
}

/* TDdispFS, DispInHalfSpace.c:153-302.  X in EFCS (ENU); slip (by=Ss, bz=Ds, bx=Ts). */
V3 td_disp_fs(const D3 X[3], const double P1[3], const double P2[3], const double P3[3],
              double by, double bz, double bx, double nu)
{
    double vn[3], vs[3], vd[3];
    td_frame(P1, P2, P3, true, vn, vs, vd);
    D3 dX[3] = {X[0] - P2[0], X[1] - P2[1], X[2] - P2[2]};
    D3 x = vn[0] * dX[0] + vn[1] * dX[1] + vn[2] * dX[2];
    D3 y = vs[0] * dX[0] + vs[1] * dX[1] + vs[2] * dX[2];
    D3 z = vd[0] * dX[0] + vd[1] * dX[1] + vd[2] * dX[2];
    double q1[3] = {P1[0] - P2[0], P1[1] - P2[1], P1[2] - P2[2]};
    double q3[3] = {P3[0] - P2[0], P3[1] - P2[1], P3[2] - P2[2]};
    double p1[3], p2[3] = {0, 0, 0}, p3[3];
    for (int r = 0; r < 3; r++) {
        const double *row = r == 0 ? vn : (r == 1 ? vs : vd);
        p1[r] = row[0] * q1[0] + row[1] * q1[1] + row[2] * q1[2];
        p3[r] = row[0] * q3[0] + row[1] * q3[1] + row[2] * q3[2];
    }
    double e12[3], e13[3], e23[3], n;
    n = std::sqrt((p2[0] - p1[0]) * (p2[0] - p1[0]) + (p2[1] - p1[1]) * (p2[1] - p1[1]) + (p2[2] - p1[2]) * (p2[2] - p1[2]));
    for (int k = 0; k < 3; k++) e12[k] = (p2[k] - p1[k]) / n;
    n = std::sqrt((p3[0] - p1[0]) * (p3[0] - p1[0]) + (p3[1] - p1[1]) * (p3[1] - p1[1]) + (p3[2] - p1[2]) * (p3[2] - p1[2]));
    for (int k = 0; k < 3; k++) e13[k] = (p3[k] - p1[k]) / n;
    n = std::sqrt((p3[0] - p2[0]) * (p3[0] - p2[0]) + (p3[1] - p2[1]) * (p3[1] - p2[1]) + (p3[2] - p2[2]) * (p3[2] - p2[2]));
    for (int k = 0; k < 3; k++) e23[k] = (p3[k] - p2[k]) / n;
    double A = std::acos(e12[0] * e13[0] + e12[1] * e13[1] + e12[2] * e13[2]);
    double B = std::acos(-e12[0] * e23[0] - e12[1] * e23[1] - e12[2] * e23[2]);
    double C = std::acos(e23[0] * e13[0] + e23[1] * e13[1] + e23[2] * e13[2]);
    int mode = tri_mode(y.v, z.v, x.v, p1[1], p1[2], p2[1], p2[2], p3[1], p3[2]);
    V3 d1, d2, d3, out;
    if (mode == 1) {
        double m13[3] = {-e13[0], -e13[1], -e13[2]};
        d1 = td_setup(x, y, z, A, bx, by, bz, nu, p1, m13);
        d2 = td_setup(x, y, z, B, bx, by, bz, nu, p2, e12);
        d3 = td_setup(x, y, z, C, bx, by, bz, nu, p3, e23);
    } else if (mode == -1) {
        double m12[3] = {-e12[0], -e12[1], -e12[2]}, m23[3] = {-e23[0], -e23[1], -e23[2]};
        d1 = td_setup(x, y, z, A, bx, by, bz, nu, p1, e13);
        d2 = td_setup(x, y, z, B, bx, by, bz, nu, p2, m12);
        d3 = td_setup(x, y, z, C, bx, by, bz, nu, p3, m23);
    } else {
        for (int k = 0; k < 3; k++) out.c[k] = D3(NAN, NAN, NAN, NAN);
        return out;
    }
    D3 dc[3];
    for (int k = 0; k < 3; k++) dc[k] = d1.c[k] + d2.c[k] + d3.c[k];
    /* Burgers function of the whole TD (solid angle) */
    D3 a[3] = {-x, p1[1] - y, p1[2] - z};
    D3 b[3] = {-x, -y, -z};
    D3 c[3] = {-x, p3[1] - y, p3[2] - z};
    D3 na = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    D3 nb = sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]);
    D3 nc = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    D3 num = a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) + a[2] * (b[0] * c[1] - b[1] * c[0]);
    D3 den = na * nb * nc + (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) * nc
           + (a[0] * c[0] + a[1] * c[1] + a[2] * c[2]) * nb + (b[0] * c[0] + b[1] * c[1] + b[2] * c[2]) * na;
    D3 Fi = -2.0 * atan2(num, den) / 4.0 / PI;
    dc[0] += bx * Fi;
    dc[1] += by * Fi;
    dc[2] += bz * Fi;
    for (int k = 0; k < 3; k++) out.c[k] = vn[k] * dc[0] + vs[k] * dc[1] + vd[k] * dc[2];
    return out;
}

/* AngDisDispFSC, DispInHalfSpace.c:577-617 */
V3 ang_dis_disp_fsc(const D3 &y1, const D3 &y2, const D3 &y3, double beta, double b1,
                    double b2, double b3, double nu, double a)
{
    double sinB = std::sin(beta), cosB = std::cos(beta), cotB = cosB / sinB;
    D3 y3b = y3 + 2.0 * a;
    D3 z1b = y1 * cosB + y3b * sinB;
    D3 z3b = -y1 * sinB + y3b * cosB;
    D3 rb = sqrt(y1 * y1 + y2 * y2 + y3b * y3b);
    D3 Fib = 2.0 * atan(-y2 / (-(rb + y3b) * (std::cos(beta / 2.0) / std::sin(beta / 2.0)) + y1));
    double n12 = 1.0 - 2.0 * nu, n1 = 1.0 - nu, cot2 = cotB * cotB;
    double k = 1.0 / 4.0 / PI / n1;
    D3 ry = rb + y3b, rz = rb + z3b, w = rb * cosB + y3b, ya = y3b - a;
    D3 lry = log(ry), lrz = log(rz);
    D3 rb2 = rb * rb, rb3 = rb2 * rb;
    D3 cpa = cosB + a / rb;

    D3 v1b1 = b1 * k * (-2.0 * n1 * n12 * Fib * cot2 + n12 * y2 / ry * ((n12 - a / rb) * cotB - y1 / ry * (nu + a / rb))
              + n12 * y2 * cosB * cotB / rz * cpa + a * y2 * ya * cotB / rb3
              + y2 * ya / (rb * ry) * (-n12 * cotB + y1 / ry * (2.0 * nu + a / rb) + a * y1 / rb2)
              + y2 * ya / (rb * rz) * (cosB / rz * (w * (n12 * cosB - a / rb) * cotB + 2.0 * n1 * (rb * sinB - y1) * cosB)
                                       - a * y3b * cosB * cotB / rb2));
    D3 v2b1 = b1 * k * (n12 * ((2.0 * n1 * cot2 - nu) * lry - (2.0 * n1 * cot2 + n12) * cosB * lrz)
              - n12 / ry * (y1 * cotB * (n12 - a / rb) + nu * y3b - a + y2 * y2 / ry * (nu + a / rb))
              - n12 * z1b * cotB / rz * cpa - a * y1 * ya * cotB / rb3
              + ya / ry * (-2.0 * nu + 1.0 / rb * (n12 * y1 * cotB - a) + y2 * y2 / (rb * ry) * (2.0 * nu + a / rb) + a * y2 * y2 / rb3)
              + ya / rz * (cosB * cosB - 1.0 / rb * (n12 * z1b * cotB + a * cosB) + a * y3b * z1b * cotB / rb3
                           - 1.0 / (rb * rz) * (y2 * y2 * cosB * cosB - a * z1b * cotB / rb * w)));
    D3 v3b1 = b1 * k * (2.0 * n1 * ((n12 * Fib * cotB) + (y2 / ry * (2.0 * nu + a / rb)) - (y2 * cosB / rz * cpa))
              + y2 * ya / rb * (2.0 * nu / ry + a / rb2)
              + y2 * ya * cosB / (rb * rz) * (n12 - w / rz * cpa - a * y3b / rb2));
    D3 v1b2 = b2 * k * (n12 * ((2.0 * n1 * cot2 + nu) * lry - (2.0 * n1 * cot2 + 1.0) * cosB * lrz)
              + n12 / ry * (-n12 * y1 * cotB + nu * y3b - a + a * y1 * cotB / rb + y1 * y1 / ry * (nu + a / rb))
              - n12 * cotB / rz * (z1b * cosB - a * (rb * sinB - y1) / (rb * cosB)) - a * y1 * ya * cotB / rb3
              + ya / ry * (2.0 * nu + 1.0 / rb * (n12 * y1 * cotB + a) - y1 * y1 / (rb * ry) * (2.0 * nu + a / rb) - a * y1 * y1 / rb3)
              + ya * cotB / rz * (-cosB * sinB + a * y1 * y3b / (rb3 * cosB)
                                  + (rb * sinB - y1) / rb * (2.0 * n1 * cosB - w / rz * (1.0 + a / (rb * cosB)))));
    D3 v2b2 = b2 * k * (2.0 * n1 * n12 * Fib * cot2 + n12 * y2 / ry * (-(n12 - a / rb) * cotB + y1 / ry * (nu + a / rb))
              - n12 * y2 * cotB / rz * (1.0 + a / (rb * cosB)) - a * y2 * ya * cotB / rb3
              + y2 * ya / (rb * ry) * (n12 * cotB - 2.0 * nu * y1 / ry - a * y1 / rb * (1.0 / rb + 1.0 / ry))
              + y2 * ya * cotB / (rb * rz) * (-2.0 * n1 * cosB + w / rz * (1.0 + a / (rb * cosB)) + a * y3b / (rb2 * cosB)));
    D3 v3b2 = b2 * k * (-2.0 * n1 * n12 * cotB * (lry - cosB * lrz) - 2.0 * n1 * y1 / ry * (2.0 * nu + a / rb)
              + 2.0 * n1 * z1b / rz * cpa + ya / rb * (n12 * cotB - 2.0 * nu * y1 / ry - a * y1 / rb2)
              - ya / rz * (cosB * sinB + w * cotB / rb * (2.0 * n1 * cosB - w / rz)
                           + a / rb * (sinB - y3b * z1b / rb2 - z1b * w / (rb * rz))));
    D3 v1b3 = b3 * k * (n12 * (y2 / ry * (1.0 + a / rb) - y2 * cosB / rz * cpa) - y2 * ya / rb * (a / rb2 + 1.0 / ry)
              + y2 * ya * cosB / (rb * rz) * (w / rz * cpa + a * y3b / rb2));
    D3 v2b3 = b3 * k * (n12 * (-sinB * lrz - y1 / ry * (1.0 + a / rb) + z1b / rz * cpa)
              + y1 * ya / rb * (a / rb2 + 1.0 / ry)
              - ya / rz * (sinB * (cosB - a / rb) + z1b / rb * (1.0 + a * y3b / rb2)
                           - 1.0 / (rb * rz) * (y2 * y2 * cosB * sinB - a * z1b / rb * w)));
    D3 v3b3 = b3 * k * (2.0 * n1 * Fib + 2.0 * n1 * (y2 * sinB / rz * cpa)
              + y2 * ya * sinB / (rb * rz) * (1.0 + w / rz * cpa + a * y3b / rb2));
    V3 o;
    o.c[0] = v1b1 + v1b2 + v1b3;
    o.c[1] = v2b1 + v2b2 + v2b3;
    o.c[2] = v3b1 + v3b2 + v3b3;
    return o;
}

/* AngSetupFSC (displacement, DispInHalfSpace.c:462-539) with the configuration-I
   frame of AngSetupFSC_S (StrainInHalfSpace.c:596-686). */
V3 ang_setup_fsc(const D3 X[3], double bX, double bY, double bZ, const double PA[3],
                 const double PB[3], double nu)
{
    V3 out;
    double sv[3] = {PB[0] - PA[0], PB[1] - PA[1], PB[2] - PA[2]};
    double l = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
    double beta = std::acos(-sv[2] / l);
    if (std::fabs(beta) < DBL_EPSILON || std::fabs(PI - beta) < DBL_EPSILON) {
        for (int k = 0; k < 3; k++) out.c[k] = D3(0.0);
        return out;
    }
    double ey1[3] = {sv[0], sv[1], 0.0};
    double n1 = std::sqrt(ey1[0] * ey1[0] + ey1[1] * ey1[1]);
    ey1[0] /= n1; ey1[1] /= n1;
    double ey3[3] = {0.0, 0.0, -1.0};
    double ey2[3] = {ey3[1] * ey1[2] - ey3[2] * ey1[1], ey3[2] * ey1[0] - ey3[0] * ey1[2],
                     ey3[0] * ey1[1] - ey3[1] * ey1[0]};
    double n2 = std::sqrt(ey2[0] * ey2[0] + ey2[1] * ey2[1] + ey2[2] * ey2[2]);
    for (int k = 0; k < 3; k++) ey2[k] /= n2;
    /* A has columns ey1, ey2, ey3 (symmetric up to rounding); y = A (X - PA) */
    double Am[3][3] = {{ey1[0], ey2[0], ey3[0]}, {ey1[1], ey2[1], ey3[1]}, {ey1[2], ey2[2], ey3[2]}};
    D3 dX[3] = {X[0] - PA[0], X[1] - PA[1], X[2] - PA[2]};
    D3 yA[3], yB[3];
    double sA[3], bA[3];
    for (int r = 0; r < 3; r++) {
        yA[r] = Am[r][0] * dX[0] + Am[r][1] * dX[1] + Am[r][2] * dX[2];
        sA[r] = Am[r][0] * sv[0] + Am[r][1] * sv[1] + Am[r][2] * sv[2];
        bA[r] = Am[r][0] * bX + Am[r][1] * bY + Am[r][2] * bZ;
    }
    for (int r = 0; r < 3; r++) yB[r] = yA[r] - sA[r];
    V3 vA, vB;
    if (beta * yA[0].v >= 0.0) {
        V3 a = ang_dis_disp_fsc(-yA[0], -yA[1], yA[2], PI - beta, -bA[0], -bA[1], bA[2], nu, -PA[2]);
        V3 b = ang_dis_disp_fsc(-yB[0], -yB[1], yB[2], PI - beta, -bA[0], -bA[1], bA[2], nu, -PB[2]);
        vA.c[0] = -a.c[0]; vA.c[1] = -a.c[1]; vA.c[2] = a.c[2];
        vB.c[0] = -b.c[0]; vB.c[1] = -b.c[1]; vB.c[2] = b.c[2];
    } else {
        vA = ang_dis_disp_fsc(yA[0], yA[1], yA[2], beta, bA[0], bA[1], bA[2], nu, -PA[2]);
        vB = ang_dis_disp_fsc(yB[0], yB[1], yB[2], beta, bA[0], bA[1], bA[2], nu, -PB[2]);
    }
    D3 dv[3] = {vB.c[0] - vA.c[0], vB.c[1] - vA.c[1], vB.c[2] - vA.c[2]};
    /* back to EFCS with the transposed frame (rows ey1, ey2, ey3), as the strain
       routine's TensTrans(.., A_t) does */
    for (int r = 0; r < 3; r++) out.c[r] = Am[0][r] * dv[0] + Am[1][r] * dv[1] + Am[2][r] * dv[2];
    return out;
}

/* TDdisp_HarFunc, DispInHalfSpace.c:306-372 */
V3 td_disp_harm(const D3 X[3], const double P1[3], const double P2[3], const double P3[3],
                double by, double bz, double bx, double nu)
{
    double vn[3], vs[3], vd[3];
    td_frame(P1, P2, P3, false, vn, vs, vd);
    double b[3];
    for (int k = 0; k < 3; k++) b[k] = vn[k] * bx + vs[k] * by + vd[k] * bz;
    V3 s1 = ang_setup_fsc(X, b[0], b[1], b[2], P1, P2, nu);
    V3 s2 = ang_setup_fsc(X, b[0], b[1], b[2], P2, P3, nu);
    V3 s3 = ang_setup_fsc(X, b[0], b[1], b[2], P3, P1, nu);
    V3 o;
    for (int k = 0; k < 3; k++) o.c[k] = s1.c[k] + s2.c[k] + s3.c[k];
    return o;
}

/* displacement gradient -> stress in the C routine's order xx,xy,xz,yy,yz,zz */
void grad_to_stress(const V3 &u, double mu, double lambda, double s[6])
{
    double exx = u.c[0].d[0], eyy = u.c[1].d[1], ezz = u.c[2].d[2];
    double exy = 0.5 * (u.c[0].d[1] + u.c[1].d[0]);
    double exz = 0.5 * (u.c[0].d[2] + u.c[2].d[0]);
    double eyz = 0.5 * (u.c[1].d[2] + u.c[2].d[1]);
    double kk = exx + eyy + ezz;
    s[0] = 2.0 * mu * exx + lambda * kk;
    s[1] = 2.0 * mu * exy;
    s[2] = 2.0 * mu * exz;
    s[3] = 2.0 * mu * eyy + lambda * kk;
    s[4] = 2.0 * mu * eyz;
    s[5] = 2.0 * mu * ezz + lambda * kk;
}

} // namespace

/* straininhalfspace_ semantics (ENU in, xx,xy,xz,yy,yz,zz stress out) */
static void nw15_enu(double X, double Y, double Z, const double P1[3], const double P2[3],
                     const double P3[3], double Ss, double Ds, double Ts, double mu,
                     double lambda, double out[6])
{
    double nu = lambda / (lambda + mu) / 2.0;
    D3 Xd[3] = {D3::var(X, 0), D3::var(Y, 1), D3::var(Z, 2)};
    double M1[3] = {P1[0], P1[1], -P1[2]}, M2[3] = {P2[0], P2[1], -P2[2]}, M3[3] = {P3[0], P3[1], -P3[2]};
    double sm[6], sh[6], si[6];
    grad_to_stress(td_disp_fs(Xd, P1, P2, P3, Ss, Ds, Ts, nu), mu, lambda, sm);
    grad_to_stress(td_disp_harm(Xd, P1, P2, P3, Ss, Ds, Ts, nu), mu, lambda, sh);
    grad_to_stress(td_disp_fs(Xd, M1, M2, M3, Ss, Ds, Ts, nu), mu, lambda, si);
    if (M1[2] == 0.0 && M2[2] == 0.0 && M3[2] == 0.0) { si[4] = -si[4]; si[5] = -si[5]; }
    for (int k = 0; k < 6; k++) out[k] = sm[k] + si[k] + sh[k];
}

extern "C" void orc_nw15_stress(double x1, double x2, double x3, const double P1[3],
                                const double P2[3], const double P3[3], double s, double d,
                                double t, double G, double lambda, double sig[6])
{
    double Q1[3] = {P1[1], P1[0], -P1[2]}, Q2[3] = {P2[1], P2[0], -P2[2]}, Q3[3] = {P3[1], P3[0], -P3[2]};
    double e[6];
    nw15_enu(x2, x1, -x3, Q1, Q2, Q3, s, -d, t, G, lambda, e);
    sig[0] = e[3];
    sig[1] = e[1];
    sig[2] = -e[4];
    sig[3] = e[0];
    sig[4] = -e[2];
    sig[5] = e[5];
}

/* computeDisplacementNikkhoo15 (nikkhoo15.f90:324-367) over TDdispHS
   (DispInHalfSpace.c:27-147): the values of the same displacement fields whose
   gradients give the stress; NED in and out, dip slip negated. */
extern "C" void orc_nw15_disp(double x1, double x2, double x3, const double P1[3], const double P2[3],
                              const double P3[3], double s, double d, double t, double G, double lambda,
                              double u[3])
{
    const double nu = lambda / (lambda + G) / 2.0;
    const double Q1[3] = {P1[1], P1[0], -P1[2]}, Q2[3] = {P2[1], P2[0], -P2[2]}, Q3[3] = {P3[1], P3[0], -P3[2]};
    const double M1[3] = {Q1[0], Q1[1], -Q1[2]}, M2[3] = {Q2[0], Q2[1], -Q2[2]}, M3[3] = {Q3[0], Q3[1], -Q3[2]};
    D3 Xd[3] = {D3::var(x2, 0), D3::var(x1, 1), D3::var(-x3, 2)};
    V3 ms = td_disp_fs(Xd, Q1, Q2, Q3, s, -d, t, nu);
    V3 hs = td_disp_harm(Xd, Q1, Q2, Q3, s, -d, t, nu);
    V3 is = td_disp_fs(Xd, M1, M2, M3, s, -d, t, nu);
    const bool surf = M1[2] == 0.0 && M2[2] == 0.0 && M3[2] == 0.0;
    double e[3];
    for (int k = 0; k < 3; k++) {
        double iv = is.c[k].v;
        if (surf && k == 2) iv = -iv;
        e[k] = ms.c[k].v + hs.c[k].v + iv;
        if (surf) e[k] = -e[k];
    }
    u[0] = e[1];
    u[1] = e[0];
    u[2] = -e[2];
}

/* computeReferenceSystemNikkhoo15 / Stuart97, nikkhoo15.f90:50-101 */
extern "C" void orc_tri_frames(int ns, int nve, const double *v, const int *i1, const int *i2,
                               const int *i3, double *sv, double *dv, double *nv, double *xc)
{
    (void)nve;
    for (int j = 0; j < ns; j++) {
        const double *A = v + 3L * (i1[j] - 1), *B = v + 3L * (i2[j] - 1), *C = v + 3L * (i3[j] - 1);
        double *n = nv + 3L * j, *s = sv + 3L * j, *d = dv + 3L * j;
        n[0] = (B[1] - A[1]) * (C[2] - A[2]) - (B[2] - A[2]) * (C[1] - A[1]);
        n[1] = (B[2] - A[2]) * (C[0] - A[0]) - (B[0] - A[0]) * (C[2] - A[2]);
        n[2] = (B[0] - A[0]) * (C[1] - A[1]) - (B[1] - A[1]) * (C[0] - A[0]);
        double norm = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int k = 0; k < 3; k++) n[k] = n[k] / norm;
        if (0.0 < n[2]) for (int k = 0; k < 3; k++) n[k] = -n[k];
        s[0] = std::cos(std::atan2(n[0], n[1]));
        s[1] = -std::sin(std::atan2(n[0], n[1]));
        s[2] = 0.0;
        d[0] = n[1] * s[2] - n[2] * s[1];
        d[1] = n[2] * s[0] - n[0] * s[2];
        d[2] = n[0] * s[1] - n[1] * s[0];
        for (int k = 0; k < 3; k++) xc[3L * j + k] = (A[k] + B[k] + C[k]) / 3.0;
    }
}
