/*
 * Oracle: Barbot, Moore & Lambert (2017) vertical strain volume.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference (computeStressVerticalStrainVolume, fortran/3d/src/
 * strainvolume.f90:1042-4640) evaluates hand-derived derivative integrals and
 * cannot be built here (no Fortran compiler).  This restatement takes the
 * published displacement integrals (computeDisplacementVerticalStrainVolume,
 * strainvolume.f90:215-991, as coded in unicycle_b200/csrc/bml17_disp.h) and
 * differentiates them NUMERICALLY -- Richardson-extrapolated central
 * differences -- independently of the device path, which differentiates them
 * exactly with dual numbers.  The integrals cancel heavily (sums of terms up to
 * ~1e6 times the result), so the displacements are evaluated in x87 extended
 * precision (long double, 64-bit significand): a binary64 difference quotient
 * would carry errors near 1e-6 of the stress, the extended one about 1e-9.  Strain rotation, eigenstrain removal and Hooke's
 * law follow strainvolume.f90:1108-1140.  Pins: physical identities (the
 * free surface is traction free, a cuboid split in two sums to the whole, a
 * thin cuboid in shear matches an Okada dislocation), tests/test_oracle.py.
 */
#include <cmath>
#include <cstdlib>
#include "oracle.h"

typedef long double xreal;
static inline xreal sv_sqrt(xreal a) { return sqrtl(a); }
static inline xreal sv_log(xreal a) { return logl(a); }
static inline xreal sv_atan(xreal a) { return atanl(a); }
static inline xreal sv_atan2(xreal y, xreal x) { return atan2l(y, x); }
static inline double sv_val(xreal a) { return (double)a; }

#include "../unicycle_b200/csrc/bml17_disp.h"

namespace {

/* u_i for eigenstrain eps (cuboid frame), observation in the cuboid frame */
void disp(xreal x1p, xreal x2p, xreal x3, double q3, double L, double T, double W, const double eps[6],
          double G, double nu, xreal u[3])
{
    xreal uq[6][3];
    bml17::displacement<-1, xreal>(x1p, x2p, x3, q3, L, T, W, nu, G, uq);
    for (int i = 0; i < 3; i++) {
        xreal s = 0.0L;
        for (int q = 0; q < 6; q++) s += eps[q] * uq[q][i];
        u[i] = s;
    }
}

double heav(double x) { return (0.0 < x) ? 1.0 : 0.0; }
double omega(double x) { return heav(x + 0.5) - heav(x - 0.5); }
double sbox(double x) { return omega(x - 0.5); }

}  // namespace

extern "C" void orc_bml17_stress(double x1, double x2, double x3, double q1, double q2, double q3,
                                 double L, double T, double W, double theta, const double eps[6],
                                 double G, double nu, double sig[6])
{
    const double ct = std::cos(theta), st = std::sin(theta);
    const double x1p = (x1 - q1) * ct + (x2 - q2) * st;
    const double x2p = -(x1 - q1) * st + (x2 - q2) * ct;
    const xreal h = 1.0e-3L * std::fmin(L, std::fmin(T, W));
    double grad[3][3];  /* grad[i][d] = d u_i / d x_d (cuboid frame) */
    for (int d = 0; d < 3; d++) {
        xreal up1[3], um1[3], up2[3], um2[3];
        xreal p[3] = {x1p, x2p, x3};
        if (d == 2 && x3 < 4 * h) {
            /* next to the free surface: one-sided fourth-order stencil below it */
            xreal f[5][3];
            for (int k = 0; k < 5; k++) disp(x1p, x2p, x3 + k * h, q3, L, T, W, eps, G, nu, f[k]);
            for (int i = 0; i < 3; i++)
                grad[i][2] = (double)((-25.0L * f[0][i] + 48.0L * f[1][i] - 36.0L * f[2][i] + 16.0L * f[3][i] -
                                       3.0L * f[4][i]) / (12.0L * h));
            continue;
        }
        p[d] += h;       disp(p[0], p[1], p[2], q3, L, T, W, eps, G, nu, up1);
        p[d] -= 2 * h;   disp(p[0], p[1], p[2], q3, L, T, W, eps, G, nu, um1);
        p[d] += 3 * h;   disp(p[0], p[1], p[2], q3, L, T, W, eps, G, nu, up2);
        p[d] -= 4 * h;   disp(p[0], p[1], p[2], q3, L, T, W, eps, G, nu, um2);
        for (int i = 0; i < 3; i++) {
            const xreal d1 = (up1[i] - um1[i]) / (2 * h);
            const xreal d2 = (up2[i] - um2[i]) / (4 * h);
            grad[i][d] = (double)((4.0L * d1 - d2) / 3.0L);
        }
    }
    const double lambda = G * 2.0 * nu / (1 - 2 * nu);
    const double e11p = grad[0][0], e22p = grad[1][1], e33 = grad[2][2];
    const double e12p = (grad[0][1] + grad[1][0]) / 2, e13p = (grad[0][2] + grad[2][0]) / 2;
    const double e23p = (grad[1][2] + grad[2][1]) / 2;
    double e11 = (ct * e11p - st * e12p) * ct - (ct * e12p - st * e22p) * st;
    double e12 = (ct * e11p - st * e12p) * st + (ct * e12p - st * e22p) * ct;
    double e13 = ct * e13p - st * e23p;
    double e22 = (st * e11p + ct * e12p) * st + (st * e12p + ct * e22p) * ct;
    double e23 = st * e13p + ct * e23p;
    double e33r = e33;
    const double p11 = eps[0], p12 = eps[1], p13 = eps[2], p22 = eps[3], p23 = eps[4], p33 = eps[5];
    const double eps11 = (ct * p11 - st * p12) * ct - (ct * p12 - st * p22) * st;
    const double eps12 = (ct * p11 - st * p12) * st + (ct * p12 - st * p22) * ct;
    const double eps13 = ct * p13 - st * p23;
    const double eps22 = (st * p11 + ct * p12) * st + (st * p12 + ct * p22) * ct;
    const double eps23 = st * p13 + ct * p23;
    const double inside = sbox(x1p / L) * omega(x2p / T) * sbox((x3 - q3) / W);
    e11 -= eps11 * inside;
    e12 -= eps12 * inside;
    e13 -= eps13 * inside;
    e22 -= eps22 * inside;
    e23 -= eps23 * inside;
    e33r -= p33 * inside;
    const double kk = e11 + e22 + e33r;
    sig[0] = lambda * kk + 2 * G * e11;
    sig[1] = 2 * G * e12;
    sig[2] = 2 * G * e13;
    sig[3] = lambda * kk + 2 * G * e22;
    sig[4] = 2 * G * e23;
    sig[5] = lambda * kk + 2 * G * e33r;
}

/* computeReferenceSystemVerticalStrainVolume, strainvolume.f90:135-163 */
extern "C" void orc_vol_frames(int ns, const double *x, const double *L, const double *W,
                               const double *strike, double *sv, double *dv, double *nv,
                               double *xc)
{
    for (int i = 0; i < ns; i++) {
        sv[3 * i + 0] = std::cos(strike[i]);
        sv[3 * i + 1] = std::sin(strike[i]);
        sv[3 * i + 2] = 0.0;
        dv[3 * i + 0] = 0.0;
        dv[3 * i + 1] = 0.0;
        dv[3 * i + 2] = -1.0;
        nv[3 * i + 0] = -std::sin(strike[i]);
        nv[3 * i + 1] = +std::cos(strike[i]);
        nv[3 * i + 2] = -0.0;
        for (int k = 0; k < 3; k++)
            xc[3 * i + k] = x[3 * i + k] + L[i] / 2 * sv[3 * i + k] - W[i] / 2 * dv[3 * i + k];
    }
}

/* displacement for tests (cuboid-frame observation, eigenstrain eps) */
extern "C" void orc_bml17_disp(double x1p, double x2p, double x3, double q3, double L, double T, double W,
                               const double eps[6], double G, double nu, double u[3])
{
    xreal ux[3];
    disp(x1p, x2p, x3, q3, L, T, W, eps, G, nu, ux);
    for (int i = 0; i < 3; i++) u[i] = (double)ux[i];
}

/* computeDisplacementVerticalStrainVolume, strainvolume.f90:215-991:
   displacement (north, east, down) at x from eigenstrain eps (cuboid frame) */
extern "C" void orc_bml17_disp_ned(double x1, double x2, double x3, double q1, double q2, double q3, double L,
                                   double T, double W, double theta, const double eps[6], double G, double nu,
                                   double u[3])
{
    const double ct = std::cos(theta), st = std::sin(theta);
    const double x1p = (x1 - q1) * ct + (x2 - q2) * st;
    const double x2p = -(x1 - q1) * st + (x2 - q2) * ct;
    xreal up[3];
    disp(x1p, x2p, x3, q3, L, T, W, eps, G, nu, up);
    u[0] = (double)up[0] * ct - (double)up[1] * st;
    u[1] = (double)up[0] * st + (double)up[1] * ct;
    u[2] = (double)up[2];
}
