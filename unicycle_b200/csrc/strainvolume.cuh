// Barbot, Moore & Lambert (2017) vertical cuboid strain volume, device side:
// stress at a receiver due to the six unit anelastic eigenstrains of one
// cuboid, all at once.
//
// Follows computeStressVerticalStrainVolume (fortran/3d/src/strainvolume.f90:
// 1042-1140): rotate the receiver into the cuboid frame, form the displacement
// gradient, rotate the strain back, remove the eigenstrain inside the cuboid
// (1124-1131), Hooke with lambda = 2 G nu / (1 - 2 nu).  The gradient is the
// exact derivative of the published displacement integrals (bml17_disp.h),
// evaluated on dual numbers, one displacement component per pass so that the
// live state of each pass stays in registers.
#pragma once
#include <cuda_runtime.h>
#include "dual.cuh"

namespace ucg {

// scalar hooks of bml17_disp.h for the three-direction dual
__device__ __forceinline__ Dd sv_sqrt(Dd a) { return dsqrt(a); }
__device__ __forceinline__ Dd sv_log(Dd a) { return dlog(a); }
__device__ __forceinline__ Dd sv_atan(Dd a) { return datan(a); }
__device__ __forceinline__ Dd sv_atan2(Dd y, Dd x) { return datan2(y, x); }
__device__ __forceinline__ double sv_val(Dd a) { return a.v; }

}  // namespace ucg

// and for plain doubles (observation-point displacements); declared in the
// integrals' namespace so that the unqualified calls there find them
namespace bml17 {
__host__ __device__ __forceinline__ double sv_sqrt(double a) { return sqrt(a); }
__host__ __device__ __forceinline__ double sv_log(double a) { return log(a); }
__host__ __device__ __forceinline__ double sv_atan(double a) { return atan(a); }
__host__ __device__ __forceinline__ double sv_atan2(double y, double x) { return atan2(y, x); }
__host__ __device__ __forceinline__ double sv_val(double a) { return a; }
}  // namespace bml17

#include "bml17_disp.h"

namespace ucg {

constexpr bool kVolumesBuilt = true;

enum : int { SV_Q1 = 0, SV_Q2, SV_Q3, SV_L, SV_T, SV_W, SV_C, SV_S, SV_SIZE };

struct SvRec {
    const double *__restrict__ base;
    long stride;
    __device__ __forceinline__ double operator[](int f) const { return __ldg(base + (long)f * stride); }
};

inline void sv_prepare(const double *x, double L, double T, double W, double strike, double *r)
{
    r[SV_Q1] = x[0]; r[SV_Q2] = x[1]; r[SV_Q3] = x[2];
    r[SV_L] = L; r[SV_T] = T; r[SV_W] = W;
    r[SV_C] = cos(strike); r[SV_S] = sin(strike);
}

// boxcar functions of strainvolume.f90:53-84
__device__ __forceinline__ double sv_heaviside(double x) { return (0.0 < x) ? 1.0 : 0.0; }
__device__ __forceinline__ double sv_omega(double x) { return sv_heaviside(x + 0.5) - sv_heaviside(x - 0.5); }
__device__ __forceinline__ double sv_s(double x) { return sv_omega(x - 0.5); }

template <int COMP>
__device__ __forceinline__ void sv_grad_pass(double x1p, double x2p, double x3, const SvRec &R, double mu,
                                             double nu, double g[6][3][3])
{
    const Dd X1{x1p, 1.0, 0.0, 0.0}, X2{x2p, 0.0, 1.0, 0.0}, X3{x3, 0.0, 0.0, 1.0};
    Dd u[6][3];
    bml17::displacement<COMP>(X1, X2, X3, R[SV_Q3], R[SV_L], R[SV_T], R[SV_W], nu, mu, u);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        g[q][COMP][0] = u[q][COMP].x;
        g[q][COMP][1] = u[q][COMP].y;
        g[q][COMP][2] = u[q][COMP].z;
    }
}

// sig[q][0..5] = s11, s12, s13, s22, s23, s33 (NED) for unit eigenstrain q
// (11, 12, 13, 22, 23, 33 in the cuboid frame)
__device__ inline void sv_pair_stress(const double *rc, const SvRec &R, double mu, double nu, double sig[6][6])
{
    const double ct = R[SV_C], st = R[SV_S];
    const double x1 = rc[0], x2 = rc[1], x3 = rc[2];
    const double x1p = (x1 - R[SV_Q1]) * ct + (x2 - R[SV_Q2]) * st;
    const double x2p = -(x1 - R[SV_Q1]) * st + (x2 - R[SV_Q2]) * ct;
    double g[6][3][3];
    sv_grad_pass<0>(x1p, x2p, x3, R, mu, nu, g);
    sv_grad_pass<1>(x1p, x2p, x3, R, mu, nu, g);
    sv_grad_pass<2>(x1p, x2p, x3, R, mu, nu, g);
    const double lambda = mu * 2.0 * nu / (1.0 - 2.0 * nu);
    const double inside = sv_s(x1p / R[SV_L]) * sv_omega(x2p / R[SV_T]) * sv_s((x3 - R[SV_Q3]) / R[SV_W]);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const double e11p = g[q][0][0], u12 = g[q][0][1], u13 = g[q][0][2];
        const double u21 = g[q][1][0], e22p = g[q][1][1], u23 = g[q][1][2];
        const double u31 = g[q][2][0], u32 = g[q][2][1], e33 = g[q][2][2];
        const double e12p = (u12 + u21) / 2, e13p = (u13 + u31) / 2, e23p = (u23 + u32) / 2;
        // strainvolume.f90:1108-1122
        double e11 = (ct * e11p - st * e12p) * ct - (ct * e12p - st * e22p) * st;
        double e12 = (ct * e11p - st * e12p) * st + (ct * e12p - st * e22p) * ct;
        double e13 = ct * e13p - st * e23p;
        double e22 = (st * e11p + ct * e12p) * st + (st * e12p + ct * e22p) * ct;
        double e23 = st * e13p + ct * e23p;
        double e33r = e33;
        // unit eigenstrain q in the cuboid frame, rotated the same way
        const double p11 = q == 0, p12 = q == 1, p13 = q == 2, p22 = q == 3, p23 = q == 4, p33 = q == 5;
        const double eps11 = (ct * p11 - st * p12) * ct - (ct * p12 - st * p22) * st;
        const double eps12 = (ct * p11 - st * p12) * st + (ct * p12 - st * p22) * ct;
        const double eps13 = ct * p13 - st * p23;
        const double eps22 = (st * p11 + ct * p12) * st + (st * p12 + ct * p22) * ct;
        const double eps23 = st * p13 + ct * p23;
        const double eps33 = p33;
        e11 = e11 - eps11 * inside;
        e12 = e12 - eps12 * inside;
        e13 = e13 - eps13 * inside;
        e22 = e22 - eps22 * inside;
        e23 = e23 - eps23 * inside;
        e33r = e33r - eps33 * inside;
        const double kk = e11 + e22 + e33r;
        sig[q][0] = lambda * kk + 2 * mu * e11;
        sig[q][1] = 2 * mu * e12;
        sig[q][2] = 2 * mu * e13;
        sig[q][3] = lambda * kk + 2 * mu * e22;
        sig[q][4] = 2 * mu * e23;
        sig[q][5] = lambda * kk + 2 * mu * e33r;
    }
}

// Displacement (north, east, down) at xr (NED) for the six unit eigenstrains
// of one cuboid (computeDisplacementVerticalStrainVolume, strainvolume.f90:
// 215-991): the receiver rotated into the cuboid frame, the 8-corner sum of
// the displacement integrals, the horizontal components rotated back.
__device__ inline void sv_pair_disp(const double xr[3], const SvRec &R, double mu, double nu, double u[6][3])
{
    const double ct = R[SV_C], st = R[SV_S];
    const double x1p = (xr[0] - R[SV_Q1]) * ct + (xr[1] - R[SV_Q2]) * st;
    const double x2p = -(xr[0] - R[SV_Q1]) * st + (xr[1] - R[SV_Q2]) * ct;
    double up[6][3];
    bml17::displacement<-1, double>(x1p, x2p, xr[2], R[SV_Q3], R[SV_L], R[SV_T], R[SV_W], nu, mu, up);
#pragma unroll
    for (int q = 0; q < 6; q++) {
        u[q][0] = up[q][0] * ct - up[q][1] * st;
        u[q][1] = up[q][0] * st + up[q][1] * ct;
        u[q][2] = up[q][2];
    }
}

}  // namespace ucg
