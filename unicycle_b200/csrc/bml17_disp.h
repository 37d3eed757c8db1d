// Displacement due to uniform anelastic eigenstrain in a vertical cuboid in an
// elastic half-space: the closed-form indefinite integrals J_ijkl ("James
// integrals") of Barbot, Moore & Lambert (2017), Bull. Seism. Soc. Am. 107(2),
// as evaluated by computeDisplacementVerticalStrainVolume
// (fortran/3d/src/strainvolume.f90:215-991).  The integrals are the published
// closed forms and therefore have to be the same expressions; they are grouped
// here by their recurring sub-terms (d1 = x1'-y1, d2 = x2'-y2, dm = x3-y3,
// dp = x3+y3, r1, r2) and templated on the scalar type, so that evaluating them
// on dual numbers seeded with the observation point gives the exact
// displacement gradient (the reference evaluates hand-derived derivative
// integrals instead, strainvolume.f90:1042-4640).
//
// Requirements on T: arithmetic with T and double, and the free functions
// sv_sqrt, sv_log, sv_atan, sv_atan2 and sv_val (value as double).
#pragma once

#ifndef SV_HD
#ifdef __CUDACC__
#define SV_HD __host__ __device__ __forceinline__
#else
#define SV_HD inline
#endif
#endif

namespace bml17 {

// reference helpers, strainvolume.f90:91-120 and macros.f90:7
template <class T> SV_HD T xlogy(const T &x, const T &y)
{
    // 0*log(0) = 0; where the coefficient vanishes the derivative keeps the
    // x' log(y) part whenever log(y) is finite
    if (sv_val(x) == 0.0) {
        if (sv_val(y) > 0.0) return x * sv_log(y);
        return x * 0.0;
    }
    return x * sv_log(y);
}

template <class T> SV_HD T atan3(const T &y, const T &x)
{
    // atan2 with the limit value at x = 0; the derivative is the same as atan2's
    if (sv_val(x) == 0.0) {
        const double h = 1.5707963267948966;
        T r = sv_atan2(y, x);     // supplies the derivative
        return r + ((sv_val(y) >= 0.0 ? h : -h) - sv_val(r));
    }
    return sv_atan(y / x);
}

template <class T> SV_HD T acoth(const T &X)
{
    // 0.5 * Re(log(X+1) - log(X-1)) = 0.5 * (log|X+1| - log|X-1|)
    T a = X + 1.0, b = X - 1.0;
    if (sv_val(a) < 0.0) a = -a;
    if (sv_val(b) < 0.0) b = -b;
    return 0.5 * (sv_log(a) - sv_log(b));
}

// The 27 integrals at one corner (y1, y2, y3) of the cuboid, observation point
// (x1, x2, x3) in the cuboid frame (x1', x2', depth).  Each integral J_ijk
// (i, j in {1,2,3}, k in {12,13,23}) is handed to emit(i-1, j-1, k-index, J) as
// soon as it is formed, so callers can fold it into their sums without holding
// all 27 at once.
template <class T, class F>
SV_HD void corner(const T &x1, const T &x2, const T &x3, double y1, double y2, double y3, double nu,
                  double G, F &&emit)
{
    const double PI = 3.141592653589793115997963468544185161;
    const double c = (1.0 / 16.0) / (1.0 - nu) / PI / G;
    const T d1 = x1 - y1, d2 = x2 - y2, dm = x3 - y3, dp = x3 + y3;
    const T r1 = sv_sqrt(d1 * d1 + d2 * d2 + dm * dm);
    const T r2 = sv_sqrt(d1 * d1 + d2 * d2 + dp * dp);
    const T ir2 = 1.0 / r2;
    const double nm = -1.0 + nu;          // (-1+nu)
    const double n2 = -1.0 + 2.0 * nu;    // (-1+2nu)
    const T d11 = d1 * d1, d22 = d2 * d2, dpp = dp * dp;
    const T s12 = d11 + d22;              // (x1-y1)^2 + (x2-y2)^2
    const T s13 = d11 + dpp;              // (x1-y1)^2 + (x3+y3)^2
    const T s23 = d22 + dpp;              // (x2-y2)^2 + (x3+y3)^2
    // recurring bracket: -(n-1)(2n-1) r2^2 (x3+y3) + (n-1)(2n-1) r2 y3 (2x3+y3) + x3 (s12 + x3 (x3+y3))
    const T Bq = -(nm * n2) * r2 * r2 * dp + nm * n2 * r2 * y3 * (2.0 * x3 + y3) + x3 * (s12 + x3 * dp);

    // J1112, strainvolume.f90:344-367
    emit(0, 0, 0, T(c * (2.0 * ir2 * x3 * d1 * d2 * y3 / s13
        - 4.0 * nm * n2 * dp * atan3(d2, d1)
        - x3 * sv_atan2(x3, d1) - 3.0 * x3 * sv_atan2(3.0 * x3, d1)
        + 4.0 * nu * x3 * sv_atan2(-nu * x3, d1)
        + 4.0 * nm * n2 * dp * sv_atan2(r2 * (-d1), d2 * dp)
        - 4.0 * nm * dm * sv_atan2(r1 * dm, d1 * d2)
        + 3.0 * y3 * sv_atan2(T(-3.0 * y3), d1) - y3 * sv_atan2(T(y3), d1)
        - 4.0 * nu * y3 * sv_atan2(T(nu * y3), d1)
        - 4.0 * nm * dp * sv_atan2(r2 * dp, d1 * d2)
        + xlogy(-(-3.0 + 4.0 * nu) * d1, r1 + d2)
        + xlogy((5.0 + 4.0 * nu * (-3.0 + 2.0 * nu)) * d1, r2 + d2)
        + xlogy(-4.0 * nm * d2, r1 + d1)
        + xlogy(-4.0 * nm * d2, r2 + d1))));
    // J1113, strainvolume.f90:373-396
    emit(0, 0, 1, T(c * (2.0 * ir2 * d1 / s12 * Bq
        + x2 * sv_atan2(-x2, d1) - 3.0 * x2 * sv_atan2(3.0 * x2, d1)
        + 4.0 * nu * x2 * sv_atan2(-nu * x2, d1)
        - 4.0 * nm * d2 * sv_atan2(r1 * d2, d1 * dm)
        + 4.0 * nm * d2 * sv_atan2(r2 * d2, d1 * dp)
        + 3.0 * y2 * sv_atan2(T(-3.0 * y2), d1) - y2 * sv_atan2(T(y2), d1)
        - 4.0 * nu * y2 * sv_atan2(T(nu * y2), d1)
        + xlogy(-(-3.0 + 4.0 * nu) * d1, r1 + dm)
        + xlogy(-(3.0 - 6.0 * nu + 4.0 * nu * nu) * d1, r2 + dp)
        + xlogy(-4.0 * nm * dm, r1 + d1)
        + xlogy(4.0 * nm * dp, r2 + d1))));
    // J1123, strainvolume.f90:402-430
    emit(0, 0, 2, T(c * (-2.0 * ir2 / s12 * d2 / s13
            * (x3 * ((x3 * x3 + d11) * (x3 * x3 + d11 + d22) + x3 * (3.0 * x3 * x3 + 2.0 * d11 + d22) * y3
                     + 3.0 * x3 * x3 * y3 * y3 + x3 * y3 * y3 * y3)
               - nm * n2 * r2 * r2 * dp * s13 + nm * n2 * r2 * y3 * (2.0 * x3 + y3) * s13)
        + 2.0 * nm * n2 * d1 * atan3(d1, d2)
        + x1 * sv_atan2(-x1, d2) - 3.0 * x1 * sv_atan2(3.0 * x1, d2)
        + 4.0 * nu * x1 * sv_atan2(-nu * x1, d2)
        + 3.0 * y1 * sv_atan2(T(-3.0 * y1), d2) - y1 * sv_atan2(T(y1), d2)
        - 4.0 * nu * y1 * sv_atan2(T(nu * y1), d2)
        + 2.0 * n2 * d1 * sv_atan2(r1 * (-d1), d2 * dm)
        + 2.0 * (1.0 - 2.0 * nu) * (1.0 - 2.0 * nu) * d1 * sv_atan2(r2 * (-d1), d2 * dp)
        + xlogy(-2.0 * x3, r2 - d2)
        + xlogy(-(-3.0 + 4.0 * nu) * d2, r1 + dm)
        + xlogy(-(3.0 - 6.0 * nu + 4.0 * nu * nu) * d2, r2 + dp)
        + xlogy(-(-3.0 + 4.0 * nu) * dm, r1 + d2)
        + xlogy(-(5.0 + 4.0 * nu * (-3.0 + 2.0 * nu)) * dp, r2 + d2))));
    // J2112 = J1212, strainvolume.f90:436-448, 560-572
    const T j2112 = c * (-r1 + (1.0 + 8.0 * nm * nu) * r2 - 2.0 * ir2 * x3 * y3
        + xlogy(-4.0 * nm * n2 * dp, r2 + dp));
    emit(1, 0, 0, T(j2112));
    emit(0, 1, 0, T(j2112));
    // J2113 = J1213, strainvolume.f90:454-469, 578-593
    const T j2113 = c * (2.0 * ir2 / s12 * d2 * Bq
        + xlogy(-(-1.0 - 2.0 * nu + 4.0 * nu * nu) * d2, r2 + dp)
        + xlogy(-d2, r1 + dm));
    emit(1, 0, 1, T(j2113));
    emit(0, 1, 1, T(j2113));
    // J2123 = J1223, strainvolume.f90:475-490, 599-614
    const T j2123 = c * (2.0 * ir2 * d1 / s12 * Bq
        + xlogy(-(-1.0 - 2.0 * nu + 4.0 * nu * nu) * d1, r2 + dp)
        + xlogy(-d1, r1 + dm));
    emit(1, 0, 2, T(j2123));
    emit(0, 1, 2, T(j2123));
    // J3112, strainvolume.f90:496-513
    emit(2, 0, 0, T(-c * (-2.0 * ir2 * x3 * d2 * y3 * dp / s13
        + 4.0 * nm * n2 * d1 * atan3(d1, d2)
        + 4.0 * nm * n2 * d1 * sv_atan2(r2 * (-d1), d2 * dp)
        + xlogy(-4.0 * nm * n2 * d2, r2 + dp)
        + xlogy(dm, r1 + d2)
        + xlogy(-x3 - 7.0 * y3 - 8.0 * nu * nu * dp + 8.0 * nu * (x3 + 2.0 * y3), r2 + d2))));
    // J3113, strainvolume.f90:519-532
    emit(2, 0, 1, T(-c * (r1 + (-1.0 - 8.0 * nm * nu) * r2 - 2.0 * ir2 * x3 * y3
        + 2.0 * (-3.0 + 4.0 * nu) * x3 * acoth(ir2 * dp)
        + xlogy(2.0 * (3.0 * x3 + 2.0 * y3 - 6.0 * nu * dp + 4.0 * nu * nu * dp), r2 + dp))));
    // J3123, strainvolume.f90:538-554
    emit(2, 0, 2, T(-c * (2.0 * ir2 * x3 * d1 * d2 * y3 / s13
        + 4.0 * nm * n2 * dp * atan3(d2, d1)
        + 4.0 * n2 * (nu * x3 + nm * y3) * sv_atan2(r2 * d1, d2 * dp)
        + xlogy(d1, r1 + d2)
        + xlogy(-(1.0 + 8.0 * nm * nu) * d1, r2 + d2))));
    // J2212, strainvolume.f90:620-643
    emit(1, 1, 0, T(c * (2.0 * ir2 * x3 * d1 * d2 * y3 / s23
        - 4.0 * nm * n2 * dp * atan3(d1, d2)
        - x3 * sv_atan2(x3, d1) - 3.0 * x3 * sv_atan2(3.0 * x3, d1)
        + 4.0 * nu * x3 * sv_atan2(-nu * x3, d1)
        + 4.0 * nm * n2 * dp * sv_atan2(r2 * (-d2), d1 * dp)
        - 4.0 * nm * dm * sv_atan2(r1 * dm, d1 * d2)
        + 3.0 * y3 * sv_atan2(T(-3.0 * y3), d1) - y3 * sv_atan2(T(y3), d1)
        - 4.0 * nu * y3 * sv_atan2(T(nu * y3), d1)
        - 4.0 * nm * dp * sv_atan2(r2 * dp, d1 * d2)
        + xlogy(-4.0 * nm * d1, r1 + d2)
        + xlogy(-4.0 * nm * d1, r2 + d2)
        + xlogy(-(-3.0 + 4.0 * nu) * d2, r1 + d1)
        + xlogy((5.0 + 4.0 * nu * (-3.0 + 2.0 * nu)) * d2, r2 + d1))));
    // J2213, strainvolume.f90:649-677
    emit(1, 1, 1, T(c * (-2.0 * ir2 * d1 / s12 / s23
            * (x3 * ((x3 * x3 + d22) * (x3 * x3 + d11 + d22) + x3 * (3.0 * x3 * x3 + d11 + 2.0 * d22) * y3
                     + 3.0 * x3 * x3 * y3 * y3 + x3 * y3 * y3 * y3)
               - nm * n2 * r2 * r2 * dp * s23 + nm * n2 * r2 * y3 * (2.0 * x3 + y3) * s23)
        + 2.0 * nm * n2 * d2 * atan3(d2, d1)
        + x2 * sv_atan2(-x2, d1) - 3.0 * x2 * sv_atan2(3.0 * x2, d1)
        + 4.0 * nu * x2 * sv_atan2(-nu * x2, d1)
        + 3.0 * y2 * sv_atan2(T(-3.0 * y2), d1) - y2 * sv_atan2(T(y2), d1)
        - 4.0 * nu * y2 * sv_atan2(T(nu * y2), d1)
        + 2.0 * n2 * d2 * sv_atan2(r1 * (-d2), d1 * dm)
        + 2.0 * (1.0 - 2.0 * nu) * (1.0 - 2.0 * nu) * d2 * sv_atan2(r2 * (-d2), d1 * dp)
        + xlogy(-2.0 * x3, r2 - d1)
        + xlogy(-(-3.0 + 4.0 * nu) * d1, r1 + dm)
        + xlogy(-(3.0 - 6.0 * nu + 4.0 * nu * nu) * d1, r2 + dp)
        + xlogy(-(-3.0 + 4.0 * nu) * dm, r1 + d1)
        + xlogy(-(5.0 + 4.0 * nu * (-3.0 + 2.0 * nu)) * dp, r2 + d1))));
    // J2223, strainvolume.f90:683-706
    emit(1, 1, 2, T(c * (2.0 * ir2 / s12 * d2 * Bq
        + x1 * sv_atan2(-x1, d2) - 3.0 * x1 * sv_atan2(3.0 * x1, d2)
        + 4.0 * nu * x1 * sv_atan2(-nu * x1, d2)
        - 4.0 * nm * d1 * sv_atan2(r1 * d1, d2 * dm)
        + 4.0 * nm * d1 * sv_atan2(r2 * d1, d2 * dp)
        + 3.0 * y1 * sv_atan2(T(-3.0 * y1), d2) - y1 * sv_atan2(T(y1), d2)
        - 4.0 * nu * y1 * sv_atan2(T(nu * y1), d2)
        + xlogy(-(-3.0 + 4.0 * nu) * d2, r1 + dm)
        + xlogy(-(3.0 - 6.0 * nu + 4.0 * nu * nu) * d2, r2 + dp)
        + xlogy(-4.0 * nm * dm, r1 + d2)
        + xlogy(4.0 * nm * dp, r2 + d2))));
    // J3212, strainvolume.f90:712-729
    emit(2, 1, 0, T(-c * (-2.0 * ir2 * x3 * d1 * y3 * dp / s23
        + 4.0 * nm * n2 * d2 * atan3(d2, d1)
        + 4.0 * nm * n2 * d2 * sv_atan2(r2 * (-d2), d1 * dp)
        + xlogy(-4.0 * nm * n2 * d1, r2 + dp)
        + xlogy(dm, r1 + d1)
        + xlogy(-x3 - 7.0 * y3 - 8.0 * nu * nu * dp + 8.0 * nu * (x3 + 2.0 * y3), r2 + d1))));
    // J3213, strainvolume.f90:735-751
    emit(2, 1, 1, T(-c * (2.0 * ir2 * x3 * d1 * d2 * y3 / s23
        + 4.0 * nm * n2 * dp * atan3(d1, d2)
        + 4.0 * n2 * (nu * x3 + nm * y3) * sv_atan2(r2 * d2, d1 * dp)
        + xlogy(d2, r1 + d1)
        + xlogy(-(1.0 + 8.0 * nm * nu) * d2, r2 + d1))));
    // J3223, strainvolume.f90:757-770
    emit(2, 1, 2, T(-c * (r1 + (-1.0 - 8.0 * nm * nu) * r2 - 2.0 * ir2 * x3 * y3
        + 2.0 * (-3.0 + 4.0 * nu) * x3 * acoth(ir2 * dp)
        + xlogy(2.0 * (3.0 * x3 + 2.0 * y3 - 6.0 * nu * dp + 4.0 * nu * nu * dp), r2 + dp))));
    // J1312, strainvolume.f90:776-793
    emit(0, 2, 0, T(-c * (2.0 * ir2 * x3 * d2 * y3 * dp / s13
        - 4.0 * nm * n2 * d1 * atan3(d1, d2)
        + 4.0 * nm * n2 * d1 * sv_atan2(r2 * d1, d2 * dp)
        + xlogy(4.0 * nm * n2 * d2, r2 + dp)
        + xlogy(dm, r1 + d2)
        + xlogy((7.0 + 8.0 * (-2.0 + nu) * nu) * x3 + y3 + 8.0 * nm * nu * y3, r2 + d2))));
    // J1313, strainvolume.f90:799-812
    emit(0, 2, 1, T(-c * (r1 + ir2 * ((7.0 + 8.0 * (-2.0 + nu) * nu) * r2 * r2 + 2.0 * x3 * y3)
        + 2.0 * (-3.0 + 4.0 * nu) * x3 * acoth(ir2 * dp)
        + xlogy(2.0 * (-3.0 * x3 - 2.0 * y3 + 6.0 * nu * dp - 4.0 * nu * nu * dp), r2 + dp))));
    // J1323, strainvolume.f90:818-834
    emit(0, 2, 2, T(-c * (-2.0 * ir2 * x3 * d1 * d2 * y3 / s13
        - 4.0 * nm * n2 * dp * atan3(d2, d1)
        - 4.0 * nm * (-3.0 * x3 - y3 + 2.0 * nu * dp) * sv_atan2(r2 * d1, d2 * dp)
        + xlogy(d1, r1 + d2)
        + xlogy((7.0 + 8.0 * (-2.0 + nu) * nu) * d1, r2 + d2))));
    // J2312, strainvolume.f90:840-857
    emit(1, 2, 0, T(-c * (2.0 * ir2 * x3 * d1 * y3 * dp / s23
        - 4.0 * nm * n2 * d2 * atan3(d2, d1)
        + 4.0 * nm * n2 * d2 * sv_atan2(r2 * d2, d1 * dp)
        + xlogy(4.0 * nm * n2 * d1, r2 + dp)
        + xlogy(dm, r1 + d1)
        + xlogy((7.0 + 8.0 * (-2.0 + nu) * nu) * x3 + y3 + 8.0 * nm * nu * y3, r2 + d1))));
    // J2313, strainvolume.f90:863-879
    emit(1, 2, 1, T(-c * (-2.0 * ir2 * x3 * d1 * d2 * y3 / s23
        - 4.0 * nm * n2 * dp * atan3(d1, d2)
        - 4.0 * nm * (-3.0 * x3 - y3 + 2.0 * nu * dp) * sv_atan2(r2 * d2, d1 * dp)
        + xlogy(d2, r1 + d1)
        + xlogy((7.0 + 8.0 * (-2.0 + nu) * nu) * d2, r2 + d1))));
    // J2323, strainvolume.f90:885-898
    emit(1, 2, 2, T(-c * (r1 + ir2 * ((7.0 + 8.0 * (-2.0 + nu) * nu) * r2 * r2 + 2.0 * x3 * y3)
        + 2.0 * (-3.0 + 4.0 * nu) * x3 * acoth(ir2 * dp)
        + xlogy(2.0 * (-3.0 * x3 - 2.0 * y3 + 6.0 * nu * dp - 4.0 * nu * nu * dp), r2 + dp))));
    // J3312, strainvolume.f90:904-929
    emit(2, 2, 0, T(c * (2.0 * ir2 * x3 * d1 * d2 * y3 / s13 / s23 * (d11 + d22 + 2.0 * dpp)
        - 3.0 * x3 * sv_atan2(3.0 * x3, d1) - 5.0 * x3 * sv_atan2(5.0 * x3, d2)
        + 12.0 * nu * x3 * sv_atan2(-3.0 * nu * x3, d2) + 4.0 * nu * x3 * sv_atan2(-nu * x3, d1)
        - 8.0 * nu * nu * x3 * sv_atan2(nu * nu * x3, d2)
        + 3.0 * y3 * sv_atan2(T(-3.0 * y3), d1) - 5.0 * y3 * sv_atan2(T(5.0 * y3), d2)
        + 12.0 * nu * y3 * sv_atan2(T(-3.0 * nu * y3), d2) - 4.0 * nu * y3 * sv_atan2(T(nu * y3), d1)
        - 8.0 * nu * nu * y3 * sv_atan2(T(nu * nu * y3), d2)
        + 2.0 * n2 * dm * sv_atan2(r1 * (-dm), d1 * d2)
        + 2.0 * (1.0 - 2.0 * nu) * (1.0 - 2.0 * nu) * dp * sv_atan2(r2 * dp, d1 * d2)
        + xlogy(-(-3.0 + 4.0 * nu) * d1, r1 + d2)
        + xlogy((5.0 + 4.0 * nu * (-3.0 + 2.0 * nu)) * d1, r2 + d2)
        + xlogy(-(-3.0 + 4.0 * nu) * d2, r1 + d1)
        + xlogy((5.0 + 4.0 * nu * (-3.0 + 2.0 * nu)) * d2, r2 + d1))));
    // J3313, strainvolume.f90:935-959
    emit(2, 2, 1, T(c * (2.0 * ir2 * x3 * d1 * y3 * dp / s23
        + 5.0 * x2 * sv_atan2(-5.0 * x2, d1) - 3.0 * x2 * sv_atan2(3.0 * x2, d1)
        + 4.0 * nu * x2 * sv_atan2(-nu * x2, d1) - 12.0 * nu * x2 * sv_atan2(3.0 * nu * x2, d1)
        + 8.0 * nu * nu * x2 * sv_atan2(-nu * nu * x2, d1)
        - 4.0 * nm * d2 * sv_atan2(r1 * d2, d1 * dm)
        - 8.0 * nm * nm * d2 * sv_atan2(r2 * d2, d1 * dp)
        + 3.0 * y2 * sv_atan2(T(-3.0 * y2), d1) - 5.0 * y2 * sv_atan2(T(5.0 * y2), d1)
        + 12.0 * nu * y2 * sv_atan2(T(-3.0 * nu * y2), d1) - 4.0 * nu * y2 * sv_atan2(T(nu * y2), d1)
        - 8.0 * nu * nu * y2 * sv_atan2(T(nu * nu * y2), d1)
        + xlogy(-4.0 * x3, r2 - d1)
        + xlogy(-4.0 * nm * d1, r1 + dm)
        + xlogy(-8.0 * nm * nm * d1, r2 + dp)
        + xlogy(-(-3.0 + 4.0 * nu) * dm, r1 + d1)
        + xlogy(-7.0 * x3 - 5.0 * y3 + 12.0 * nu * dp - 8.0 * nu * nu * dp, r2 + d1))));
    // J3323, strainvolume.f90:965-989
    emit(2, 2, 2, T(c * (2.0 * ir2 * x3 * d2 * y3 * dp / s13
        + 5.0 * x1 * sv_atan2(-5.0 * x1, d2) - 3.0 * x1 * sv_atan2(3.0 * x1, d2)
        + 4.0 * nu * x1 * sv_atan2(-nu * x1, d2) - 12.0 * nu * x1 * sv_atan2(3.0 * nu * x1, d2)
        + 8.0 * nu * nu * x1 * sv_atan2(-nu * nu * x1, d2)
        - 4.0 * nm * d1 * sv_atan2(r1 * d1, d2 * dm)
        - 8.0 * nm * nm * d1 * sv_atan2(r2 * d1, d2 * dp)
        + 3.0 * y1 * sv_atan2(T(-3.0 * y1), d2) - 5.0 * y1 * sv_atan2(T(5.0 * y1), d2)
        + 12.0 * nu * y1 * sv_atan2(T(-3.0 * nu * y1), d2) - 4.0 * nu * y1 * sv_atan2(T(nu * y1), d2)
        - 8.0 * nu * nu * y1 * sv_atan2(T(nu * nu * y1), d2)
        + xlogy(-4.0 * x3, r2 - d2)
        + xlogy(-4.0 * nm * d2, r1 + dm)
        + xlogy(-8.0 * nm * nm * d2, r2 + dp)
        + xlogy(-(-3.0 + 4.0 * nu) * dm, r1 + d2)
        + xlogy(-7.0 * x3 - 5.0 * y3 + 12.0 * nu * dp - 8.0 * nu * nu * dp, r2 + d2))));
}

// Displacement (u1', u2', u3) in the cuboid frame for unit eigenstrain component
// q (0..5: 11, 12, 13, 22, 23, 33), all six at once: u[q][i].
// IU1..IU3 of strainvolume.f90:296-338 and the 8-corner sum of 254-261.
// COMP = 0, 1, 2 forms displacement component COMP+1 only (the other
// integrals are not evaluated); COMP = -1 forms all three.
template <int COMP = -1, class T>
SV_HD void displacement(const T &x1, const T &x2, const T &x3, double q3, double L, double Tk,
                        double W, double nu, double G, T u[6][3])
{
    const double lambda = G * 2.0 * nu / (1.0 - 2.0 * nu);
    for (int q = 0; q < 6; q++)
        for (int i = 0; i < 3; i++) u[q][i] = T(0.0);
    // corners and signs of the 8-term sum
    const double cy1[8] = {L, L, L, L, 0.0, 0.0, 0.0, 0.0};
    const double cy2[8] = {Tk / 2, -Tk / 2, -Tk / 2, Tk / 2, Tk / 2, -Tk / 2, -Tk / 2, Tk / 2};
    const double cy3[8] = {q3 + W, q3 + W, q3, q3, q3 + W, q3 + W, q3, q3};
    const double sg[8] = {1.0, -1.0, 1.0, -1.0, -1.0, 1.0, -1.0, 1.0};
    const double l2g = lambda + 2.0 * G, g2 = 2.0 * G;
    for (int k = 0; k < 8; k++) {
        const double sgk = sg[k];
        // IU_i = (lam ekk + 2G e11) Ji123 + 2G e12 (Ji223 + Ji113) + 2G e13 (Ji323 + Ji112)
        //      + (lam ekk + 2G e22) Ji213 + 2G e23 (Ji212 + Ji313) + (lam ekk + 2G e33) Ji312
        // for the six unit eigenstrains q = 11, 12, 13, 22, 23, 33
        corner(x1, x2, x3, cy1[k], cy2[k], cy3[k], nu, G, [&](int i, int j, int kk, const T &J) {
            if (COMP >= 0 && i != COMP) return;
            const T sJ = sgk * J;
            const int jk = 3 * j + kk;
            switch (jk) {
            case 2:  // J_i123
                u[0][i] = u[0][i] + l2g * sJ; u[3][i] = u[3][i] + lambda * sJ; u[5][i] = u[5][i] + lambda * sJ;
                break;
            case 4:  // J_i213
                u[0][i] = u[0][i] + lambda * sJ; u[3][i] = u[3][i] + l2g * sJ; u[5][i] = u[5][i] + lambda * sJ;
                break;
            case 6:  // J_i312
                u[0][i] = u[0][i] + lambda * sJ; u[3][i] = u[3][i] + lambda * sJ; u[5][i] = u[5][i] + l2g * sJ;
                break;
            case 5:  // J_i223
            case 1:  // J_i113
                u[1][i] = u[1][i] + g2 * sJ;
                break;
            case 8:  // J_i323
            case 0:  // J_i112
                u[2][i] = u[2][i] + g2 * sJ;
                break;
            case 3:  // J_i212
            case 7:  // J_i313
                u[4][i] = u[4][i] + g2 * sJ;
                break;
            }
        });
    }
}

}  // namespace bml17
