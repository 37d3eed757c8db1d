/*
 * Forward-mode dual numbers carrying a value and its gradient with respect to
 * the three observation coordinates.  Used by the oracle to differentiate the
 * closed-form displacement fields of Nikkhoo & Walter (2015) and Barbot et al.
 * (2017) exactly (to rounding), giving displacement gradients, strains and
 * stresses without transcribing the reference's expanded derivative formulas.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#ifndef UCG_ORACLE_DUAL3_H
#define UCG_ORACLE_DUAL3_H
#include <cmath>

struct D3 {
    double v, d[3];
    D3() : v(0), d{0, 0, 0} {}
    D3(double c) : v(c), d{0, 0, 0} {}
    D3(double c, double a, double b, double e) : v(c), d{a, b, e} {}
    static D3 var(double c, int k) { D3 r(c); r.d[k] = 1.0; return r; }
};

inline D3 operator+(const D3 &a, const D3 &b) { return D3(a.v + b.v, a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2]); }
inline D3 operator-(const D3 &a, const D3 &b) { return D3(a.v - b.v, a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2]); }
inline D3 operator-(const D3 &a) { return D3(-a.v, -a.d[0], -a.d[1], -a.d[2]); }
inline D3 operator*(const D3 &a, const D3 &b)
{
    return D3(a.v * b.v, a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1], a.d[2] * b.v + a.v * b.d[2]);
}
inline D3 operator/(const D3 &a, const D3 &b)
{
    double q = a.v / b.v;
    return D3(q, (a.d[0] - q * b.d[0]) / b.v, (a.d[1] - q * b.d[1]) / b.v, (a.d[2] - q * b.d[2]) / b.v);
}
inline D3 operator+(const D3 &a, double c) { return D3(a.v + c, a.d[0], a.d[1], a.d[2]); }
inline D3 operator+(double c, const D3 &a) { return a + c; }
inline D3 operator-(const D3 &a, double c) { return D3(a.v - c, a.d[0], a.d[1], a.d[2]); }
inline D3 operator-(double c, const D3 &a) { return D3(c - a.v, -a.d[0], -a.d[1], -a.d[2]); }
inline D3 operator*(const D3 &a, double c) { return D3(a.v * c, a.d[0] * c, a.d[1] * c, a.d[2] * c); }
inline D3 operator*(double c, const D3 &a) { return a * c; }
inline D3 operator/(const D3 &a, double c) { return D3(a.v / c, a.d[0] / c, a.d[1] / c, a.d[2] / c); }
inline D3 operator/(double c, const D3 &a)
{
    double q = c / a.v, s = -q / a.v;
    return D3(q, s * a.d[0], s * a.d[1], s * a.d[2]);
}
inline D3 &operator+=(D3 &a, const D3 &b) { a = a + b; return a; }
inline D3 &operator-=(D3 &a, const D3 &b) { a = a - b; return a; }

inline D3 chain(const D3 &a, double f, double fp) { return D3(f, fp * a.d[0], fp * a.d[1], fp * a.d[2]); }
inline D3 sqrt(const D3 &a) { double s = std::sqrt(a.v); return chain(a, s, 0.5 / s); }
inline D3 log(const D3 &a) { return chain(a, std::log(a.v), 1.0 / a.v); }
inline D3 atan(const D3 &a) { return chain(a, std::atan(a.v), 1.0 / (1.0 + a.v * a.v)); }
inline D3 atan2(const D3 &y, const D3 &x)
{
    double r2 = x.v * x.v + y.v * y.v;
    double f = std::atan2(y.v, x.v);
    return D3(f, (x.v * y.d[0] - y.v * x.d[0]) / r2, (x.v * y.d[1] - y.v * x.d[1]) / r2,
              (x.v * y.d[2] - y.v * x.d[2]) / r2);
}
inline D3 sq(const D3 &a) { return a * a; }
inline D3 cube(const D3 &a) { return a * a * a; }

#endif
