// Forward-mode dual numbers for device code: a value and its gradient with
// respect to the three observation coordinates.  Evaluating a closed-form
// displacement field on these yields its exact displacement gradient (to
// rounding), from which strain and stress follow.
#pragma once
#include <cuda_runtime.h>

namespace ucg {

struct Dd {
    double v, x, y, z;
    Dd() = default;
    __host__ __device__ constexpr Dd(double c) : v(c), x(0.0), y(0.0), z(0.0) {}
    __host__ __device__ constexpr Dd(double c, double a, double b, double e) : v(c), x(a), y(b), z(e) {}
};

__device__ __forceinline__ Dd dd(double c) { return Dd{c, 0.0, 0.0, 0.0}; }
__device__ __forceinline__ Dd operator+(Dd a, Dd b) { return Dd{a.v + b.v, a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ Dd operator-(Dd a, Dd b) { return Dd{a.v - b.v, a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Dd operator-(Dd a) { return Dd{-a.v, -a.x, -a.y, -a.z}; }
__device__ __forceinline__ Dd operator*(Dd a, Dd b)
{
    return Dd{a.v * b.v, a.x * b.v + a.v * b.x, a.y * b.v + a.v * b.y, a.z * b.v + a.v * b.z};
}
__device__ __forceinline__ Dd operator+(Dd a, double c) { return Dd{a.v + c, a.x, a.y, a.z}; }
__device__ __forceinline__ Dd operator+(double c, Dd a) { return Dd{a.v + c, a.x, a.y, a.z}; }
__device__ __forceinline__ Dd operator-(Dd a, double c) { return Dd{a.v - c, a.x, a.y, a.z}; }
__device__ __forceinline__ Dd operator-(double c, Dd a) { return Dd{c - a.v, -a.x, -a.y, -a.z}; }
__device__ __forceinline__ Dd operator*(Dd a, double c) { return Dd{a.v * c, a.x * c, a.y * c, a.z * c}; }
__device__ __forceinline__ Dd operator*(double c, Dd a) { return Dd{a.v * c, a.x * c, a.y * c, a.z * c}; }
// reciprocal carries one division; quotients multiply by it
__device__ __forceinline__ Dd rcp(Dd a)
{
    double r = 1.0 / a.v, s = -r * r;
    return Dd{r, s * a.x, s * a.y, s * a.z};
}
__device__ __forceinline__ Dd operator/(Dd a, Dd b)
{
    double r = 1.0 / b.v, q = a.v * r;
    return Dd{q, (a.x - q * b.x) * r, (a.y - q * b.y) * r, (a.z - q * b.z) * r};
}
__device__ __forceinline__ Dd operator/(Dd a, double c)
{
    double r = 1.0 / c;
    return Dd{a.v * r, a.x * r, a.y * r, a.z * r};
}
__device__ __forceinline__ Dd operator/(double c, Dd a)
{
    double r = 1.0 / a.v, q = c * r, s = -q * r;
    return Dd{q, s * a.x, s * a.y, s * a.z};
}
__device__ __forceinline__ Dd dsqrt(Dd a)
{
    double s = sqrt(a.v), h = 0.5 / s;
    return Dd{s, h * a.x, h * a.y, h * a.z};
}
__device__ __forceinline__ Dd dlog(Dd a)
{
    double r = 1.0 / a.v;
    return Dd{log(a.v), r * a.x, r * a.y, r * a.z};
}
__device__ __forceinline__ Dd datan(Dd a)
{
    double r = 1.0 / (1.0 + a.v * a.v);
    return Dd{atan(a.v), r * a.x, r * a.y, r * a.z};
}
__device__ __forceinline__ Dd datan2(Dd y, Dd x)
{
    double r = 1.0 / (x.v * x.v + y.v * y.v);
    return Dd{atan2(y.v, x.v), (x.v * y.x - y.v * x.x) * r, (x.v * y.y - y.v * x.y) * r,
              (x.v * y.z - y.v * x.z) * r};
}
// gradient-only variants: the value of the log / arctangent is not needed when
// only the gradient of the field is formed (the value never feeds back into a
// product), which saves the transcendental evaluation.
__device__ __forceinline__ Dd dlog_g(Dd a)
{
    double r = 1.0 / a.v;
    return Dd{0.0, r * a.x, r * a.y, r * a.z};
}
__device__ __forceinline__ Dd datan_g(Dd a)
{
    double r = 1.0 / (1.0 + a.v * a.v);
    return Dd{0.0, r * a.x, r * a.y, r * a.z};
}
__device__ __forceinline__ Dd datan2_g(Dd y, Dd x)
{
    double r = 1.0 / (x.v * x.v + y.v * y.v);
    return Dd{0.0, (x.v * y.x - y.v * x.x) * r, (x.v * y.y - y.v * x.y) * r,
              (x.v * y.z - y.v * x.z) * r};
}

// square root and its reciprocal from one square root and one division
__device__ __forceinline__ void dsqrt_inv(Dd a, Dd &s, Dd &is)
{
    const double q = sqrt(a.v), r = 1.0 / q, h = 0.5 * r, g = -r * r * h;
    s = Dd{q, h * a.x, h * a.y, h * a.z};
    is = Dd{r, g * a.x, g * a.y, g * a.z};
}
// gradient-only logarithm of a, given ia = 1 / a (already formed)
__device__ __forceinline__ Dd dlog_gi(Dd a, Dd ia) { return Dd{0.0, ia.v * a.x, ia.v * a.y, ia.v * a.z}; }
// gradient-only arctangent of n / d: (d n' - n d') / (n^2 + d^2), one division
__device__ __forceinline__ Dd datan_q_g(Dd n, Dd d) { return datan2_g(n, d); }

// Single-direction dual: a value and one directional derivative.  Evaluating a
// field once per coordinate direction with these keeps half the live state of
// the three-direction type, which matters for the longest expressions.
struct Dd1 {
    double v, d;
    Dd1() = default;
    __host__ __device__ constexpr Dd1(double c) : v(c), d(0.0) {}
    __host__ __device__ constexpr Dd1(double c, double e) : v(c), d(e) {}
};
__device__ __forceinline__ Dd1 operator+(Dd1 a, Dd1 b) { return Dd1{a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dd1 operator-(Dd1 a, Dd1 b) { return Dd1{a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dd1 operator-(Dd1 a) { return Dd1{-a.v, -a.d}; }
__device__ __forceinline__ Dd1 operator*(Dd1 a, Dd1 b) { return Dd1{a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dd1 operator+(Dd1 a, double c) { return Dd1{a.v + c, a.d}; }
__device__ __forceinline__ Dd1 operator+(double c, Dd1 a) { return Dd1{a.v + c, a.d}; }
__device__ __forceinline__ Dd1 operator-(Dd1 a, double c) { return Dd1{a.v - c, a.d}; }
__device__ __forceinline__ Dd1 operator-(double c, Dd1 a) { return Dd1{c - a.v, -a.d}; }
__device__ __forceinline__ Dd1 operator*(Dd1 a, double c) { return Dd1{a.v * c, a.d * c}; }
__device__ __forceinline__ Dd1 operator*(double c, Dd1 a) { return Dd1{a.v * c, a.d * c}; }
__device__ __forceinline__ Dd1 rcp(Dd1 a)
{
    double r = 1.0 / a.v;
    return Dd1{r, -r * r * a.d};
}
__device__ __forceinline__ Dd1 operator/(Dd1 a, Dd1 b)
{
    double r = 1.0 / b.v, q = a.v * r;
    return Dd1{q, (a.d - q * b.d) * r};
}
__device__ __forceinline__ Dd1 operator/(Dd1 a, double c)
{
    double r = 1.0 / c;
    return Dd1{a.v * r, a.d * r};
}
__device__ __forceinline__ Dd1 operator/(double c, Dd1 a)
{
    double r = 1.0 / a.v, q = c * r;
    return Dd1{q, -q * r * a.d};
}
__device__ __forceinline__ Dd1 dsqrt(Dd1 a)
{
    double s = sqrt(a.v);
    return Dd1{s, 0.5 / s * a.d};
}
__device__ __forceinline__ Dd1 dlog_g(Dd1 a) { return Dd1{0.0, a.d / a.v}; }
__device__ __forceinline__ Dd1 datan_g(Dd1 a) { return Dd1{0.0, a.d / (1.0 + a.v * a.v)}; }

__device__ __forceinline__ void dsqrt_inv(Dd1 a, Dd1 &s, Dd1 &is)
{
    const double q = sqrt(a.v), r = 1.0 / q, h = 0.5 * r * a.d;
    s = Dd1{q, h};
    is = Dd1{r, -r * r * h};
}
__device__ __forceinline__ Dd1 dlog_gi(Dd1 a, Dd1 ia) { return Dd1{0.0, ia.v * a.d}; }
__device__ __forceinline__ Dd1 datan_q_g(Dd1 n, Dd1 d)
{
    return Dd1{0.0, (d.v * n.d - n.v * d.d) / (n.v * n.v + d.v * d.v)};
}

// Plain value: the same closed forms evaluated for the displacement itself
// (observation-point displacements).  The "gradient-only" forms of the dual
// types above skip the value of a logarithm or arctangent; for this type the
// value is all there is, so they evaluate it.
struct Dv {
    double v;
    Dv() = default;
    __host__ __device__ constexpr Dv(double c) : v(c) {}
};
__device__ __forceinline__ Dv operator+(Dv a, Dv b) { return Dv{a.v + b.v}; }
__device__ __forceinline__ Dv operator-(Dv a, Dv b) { return Dv{a.v - b.v}; }
__device__ __forceinline__ Dv operator-(Dv a) { return Dv{-a.v}; }
__device__ __forceinline__ Dv operator*(Dv a, Dv b) { return Dv{a.v * b.v}; }
__device__ __forceinline__ Dv operator+(Dv a, double c) { return Dv{a.v + c}; }
__device__ __forceinline__ Dv operator+(double c, Dv a) { return Dv{c + a.v}; }
__device__ __forceinline__ Dv operator-(Dv a, double c) { return Dv{a.v - c}; }
__device__ __forceinline__ Dv operator-(double c, Dv a) { return Dv{c - a.v}; }
__device__ __forceinline__ Dv operator*(Dv a, double c) { return Dv{a.v * c}; }
__device__ __forceinline__ Dv operator*(double c, Dv a) { return Dv{c * a.v}; }
__device__ __forceinline__ Dv rcp(Dv a) { return Dv{1.0 / a.v}; }
__device__ __forceinline__ Dv operator/(Dv a, Dv b) { return Dv{a.v / b.v}; }
__device__ __forceinline__ Dv operator/(Dv a, double c) { return Dv{a.v / c}; }
__device__ __forceinline__ Dv operator/(double c, Dv a) { return Dv{c / a.v}; }
__device__ __forceinline__ Dv dsqrt(Dv a) { return Dv{sqrt(a.v)}; }
__device__ __forceinline__ Dv dlog_g(Dv a) { return Dv{log(a.v)}; }
__device__ __forceinline__ Dv datan_g(Dv a) { return Dv{atan(a.v)}; }
__device__ __forceinline__ Dv datan2_g(Dv y, Dv x) { return Dv{atan2(y.v, x.v)}; }

// the value forms: the square root and its reciprocal, the logarithm itself,
// and the arctangent of the quotient as written (not atan2: the value keeps
// the closed form's branch)
__device__ __forceinline__ void dsqrt_inv(Dv a, Dv &s, Dv &is)
{
    s = Dv{sqrt(a.v)};
    is = Dv{1.0 / s.v};
}
__device__ __forceinline__ Dv dlog_gi(Dv a, Dv) { return Dv{log(a.v)}; }
__device__ __forceinline__ Dv datan_q_g(Dv n, Dv d) { return Dv{atan(n.v / d.v)}; }

}  // namespace ucg
