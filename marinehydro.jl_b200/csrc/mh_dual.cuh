// Forward-mode dual numbers with ND tangent directions, for exact
// derivatives of the panel-pair functions along geometry and frequency
// directions (the adjoint contraction kernels).  `val(x)` gives the value
// part; branches of the pair functions test values only, as the reference's
// Julia code does under ForwardDiff.
#pragma once
#include <cuda_runtime.h>

namespace mh {

// The dual overloads below live in mh; these keep the double ones visible
// to unqualified calls made inside mh.
using ::atan2;
using ::exp;
using ::fabs;
using ::fma;
using ::hypot;
using ::j0;
using ::j1;
using ::log;
using ::sincos;
using ::sqrt;
using ::y0;
using ::y1;

template <int ND>
struct dualn {
    double v;
    double d[ND];
};

__device__ __forceinline__ double val(double x) { return x; }
template <int ND>
__device__ __forceinline__ double val(const dualn<ND>& x) { return x.v; }

template <int ND>
__device__ __forceinline__ dualn<ND> dconst(double v)
{
    dualn<ND> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = 0.0;
    return r;
}

// f(x) with f'(x) = fp
template <int ND>
__device__ __forceinline__ dualn<ND> dchain(const dualn<ND>& x, double f, double fp)
{
    dualn<ND> r;
    r.v = f;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = fp * x.d[k];
    return r;
}

#define MH_DUAL_BINOP(OP, VEXPR, DEXPR)                                                        \
    template <int ND>                                                                          \
    __device__ __forceinline__ dualn<ND> operator OP(const dualn<ND>& a, const dualn<ND>& b)   \
    {                                                                                          \
        dualn<ND> r;                                                                           \
        r.v = VEXPR;                                                                           \
        _Pragma("unroll") for (int k = 0; k < ND; ++k) r.d[k] = DEXPR;                          \
        return r;                                                                              \
    }
MH_DUAL_BINOP(+, a.v + b.v, a.d[k] + b.d[k])
MH_DUAL_BINOP(-, a.v - b.v, a.d[k] - b.d[k])
MH_DUAL_BINOP(*, a.v * b.v, a.d[k] * b.v + a.v * b.d[k])
#undef MH_DUAL_BINOP

template <int ND>
__device__ __forceinline__ dualn<ND> operator/(const dualn<ND>& a, const dualn<ND>& b)
{
    dualn<ND> r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}

template <int ND>
__device__ __forceinline__ dualn<ND> operator-(const dualn<ND>& a)
{
    dualn<ND> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = -a.d[k];
    return r;
}

// mixed with double
template <int ND>
__device__ __forceinline__ dualn<ND> operator+(const dualn<ND>& a, double b)
{
    dualn<ND> r = a;
    r.v += b;
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator+(double b, const dualn<ND>& a) { return a + b; }
template <int ND>
__device__ __forceinline__ dualn<ND> operator-(const dualn<ND>& a, double b) { return a + (-b); }
template <int ND>
__device__ __forceinline__ dualn<ND> operator-(double b, const dualn<ND>& a) { return (-a) + b; }
template <int ND>
__device__ __forceinline__ dualn<ND> operator*(const dualn<ND>& a, double b)
{
    dualn<ND> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> operator*(double b, const dualn<ND>& a) { return a * b; }
template <int ND>
__device__ __forceinline__ dualn<ND> operator/(const dualn<ND>& a, double b) { return a * (1.0 / b); }
template <int ND>
__device__ __forceinline__ dualn<ND> operator/(double a, const dualn<ND>& b)
{
    return dchain(b, a / b.v, -a / (b.v * b.v));
}

template <int ND>
__device__ __forceinline__ dualn<ND>& operator+=(dualn<ND>& a, const dualn<ND>& b) { return a = a + b; }
template <int ND>
__device__ __forceinline__ dualn<ND>& operator-=(dualn<ND>& a, const dualn<ND>& b) { return a = a - b; }

template <int ND>
__device__ __forceinline__ dualn<ND> sqrt(const dualn<ND>& x)
{
    const double s = ::sqrt(x.v);
    return dchain(x, s, s > 0.0 ? 0.5 / s : 0.0);
}
template <int ND>
__device__ __forceinline__ dualn<ND> exp(const dualn<ND>& x)
{
    const double e = ::exp(x.v);
    return dchain(x, e, e);
}
template <int ND>
__device__ __forceinline__ dualn<ND> log(const dualn<ND>& x) { return dchain(x, ::log(x.v), 1.0 / x.v); }
template <int ND>
__device__ __forceinline__ dualn<ND> fabs(const dualn<ND>& x) { return x.v < 0.0 ? -x : x; }
template <int ND>
__device__ __forceinline__ dualn<ND> atan2(const dualn<ND>& y, const dualn<ND>& x)
{
    dualn<ND> r;
    r.v = ::atan2(y.v, x.v);
    const double den = x.v * x.v + y.v * y.v;
    const double iv = den > 0.0 ? 1.0 / den : 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) r.d[k] = (x.v * y.d[k] - y.v * x.d[k]) * iv;
    return r;
}
template <int ND>
__device__ __forceinline__ dualn<ND> hypot(const dualn<ND>& a, const dualn<ND>& b)
{
    return sqrt(a * a + b * b);
}
template <int ND>
__device__ __forceinline__ void sincos(const dualn<ND>& x, dualn<ND>* s, dualn<ND>* c)
{
    double sv, cv;
    ::sincos(x.v, &sv, &cv);
    *s = dchain(x, sv, cv);
    *c = dchain(x, cv, -sv);
}
// Bessel functions: J0' = -J1, J1' = J0 - J1/x, Y0' = -Y1, Y1' = Y0 - Y1/x
template <int ND>
__device__ __forceinline__ dualn<ND> j0(const dualn<ND>& x) { return dchain(x, ::j0(x.v), -::j1(x.v)); }
template <int ND>
__device__ __forceinline__ dualn<ND> j1(const dualn<ND>& x)
{
    const double J1 = ::j1(x.v);
    return dchain(x, J1, x.v != 0.0 ? ::j0(x.v) - J1 / x.v : 0.5);
}
template <int ND>
__device__ __forceinline__ dualn<ND> y0(const dualn<ND>& x) { return dchain(x, ::y0(x.v), -::y1(x.v)); }
template <int ND>
__device__ __forceinline__ dualn<ND> y1(const dualn<ND>& x)
{
    const double Y1 = ::y1(x.v);
    return dchain(x, Y1, ::y0(x.v) - Y1 / x.v);
}
template <int ND>
__device__ __forceinline__ dualn<ND> fma(const dualn<ND>& a, const dualn<ND>& b, const dualn<ND>& c)
{
    return a * b + c;
}
template <int ND>
__device__ __forceinline__ dualn<ND> fma(double a, const dualn<ND>& b, const dualn<ND>& c)
{
    return a * b + c;
}

}  // namespace mh
