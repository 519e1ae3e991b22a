// Device-side Green-function arithmetic (FP64).
//
// Restates, per panel pair, the reference's
//   integral(::Rankine)                       src/green_functions/rankine.jl:24-63
//   both_integral_and_integral_gradient       src/green_functions/rankine.jl:65-123
//   RankineReflected / ...Negative            src/green_functions/rankine_reflected*.jl
//   GFWu                                      src/green_functions/wu.jl
//   ExactGuevelDelhommeau                     src/green_functions/exact_Guevel_Delhommeau.jl
//   with_reduced_coordinates(_derivative)     src/green_functions/abstract_greens_function.jl:88-155
// Bessel functions come from CUDA's j0/j1/y0/y1; the complex exponential
// integral E1 is written from Abramowitz & Stegun 5.1.11 / 5.1.22; the
// Delhommeau theta-integral uses adaptive Gauss-Kronrod (7,15) bisection
// (QUADPACK's published nodes) with an explicit per-thread interval stack.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "marinehydro_b200.h"
#include "mh_dual.cuh"

namespace mh {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kEulerGamma = 0.57721566490153286060651209008240243;

template <class T>
struct cx {
    T re, im;
};
using cplx = cx<double>;

__device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
template <class T>
__device__ __forceinline__ cx<T> operator+(const cx<T>& a, const cx<T>& b) { return {a.re + b.re, a.im + b.im}; }
template <class T>
__device__ __forceinline__ cx<T> operator-(const cx<T>& a, const cx<T>& b) { return {a.re - b.re, a.im - b.im}; }
template <class T>
__device__ __forceinline__ cx<T> operator-(const cx<T>& a) { return {-a.re, -a.im}; }
template <class T>
__device__ __forceinline__ cx<T> operator*(const cx<T>& a, const cx<T>& b)
{
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class T>
__device__ __forceinline__ cx<T> operator*(T s, const cx<T>& a) { return {s * a.re, s * a.im}; }
template <class T>
__device__ __forceinline__ cx<T> operator*(const cx<T>& a, T s) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cplx operator/(const cplx& a, double s) { return {a.re / s, a.im / s}; }
// Smith's algorithm for complex division.
__device__ __forceinline__ cplx operator/(const cplx& a, const cplx& b)
{
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, d = b.re + b.im * r;
        return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
    }
    double r = b.re / b.im, d = b.re * r + b.im;
    return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
__device__ __forceinline__ double cabs_(cplx a) { return hypot(a.re, a.im); }
__device__ __forceinline__ cplx cexp_(cplx a)
{
    double s, c, e = exp(a.re);
    sincos(a.im, &s, &c);
    return {e * c, e * s};
}
__device__ __forceinline__ cplx clog_(cplx a) { return {log(cabs_(a)), atan2(a.im, a.re)}; }

// constant of the scalar type (double or dual number)
__device__ __forceinline__ void tset(double& r, double v) { r = v; }
template <int ND>
__device__ __forceinline__ void tset(dualn<ND>& r, double v) { r = dconst<ND>(v); }
template <class T>
__device__ __forceinline__ T tconst(double v)
{
    T r;
    tset(r, v);
    return r;
}

// ---------------------------------------------------------------------------
// complex E1
// ---------------------------------------------------------------------------

// A&S 5.1.11: E1(z) = -gamma - log z - sum_{n>=1} (-z)^n / (n n!)
static __device__ __noinline__ cplx e1_series(cplx z)
{
    cplx term = mk(1.0, 0.0), sum = mk(0.0, 0.0);
    cplx mz = -z;
    for (int n = 1; n < 400; ++n) {
        term = term * mz / (double)n;
        cplx add = term / (double)n;
        sum = sum + add;
        if (cabs_(add) <= 1e-17 * cabs_(sum)) break;
    }
    return mk(-kEulerGamma, 0.0) - clog_(z) - sum;
}

// A&S 5.1.22 contracted form, modified Lentz.
static __device__ __noinline__ cplx e1_cfrac(cplx z)
{
    const double tiny = 1e-300;
    cplx b = z + mk(1.0, 0.0);
    cplx c = mk(1.0 / tiny, 0.0);
    cplx d = mk(1.0, 0.0) / b;
    cplx h = d;
    for (int i = 1; i < 2000; ++i) {
        double an = -(double)i * (double)i;
        b.re += 2.0;
        d = an * d + b;
        if (cabs_(d) < tiny) d = mk(tiny, 0.0);
        d = mk(1.0, 0.0) / d;
        c = b + mk(an, 0.0) / c;
        if (cabs_(c) < tiny) c = mk(tiny, 0.0);
        cplx del = c * d;
        h = h * del;
        if (cabs_(del - mk(1.0, 0.0)) < 1e-16) break;
    }
    return h * cexp_(-z);
}

__device__ __forceinline__ cplx expint_e1(cplx z)
{
    double az = cabs_(z);
    if (az < 2.0 || az + z.re < 4.0) return e1_series(z);
    return e1_cfrac(z);
}

// ---------------------------------------------------------------------------
// Rankine panel integrals
// ---------------------------------------------------------------------------

template <class T>
struct PanelT {
    T c[3];   // centre
    T n[3];   // unit normal
    T v[12];  // 4 vertices, v[3*a + coord]
    T area;
    T radius;
};
using Panel = PanelT<double>;

template <class T>
__device__ __forceinline__ T dot3(const T* a, const T* b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ double signd(double v) { return (double)((v > 0) - (v < 0)); }

// integral(::Rankine) (rankine.jl:24-63) and the gradient of
// both_integral_and_integral_gradient(::Rankine) (rankine.jl:65-123),
// computed in one pass over the panel edges.  The gradient is w.r.t. the
// source point; callers negate it for with_respect_to_first_variable.
template <class T>
__device__ __forceinline__ void rankine_pair(const T x[3], const PanelT<T>& p, T& integral, T grad[3])
{
    T rb[3] = {x[0] - p.c[0], x[1] - p.c[1], x[2] - p.c[2]};
    T r = sqrt(dot3(rb, rb));
    if (val(r) > 7.0 * val(p.radius)) {
        T inv3 = 1.0 / (r * r * r);
        integral = p.area / r;
        grad[0] = rb[0] * inv3 * p.area;
        grad[1] = rb[1] * inv3 * p.area;
        grad[2] = rb[2] * inv3 * p.area;
        return;
    }
    T I = tconst<T>(0.0), g0 = tconst<T>(0.0), g1 = tconst<T>(0.0), g2 = tconst<T>(0.0);
    T GZ = dot3(rb, p.n);
    T aGZ = fabs(GZ);
    double sg = signd(val(GZ));
    bool use_at = val(aGZ) >= 1e-4 * val(p.radius);
    T RR[4], DRX[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        T d0 = x[0] - p.v[3 * a], d1 = x[1] - p.v[3 * a + 1], d2 = x[2] - p.v[3 * a + 2];
        RR[a] = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        DRX[a][0] = d0 / RR[a];
        DRX[a][1] = d1 / RR[a];
        DRX[a][2] = d2 / RR[a];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int b = (a + 1) & 3;
        T e0 = p.v[3 * b] - p.v[3 * a], e1 = p.v[3 * b + 1] - p.v[3 * a + 1],
          e2 = p.v[3 * b + 2] - p.v[3 * a + 2];
        T L = sqrt(e0 * e0 + e1 * e1 + e2 * e2);
        if (val(L) >= 1e-3 * val(p.radius)) {
            T u0 = e0 / L, u1 = e1 / L, u2 = e2 / L;
            T GYX[3] = {p.n[1] * u2 - p.n[2] * u1, p.n[2] * u0 - p.n[0] * u2,
                        p.n[0] * u1 - p.n[1] * u0};
            T pa[3] = {x[0] - p.v[3 * a], x[1] - p.v[3 * a + 1], x[2] - p.v[3 * a + 2]};
            T GY = dot3(pa, GYX);
            T s = RR[b] + RR[a];
            T ANT = 2.0 * GY * L;
            T DNT = s * s - L * L + 2.0 * aGZ * s;
            T ANL = s + L;
            T DNL = s - L;
            T ALDEN = log(ANL / DNL);
            T AT = use_at ? atan2(ANT, DNT) : tconst<T>(0.0);
            // integral(): solid-angle term and log term with their own guards
            if (use_at) I -= 2.0 * aGZ * AT;
            if (fabs(val(GY)) > 1e-5) I += GY * ALDEN;
            // gradient (rankine.jl:97-110)
            T q = GY * (DNL - ANL) / (ANL * DNL);
            T den = ANT * ANT + DNT * DNT;
            T gg[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T ANLX = DRX[b][c] + DRX[a][c];
                T ANTX = 2.0 * L * GYX[c];
                T DNTX = 2.0 * (s + aGZ) * ANLX + (2.0 * sg) * s * p.n[c];
                gg[c] = ALDEN * GYX[c] - (2.0 * sg) * AT * p.n[c] + q * ANLX
                        - 2.0 * aGZ * (ANTX * DNT - DNTX * ANT) / den;
            }
            g0 -= gg[0];
            g1 -= gg[1];
            g2 -= gg[2];
        }
    }
    integral = I;
    grad[0] = g0;
    grad[1] = g1;
    grad[2] = g2;
}

// ---------------------------------------------------------------------------
// Wu et al. wave term (wu.jl)
// ---------------------------------------------------------------------------

template <class T>
__device__ __forceinline__ T wu_dFuncC(const T& t)  // wu.jl:51-66
{
    T g = (3168.35 + -1590.27 * t) * t;
    g = (-2318.58 + g) * t;
    g = (847.8 + g) * t;
    g = (-148.24 + g) * t;
    return 14.19 + g;
}
template <class T>
__device__ __forceinline__ T wu_dFuncB(const T& t)  // wu.jl:69-92
{
    T g = (-76209.82 + 19923.28 * t) * t;
    g = (118879.26 + g) * t;
    g = (-97014.11 + g) * t;
    g = (44270.15 + g) * t;
    g = (-11336.19 + g) * t;
    g = (1565.35 + g) * t;
    g = (-76.765 + g) * t;
    g = (2.894 + g) * t;
    return 1.11 + g;
}
template <class T>
__device__ __forceinline__ T wu_dFuncA(const T& t)  // wu.jl:94-117
{
    T g = (-46688.0 + 12622.25 * t) * t;
    g = (68220.87 + g) * t;
    g = (-48811.41 + g) * t;
    g = (16370.75 + g) * t;
    g = (-1187.71 + g) * t;
    g = (-754.85 + g) * t;
    g = (249.69 + g) * t;
    g = (-24.53 + g) * t;
    return 2.948 + g;
}
template <class T>
__device__ __forceinline__ T wu_FuncD(const T& t)  // wu.jl:159-182
{
    T g = (128170.2 + -33744.6 * t) * t;
    g = (-205690.43 + g) * t;
    g = (181856.75 + g) * t;
    g = (-96293.05 + g) * t;
    g = (31127.39 + g) * t;
    g = (-6072.07 + g) * t;
    g = (667.16 + g) * t;
    g = (-40.97 + g) * t;
    return 0.632 + g;
}
template <class T>
__device__ __forceinline__ T wu_FuncC(const T& t)  // wu.jl:184-203
{
    T g = (9136.4 + -3272.62 * t) * t;
    g = (-9844.35 + g) * t;
    g = (5155.67 + g) * t;
    g = (-1397.89 + g) * t;
    g = (209.653 + g) * t;
    g = (-9.747 + g) * t;
    return 1.268 + g;
}
template <class T>
__device__ __forceinline__ T wu_FuncB(const T& t)  // wu.jl:205-228
{
    T g = (-29030.24 + 7671.22 * t) * t;
    g = (44894.06 + g) * t;
    g = (-36618.81 + g) * t;
    g = (17137.74 + g) * t;
    g = (-4780.77 + g) * t;
    g = (796.534 + g) * t;
    g = (-67.92 + g) * t;
    g = (5.737 + g) * t;
    return 0.938 + g;
}
template <class T>
__device__ __forceinline__ T wu_FuncA(const T& t)  // wu.jl:230-253
{
    T g = (21859.0 + -4838.6 * t) * t;
    g = (-41592.9 + g) * t;
    g = (42002.57 + g) * t;
    g = (-24314.21 + g) * t;
    g = (8418.94 + g) * t;
    g = (-1763.96 + g) * t;
    g = (215.896 + g) * t;
    g = (-13.328 + g) * t;
    return 1.21 + g;
}

template <class T>
__device__ __forceinline__ T struve_h0(const T& xx)  // wu.jl:295-327
{
    if (val(xx) <= 3.0) {
        T yy = (xx / 3.0) * (xx / 3.0);
        T h = 1.909859164 + (-1.909855001 + (0.687514637 + (-0.126164557
                   + (0.013828813 + -0.000876918 * yy) * yy) * yy) * yy) * yy;
        return h * (xx / 3.0);
    }
    T yy = (3.0 / xx) * (3.0 / xx);
    T c1 = 2.0 * (0.99999906 + (4.77228920 + (3.85542044 + 0.32303607 * yy) * yy) * yy);
    T c2 = kPi * xx * (1.0 + (4.88331068 + (4.28957333 + 0.52120508 * yy) * yy) * yy);
    return c1 / c2 + y0(xx);
}

template <class T>
__device__ __forceinline__ T struve_h1(const T& xx)  // wu.jl:331-362
{
    if (val(xx) <= 3.0) {
        T yy = (xx / 3.0) * (xx / 3.0);
        return (1.909859286 + (-1.145914713 + (0.294656958 + (-0.042070508
                + (0.003785727 + -0.000207183 * yy) * yy) * yy) * yy) * yy) * yy;
    }
    T yy = (3.0 / xx) * (3.0 / xx);
    T c1 = 2.0 * (1.00000004 + (3.92205313 + (2.64893033 + 0.27450895 * yy) * yy) * yy);
    T c2 = kPi * (1.0 + (3.81095112 + (2.26216956 + 0.10885141 * yy) * yy) * yy);
    return c1 / c2 + y1(xx);
}

// (G, dG/dh, dG/dv) of the Wu wave term, wu.jl:19-30; out = 3 complex.
template <class T>
__device__ __forceinline__ void wu_dimless(const T& hh, const T& vv, cx<T> out[3])
{
    T dd = sqrt(hh * hh + vv * vv);
    T alpha = -vv / dd;
    T beta = hh / dd;
    T rho = dd / (1.0 + dd);
    T ev = exp(vv);
    T om = 1.0 - rho;
    T om3 = om * om * om;
    T dd3 = dd * dd * dd;
    // GF_Func_Lp / GF_Func_L0 (wu.jl:266-293)
    T RR = (1.0 - beta) * wu_FuncA(rho);
    RR -= beta * wu_FuncB(rho);
    RR -= alpha * wu_FuncC(rho) / (1.0 + 6.0 * alpha * rho * (1.0 - rho));
    RR += beta * (1.0 - beta) * wu_FuncD(rho);
    T Lp = rho * om3 * RR;
    const double gama = 0.5772156649;
    T PP = log(0.5 * (dd - vv)) + gama - 2.0 * dd * dd;
    PP = ev * PP;
    PP = PP + dd * dd - vv;
    T L0 = 2.0 * PP / (1.0 + dd3) + 2.0 * Lp;
    // GF_Func_Lsp / GF_Func_Ls (wu.jl:131-157)
    T RS = beta * wu_dFuncA(rho);
    RS -= (1.0 - alpha) * wu_dFuncB(rho);
    RS += beta * (1.0 - beta) * rho * (1.0 - 2.0 * rho) * wu_dFuncC(rho);
    T Lsp = rho * om3 * RS;
    T PS = (beta + hh) / (dd - vv);
    PS = PS - 2.0 * beta + 2.0 * ev * dd - hh;
    T QS = exp(-dd) * (1.0 - beta);
    QS = QS * (1.0 + dd / (1.0 + dd3));
    T Ls = 2.0 * PS / (1.0 + dd3) - 4.0 * QS + 2.0 * Lsp;
    // W, Wh (wu.jl:122-129, :257-264)
    T H0 = struve_h0(hh), J0 = j0(hh), H1 = struve_h1(hh), J1 = j1(hh);
    T G_re = -L0 - (2.0 * kPi) * H0 * ev;
    T G_im = (2.0 * kPi) * J0 * ev;
    out[0] = cx<T>{G_re, G_im};
    out[1] = cx<T>{-Ls - (2.0 * kPi) * (2.0 / kPi - H1) * ev, (-2.0 * kPi) * J1 * ev};
    out[2] = cx<T>{G_re + 2.0 / dd, G_im};
}

// ---------------------------------------------------------------------------
// exact Guevel-Delhommeau wave term
// ---------------------------------------------------------------------------

// Integrands of _dimless_wave_term and _d_dimless_wave_term_dr
// (exact_Guevel_Delhommeau.jl:16-23, :36-43).
__device__ __forceinline__ void delh_integrand(double theta, double r, double z, double f[4])
{
    double c = cos(theta);
    cplx zeta = mk(z, r * c);
    cplx ez = cexp_(zeta);
    cplx e1 = expint_e1(zeta);
    cplx j = ez * mk(e1.re / kPi, e1.im / kPi + 1.0);
    f[0] = j.re;
    f[1] = ez.re;
    cplx t = j - mk(1.0, 0.0) / (kPi * zeta);
    // Re(i c t) = -c Im t ; Re(i c e^zeta) = -c Im e^zeta
    f[2] = -c * t.im;
    f[3] = -c * ez.im;
}

// Gauss-Kronrod (7,15) rule on [-1, 1]: QUADPACK's published qk15 nodes and
// weights (statically initialised, one copy per translation unit).
static __constant__ double c_xgk[8] = {
    0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
    0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
    0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
    0.207784955007898467600689403773245, 0.0};
static __constant__ double c_wgk[8] = {
    0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
    0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
    0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
    0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
static __constant__ double c_wg[4] = {
    0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
    0.381830050505118944950369775488975, 0.417959183673469387755102040816327};

__device__ __forceinline__ void delh_gk15(double a, double b, double r, double z, double res[4],
                                          double& err)
{
    double c = 0.5 * (a + b), h = 0.5 * (b - a);
    double rk[4], rg[4], f[4];
    delh_integrand(c, r, z, f);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        rk[q] = c_wgk[7] * f[q];
        rg[q] = c_wg[3] * f[q];
    }
    for (int j = 0; j < 7; ++j) {
        double f1[4], f2[4];
        delh_integrand(c - h * c_xgk[j], r, z, f1);
        delh_integrand(c + h * c_xgk[j], r, z, f2);
        double wk = c_wgk[j];
        double wgj = (j & 1) ? c_wg[j >> 1] : 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double s = f1[q] + f2[q];
            rk[q] += wk * s;
            rg[q] += wgj * s;
        }
    }
    double e = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        res[q] = rk[q] * h;
        double d = fabs((rk[q] - rg[q]) * h);
        e = fmax(e, d);
    }
    err = e;
}

// (G, dG/dr, dG/dz) of the exact wave term; the theta-integral is adaptive
// Gauss-Kronrod bisection with the same acceptance rule as the CPU oracle.
static __device__ __noinline__ void delh_dimless(double r, double z, cplx out[3])
{
    const double half_pi = 0.5 * kPi;
    double est[4], err;
    delh_gk15(0.0, half_pi, r, z, est, err);
    double scale = fmax(fmax(fabs(est[0]), fabs(est[1])), fmax(fabs(est[2]), fabs(est[3])));
    double tol = fmax(1e-15, 1e-13 * scale) / half_pi;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (err <= tol * half_pi) {
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = est[q];
    } else {
        constexpr int kStack = 52;
        constexpr int kMaxIntervals = 4096;
        double sa[kStack], sb[kStack];
        int sd[kStack];
        int sp = 0;
        int processed = 0;  // hard cap: a NaN error estimate must not bisect forever
        double m = 0.5 * half_pi;
        sa[sp] = m; sb[sp] = half_pi; sd[sp] = 1; ++sp;
        sa[sp] = 0.0; sb[sp] = m; sd[sp] = 1; ++sp;
        while (sp > 0) {
            --sp;
            double a = sa[sp], b = sb[sp];
            int d = sd[sp];
            double res[4], e;
            delh_gk15(a, b, r, z, res, e);
            if (e <= tol * (b - a) || d >= 48 || sp + 2 > kStack || ++processed > kMaxIntervals) {
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[q] += res[q];
            } else {
                double mm = 0.5 * (a + b);
                sa[sp] = mm; sb[sp] = b; sd[sp] = d + 1; ++sp;
                sa[sp] = a; sb[sp] = mm; sd[sp] = d + 1; ++sp;
            }
        }
    }
    out[0] = mk(4.0 * acc[0], 4.0 * acc[1]);
    out[1] = mk(4.0 * acc[2], 4.0 * acc[3]);
    out[2] = mk(out[0].re + 2.0 / hypot(r, z), out[0].im);
}

}  // namespace mh

#include "mh_table.cuh"

namespace mh {

// ---------------------------------------------------------------------------
// reduced coordinates and the per-pair sum over Green-function terms
// ---------------------------------------------------------------------------

// Exact wave term in the T arithmetic: the double quadrature, or for dual
// numbers its value with derivatives from dG/dr, dG/dz = G + 2/R and, for
// the second derivatives, G_zz = G_z - 2z/R^3, G_rz = G_r - 2r/R^3 and the
// harmonic identity G_rr = -G_r/r - G_zz (the wave part solves Laplace's
// equation), G_rr(0, z) = -G_zz/2.
__device__ __forceinline__ void delh_exact_t(const double& r, const double& z, cplx out[3])
{
    delh_dimless(r, z, out);
}
template <int ND>
__device__ __forceinline__ void delh_exact_t(const dualn<ND>& r, const dualn<ND>& z,
                                             cx<dualn<ND>> out[3])
{
    cplx o[3];
    delh_dimless(r.v, z.v, o);
    const double R = hypot(r.v, z.v), R3 = R * R * R;
    cplx gzz = o[2] - mk(2.0 * z.v / R3, 0.0);
    cplx grz = o[1] - mk(2.0 * r.v / R3, 0.0);
    cplx grr = (r.v > 0.0) ? -(o[1] / r.v) - gzz : mk(-0.5 * gzz.re, -0.5 * gzz.im);
    const cplx d[3][2] = {{o[1], o[2]}, {grr, grz}, {grz, gzz}};  // (d/dr, d/dz) of G, G_r, G_z
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        out[q].re.v = o[q].re;
        out[q].im.v = o[q].im;
#pragma unroll
        for (int k = 0; k < ND; ++k) {
            out[q].re.d[k] = d[q][0].re * r.d[k] + d[q][1].re * z.d[k];
            out[q].im.d[k] = d[q][0].im * r.d[k] + d[q][1].im * z.d[k];
        }
    }
}

// Table evaluation in the T arithmetic (the double version is
// delh_dimless_table); derivatives are those of the Chebyshev interpolant.
template <int NU, int NV, class T>
__device__ __forceinline__ T cheb2d_t(const double* __restrict__ c, const T& u, const T& v)
{
    T a1 = tconst<T>(0.0), a2 = tconst<T>(0.0), s0 = tconst<T>(0.0);
#pragma unroll 1
    for (int i = NU - 1; i >= 0; --i) {
        const double* ci = c + i * NV;
        T b1 = tconst<T>(0.0), b2 = tconst<T>(0.0);
#pragma unroll 4
        for (int j = NV - 1; j >= 1; --j) {
            T t = 2.0 * v * b1 + (__ldg(ci + j) - b2);
            b2 = b1;
            b1 = t;
        }
        T si = v * b1 + (__ldg(ci) - b2);
        if (i >= 1) {
            T t = 2.0 * u * a1 + (si - a2);
            a2 = a1;
            a1 = t;
        } else {
            s0 = u * a1 + (si - a2);
        }
    }
    return s0;
}

template <class T>
__device__ __forceinline__ void delh_table_t(const double* __restrict__ tab, const T& r, const T& z,
                                             cx<T> out[3])
{
    const T az = -z;
    const T R = hypot(r, z);
    T B, C;
    if (!(val(az) >= 0.0)) {
        delh_exact_t(r, z, out);
        return;
    }
    if (val(R) < kTabRPolar) {
        T alpha = atan2(r, az);
        T u = R * (2.0 / kTabRPolar) - 1.0;
        T v = alpha * (4.0 / kPi) - 1.0;
        B = cheb2d_t<kTabNU, kTabNV>(tab, u, v);
        C = cheb2d_t<kTabNU, kTabNV>(tab + kTabPolarFn, u, v);
    } else if (val(r) < kTabExtent && val(az) < kTabExtent) {
        int ir = min((int)(val(r) / kTabH), kTabNCell - 1);
        int iz = min((int)(val(az) / kTabH), kTabNCell - 1);
        const double* c = tab + kTabPolarWords + (iz * kTabNCell + ir) * kTabCellWords;
        T u = (r - ir * kTabH) * (2.0 / kTabH) - 1.0;
        T v = (az - iz * kTabH) * (2.0 / kTabH) - 1.0;
        B = cheb2d_t<kTabNC, kTabNC>(c, u, v);
        C = cheb2d_t<kTabNC, kTabNC>(c + kTabNC * kTabNC, u, v);
    } else {
        delh_exact_t(r, z, out);
        return;
    }
    const T e = exp(z);
    const T J0 = j0(r), J1 = j1(r);
    const T L = log(0.5 * (R + az));
    const T G_re = -2.0 * e * J0 * L + B;
    const T G_im = (2.0 * kPi) * e * J0;
    out[0] = cx<T>{G_re, G_im};
    out[1] = cx<T>{2.0 * e * J1 * L - 2.0 * e * J0 * r / (R * (R + az)) + C, (-2.0 * kPi) * e * J1};
    out[2] = cx<T>{G_re + 2.0 / R, G_im};
}

// k*G*area and the k-scaled gradient * area (abstract_greens_function.jl:88-155,
// one-point rule wu.jl:33-47 / exact_Guevel_Delhommeau.jl:61-75).
template <bool kDelh, class T>
__device__ __forceinline__ void wave_pair(const T x[3], const PanelT<T>& p, const T& k, bool wrt_first,
                                          const double* tab, cx<T>& s, cx<T> g[3])
{
    T dx = x[0] - p.c[0], dy = x[1] - p.c[1];
    T dis2 = dx * dx + dy * dy;
    const double purt = 1e-18;
    T dis = (val(dis2) == 0.0) ? sqrt(dis2 + purt * purt) - purt : sqrt(dis2);
    T r = k * dis;
    T z = k * (x[2] + p.c[2]);
    cx<T> o[3];
    if (kDelh) {
        if constexpr (std::is_same<T, double>::value) {
            if (tab) delh_dimless_table(tab, r, z, o);
            else delh_dimless(r, z, o);
        } else {
            if (tab) delh_table_t(tab, r, z, o);
            else delh_exact_t(r, z, o);
        }
    } else {
        wu_dimless(r, z, o);
    }
    T d1 = tconst<T>(0.0), d2 = tconst<T>(0.0);
    if (fabs(val(r)) > 1e-6) {
        T f = k * k / r;
        d1 = wrt_first ? f * dx : -(f * dx);
        d2 = wrt_first ? f * dy : -(f * dy);
    }
    T ka = k * p.area;
    s = ka * o[0];
    g[0] = (ka * d1) * o[1];
    g[1] = (ka * d2) * o[1];
    g[2] = (ka * k) * o[2];
}

// Sum over the Green-function tuple of integral / integral_gradient.
template <class T>
__device__ __forceinline__ void pair_integrals(const T x[3], const PanelT<T>& p, const T& k,
                                               uint32_t mask, bool wrt_first, const double* tab,
                                               cx<T>& s, cx<T> g[3])
{
    const T zero = tconst<T>(0.0);
    s = cx<T>{zero, zero};
    g[0] = g[1] = g[2] = cx<T>{zero, zero};
    if (mask & MH_GF_RANKINE) {
        T I, gr[3];
        rankine_pair(x, p, I, gr);
        double sg = wrt_first ? -1.0 : 1.0;
        s.re += I;
        g[0].re += sg * gr[0];
        g[1].re += sg * gr[1];
        g[2].re += sg * gr[2];
    }
    uint32_t refl = mask & (MH_GF_RANKINE_REFLECTED | MH_GF_RANKINE_REFLECTED_NEGATIVE);
    if (refl == MH_GF_RANKINE_REFLECTED || refl == MH_GF_RANKINE_REFLECTED_NEGATIVE) {
        double sgn = (refl == MH_GF_RANKINE_REFLECTED) ? 1.0 : -1.0;
        T xr[3] = {x[0], x[1], -x[2]};
        T I, gr[3];
        rankine_pair(xr, p, I, gr);
        double sg = wrt_first ? -1.0 : 1.0;
        double sz = wrt_first ? -1.0 : 1.0;  // vertical_reflection for wrt_first
        s.re += sgn * I;
        g[0].re += (sgn * sg) * gr[0];
        g[1].re += (sgn * sg) * gr[1];
        g[2].re += (sgn * sg * sz) * gr[2];
    }
    if (mask & MH_GF_WU) {
        cx<T> sw, gw[3];
        wave_pair<false>(x, p, k, wrt_first, tab, sw, gw);
        s = s + sw;
        g[0] = g[0] + gw[0];
        g[1] = g[1] + gw[1];
        g[2] = g[2] + gw[2];
    }
    if (mask & MH_GF_DELHOMMEAU) {
        cx<T> sw, gw[3];
        wave_pair<true>(x, p, k, wrt_first, tab, sw, gw);
        s = s + sw;
        g[0] = g[0] + gw[0];
        g[1] = g[1] + gw[1];
        g[2] = g[2] + gw[2];
    }
}

}  // namespace mh
