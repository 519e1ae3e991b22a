/*
 * FP64 CPU oracle: plain-C restatement of MarineHydro.jl's Green functions,
 * panel integrals and influence-matrix assembly.
 *
 * TEST INFRASTRUCTURE ONLY -- the checker of the CUDA library and the timed
 * CPU baseline.  The product path never links or calls this file.
 *
 * Every function cites the reference file:line it restates (paths inside the
 * MarineHydro.jl repository).  Third-party arithmetic the reference reaches
 * through Julia packages is restated from published methods:
 *   - SpecialFunctions.jl v2.7.1 `expint` (complex E1): Abramowitz & Stegun
 *     5.1.11 (ascending series) and 5.1.22 (continued fraction, evaluated by
 *     the modified Lentz method);
 *   - SpecialFunctions.jl `besselj0/besselj1/bessely0/bessely1`: the C
 *     library's j0/j1/y0/y1;
 *   - Integrals.jl v4.10 + HCubature v1.8 adaptive 1-D quadrature: adaptive
 *     Gauss-Kronrod (7,15) bisection to a tighter tolerance than the
 *     reference's default (so the oracle is at least as accurate).
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stddef.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI 3.14159265358979323846264338327950288
#define EULER_GAMMA 0.57721566490153286060651209008240243

/* ------------------------------------------------------------------------ */
/* complex E1                                                               */
/* ------------------------------------------------------------------------ */

/* A&S 5.1.11: E1(z) = -gamma - log z - sum_{n>=1} (-z)^n / (n n!) */
static double complex e1_series(double complex z)
{
    double complex term = 1.0, sum = 0.0;
    for (int n = 1; n < 400; ++n) {
        term *= -z / (double)n;
        double complex add = term / (double)n;
        sum += add;
        if (cabs(add) <= 1e-17 * cabs(sum)) break;
    }
    return -EULER_GAMMA - clog(z) - sum;
}

/* A&S 5.1.22, contracted (even) form, modified Lentz:
 * E1(z) = e^{-z} / (z+1 - 1/(z+3 - 4/(z+5 - 9/(z+7 - ...)))) */
static double complex e1_cfrac(double complex z)
{
    const double tiny = 1e-300;
    double complex b = z + 1.0;
    double complex c = 1.0 / tiny;
    double complex d = 1.0 / b;
    double complex h = d;
    for (int i = 1; i < 2000; ++i) {
        double an = -(double)i * (double)i;
        b += 2.0;
        d = an * d + b;
        if (cabs(d) < tiny) d = tiny;
        d = 1.0 / d;
        c = b + an / c;
        if (cabs(c) < tiny) c = tiny;
        double complex del = c * d;
        h *= del;
        if (cabs(del - 1.0) < 1e-16) break;
    }
    return h * cexp(-z);
}

/* The series loses about exp(|z| + Re z) in relative accuracy to
 * cancellation; the continued fraction converges fast away from the
 * negative real axis.  Pick by that loss. */
static double complex e1c(double complex z)
{
    double az = cabs(z);
    if (az < 2.0 || az + creal(z) < 4.0) return e1_series(z);
    return e1_cfrac(z);
}

void orc_expint_e1(double zr, double zi, double out[2])
{
    double complex v = e1c(zr + I * zi);
    out[0] = creal(v);
    out[1] = cimag(v);
}

/* ------------------------------------------------------------------------ */
/* Rankine                                                                  */
/* ------------------------------------------------------------------------ */

static inline double dot3(const double a[3], const double b[3])
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline void cross3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double norm3(const double a[3]) { return sqrt(dot3(a, a)); }
static inline double signd(double v) { return (v > 0) - (v < 0); } /* Julia sign(0)=0 */

/* rankine.jl:24-63  integral(::Rankine, e1, e2) */
double orc_rankine_integral(const double x[3], const double center[3],
                            const double normal[3], const double verts[12],
                            double area, double radius)
{
    double rb[3] = {x[0] - center[0], x[1] - center[1], x[2] - center[2]};
    double r = norm3(rb);
    if (r > 7.0 * radius) return area / r; /* rankine.jl:33-34 */
    double integral = 0.0;
    double GZ = dot3(rb, normal);
    double RR[4];
    for (int a = 0; a < 4; ++a) {
        double d[3] = {x[0] - verts[3 * a], x[1] - verts[3 * a + 1], x[2] - verts[3 * a + 2]};
        RR[a] = norm3(d);
    }
    for (int a = 0; a < 4; ++a) {
        int b = (a + 1) & 3;
        const double* va = verts + 3 * a;
        const double* vb = verts + 3 * b;
        double e[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
        double L = norm3(e);
        if (L >= 1e-3 * radius) { /* rankine.jl:45 */
            double u[3] = {e[0] / L, e[1] / L, e[2] / L};
            double gyx[3];
            cross3(normal, u, gyx);
            double pa[3] = {x[0] - va[0], x[1] - va[1], x[2] - va[2]};
            double GY = dot3(pa, gyx);
            if (fabs(GZ) >= 1e-4 * radius) { /* rankine.jl:47-51 */
                double ANT = 2.0 * GY * L;
                double s = RR[b] + RR[a];
                double DNT = s * s - L * L + 2.0 * fabs(GZ) * s;
                integral -= 2.0 * fabs(GZ) * atan2(ANT, DNT);
            }
            if (fabs(GY) > 1e-5) { /* rankine.jl:53-57 */
                double ANL = RR[b] + RR[a] + L;
                double DNL = RR[b] + RR[a] - L;
                integral += GY * log(ANL / DNL);
            }
        }
    }
    return integral;
}

/* rankine.jl:65-123  both_integral_and_integral_gradient(::Rankine, ...)
 * (the returned integral omits the solid-angle term, as the reference's
 * does; the assembly only uses the gradient from this routine). */
void orc_rankine_both(const double x[3], const double center[3],
                      const double normal[3], const double verts[12],
                      double area, double radius, int wrt_first,
                      double* integral_out, double grad[3])
{
    double rb[3] = {x[0] - center[0], x[1] - center[1], x[2] - center[2]};
    double r = norm3(rb);
    double integral = 0.0;
    double g[3] = {0.0, 0.0, 0.0};
    if (r > 7.0 * radius) { /* rankine.jl:73-76 */
        double inv3 = 1.0 / (r * r * r);
        integral = area / r;
        g[0] = rb[0] * inv3 * area;
        g[1] = rb[1] * inv3 * area;
        g[2] = rb[2] * inv3 * area;
    } else {
        double GZ = dot3(rb, normal);
        double RR[4], DRX[4][3];
        for (int a = 0; a < 4; ++a) {
            double d[3] = {x[0] - verts[3 * a], x[1] - verts[3 * a + 1], x[2] - verts[3 * a + 2]};
            RR[a] = norm3(d);
            DRX[a][0] = d[0] / RR[a];
            DRX[a][1] = d[1] / RR[a];
            DRX[a][2] = d[2] / RR[a];
        }
        for (int a = 0; a < 4; ++a) {
            int b = (a + 1) & 3;
            const double* va = verts + 3 * a;
            const double* vb = verts + 3 * b;
            double e[3] = {vb[0] - va[0], vb[1] - va[1], vb[2] - va[2]};
            double L = norm3(e);
            if (L >= 1e-3 * radius) {
                double u[3] = {e[0] / L, e[1] / L, e[2] / L};
                double GYX[3];
                cross3(normal, u, GYX);
                double pa[3] = {x[0] - va[0], x[1] - va[1], x[2] - va[2]};
                double GY = dot3(pa, GYX);
                double s = RR[b] + RR[a];
                double ANT = 2.0 * GY * L;
                double DNT = s * s - L * L + 2.0 * fabs(GZ) * s;
                double ANL = s + L;
                double DNL = s - L;
                double ALDEN = log(ANL / DNL);
                double AT = (fabs(GZ) >= 1e-4 * radius) ? atan2(ANT, DNT) : 0.0;
                double sg = signd(GZ);
                double q = GY * (DNL - ANL) / (ANL * DNL);
                double den = ANT * ANT + DNT * DNT;
                for (int c = 0; c < 3; ++c) {
                    double ANLX = DRX[b][c] + DRX[a][c];
                    double ANTX = 2.0 * L * GYX[c];
                    double DNTX = 2.0 * (s + fabs(GZ)) * ANLX + 2.0 * sg * s * normal[c];
                    g[c] -= ALDEN * GYX[c] - 2.0 * sg * AT * normal[c] + q * ANLX
                            - 2.0 * fabs(GZ) * (ANTX * DNT - DNTX * ANT) / den;
                }
                integral += GY * ALDEN;
            }
        }
    }
    double sgn = wrt_first ? -1.0 : 1.0; /* rankine.jl:118-122 */
    *integral_out = integral;
    grad[0] = sgn * g[0];
    grad[1] = sgn * g[1];
    grad[2] = sgn * g[2];
}

/* ------------------------------------------------------------------------ */
/* Wu et al. wave term (wu.jl)                                              */
/* ------------------------------------------------------------------------ */

/* wu.jl:51-66 */
static double wu_dFuncC(double t)
{
    double g = (3168.35 + -1590.27 * t) * t;
    g = (-2318.58 + g) * t;
    g = (847.8 + g) * t;
    g = (-148.24 + g) * t;
    return 14.19 + g;
}
/* wu.jl:69-92 */
static double wu_dFuncB(double t)
{
    double g = (-76209.82 + 19923.28 * t) * t;
    g = (118879.26 + g) * t;
    g = (-97014.11 + g) * t;
    g = (44270.15 + g) * t;
    g = (-11336.19 + g) * t;
    g = (1565.35 + g) * t;
    g = (-76.765 + g) * t;
    g = (2.894 + g) * t;
    return 1.11 + g;
}
/* wu.jl:94-117 */
static double wu_dFuncA(double t)
{
    double g = (-46688.0 + 12622.25 * t) * t;
    g = (68220.87 + g) * t;
    g = (-48811.41 + g) * t;
    g = (16370.75 + g) * t;
    g = (-1187.71 + g) * t;
    g = (-754.85 + g) * t;
    g = (249.69 + g) * t;
    g = (-24.53 + g) * t;
    return 2.948 + g;
}
/* wu.jl:159-182 */
static double wu_FuncD(double t)
{
    double g = (128170.2 + -33744.6 * t) * t;
    g = (-205690.43 + g) * t;
    g = (181856.75 + g) * t;
    g = (-96293.05 + g) * t;
    g = (31127.39 + g) * t;
    g = (-6072.07 + g) * t;
    g = (667.16 + g) * t;
    g = (-40.97 + g) * t;
    return 0.632 + g;
}
/* wu.jl:184-203 */
static double wu_FuncC(double t)
{
    double g = (9136.4 + -3272.62 * t) * t;
    g = (-9844.35 + g) * t;
    g = (5155.67 + g) * t;
    g = (-1397.89 + g) * t;
    g = (209.653 + g) * t;
    g = (-9.747 + g) * t;
    return 1.268 + g;
}
/* wu.jl:205-228 */
static double wu_FuncB(double t)
{
    double g = (-29030.24 + 7671.22 * t) * t;
    g = (44894.06 + g) * t;
    g = (-36618.81 + g) * t;
    g = (17137.74 + g) * t;
    g = (-4780.77 + g) * t;
    g = (796.534 + g) * t;
    g = (-67.92 + g) * t;
    g = (5.737 + g) * t;
    return 0.938 + g;
}
/* wu.jl:230-253 */
static double wu_FuncA(double t)
{
    double g = (21859.0 + -4838.6 * t) * t;
    g = (-41592.9 + g) * t;
    g = (42002.57 + g) * t;
    g = (-24314.21 + g) * t;
    g = (8418.94 + g) * t;
    g = (-1763.96 + g) * t;
    g = (215.896 + g) * t;
    g = (-13.328 + g) * t;
    return 1.21 + g;
}

/* wu.jl:295-327 */
static double struve_h0(double xx)
{
    if (xx <= 3.0) {
        double yy = (xx / 3.0) * (xx / 3.0);
        double h = 1.909859164 + (-1.909855001 + (0.687514637 + (-0.126164557
                   + (0.013828813 + -0.000876918 * yy) * yy) * yy) * yy) * yy;
        return h * (xx / 3.0);
    }
    double yy = (3.0 / xx) * (3.0 / xx);
    double c1 = 2.0 * (0.99999906 + (4.77228920 + (3.85542044 + 0.32303607 * yy) * yy) * yy);
    double c2 = PI * xx * (1.0 + (4.88331068 + (4.28957333 + 0.52120508 * yy) * yy) * yy);
    return c1 / c2 + y0(xx);
}

/* wu.jl:331-362 */
static double struve_h1(double xx)
{
    if (xx <= 3.0) {
        double yy = (xx / 3.0) * (xx / 3.0);
        return (1.909859286 + (-1.145914713 + (0.294656958 + (-0.042070508
                + (0.003785727 + -0.000207183 * yy) * yy) * yy) * yy) * yy) * yy;
    }
    double yy = (3.0 / xx) * (3.0 / xx);
    double c1 = 2.0 * (1.00000004 + (3.92205313 + (2.64893033 + 0.27450895 * yy) * yy) * yy);
    double c2 = PI * (1.0 + (3.81095112 + (2.26216956 + 0.10885141 * yy) * yy) * yy);
    return c1 / c2 + y1(xx);
}

/* wu.jl:266-280 */
static double wu_Lp(double alpha, double beta, double rho)
{
    double A = wu_FuncA(rho), B = wu_FuncB(rho), C = wu_FuncC(rho), D = wu_FuncD(rho);
    double RR = (1.0 - beta) * A;
    RR -= beta * B;
    RR -= alpha * C / (1.0 + 6.0 * alpha * rho * (1.0 - rho));
    RR += beta * (1.0 - beta) * D;
    double om = 1.0 - rho;
    return rho * om * om * om * RR;
}
/* wu.jl:282-293 */
static double wu_L0(double vv, double dd, double alpha, double beta, double rho)
{
    const double gama = 0.5772156649;
    double PP = log(0.5 * (dd - vv)) + gama - 2.0 * dd * dd;
    PP = exp(vv) * PP;
    PP = PP + dd * dd - vv;
    double Lp = wu_Lp(alpha, beta, rho);
    return 2.0 * PP / (1.0 + dd * dd * dd) + 2.0 * Lp;
}
/* wu.jl:131-143 */
static double wu_Lsp(double alpha, double beta, double rho)
{
    double A = wu_dFuncA(rho), B = wu_dFuncB(rho), C = wu_dFuncC(rho);
    double RR = beta * A;
    RR -= (1.0 - alpha) * B;
    RR += beta * (1.0 - beta) * rho * (1.0 - 2.0 * rho) * C;
    double om = 1.0 - rho;
    return rho * om * om * om * RR;
}
/* wu.jl:145-157 */
static double wu_Ls(double hh, double vv, double dd, double alpha, double beta, double rho)
{
    double PS = (beta + hh) / (dd - vv);
    PS = PS - 2.0 * beta + 2.0 * exp(vv) * dd - hh;
    double QS = exp(-dd) * (1.0 - beta);
    QS = QS * (1.0 + dd / (1.0 + dd * dd * dd));
    double Lsp = wu_Lsp(alpha, beta, rho);
    return 2.0 * PS / (1.0 + dd * dd * dd) - 4.0 * QS + 2.0 * Lsp;
}

/* wu.jl:19-30 (G, dG/dh, dG/dv); W (wu.jl:257-264) and Wh (wu.jl:122-129) */
void orc_wu_dimless(double hh, double vv, double out[6])
{
    double dd = sqrt(hh * hh + vv * vv);
    double alpha = -vv / dd;
    double beta = hh / dd;
    double rho = dd / (1.0 + dd);
    double ev = exp(vv);
    double H0 = struve_h0(hh), J0 = j0(hh);
    double H1 = struve_h1(hh), J1 = j1(hh);
    /* W = 2 pi (H0 - i J0) e^v ;  Wh = 2 pi (2/pi - H1 + i J1) e^v */
    double W_re = 2.0 * PI * H0 * ev, W_im = -2.0 * PI * J0 * ev;
    double Wh_re = 2.0 * PI * (2.0 / PI - H1) * ev, Wh_im = 2.0 * PI * J1 * ev;
    double L0 = wu_L0(vv, dd, alpha, beta, rho);
    double Ls = wu_Ls(hh, vv, dd, alpha, beta, rho);
    double G_re = -L0 - W_re, G_im = -W_im;
    out[0] = G_re;
    out[1] = G_im;
    out[2] = -Ls - Wh_re;
    out[3] = -Wh_im;
    out[4] = G_re + 2.0 / dd;
    out[5] = G_im;
}

/* ------------------------------------------------------------------------ */
/* Exact Guevel-Delhommeau wave term (exact_Guevel_Delhommeau.jl)           */
/* ------------------------------------------------------------------------ */

/* Integrands of _dimless_wave_term (:16-23) and _d_dimless_wave_term_dr
 * (:36-43): out = (Gp.re, Gp.im, dGp.re, dGp.im) */
static void delh_integrand(double theta, double r, double z, double out[4])
{
    double c = cos(theta);
    double complex zeta = z + I * (r * c);
    double complex ez = cexp(zeta);
    double complex j = ez * (e1c(zeta) / PI + I);
    out[0] = creal(j);
    out[1] = creal(ez);
    out[2] = creal(I * c * (j - 1.0 / (PI * zeta)));
    out[3] = creal(I * c * ez);
}

/* Gauss-Kronrod (7,15) nodes and weights on [-1, 1] (QUADPACK qk15). */
static const double xgk[8] = {
    0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
    0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
    0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
    0.207784955007898467600689403773245, 0.0};
static const double wgk[8] = {
    0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
    0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
    0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
    0.204432940075298892414161999234649, 0.209482141084727828012999174891714};
static const double wg[4] = {
    0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
    0.381830050505118944950369775488975, 0.417959183673469387755102040816327};

static void gk15(double a, double b, double r, double z, double res[4], double* err)
{
    double c = 0.5 * (a + b), h = 0.5 * (b - a);
    double rk[4] = {0, 0, 0, 0}, rg[4] = {0, 0, 0, 0};
    double f[4];
    delh_integrand(c, r, z, f);
    for (int q = 0; q < 4; ++q) {
        rk[q] = wgk[7] * f[q];
        rg[q] = wg[3] * f[q];
    }
    for (int j = 0; j < 7; ++j) {
        double f1[4], f2[4];
        delh_integrand(c - h * xgk[j], r, z, f1);
        delh_integrand(c + h * xgk[j], r, z, f2);
        for (int q = 0; q < 4; ++q) {
            rk[q] += wgk[j] * (f1[q] + f2[q]);
            if (j & 1) rg[q] += wg[j / 2] * (f1[q] + f2[q]);
        }
    }
    double e = 0.0;
    for (int q = 0; q < 4; ++q) {
        res[q] = rk[q] * h;
        double d = fabs((rk[q] - rg[q]) * h);
        if (d > e) e = d;
    }
    *err = e;
}

/* Depth-first bisection; *budget caps the number of intervals processed so
 * that a NaN error estimate cannot bisect forever. */
static void adapt(double a, double b, double r, double z, double tol_per_len,
                  int depth, double acc[4], int* budget)
{
    double res[4], err;
    gk15(a, b, r, z, res, &err);
    if (err <= tol_per_len * (b - a) || depth >= 48 || --(*budget) < 0) {
        for (int q = 0; q < 4; ++q) acc[q] += res[q];
        return;
    }
    double m = 0.5 * (a + b);
    adapt(a, m, r, z, tol_per_len, depth + 1, acc, budget);
    adapt(m, b, r, z, tol_per_len, depth + 1, acc, budget);
}

/* exact_Guevel_Delhommeau.jl:15-26 (G), :35-46 (dG/dr), :52-59 (dG/dz) */
void orc_delhommeau_dimless(double r, double z, double out[6])
{
    double est[4], err;
    gk15(0.0, 0.5 * PI, r, z, est, &err);
    double scale = 0.0;
    for (int q = 0; q < 4; ++q)
        if (fabs(est[q]) > scale) scale = fabs(est[q]);
    double tol = fmax(1e-15, 1e-13 * scale) / (0.5 * PI);
    double acc[4] = {0, 0, 0, 0};
    int budget = 4097;
    adapt(0.0, 0.5 * PI, r, z, tol, 0, acc, &budget);
    out[0] = 4.0 * acc[0];
    out[1] = 4.0 * acc[1];
    out[2] = 4.0 * acc[2];
    out[3] = 4.0 * acc[3];
    out[4] = out[0] + 2.0 / hypot(r, z);
    out[5] = out[1];
}

/* ------------------------------------------------------------------------ */
/* Reduced coordinates (abstract_greens_function.jl:88-155)                 */
/* ------------------------------------------------------------------------ */

typedef void (*dimless_fn)(double r, double z, double out[6]);

/* Returns k*G in s[2] and the k-scaled gradient in g[6] (complex 3-vector),
 * both multiplied by the source area (one-point rule, wu.jl:33-47). */
static void wave_term(dimless_fn fn, const double x[3], const double xi[3],
                      double k, double area, int wrt_first, double s[2], double g[6])
{
    double dx = x[0] - xi[0], dy = x[1] - xi[1];
    double dis2 = dx * dx + dy * dy;
    const double purt = 1e-18;
    double dis = (dis2 == 0.0) ? sqrt(dis2 + purt * purt) - purt : sqrt(dis2);
    double r = k * dis;
    double z = k * (x[2] + xi[2]);
    double o[6];
    fn(r, z, o);
    double d1 = 0.0, d2 = 0.0;
    if (fabs(r) > 1e-6) {
        double f = k * k / r;
        d1 = wrt_first ? f * dx : -f * dx;
        d2 = wrt_first ? f * dy : -f * dy;
    }
    double dz = k;
    s[0] = k * o[0] * area;
    s[1] = k * o[1] * area;
    g[0] = k * d1 * o[2] * area;
    g[1] = k * d1 * o[3] * area;
    g[2] = k * d2 * o[2] * area;
    g[3] = k * d2 * o[3] * area;
    g[4] = k * dz * o[4] * area;
    g[5] = k * dz * o[5] * area;
}

/* Sum over the GF tuple (abstract_greens_function.jl:49,65) of integral and
 * integral_gradient; reflected terms per rankine_reflected.jl:19-35 and
 * rankine_reflected_negative.jl:11-17. */
void orc_pair_integrals(const double x[3],
                        const double center[3], const double normal[3],
                        const double verts[12], double area, double radius,
                        double k, uint32_t gf_mask, int wrt_first,
                        double s[2], double g[6])
{
    memset(s, 0, 2 * sizeof(double));
    memset(g, 0, 6 * sizeof(double));
    if (gf_mask & ORC_GF_RANKINE) {
        double I0, gr[3], dummy;
        I0 = orc_rankine_integral(x, center, normal, verts, area, radius);
        orc_rankine_both(x, center, normal, verts, area, radius, wrt_first, &dummy, gr);
        s[0] += I0;
        g[0] += gr[0];
        g[2] += gr[1];
        g[4] += gr[2];
    }
    uint32_t refl = gf_mask & (ORC_GF_RANKINE_REFLECTED | ORC_GF_RANKINE_REFL_NEG);
    if (refl == ORC_GF_RANKINE_REFLECTED || refl == ORC_GF_RANKINE_REFL_NEG) {
        double sg = (refl == ORC_GF_RANKINE_REFLECTED) ? 1.0 : -1.0;
        double xr[3] = {x[0], x[1], -x[2]};
        double I0, gr[3], dummy;
        I0 = orc_rankine_integral(xr, center, normal, verts, area, radius);
        orc_rankine_both(xr, center, normal, verts, area, radius, wrt_first, &dummy, gr);
        if (wrt_first) gr[2] = -gr[2]; /* vertical_reflection, rankine_reflected.jl:31-35 */
        s[0] += sg * I0;
        g[0] += sg * gr[0];
        g[2] += sg * gr[1];
        g[4] += sg * gr[2];
    }
    if (gf_mask & ORC_GF_WU) {
        double sw[2], gw[6];
        wave_term(orc_wu_dimless, x, center, k, area, wrt_first, sw, gw);
        s[0] += sw[0];
        s[1] += sw[1];
        for (int q = 0; q < 6; ++q) g[q] += gw[q];
    }
    if (gf_mask & ORC_GF_DELHOMMEAU) {
        double sw[2], gw[6];
        wave_term(orc_delhommeau_dimless, x, center, k, area, wrt_first, sw, gw);
        s[0] += sw[0];
        s[1] += sw[1];
        for (int q = 0; q < 6; ++q) g[q] += gw[q];
    }
}

/* ------------------------------------------------------------------------ */
/* Assembly (matrix_assembly.jl:4-42)                                       */
/* ------------------------------------------------------------------------ */

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_assemble_columns(int64_t n, int64_t nv,
                         const double* centers, const double* normals,
                         const double* areas, const double* radii,
                         const double* vertices, const int64_t* faces,
                         double k, uint32_t gf_mask, int direct,
                         int64_t j0c, int64_t j1c,
                         double* S_out, double* D_out, int nthreads)
{
    if (n <= 0 || nv <= 0 || !centers || !normals || !areas || !radii || !vertices || !faces)
        return 1;
    if (j0c < 0 || j1c > n || j0c > j1c) return 1;
    for (int64_t i = 0; i < 4 * n; ++i)
        if (faces[i] < 0 || faces[i] >= nv) return 1;
    const double inv4pi = 1.0 / (4.0 * PI); /* -1/2tau, tau = 2pi (MarineHydro.jl:11) */
    int wrt_first = !direct;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t j = j0c; j < j1c; ++j) {
        double cj[3] = {centers[j], centers[n + j], centers[2 * n + j]};
        double nj[3] = {normals[j], normals[n + j], normals[2 * n + j]};
        double vj[12];
        for (int a = 0; a < 4; ++a) {
            int64_t vi = faces[j + n * a];
            vj[3 * a + 0] = vertices[vi];
            vj[3 * a + 1] = vertices[nv + vi];
            vj[3 * a + 2] = vertices[2 * nv + vi];
        }
        for (int64_t i = 0; i < n; ++i) {
            double xi[3] = {centers[i], centers[n + i], centers[2 * n + i]};
            double s[2], g[6];
            orc_pair_integrals(xi, cj, nj, vj, areas[j], radii[j], k, gf_mask, wrt_first, s, g);
            int64_t o = 2 * (i + n * j);
            if (S_out) {
                S_out[o] = -inv4pi * s[0];
                S_out[o + 1] = -inv4pi * s[1];
            }
            if (D_out) {
                const double* nn = nj;
                double ni[3];
                if (!direct) {
                    ni[0] = normals[i];
                    ni[1] = normals[n + i];
                    ni[2] = normals[2 * n + i];
                    nn = ni;
                }
                double dre = nn[0] * g[0] + nn[1] * g[2] + nn[2] * g[4];
                double dim = nn[0] * g[1] + nn[1] * g[3] + nn[2] * g[5];
                D_out[o] = (i == j ? 0.5 : 0.0) - inv4pi * dre;
                D_out[o + 1] = -inv4pi * dim;
            }
        }
    }
    return 0;
}

int orc_assemble(int64_t n, int64_t nv,
                 const double* centers, const double* normals,
                 const double* areas, const double* radii,
                 const double* vertices, const int64_t* faces,
                 double k, uint32_t gf_mask, int direct,
                 double* S_out, double* D_out, int nthreads)
{
    return orc_assemble_columns(n, nv, centers, normals, areas, radii, vertices, faces,
                                k, gf_mask, direct, 0, n, S_out, D_out, nthreads);
}
