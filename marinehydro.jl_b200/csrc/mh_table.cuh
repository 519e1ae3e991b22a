// Tabulated Guevel-Delhommeau wave term.
//
// The reference evaluates the dimensionless wave term of the infinite-depth
// Green function by adaptive quadrature per panel pair
// (src/green_functions/exact_Guevel_Delhommeau.jl:15-59).  With
// R = sqrt(r^2 + z^2), z < 0, the term separates into closed-form parts and
// one smooth remainder:
//
//   Im G    =  2 pi e^z J0(r)
//   Re G    = -2 e^z J0(r) log((R + |z|)/2) + B(r, z)
//   Im dG/dr = -2 pi e^z J1(r)
//   Re dG/dr =  2 e^z J1(r) log((R+|z|)/2) - 2 e^z J0(r) r / (R (R+|z|)) + C(r, z)
//   dG/dz   =  G + 2/R                              (exact_Guevel_Delhommeau.jl:56)
//
// (the log coefficient is the generating function sum_m (-R)^m P_m(|z|/R)/m!
// = e^z J0(r) of the log-moments of e^zeta E1(zeta)).  B and C are smooth
// in polar coordinates (R, alpha = atan2(r, |z|)) near the origin and in
// (r, |z|) away from it, so they are tabulated as 2-D Chebyshev series:
//   - one polar patch, R in [0, 2), alpha in [0, pi/2], fitted at 24 x 24
//     nodes, holding B, C and also E0 = e^z J0(r), E1 = e^z J1(r) (smooth;
//     used by the frequency-batched evaluation, which contracts the alpha
//     direction once per panel pair and then needs only 1-D series in R per
//     frequency).  Degree 14 in R and 21 in alpha are kept: the fitted
//     coefficients beyond them are at the rounding level (|c| < 5e-15 for
//     all four functions);
//   - Cartesian cells of 0.5 x 0.5 over r, |z| in [0, 16), degree 12 x 12,
//     for R >= 2 (every cell touching R < 1 lies inside the polar patch).
// Points outside the table fall back to the adaptive quadrature.  The node
// values are computed on the device with the FP64 quadrature; the table's
// error against it is ~1e-12 absolute.
#pragma once
// Included from mh_device.cuh after the quadrature routines it falls back to.

namespace mh {

constexpr int kTabNP = 24;          // polar patch nodes per direction (fit)
constexpr int kTabNU = 15;          // polar coefficients kept in R (rows)
constexpr int kTabNV = 22;          // polar coefficients kept in alpha (columns)
constexpr int kTabNC = 12;          // Cartesian cell degree
constexpr double kTabRPolar = 2.0;  // polar patch radius
constexpr double kTabH = 0.5;       // Cartesian cell size
constexpr int kTabNCell = 32;       // cells per direction -> extent 16
constexpr double kTabExtent = kTabH * kTabNCell;
constexpr int kTabPolarFn = kTabNU * kTabNV;                   // one polar function
constexpr int kTabPolarWords = 4 * kTabPolarFn;                 // B, C, E0, E1
constexpr int kTabCellWords = 2 * kTabNC * kTabNC;             // B then C
// The polar functions once more with the R direction in the monomial basis:
// row m holds the coefficient of u^m (u = 2 R / kTabRPolar - 1), columns
// still Chebyshev in alpha.  After the alpha contraction each function is a
// degree-14 polynomial in u whose monomial coefficients sum to less than 6
// in absolute value (the Chebyshev coefficients decay faster than the basis
// change grows them), so Horner's rule in u is as accurate as Clenshaw's
// recurrence and takes one FMA per term instead of two operations.
constexpr int kTabMonoOff = kTabPolarWords + kTabNCell * kTabNCell * kTabCellWords;
constexpr int kTabWords = kTabMonoOff + kTabPolarWords;

// sum_i sum_j c[i*NV + j] T_i(u) T_j(v), i < NU, j < NV, by nested Clenshaw
// recurrences (rows in v, then the row sums in u); a few registers instead
// of NU + NV basis values.
template <int NU, int NV>
__device__ __forceinline__ double cheb2d(const double* __restrict__ c, double u, double v)
{
    double a1 = 0.0, a2 = 0.0, s0 = 0.0;
#pragma unroll 1
    for (int i = NU - 1; i >= 0; --i) {
        const double* ci = c + i * NV;
        double b1 = 0.0, b2 = 0.0;
#pragma unroll
        for (int j = NV - 1; j >= 1; --j) {
            const double t = fma(2.0 * v, b1, __ldg(ci + j) - b2);
            b2 = b1;
            b1 = t;
        }
        const double si = fma(v, b1, __ldg(ci) - b2);
        if (i >= 1) {
            const double t = fma(2.0 * u, a1, si - a2);
            a2 = a1;
            a1 = t;
        } else {
            s0 = fma(u, a1, si - a2);
        }
    }
    return s0;
}

// (G, dG/dr, dG/dz) from the table (falls back to quadrature outside it).
__device__ __noinline__ static void delh_dimless_table(const double* __restrict__ tab, double r, double z,
                                                   cplx out[3])
{
    const double az = -z;
    const double R = hypot(r, z);
    double B, C;
    if (!(az >= 0.0)) {  // above the free surface or NaN: not tabulated
        delh_dimless(r, z, out);
        return;
    }
    if (R < kTabRPolar) {
        double alpha = atan2(r, az);
        double u = 2.0 * R / kTabRPolar - 1.0;
        double v = 4.0 * alpha / kPi - 1.0;
        B = cheb2d<kTabNU, kTabNV>(tab, u, v);
        C = cheb2d<kTabNU, kTabNV>(tab + kTabPolarFn, u, v);
    } else if (r < kTabExtent && az < kTabExtent) {
        int ir = min((int)(r / kTabH), kTabNCell - 1);
        int iz = min((int)(az / kTabH), kTabNCell - 1);
        const double* c = tab + kTabPolarWords + (iz * kTabNCell + ir) * kTabCellWords;
        double u = 2.0 * (r - ir * kTabH) / kTabH - 1.0;
        double v = 2.0 * (az - iz * kTabH) / kTabH - 1.0;
        B = cheb2d<kTabNC, kTabNC>(c, u, v);
        C = cheb2d<kTabNC, kTabNC>(c + kTabNC * kTabNC, u, v);
    } else {
        delh_dimless(r, z, out);
        return;
    }
    const double e = exp(z);
    const double J0 = j0(r), J1 = j1(r);
    const double L = log(0.5 * (R + az));
    const double G_re = -2.0 * e * J0 * L + B;
    const double G_im = 2.0 * kPi * e * J0;
    out[0] = mk(G_re, G_im);
    out[1] = mk(2.0 * e * J1 * L - 2.0 * e * J0 * r / (R * (R + az)) + C, -2.0 * kPi * e * J1);
    out[2] = mk(G_re + 2.0 / R, G_im);
}

}  // namespace mh
