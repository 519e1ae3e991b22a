// Batched hydrodynamic coefficients: many frequencies of one mesh, every
// radiating degree of freedom and every incident-wave heading at once.
//
// Replaces the reference's problem loop (src/solve.jl:4-21 over
// src/problems_and_results.jl:70-100, assembled per problem) with one call:
//
//   FP64 (MH_PRECISION_FP64): per frequency, FP64 assembly of S and D (or K),
//     S*BC with cuBLAS, zgetrf/zgetrs from cuSOLVER, force reduction.
//   mixed (MH_PRECISION_MIXED): the frequency-independent Rankine part of S
//     and D once per call; per frequency the wave part is added in FP64 and
//     written twice, an FP64 master copy for residuals and an FP32 copy that
//     is LU-factorised without pivoting (batched over frequencies); FP64
//     iterative refinement r = b - D x, x += LU^-1 r until
//     max|r|/max|b| <= tol per right-hand side.  A problem whose FP32 LU
//     meets a bad pivot or does not converge is re-solved with the pivoted
//     FP64 LU (counted in mh_batch_info.n_fallback).
#include <cuComplex.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mh_device.cuh"
#include "mh_internal.h"

namespace mh {
namespace {

constexpr int kRows = 128;
constexpr int kCols = 16;
constexpr double kInv4Pi = 1.0 / (4.0 * kPi);
constexpr size_t kBatchBytes = 16ull << 30;  // device memory budget of one frequency chunk
constexpr int kAllwMinFreqs = 6;  // chunks this large use the frequency-batched Delhommeau pass

__device__ __forceinline__ void load_panel_field(Panel& p, int f, double v)
{
    if (f < 3) p.c[f] = v;
    else if (f < 6) p.n[f - 3] = v;
    else if (f == G_AREA) p.area = v;
    else if (f == G_RADIUS) p.radius = v;
    else p.v[f - G_V] = v;
}

__device__ __forceinline__ void stage_panels(Panel* sp, const double* __restrict__ geom, int64_t n,
                                             int64_t j0)
{
    for (int t = threadIdx.x; t < kCols * G_NFIELDS; t += blockDim.x) {
        int f = t / kCols, jj = t % kCols;
        int64_t j = j0 + jj;
        load_panel_field(sp[jj], f, (j < n) ? geom[(int64_t)f * n + j] : 0.0);
    }
}

// Rankine / reflected terms (real, frequency independent), with the -1/(4 pi)
// factor and the 1/2 diagonal of D already applied.
__global__ void __launch_bounds__(kRows)
k_rankine_real(const double* __restrict__ geom, int64_t n, uint32_t mask, int direct,
               double* __restrict__ SR, double* __restrict__ DR)
{
    __shared__ Panel sp[kCols];
    const int64_t j0 = (int64_t)blockIdx.y * kCols;
    stage_panels(sp, geom, n, j0);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kRows + threadIdx.x;
    if (i >= n) return;
    const double x[3] = {geom[G_CX * n + i], geom[G_CY * n + i], geom[G_CZ * n + i]};
    const double ni[3] = {geom[G_NX * n + i], geom[G_NY * n + i], geom[G_NZ * n + i]};
    const int jend = (int)min((int64_t)kCols, n - j0);
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        cplx s, g[3];
        pair_integrals(x, p, 0.0, mask, !direct, nullptr, s, g);
        const double* nn = direct ? p.n : ni;
        const int64_t o = j * n + i;
        SR[o] = -kInv4Pi * s.re;
        DR[o] = (i == j ? 0.5 : 0.0) - kInv4Pi * (nn[0] * g[0].re + nn[1] * g[1].re + nn[2] * g[2].re);
    }
}

// Per frequency z = blockIdx.z: S = SR + wave, D = DR + wave, written as FP64
// complex (S64, D64) and the FP32 LU copy of D (Dlo).
template <bool kDelh>
__global__ void __launch_bounds__(kRows)
k_wave_batch(const double* __restrict__ geom, int64_t n, int direct, const double* __restrict__ tab,
             const double* __restrict__ kvec, const double* __restrict__ SR,
             const double* __restrict__ DR, double2* __restrict__ S64, double2* __restrict__ D64,
             float2* __restrict__ Dlo, double2* __restrict__ tape)
{
    __shared__ Panel sp[kCols];
    const int64_t j0 = (int64_t)blockIdx.y * kCols;
    stage_panels(sp, geom, n, j0);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kRows + threadIdx.x;
    if (i >= n) return;
    const double k = kvec[blockIdx.z];
    const int64_t mat = (int64_t)blockIdx.z * n * n;
    const double x[3] = {geom[G_CX * n + i], geom[G_CY * n + i], geom[G_CZ * n + i]};
    const double ni[3] = {geom[G_NX * n + i], geom[G_NY * n + i], geom[G_NZ * n + i]};
    const int jend = (int)min((int64_t)kCols, n - j0);
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        cplx s, g[3];
        wave_pair<kDelh>(x, p, k, !direct, tab, s, g);
        const double* nn = direct ? p.n : ni;
        const int64_t o = j * n + i;
        if (kDelh && tape) {  // (G, G_r) for the adjoint of the same call
            const double dx = x[0] - p.c[0], dy = x[1] - p.c[1], dis2 = dx * dx + dy * dy;
            const double dis = (dis2 == 0.0) ? sqrt(dis2 + 1e-36) - 1e-18 : sqrt(dis2);
            cplx G[3];
            if (tab) delh_dimless_table(tab, k * dis, k * (x[2] + p.c[2]), G);
            else delh_dimless(k * dis, k * (x[2] + p.c[2]), G);
            tape[2 * (mat + o)] = make_double2(G[0].re, G[0].im);
            tape[2 * (mat + o) + 1] = make_double2(G[1].re, G[1].im);
        }
        double sr = SR[o] - kInv4Pi * s.re, si = -kInv4Pi * s.im;
        double dr = DR[o] - kInv4Pi * (nn[0] * g[0].re + nn[1] * g[1].re + nn[2] * g[2].re);
        double di = -kInv4Pi * (nn[0] * g[0].im + nn[1] * g[1].im + nn[2] * g[2].im);
        S64[mat + o] = make_double2(sr, si);
        D64[mat + o] = make_double2(dr, di);
        Dlo[mat + o] = make_float2((float)dr, (float)di);
    }
}

// Frequency-batched tabulated Delhommeau term.  Every frequency of the chunk
// sees the same panel pair, so the pair's polar angle alpha is fixed and only
// R = k d moves: the alpha direction of the four polar tables (B, C,
// E0 = e^z J0(r), E1 = e^z J1(r)) is contracted once per pair into
// w_q[i] = sum_j c_q[i][j] T_j(v(alpha)) (shared memory), and each frequency
// then evaluates four 1-D Chebyshev series in R (Clenshaw) with no
// transcendental calls; the log term splits as log(k) + log((d + |zeta|)/2).
// The series in R use the table's monomial-in-u copy (Horner's rule, four
// frequencies per pass).
// Frequencies at which the pair leaves the polar patch use the full table.
// Same arithmetic as wave_pair<true> up to reassociation (~1e-16).
// One pair of the frequency-batched pass and its output: S, D (FP64 and the
// FP32 copy of D) and the tape of frequency z from the dimensionless
// (G, G_r, G_z) in o3.
struct AllwPair {
    double dx, dy, rho, inv_rho, area, sr, dr;
    double n0, n1, n2;  // the normal of D (source panel when direct), held in registers
    int64_t o;          // pair offset j * n + i
    bool wrt_first;
};

__device__ __forceinline__ void allw_emit(const AllwPair& q, int z, double k, const cplx o3[3], int64_t nn,
                                          double2* __restrict__ S64, double2* __restrict__ D64,
                                          float2* __restrict__ Dlo, double2* __restrict__ tape)
{
    const double r = k * q.rho;
    double d1 = 0.0, d2 = 0.0;
    if (fabs(r) > 1e-6) {
        const double f = k * q.inv_rho;  // k^2 / r
        d1 = q.wrt_first ? f * q.dx : -f * q.dx;
        d2 = q.wrt_first ? f * q.dy : -f * q.dy;
    }
    const double ka = k * q.area;
    const cplx s = ka * o3[0];
    const cplx g0 = (ka * d1) * o3[1], g1 = (ka * d2) * o3[1], g2 = (ka * k) * o3[2];
    const double Sr = q.sr - kInv4Pi * s.re, Si = -kInv4Pi * s.im;
    const double Dr = q.dr - kInv4Pi * (q.n0 * g0.re + q.n1 * g1.re + q.n2 * g2.re);
    const double Di = -kInv4Pi * (q.n0 * g0.im + q.n1 * g1.im + q.n2 * g2.im);
    const int64_t m = (int64_t)z * nn + q.o;
    S64[m] = make_double2(Sr, Si);
    D64[m] = make_double2(Dr, Di);
    Dlo[m] = make_float2((float)Dr, (float)Di);
    if (tape) {  // (G, G_r) for the adjoint of the same call
        tape[2 * m] = make_double2(o3[0].re, o3[0].im);
        tape[2 * m + 1] = make_double2(o3[1].re, o3[1].im);
    }
}

// The four polar functions' monomial-in-u coefficients in constant memory:
// every lane of the alpha contraction reads the same coefficient, which the
// constant cache broadcasts.  Copied from the context's table before each
// launch; every context builds the same table, so concurrent copies write
// identical bytes.
__constant__ double c_polar_mono[4 * kTabPolarFn];
// The same coefficients rounded to FP32 (the FP32 alpha contraction).
__constant__ float c_polar_mono_f[4 * kTabPolarFn];

template <typename CT>
__device__ __forceinline__ CT polar_coef(int i);
template <>
__device__ __forceinline__ double polar_coef<double>(int i) { return c_polar_mono[i]; }
template <>
__device__ __forceinline__ float polar_coef<float>(int i) { return c_polar_mono_f[i]; }

constexpr int kWT = 128;  // threads (rows) per CTA of k_wave_delh_allw
constexpr int kAllwMaxFreqs = 128;  // frequencies per launch of k_wave_delh_allw
// k, log k and 1/k per frequency, then the contracted series of every row
// in the type HT of the per-frequency Horner pass (the polar coefficients
// are read from constant memory)
template <typename HT>
constexpr size_t wave_allw_smem()
{
    return sizeof(double) * 3 * kAllwMaxFreqs + sizeof(HT) * 4 * kTabNU * kWT;
}
constexpr size_t kWaveAllwSmem = wave_allw_smem<double>();

__global__ void k_coef_to_f32(const double* __restrict__ a, float* __restrict__ b, int count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) b[t] = (float)a[t];
}

__device__ __forceinline__ double hfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float hfma(float a, float b, float c) { return fmaf(a, b, c); }

// HT: the type of the per-frequency Horner series in R; CT: the type of the
// alpha contraction (double, or float in the reduced-precision levels of the
// mixed path, mh_ctx_set_wave_series_fp32).  The pair geometry, the log
// terms and everything after the series stay in FP64.
template <typename HT, typename CT>
__global__ void __launch_bounds__(kWT, 3)
k_wave_delh_allw(const double* __restrict__ geom, int64_t n, int direct, const double* __restrict__ tab,
                 const double* __restrict__ kvec, int nb, const double* __restrict__ SR,
                 const double* __restrict__ DR, double2* __restrict__ S64, double2* __restrict__ D64,
                 float2* __restrict__ Dlo, double2* __restrict__ tape, int* __restrict__ fall)
{
    extern __shared__ double wsm[];
    double* logk = wsm;                            // [nb]
    double* invk = logk + kAllwMaxFreqs;           // [nb], nb <= kAllwMaxFreqs
    double* ksm = invk + kAllwMaxFreqs;            // [nb]
    HT* w = reinterpret_cast<HT*>(ksm + kAllwMaxFreqs);  // [4 * NU][kWT]
    __shared__ Panel sp[kCols];
    const int64_t j0 = (int64_t)blockIdx.y * kCols;
    stage_panels(sp, geom, n, j0);
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        ksm[t] = kvec[t];
        logk[t] = log(kvec[t]);
        invk[t] = 1.0 / kvec[t];
    }
    __syncthreads();
    const int tid = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * kWT + tid;
    if (i >= n) return;
    const int64_t nn = n * n;
    const double x[3] = {geom[G_CX * n + i], geom[G_CY * n + i], geom[G_CZ * n + i]};
    const double ni[3] = {geom[G_NX * n + i], geom[G_NY * n + i], geom[G_NZ * n + i]};
    const bool wrt_first = !direct;
    const int jend = (int)min((int64_t)kCols, n - j0);
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        const int64_t o = j * n + i;
        // pair geometry (abstract_greens_function.jl:111-131 at k = 1)
        const double dx = x[0] - p.c[0], dy = x[1] - p.c[1];
        const double dis2 = dx * dx + dy * dy;
        const double purt = 1e-18;
        const double rho = (dis2 == 0.0) ? sqrt(dis2 + purt * purt) - purt : sqrt(dis2);
        const double zeta = x[2] + p.c[2];
        const double az = -zeta;
        const double d = hypot(rho, zeta);
        const bool polar_ok = az >= 0.0;
        const double v = 4.0 * atan2(rho, az) / kPi - 1.0;
        const double lp = log(0.5 * (d + az));
        const double gp = rho / (d * (d + az));
        const double inv_d = 1.0 / d, inv_rho = rho > 0.0 ? 1.0 / rho : 0.0;
        const double sr = SR[o], dr = DR[o];
        // contract alpha: w_q[row] = sum_j c_q[row][j] T_j(v), the four
        // functions' Clenshaw recurrences interleaved (four independent
        // dependency chains per row)
        if (polar_ok) {
            const CT vc = (CT)v, v2 = (CT)(2.0 * v);
#pragma unroll 1
            for (int row = 0; row < kTabNU; ++row) {
                const int cr = row * kTabNV;
                CT b1[4] = {0, 0, 0, 0}, b2[4] = {0, 0, 0, 0};
#pragma unroll
                for (int col = kTabNV - 1; col >= 1; --col) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const CT t = hfma(v2, b1[q], polar_coef<CT>(cr + q * kTabPolarFn + col) - b2[q]);
                        b2[q] = b1[q];
                        b1[q] = t;
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    w[(q * kTabNU + row) * kWT + tid] = (HT)hfma(vc, b1[q], polar_coef<CT>(cr + q * kTabPolarFn) - b2[q]);
            }
        }
        const AllwPair q{dx, dy, rho, inv_rho, p.area, sr, dr, direct ? p.n[0] : ni[0], direct ? p.n[1] : ni[1],
                         direct ? p.n[2] : ni[2], o, wrt_first};
        // four frequencies per Horner pass: each coefficient read from shared
        // memory feeds four recurrences.  Frequencies off the polar patch are
        // only counted here: k_wave_delh_allw_rest evaluates them with the
        // full table, so this kernel makes no out-of-line call (whose calling
        // convention would cost spills on the hot path)
        constexpr int kZP = 4;
        int nfall = 0;
        for (int z0 = 0; z0 < nb; z0 += kZP) {
            const int nz = min(kZP, nb - z0);
            double kz[kZP];
            HT uz[kZP];
            bool pz[kZP];
            bool anyp = false;
#pragma unroll
            for (int t = 0; t < kZP; ++t) {
                kz[t] = ksm[z0 + (t < nz ? t : 0)];
                const double R = kz[t] * d;
                pz[t] = t < nz && polar_ok && R < kTabRPolar;
                anyp |= pz[t];
                uz[t] = (HT)(2.0 * R / kTabRPolar - 1.0);
            }
            HT val[kZP][4];
            if (anyp) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const HT c = w[(q * kTabNU + kTabNU - 1) * kWT + tid];
#pragma unroll
                    for (int t = 0; t < kZP; ++t) val[t][q] = c;
                }
#pragma unroll
                for (int row = kTabNU - 2; row >= 0; --row) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const HT c = w[(q * kTabNU + row) * kWT + tid];
#pragma unroll
                        for (int t = 0; t < kZP; ++t) val[t][q] = hfma(val[t][q], uz[t], c);
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < kZP; ++t) {
                if (t >= nz) break;
                if (!pz[t]) {
                    ++nfall;
                    continue;
                }
                const int z = z0 + t;
                const double ik = invk[z];
                const double B = (double)val[t][0], C = (double)val[t][1], E0 = (double)val[t][2],
                             E1 = (double)val[t][3];
                const double L = logk[z] + lp;
                const double G_re = -2.0 * E0 * L + B, G_im = 2.0 * kPi * E0;
                cplx o3[3];
                o3[0] = mk(G_re, G_im);
                o3[1] = mk(2.0 * E1 * L - 2.0 * E0 * gp * ik + C, -2.0 * kPi * E1);
                o3[2] = mk(G_re + 2.0 * inv_d * ik, G_im);  // 2 / R, R = k d
                allw_emit(q, z, kz[t], o3, nn, S64, D64, Dlo, tape);
            }
        }
        if (nfall) *fall = 1;
    }
}

// The frequencies k_wave_delh_allw left to the full table (pairs above the
// free surface or at R = k d >= 2); exits at once when it flagged none.  The
// test takes a margin of 1e-12 in R so that a pair on the patch edge is
// written by one kernel at least, whatever the rounding of d in each (a pair
// written by both gets this kernel's value, which runs second).
__global__ void __launch_bounds__(kWT)
k_wave_delh_allw_rest(const int* __restrict__ fall, const double* __restrict__ geom, int64_t n, int direct,
                      const double* __restrict__ tab, const double* __restrict__ kvec, int nb,
                      const double* __restrict__ SR, const double* __restrict__ DR, double2* __restrict__ S64,
                      double2* __restrict__ D64, float2* __restrict__ Dlo, double2* __restrict__ tape)
{
    if (*fall == 0) return;
    __shared__ Panel sp[kCols];
    const int64_t j0 = (int64_t)blockIdx.y * kCols;
    stage_panels(sp, geom, n, j0);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kWT + threadIdx.x;
    if (i >= n) return;
    const int64_t nn = n * n;
    const double x[3] = {geom[G_CX * n + i], geom[G_CY * n + i], geom[G_CZ * n + i]};
    const double ni[3] = {geom[G_NX * n + i], geom[G_NY * n + i], geom[G_NZ * n + i]};
    const int jend = (int)min((int64_t)kCols, n - j0);
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t o = (j0 + jj) * n + i;
        const double dx = x[0] - p.c[0], dy = x[1] - p.c[1];
        const double dis2 = dx * dx + dy * dy;
        const double purt = 1e-18;
        const double rho = (dis2 == 0.0) ? sqrt(dis2 + purt * purt) - purt : sqrt(dis2);
        const double zeta = x[2] + p.c[2];
        const double d = hypot(rho, zeta);
        const bool polar_ok = -zeta >= 0.0;
        const double* nn3 = direct ? p.n : ni;
        const AllwPair q{dx, dy, rho, rho > 0.0 ? 1.0 / rho : 0.0, p.area, SR[o], DR[o], nn3[0], nn3[1], nn3[2], o,
                         !direct};
#pragma unroll 1
        for (int z = 0; z < nb; ++z) {
            const double k = kvec[z];
            if (polar_ok && k * d < kTabRPolar * (1.0 - 1e-12)) continue;
            cplx o3[3];
            delh_dimless_table(tab, k * rho, k * zeta, o3);
            allw_emit(q, z, k, o3, nn, S64, D64, Dlo, tape);
        }
    }
}

// Copies of the Rankine part when the Green-function tuple has no wave term.
__global__ void k_no_wave_batch(int64_t nn, const double* __restrict__ SR,
                                const double* __restrict__ DR, double2* __restrict__ S64,
                                double2* __restrict__ D64, float2* __restrict__ Dlo)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nn) return;
    const int64_t mat = (int64_t)blockIdx.y * nn;
    S64[mat + t] = make_double2(SR[t], 0.0);
    D64[mat + t] = make_double2(DR[t], 0.0);
    Dlo[mat + t] = make_float2((float)DR[t], 0.f);
}

// Boundary conditions of every right-hand side of frequency blockIdx.y:
// q < ndof: radiation -i omega (n . dof_q) (src/waves.jl:89-101);
// q >= ndof: incident Airy wave of heading beta_{q-ndof} (src/waves.jl:121-142).
__global__ void k_bc_batch(const double* __restrict__ geom, int64_t n, const double* __restrict__ dofs,
                           int ndof, const double* __restrict__ betas, int nbeta,
                           const double* __restrict__ omegas, double gacc, double2* __restrict__ BC)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nrhs = ndof + nbeta;
    const double w = omegas[blockIdx.y];
    double2* out = BC + (int64_t)blockIdx.y * n * nrhs;
    const double nx = geom[G_NX * n + i], ny = geom[G_NY * n + i], nz = geom[G_NZ * n + i];
    for (int q = 0; q < ndof; ++q) {
        const double* d = dofs + (int64_t)q * 3 * n;
        double nd = nx * d[i] + ny * d[n + i] + nz * d[2 * n + i];
        out[(int64_t)q * n + i] = make_double2(0.0, -w * nd);
    }
    const double k = w * w / gacc;
    const double x = geom[G_CX * n + i], y = geom[G_CY * n + i], z = geom[G_CZ * n + i];
    const double cih = exp(k * z), f = gacc * k / w;
    for (int b = 0; b < nbeta; ++b) {
        double cb, sb, cw, sw;
        sincos(betas[b], &sb, &cb);
        sincos(k * (x * cb + y * sb), &sw, &cw);
        cplx e = mk(f * cw, f * sw);
        cplx vn = e * (cb * cih * nx) + e * (sb * cih * ny) + e * mk(0.0, -cih * nz);
        out[(int64_t)(ndof + b) * n + i] = make_double2(-vn.re, -vn.im);
    }
}

// Forces of right-hand side q of frequency z (blockIdx.x = z*nrhs + q):
// F_i = sum_j (i rho omega phi_j) * (-(n_j . dof_i,j)) * area_j for every
// influenced dof i (src/waves.jl:72-85); for diffraction right-hand sides
// also the Froude-Krylov force of the same heading (src/waves.jl:157-163).
__global__ void __launch_bounds__(256)
k_forces_batch(const double* __restrict__ geom, int64_t n, const double* __restrict__ dofs, int ndof,
               const double* __restrict__ betas, int nbeta, const double* __restrict__ omegas,
               double rho, double gacc, const double2* __restrict__ phi, double2* __restrict__ F,
               double2* __restrict__ FK)
{
    const int nrhs = ndof + nbeta;
    const int z = blockIdx.x / nrhs, q = blockIdx.x % nrhs;
    const double w = omegas[z];
    const double2* ph = phi + ((int64_t)z * nrhs + q) * n;
    const bool diff = q >= ndof;
    double fr[kMaxRhs], fi[kMaxRhs], kr[kMaxRhs], ki[kMaxRhs];
    for (int d = 0; d < ndof; ++d) fr[d] = fi[d] = kr[d] = ki[d] = 0.0;
    double k = w * w / gacc, cb = 1.0, sb = 0.0;
    if (diff) sincos(betas[q - ndof], &sb, &cb);
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const double nx = geom[G_NX * n + j], ny = geom[G_NY * n + j], nz = geom[G_NZ * n + j];
        const double a = geom[G_AREA * n + j];
        // i rho omega phi
        const double pr = -rho * w * ph[j].y, pi = rho * w * ph[j].x;
        double ar = 0.0, ai = 0.0;
        if (diff) {  // airy pressure i omega rho phi_inc = rho g e^{kz} e^{i k wbar}
            const double x = geom[G_CX * n + j], y = geom[G_CY * n + j], zz = geom[G_CZ * n + j];
            double sw, cw;
            sincos(k * (x * cb + y * sb), &sw, &cw);
            const double m = rho * gacc * exp(k * zz);
            ar = m * cw;
            ai = m * sw;
        }
        for (int d = 0; d < ndof; ++d) {
            const double* dd = dofs + (int64_t)d * 3 * n;
            const double wgt = -(nx * dd[j] + ny * dd[n + j] + nz * dd[2 * n + j]) * a;
            fr[d] += pr * wgt;
            fi[d] += pi * wgt;
            kr[d] += ar * wgt;
            ki[d] += ai * wgt;
        }
    }
    __shared__ double red[8][4 * kMaxRhs];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 0; d < ndof; ++d) {
        double v[4] = {fr[d], fi[d], kr[d], ki[d]};
        for (int c = 0; c < 4; ++c) {
            double s = v[c];
            for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
            if (lane == 0) red[warp][4 * d + c] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x < 4 * ndof) {
        double s = 0.0;
        for (int wp = 0; wp < (int)(blockDim.x >> 5); ++wp) s += red[wp][threadIdx.x];
        red[0][threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x < ndof) {
        const int d = threadIdx.x;
        F[((int64_t)z * nrhs + q) * ndof + d] = make_double2(red[0][4 * d], red[0][4 * d + 1]);
        if (diff)
            FK[((int64_t)z * nbeta + (q - ndof)) * ndof + d] =
                make_double2(red[0][4 * d + 2], red[0][4 * d + 3]);
    }
}

__global__ void k_to_f32(const double2* __restrict__ a, float2* __restrict__ b, int64_t count)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) b[t] = make_float2((float)a[t].x, (float)a[t].y);
}

__global__ void k_add_f32(double2* __restrict__ x, const float2* __restrict__ d, int64_t count)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) x[t] = make_double2(x[t].x + (double)d[t].x, x[t].y + (double)d[t].y);
}

// Batched complex matrix products with few columns in FP64 (refinement
// residuals, S b, S^H lambda), bandwidth-bound reads of the n x n matrices
// (column-major, nb of them, n*n apart), nrhs <= kMaxRhs:
// k_resid_n: R = beta B + alpha A X, one thread per row i, coalesced down the
// columns; k_resid_c: R = beta B + alpha A^H X, one warp per JW outputs j
// reading columns j (each x entry loaded once for the JW columns).  B may be R (read before written) or null when beta = 0.
// Q >= nrhs: accumulators per thread (4, 8 or 16, picked by the launcher).
template <int Q>
__global__ void __launch_bounds__(256)
k_resid_n(const double2* __restrict__ A, const double2* __restrict__ X, const double2* B, double2* R, int64_t n,
          int nrhs, double alpha, double beta, const int* done, const int* bad)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t b = blockIdx.y;
    if (i >= n) return;
    if (done && (done[b] || bad[b])) return;  // refinement: converged or marked matrices
    const double2* M = A + b * n * n;
    const double2* x = X + b * n * nrhs;
    double ar[Q], ai[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) ar[q] = ai[q] = 0.0;
#pragma unroll 4
    for (int64_t j = 0; j < n; ++j) {
        const double2 m = M[j * n + i];
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q < nrhs) {
                const double2 v = __ldg(x + (int64_t)q * n + j);
                ar[q] = fma(m.x, v.x, fma(-m.y, v.y, ar[q]));
                ai[q] = fma(m.x, v.y, fma(m.y, v.x, ai[q]));
            }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q)
        if (q < nrhs) {
            const int64_t o = b * n * nrhs + (int64_t)q * n + i;
            const double2 bo = B ? B[o] : make_double2(0.0, 0.0);
            R[o] = make_double2(beta * bo.x + alpha * ar[q], beta * bo.y + alpha * ai[q]);
        }
}

template <int Q, int JW>
__global__ void __launch_bounds__(256, 2)
k_resid_c(const double2* __restrict__ A, const double2* __restrict__ X, const double2* B, double2* R, int64_t n,
          int nrhs, double alpha, double beta, const int* done, const int* bad)
{
    const int lane = threadIdx.x & 31;
    const int64_t j0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * JW;
    const int64_t b = blockIdx.y;
    if (j0 >= n) return;  // whole warps leave together
    if (done && (done[b] || bad[b])) return;  // refinement: converged or marked matrices
    const double2* M = A + b * n * n;
    const double2* x = X + b * n * nrhs;
    int64_t jc[JW];  // columns of this warp (the last one repeated past n, not stored)
#pragma unroll
    for (int u = 0; u < JW; ++u) jc[u] = min(j0 + u, n - 1);
    double ar[JW][Q], ai[JW][Q];
#pragma unroll
    for (int u = 0; u < JW; ++u)
#pragma unroll
        for (int q = 0; q < Q; ++q) ar[u][q] = ai[u][q] = 0.0;
#pragma unroll 4
    for (int64_t i = lane; i < n; i += 32) {
        double2 m[JW];
#pragma unroll
        for (int u = 0; u < JW; ++u) m[u] = M[jc[u] * n + i];
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q < nrhs) {  // conj(m) * x, each x entry read once for JW columns
                const double2 v = __ldg(x + (int64_t)q * n + i);
#pragma unroll
                for (int u = 0; u < JW; ++u) {
                    ar[u][q] = fma(m[u].x, v.x, fma(m[u].y, v.y, ar[u][q]));
                    ai[u][q] = fma(m[u].x, v.y, fma(-m[u].y, v.x, ai[u][q]));
                }
            }
    }
#pragma unroll
    for (int u = 0; u < JW; ++u)
#pragma unroll
        for (int q = 0; q < Q; ++q)
            if (q < nrhs) {
                for (int off = 16; off > 0; off >>= 1) {
                    ar[u][q] += __shfl_down_sync(0xffffffffu, ar[u][q], off);
                    ai[u][q] += __shfl_down_sync(0xffffffffu, ai[u][q], off);
                }
                if (lane == 0 && j0 + u < n) {
                    const int64_t o = b * n * nrhs + (int64_t)q * n + j0 + u;
                    const double2 bo = B ? B[o] : make_double2(0.0, 0.0);
                    R[o] = make_double2(beta * bo.x + alpha * ar[u][q], beta * bo.y + alpha * ai[u][q]);
                }
            }
}

// Per (frequency z = blockIdx.x): max over right-hand sides of
// max_i |r_iq| / max_i |b_iq|.
__global__ void __launch_bounds__(256)
k_rel_residual(const double2* __restrict__ r, const double2* __restrict__ b, int64_t n, int nrhs,
               double* __restrict__ out, double tol, int* done, const int* bad, int* sweeps, int sweep)
{
    __shared__ double sr[256], sb[256];
    // refinement control (done != null): skip converged or marked matrices,
    // mark the ones that reach tol and count the sweeps of each
    if (done && (done[blockIdx.x] || bad[blockIdx.x])) return;
    double worst = 0.0;
    for (int q = 0; q < nrhs; ++q) {
        const int64_t off = ((int64_t)blockIdx.x * nrhs + q) * n;
        double mr = 0.0, mb = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            mr = fmax(mr, hypot(r[off + i].x, r[off + i].y));
            mb = fmax(mb, hypot(b[off + i].x, b[off + i].y));
        }
        sr[threadIdx.x] = mr;
        sb[threadIdx.x] = mb;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                sr[threadIdx.x] = fmax(sr[threadIdx.x], sr[threadIdx.x + s]);
                sb[threadIdx.x] = fmax(sb[threadIdx.x], sb[threadIdx.x + s]);
            }
            __syncthreads();
        }
        if (sb[0] > 0.0) worst = fmax(worst, sr[0] / sb[0]);
        else if (sr[0] > 0.0 || sr[0] != sr[0]) worst = INFINITY;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        worst = (worst == worst) ? worst : INFINITY;
        out[blockIdx.x] = worst;
        if (done) {
            sweeps[blockIdx.x] = sweep;
            if (worst <= tol) done[blockIdx.x] = 1;
        }
    }
}

// X += d and R32 = fp32(R) of the refinement, skipping converged or marked
// matrices (per = entries per matrix).
__global__ void k_refine_add(double2* __restrict__ x, const float2* __restrict__ d, int64_t per, int64_t count,
                             const int* __restrict__ done, const int* __restrict__ bad)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int64_t z = t / per;
    if (done[z] || bad[z]) return;
    x[t] = make_double2(x[t].x + (double)d[t].x, x[t].y + (double)d[t].y);
}

__global__ void k_refine_to_f32(const double2* __restrict__ a, float2* __restrict__ b, int64_t per, int64_t count,
                                const int* __restrict__ done, const int* __restrict__ bad)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int64_t z = t / per;
    if (done[z] || bad[z]) return;
    b[t] = make_float2((float)a[t].x, (float)a[t].y);
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------

unsigned blocks(int64_t count, int threads) { return (unsigned)((count + threads - 1) / threads); }

}  // namespace

int zgemm_strided(mh_ctx* ctx, int64_t n, int nrhs, const double2* A, const double2* B, double2* C,
                  int nb, double alpha_re, double beta_re)
{
    const cuDoubleComplex alpha = make_cuDoubleComplex(alpha_re, 0.0);
    const cuDoubleComplex beta = make_cuDoubleComplex(beta_re, 0.0);
    cublasStatus_t st = cublasZgemmStridedBatched(
        ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, nrhs, (int)n, &alpha,
        (const cuDoubleComplex*)A, (int)n, n * n, (const cuDoubleComplex*)B, (int)n, n * nrhs, &beta,
        (cuDoubleComplex*)C, (int)n, n * nrhs, nb);
    if (st != CUBLAS_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cublasZgemmStridedBatched failed (%d)", (int)st);
    return MH_OK;
}

int fp64_lu_factor(mh_ctx* ctx, int64_t n, double2* A, int* piv)
{
    int lwork = 0;
    cusolverStatus_t st = cusolverDnZgetrf_bufferSize(ctx->cusolver, (int)n, (int)n,
                                                      (cuDoubleComplex*)A, (int)n, &lwork);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrf_bufferSize failed (%d)", (int)st);
    auto* work = (cuDoubleComplex*)ws_get(ctx, WS_LWORK, sizeof(cuDoubleComplex) * (size_t)lwork);
    auto* info = (int*)ws_get(ctx, WS_INFO, sizeof(int) * 2);
    if (!work || !info) return MH_ERR_OOM;
    st = cusolverDnZgetrf(ctx->cusolver, (int)n, (int)n, (cuDoubleComplex*)A, (int)n, work, piv, info);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrf failed (%d)", (int)st);
    int h = 0;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    if (h > 0) return set_err(ctx, MH_ERR_SINGULAR, "zero pivot at column %d", h);
    return MH_OK;
}

int fp64_getrs(mh_ctx* ctx, bool conj_trans, int64_t n, const double2* LU, const int* piv, double2* B,
               int nrhs)
{
    auto* info = (int*)ws_get(ctx, WS_INFO, sizeof(int) * 2);
    if (!info) return MH_ERR_OOM;
    cusolverStatus_t st = cusolverDnZgetrs(ctx->cusolver, conj_trans ? CUBLAS_OP_C : CUBLAS_OP_N,
                                           (int)n, nrhs, (const cuDoubleComplex*)LU, (int)n, piv,
                                           (cuDoubleComplex*)B, (int)n, info + 1);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrs failed (%d)", (int)st);
    return MH_OK;
}

int fp64_lu_solve(mh_ctx* ctx, int64_t n, double2* A, double2* B, int nrhs)
{
    auto* piv = (int*)ws_get(ctx, WS_PIV, sizeof(int) * (size_t)n);
    if (!piv) return MH_ERR_OOM;
    int rc = fp64_lu_factor(ctx, n, A, piv);
    if (rc) return rc;
    return fp64_getrs(ctx, false, n, A, piv, B, nrhs);
}

namespace {

// FP64 path: one frequency at a time.
int run_fp64(const Batch& bt, const double* d_omegas, int nomega, double2* d_F, double2* d_FK)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const size_t mat = sizeof(double2) * (size_t)n * (size_t)n;
    const size_t vec = sizeof(double2) * (size_t)n * (size_t)bt.nrhs;
    auto* S = (double2*)ws_get(ctx, WS_S, mat);
    auto* D = (double2*)ws_get(ctx, WS_D, mat);
    auto* BC = (double2*)ws_get(ctx, WS_RHS, vec);
    auto* X = (double2*)ws_get(ctx, WS_PHI, vec);
    if (!S || !D || !BC || !X) return MH_ERR_OOM;
    int rc;
    const double* tab = delh_table_for(ctx, bt.mask, &rc);
    if (rc) return rc;
    std::vector<double> h_w(nomega);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h_w.data(), d_omegas, sizeof(double) * nomega,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int z = 0; z < nomega; ++z) {
        const double k = h_w[z] * h_w[z] / bt.g;
        phase_begin(ctx, PH_FP64_ASSEMBLY);
        MH_CUDA_TRY(ctx, launch_assemble_f64(ctx, bt.m, k, bt.mask, bt.direct, tab, S, D));
        phase_end(ctx, PH_FP64_ASSEMBLY);
        k_bc_batch<<<dim3(blocks(n, 256), 1), 256, 0, ctx->stream>>>(
            bt.m->geom, n, bt.d_dofs, bt.ndof, bt.d_betas, bt.nbeta, d_omegas + z, bt.g, BC);
        ctx->launches += 1;
        if (bt.direct) {
            if ((rc = zgemm_strided(ctx, n, bt.nrhs, S, BC, X, 1, 1.0, 0.0))) return rc;
            phase_begin(ctx, PH_FP64_LU);
            if ((rc = fp64_lu_solve(ctx, n, D, X, bt.nrhs))) return rc;
            phase_end(ctx, PH_FP64_LU);
        } else {
            phase_begin(ctx, PH_FP64_LU);
            if ((rc = fp64_lu_solve(ctx, n, D, BC, bt.nrhs))) return rc;
            phase_end(ctx, PH_FP64_LU);
            if ((rc = zgemm_strided(ctx, n, bt.nrhs, S, BC, X, 1, 1.0, 0.0))) return rc;
        }
        k_forces_batch<<<bt.nrhs, 256, 0, ctx->stream>>>(
            bt.m->geom, n, bt.d_dofs, bt.ndof, bt.d_betas, bt.nbeta, d_omegas + z, bt.rho, bt.g, X,
            d_F + (int64_t)z * bt.nrhs * bt.ndof, d_FK + (int64_t)z * bt.nbeta * bt.ndof);
        ctx->launches += 1;
        MH_CUDA_TRY(ctx, cudaGetLastError());
    }
    return MH_OK;
}

}  // namespace

// Mixed path for one chunk of `nb` frequencies.
int run_mixed_chunk(const Batch& bt, const double* d_omegas, const double* d_k, int nb,
                    const double* SR, const double* DR, double tol, int max_iter, double2* d_F,
                    double2* d_FK, mh_batch_info* info, FallbackStore* fb)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n, nn = n * n;
    const int nrhs = bt.nrhs;
    const int64_t nv = n * nrhs;
    auto* S64 = (double2*)ws_get(ctx, WS_S, sizeof(double2) * nn * nb);
    auto* D64 = (double2*)ws_get(ctx, WS_D, sizeof(double2) * nn * nb);
    auto* Dlo = (float2*)ws_get(ctx, WS_LO, sizeof(float2) * nn * nb);
    const bool tc = ctx->lu_backend == MH_LU_TCGEN05_F16;
    const int64_t dinv_stride = tc ? lu_dinv_stride_tc(n) : lu_dinv_stride(n);
    auto* Dinv = (float2*)ws_get(ctx, WS_DINV, sizeof(float2) * dinv_stride * nb);
    auto* T32 = (float2*)ws_get(ctx, WS_TMP32B, sizeof(float2) * n * nrhs * nb);
    auto* BC = (double2*)ws_get(ctx, WS_RHS, sizeof(double2) * nv * nb);
    auto* X = (double2*)ws_get(ctx, WS_PHI, sizeof(double2) * nv * nb);
    auto* R = (double2*)ws_get(ctx, WS_TMP, sizeof(double2) * nv * nb * 2);
    auto* R32 = (float2*)ws_get(ctx, WS_TMP32, sizeof(float2) * nv * nb);
    auto* misc = (char*)ws_get(ctx, WS_MISC, refine_ctl_bytes(nb) + 64);
    if (!S64 || !D64 || !Dlo || !Dinv || !T32 || !BC || !X || !R || !R32 || !misc) return MH_ERR_OOM;
    double2* RHS = R + nv * nb;  // right-hand side of the D (or K) system
    const RefineCtl ctl = refine_ctl(misc, nb);
    int* d_bad = ctl.bad;
    auto* d_fall = (int*)(misc + refine_ctl_bytes(nb));  // set when the frequency-batched pass left pairs to the full table
    int rc;
    const double* tab = delh_table_for(ctx, bt.mask, &rc);
    if (rc) return rc;
    // matrices
    const uint32_t wave = bt.mask & (MH_GF_WU | MH_GF_DELHOMMEAU);
    dim3 grid(blocks(n, kRows), blocks(n, kCols), (unsigned)nb);
    phase_begin(ctx, PH_WAVE);
    if (wave == MH_GF_WU)
        k_wave_batch<false><<<grid, kRows, 0, ctx->stream>>>(bt.m->geom, n, bt.direct, nullptr, d_k, SR,
                                                            DR, S64, D64, Dlo, nullptr);
    else if (wave == MH_GF_DELHOMMEAU && tab && nb >= kAllwMinFreqs) {
        const int lvl = ctx->wave_series_fp32;
        auto* wk = lvl == 2 ? k_wave_delh_allw<float, float>
                 : lvl == 1 ? k_wave_delh_allw<float, double> : k_wave_delh_allw<double, double>;
        const size_t wsm = lvl ? wave_allw_smem<float>() : wave_allw_smem<double>();
        MH_CUDA_TRY(ctx, cudaFuncSetAttribute(wk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm));
        if (lvl == 2) {  // FP32 copy of the polar coefficients for the FP32 contraction
            auto* cf = (float*)ws_get(ctx, WS_COEF32, sizeof(float) * 4 * kTabPolarFn);
            if (!cf) return MH_ERR_OOM;
            k_coef_to_f32<<<blocks(4 * kTabPolarFn, 256), 256, 0, ctx->stream>>>(tab + kTabMonoOff, cf,
                                                                                 4 * kTabPolarFn);
            ctx->launches += 1;
            MH_CUDA_TRY(ctx, cudaMemcpyToSymbolAsync(c_polar_mono_f, cf, sizeof(float) * 4 * kTabPolarFn, 0,
                                                     cudaMemcpyDeviceToDevice, ctx->stream));
        }
        MH_CUDA_TRY(ctx, cudaMemcpyToSymbolAsync(c_polar_mono, tab + kTabMonoOff, sizeof(c_polar_mono), 0,
                                                 cudaMemcpyDeviceToDevice, ctx->stream));
        for (int z = 0; z < nb; z += kAllwMaxFreqs) {
            const int m = std::min(kAllwMaxFreqs, nb - z);
            const int64_t off = (int64_t)z * nn;
            double2* tp = bt.tape ? bt.tape + 2 * off : nullptr;
            const dim3 g2(blocks(n, kWT), blocks(n, kCols));
            MH_CUDA_TRY(ctx, cudaMemsetAsync(d_fall, 0, sizeof(int), ctx->stream));
            wk<<<g2, kWT, wsm, ctx->stream>>>(bt.m->geom, n, bt.direct, tab, d_k + z, m, SR, DR, S64 + off,
                                              D64 + off, Dlo + off, tp, d_fall);
            k_wave_delh_allw_rest<<<g2, kWT, 0, ctx->stream>>>(d_fall, bt.m->geom, n, bt.direct, tab, d_k + z, m,
                                                              SR, DR, S64 + off, D64 + off, Dlo + off, tp);
            ctx->launches += 1 + (z > 0);
        }
    } else if (wave == MH_GF_DELHOMMEAU)
        k_wave_batch<true><<<grid, kRows, 0, ctx->stream>>>(bt.m->geom, n, bt.direct, tab, d_k, SR, DR,
                                                           S64, D64, Dlo, bt.tape);
    else if (wave == 0)
        k_no_wave_batch<<<dim3(blocks(nn, 256), nb), 256, 0, ctx->stream>>>(nn, SR, DR, S64, D64, Dlo);
    else
        return set_err(ctx, MH_ERR_ARG, "the mixed path takes one wave term (GFWu or Delhommeau)");
    ctx->launches += 1;
    phase_end(ctx, PH_WAVE);
    phase_begin(ctx, PH_RHS);
    k_bc_batch<<<dim3(blocks(n, 256), nb), 256, 0, ctx->stream>>>(
        bt.m->geom, n, bt.d_dofs, bt.ndof, bt.d_betas, bt.nbeta, d_omegas, bt.g, BC);
    ctx->launches += 1;
    MH_CUDA_TRY(ctx, cudaGetLastError());
    if (bt.direct) {
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, S64, n, nb, BC, nullptr, RHS, nrhs, 1.0, 0.0));
    } else {
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(RHS, BC, sizeof(double2) * nv * nb, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
    }
    phase_end(ctx, PH_RHS);
    // FP32 LU of every D (or K)
    MH_CUDA_TRY(ctx, cudaMemsetAsync(d_bad, 0, sizeof(int) * nb, ctx->stream));
    phase_begin(ctx, PH_LU);
    if (tc) {
        auto* panels = (unsigned char*)ws_get(ctx, WS_PANEL, (size_t)lu_panel_bytes_tc(n) * nb);
        if (!panels) return MH_ERR_OOM;
        MH_CUDA_TRY(ctx, launch_lu_tc(ctx, Dlo, n, nn, nb, Dinv, panels, d_bad));
    }
    else MH_CUDA_TRY(ctx, launch_lu_f32(ctx, Dlo, n, nn, nb, Dinv, d_bad));
    phase_end(ctx, PH_LU);
    phase_begin(ctx, PH_REFINE);
    RefineState h;
    if ((rc = refine_sweeps(ctx, false, n, nb, nrhs, D64, Dlo, Dinv, RHS, X, R, R32, ctl, tol, max_iter, h)))
        return rc;
    phase_end(ctx, PH_REFINE);
    info->refine_iterations = std::max(info->refine_iterations, h.most_sweeps());
    // FP64 fallback for bad (pivot, wait timeout) or unconverged problems
    for (int z = 0; z < nb; ++z) {
        if (h.ok(z)) {
            info->max_rel_residual = std::max(info->max_rel_residual, h.res[z]);
            continue;
        }
        info->n_fallback += 1;
        double2* Xz = X + (int64_t)z * nv;
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(Xz, RHS + (int64_t)z * nv, sizeof(double2) * nv,
                                         cudaMemcpyDeviceToDevice, ctx->stream));
        if (fb) {  // keep D: factor a copy and keep its pivots for the adjoint solve
            if ((rc = fallback_factor(ctx, fb, n, nb, z, D64 + (int64_t)z * nn))) return rc;
            if ((rc = fp64_getrs(ctx, false, n, fb->lu + (int64_t)z * nn, fb->piv + z * n, Xz, nrhs)))
                return rc;
        } else if ((rc = fp64_lu_solve(ctx, n, D64 + (int64_t)z * nn, Xz, nrhs))) {
            return rc;
        }
    }
    // indirect: phi = S sigma
    double2* PHI = X;
    if (!bt.direct) {
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, S64, n, nb, X, nullptr, R, nrhs, 1.0, 0.0));
        PHI = R;
    }
    phase_begin(ctx, PH_FORCES);
    k_forces_batch<<<nb * nrhs, 256, 0, ctx->stream>>>(bt.m->geom, n, bt.d_dofs, bt.ndof, bt.d_betas,
                                                        bt.nbeta, d_omegas, bt.rho, bt.g, PHI, d_F, d_FK);
    ctx->launches += 1;
    phase_end(ctx, PH_FORCES);
    MH_CUDA_TRY(ctx, cudaGetLastError());
    return MH_OK;
}

// FP64 path with the mixed path's batch structure, for one chunk of nb
// frequencies: the frequency-batched wave pass writes the FP64 S and D (the
// Rankine part SR, DR computed once per call), then cuSOLVER zgetrf/zgetrs
// factor and solve each frequency's FP64 D (or K) with partial pivoting,
// frequencies spread over several streams, the pivot checks of all
// frequencies read back once at the end.
int run_fp64_chunk(const Batch& bt, const double* d_omegas, const double* d_k, int nb, const double* SR,
                   const double* DR, double2* d_F, double2* d_FK)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n, nn = n * n;
    const int nrhs = bt.nrhs;
    const int64_t nv = n * nrhs;
    auto* S64 = (double2*)ws_get(ctx, WS_S, sizeof(double2) * nn * nb);
    auto* D64 = (double2*)ws_get(ctx, WS_D, sizeof(double2) * nn * nb);
    auto* Dlo = (float2*)ws_get(ctx, WS_LO, sizeof(float2) * nn * nb);
    auto* BC = (double2*)ws_get(ctx, WS_RHS, sizeof(double2) * nv * nb);
    auto* X = (double2*)ws_get(ctx, WS_PHI, sizeof(double2) * nv * nb);
    auto* P = (double2*)ws_get(ctx, WS_TMP, sizeof(double2) * nv * nb);
    auto* piv = (int*)ws_get(ctx, WS_PIV, sizeof(int) * (size_t)(n * nb + 2 * nb + 2));
    auto* d_fall = (int*)ws_get(ctx, WS_MISC, 64);
    if (!S64 || !D64 || !Dlo || !BC || !X || !P || !piv || !d_fall) return MH_ERR_OOM;
    int* infos = piv + n * nb;
    int rc;
    const double* tab = delh_table_for(ctx, bt.mask, &rc);
    if (rc) return rc;
    const uint32_t wave = bt.mask & (MH_GF_WU | MH_GF_DELHOMMEAU);
    phase_begin(ctx, PH_WAVE);
    if (wave == MH_GF_WU) {
        dim3 grid(blocks(n, kRows), blocks(n, kCols), (unsigned)nb);
        k_wave_batch<false><<<grid, kRows, 0, ctx->stream>>>(bt.m->geom, n, bt.direct, nullptr, d_k, SR, DR, S64,
                                                            D64, Dlo, nullptr);
        ctx->launches += 1;
    } else if (wave == MH_GF_DELHOMMEAU && tab && nb >= kAllwMinFreqs) {
        MH_CUDA_TRY(ctx, cudaFuncSetAttribute(k_wave_delh_allw<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)kWaveAllwSmem));
        MH_CUDA_TRY(ctx, cudaMemcpyToSymbolAsync(c_polar_mono, tab + kTabMonoOff, sizeof(c_polar_mono), 0,
                                                 cudaMemcpyDeviceToDevice, ctx->stream));
        for (int z = 0; z < nb; z += kAllwMaxFreqs) {
            const int m = std::min(kAllwMaxFreqs, nb - z);
            const int64_t off = (int64_t)z * nn;
            const dim3 g2(blocks(n, kWT), blocks(n, kCols));
            MH_CUDA_TRY(ctx, cudaMemsetAsync(d_fall, 0, sizeof(int), ctx->stream));
            double2* tp = bt.tape ? bt.tape + 2 * off : nullptr;
            k_wave_delh_allw<double, double><<<g2, kWT, kWaveAllwSmem, ctx->stream>>>(
                bt.m->geom, n, bt.direct, tab, d_k + z, m, SR, DR, S64 + off, D64 + off, Dlo + off, tp, d_fall);
            k_wave_delh_allw_rest<<<g2, kWT, 0, ctx->stream>>>(d_fall, bt.m->geom, n, bt.direct, tab, d_k + z, m,
                                                              SR, DR, S64 + off, D64 + off, Dlo + off, tp);
            ctx->launches += 2;
        }
    } else if (wave == MH_GF_DELHOMMEAU) {
        dim3 grid(blocks(n, kRows), blocks(n, kCols), (unsigned)nb);
        k_wave_batch<true><<<grid, kRows, 0, ctx->stream>>>(bt.m->geom, n, bt.direct, tab, d_k, SR, DR, S64, D64,
                                                           Dlo, bt.tape);
        ctx->launches += 1;
    } else if (wave == 0) {
        k_no_wave_batch<<<dim3(blocks(nn, 256), nb), 256, 0, ctx->stream>>>(nn, SR, DR, S64, D64, Dlo);
        ctx->launches += 1;
    } else {
        return set_err(ctx, MH_ERR_ARG, "the batched FP64 path takes one wave term (GFWu or Delhommeau)");
    }
    phase_end(ctx, PH_WAVE);
    MH_CUDA_TRY(ctx, cudaGetLastError());
    phase_begin(ctx, PH_RHS);
    MH_CUDA_TRY(ctx, launch_bc_batch(bt, d_omegas, nb, BC));
    if (bt.direct) MH_CUDA_TRY(ctx, launch_gemv(ctx, false, S64, n, nb, BC, nullptr, X, nrhs, 1.0, 0.0));
    else MH_CUDA_TRY(ctx, cudaMemcpyAsync(X, BC, sizeof(double2) * nv * nb, cudaMemcpyDeviceToDevice, ctx->stream));
    phase_end(ctx, PH_RHS);
    phase_begin(ctx, PH_FP64_LU);
    // one frequency per stream, kLuGroups streams (the LU groups' main
    // streams), each with its own cuSOLVER handle and workspace, so the
    // latency-bound panel factorisations of different frequencies overlap
    const int ns = std::min(kLuGroups, nb);
    for (int g = 0; g + 1 < ns; ++g)
        if (!ctx->cusolver_grp[g]) {
            if (cusolverDnCreate(&ctx->cusolver_grp[g]) != CUSOLVER_STATUS_SUCCESS) {
                ctx->cusolver_grp[g] = nullptr;
                return set_err(ctx, MH_ERR_CUDA, "cuSOLVER handle creation failed");
            }
            cusolverDnSetStream(ctx->cusolver_grp[g], ctx->grp_main[g]);
        }
    int lwork = 0;
    cusolverStatus_t st = cusolverDnZgetrf_bufferSize(ctx->cusolver, (int)n, (int)n, (cuDoubleComplex*)D64,
                                                      (int)n, &lwork);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrf_bufferSize failed (%d)", (int)st);
    auto* work = (cuDoubleComplex*)ws_get(ctx, WS_LWORK, sizeof(cuDoubleComplex) * (size_t)lwork * ns);
    if (!work) return MH_ERR_OOM;
    if (ns > 1) {
        MH_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
        for (int g = 0; g + 1 < ns; ++g) MH_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->grp_main[g], ctx->ev_fork, 0));
    }
    for (int z = 0; z < nb; ++z) {
        const int q = z % ns;
        cusolverDnHandle_t h = q ? ctx->cusolver_grp[q - 1] : ctx->cusolver;
        auto* Dz = (cuDoubleComplex*)(D64 + (int64_t)z * nn);
        st = cusolverDnZgetrf(h, (int)n, (int)n, Dz, (int)n, work + (size_t)lwork * q, piv + z * n, infos + z);
        if (st != CUSOLVER_STATUS_SUCCESS)
            return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrf failed (%d)", (int)st);
        st = cusolverDnZgetrs(h, CUBLAS_OP_N, (int)n, nrhs, Dz, (int)n, piv + z * n,
                              (cuDoubleComplex*)(X + (int64_t)z * nv), (int)n, infos + nb + z);
        if (st != CUSOLVER_STATUS_SUCCESS)
            return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrs failed (%d)", (int)st);
    }
    for (int g = 0; g + 1 < ns; ++g) {
        MH_CUDA_TRY(ctx, cudaEventRecord(ctx->grp_ev_join[g], ctx->grp_main[g]));
        MH_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->grp_ev_join[g], 0));
    }
    phase_end(ctx, PH_FP64_LU);
    double2* PHI = X;
    if (!bt.direct) {
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, S64, n, nb, X, nullptr, P, nrhs, 1.0, 0.0));
        PHI = P;
    }
    phase_begin(ctx, PH_FORCES);
    MH_CUDA_TRY(ctx, launch_forces_batch(bt, d_omegas, nb, PHI, d_F, d_FK));
    phase_end(ctx, PH_FORCES);
    std::vector<int> h(nb);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), infos, sizeof(int) * (size_t)nb, cudaMemcpyDeviceToHost, ctx->stream));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    for (int z = 0; z < nb; ++z)
        if (h[z] > 0) return set_err(ctx, MH_ERR_SINGULAR, "frequency %d: zero pivot at column %d", z, h[z]);
    return MH_OK;
}

// op(D_z)^-1 X_z for nb frequencies with the pivoted FP64 factors that
// run_fp64_chunk left in place (D64 in WS_D, pivots in WS_PIV), one frequency
// per stream as in the forward solve.
int fp64_batched_getrs(mh_ctx* ctx, bool conj_trans, int64_t n, int nb, int nrhs, double2* X)
{
    const int64_t nn = n * n, nv = n * nrhs;
    auto* D64 = (double2*)ctx->ws[WS_D];
    auto* piv = (int*)ctx->ws[WS_PIV];
    if (!D64 || !piv) return set_err(ctx, MH_ERR_ARG, "no batched FP64 factors to solve with");
    int* infos = piv + n * nb;
    const int ns = std::min(kLuGroups, nb);
    if (ns > 1) {
        MH_CUDA_TRY(ctx, cudaEventRecord(ctx->ev_fork, ctx->stream));
        for (int g = 0; g + 1 < ns; ++g) MH_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->grp_main[g], ctx->ev_fork, 0));
    }
    for (int z = 0; z < nb; ++z) {
        const int q = z % ns;
        cusolverDnHandle_t h = q ? ctx->cusolver_grp[q - 1] : ctx->cusolver;
        const cusolverStatus_t st = cusolverDnZgetrs(h, conj_trans ? CUBLAS_OP_C : CUBLAS_OP_N, (int)n, nrhs,
                                                     (const cuDoubleComplex*)(D64 + (int64_t)z * nn), (int)n,
                                                     piv + z * n, (cuDoubleComplex*)(X + (int64_t)z * nv), (int)n,
                                                     infos + nb + z);
        if (st != CUSOLVER_STATUS_SUCCESS) return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrs failed (%d)", (int)st);
    }
    for (int g = 0; g + 1 < ns; ++g) {
        MH_CUDA_TRY(ctx, cudaEventRecord(ctx->grp_ev_join[g], ctx->grp_main[g]));
        MH_CUDA_TRY(ctx, cudaStreamWaitEvent(ctx->stream, ctx->grp_ev_join[g], 0));
    }
    return MH_OK;
}

size_t refine_ctl_bytes(int nb) { return (sizeof(double) + 3 * sizeof(int)) * (size_t)nb + 16; }

RefineCtl refine_ctl(void* block, int nb)
{
    RefineCtl c;
    c.res = (double*)block;
    c.bad = (int*)(c.res + nb);
    c.done = c.bad + nb;
    c.sweeps = c.done + nb;
    return c;
}

int RefineState::most_sweeps() const
{
    int m = 0;
    for (size_t z = 0; z < sweeps.size(); ++z)
        if (!bad[z]) m = std::max(m, sweeps[z]);
    return m;
}

int refine_sweeps(mh_ctx* ctx, bool conj_trans, int64_t n, int nb, int nrhs, const double2* D64,
                  const float2* Dlo, const float2* Dinv, const double2* RHS, double2* X, double2* R, float2* R32,
                  const RefineCtl& c, double tol, int max_iter, RefineState& h)
{
    const int64_t nn = n * n, nv = n * nrhs, cnt = nv * nb;
    MH_CUDA_TRY(ctx, cudaMemsetAsync(X, 0, sizeof(double2) * cnt, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(R, RHS, sizeof(double2) * cnt, cudaMemcpyDeviceToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(c.done, 0, sizeof(int) * 2 * (size_t)nb, ctx->stream));  // done, sweeps
    const size_t bytes = (sizeof(double) + 3 * sizeof(int)) * (size_t)nb;
    std::vector<unsigned char> host(bytes);
    h.res.assign(nb, INFINITY);
    h.bad.assign(nb, 0);
    h.done.assign(nb, 0);
    h.sweeps.assign(nb, 0);
    const int dir = conj_trans ? 1 : 0;
    const int ahead = std::max(1, std::min(ctx->refine_ahead[dir], max_iter));
    int it = 0;
    while (it < max_iter) {
        // the sweeps the last call needed, then one at a time; a sweep costs
        // next to nothing on matrices that converged or are marked
        for (int s = 0, k = it == 0 ? ahead : 1; s < k && it < max_iter; ++s) {
            ++it;
            k_refine_to_f32<<<blocks(cnt, 256), 256, 0, ctx->stream>>>(R, R32, nv, cnt, c.done, c.bad);
            MH_CUDA_TRY(ctx, launch_lu_solve_persist(ctx, ctx->lu_backend, conj_trans, Dlo, n, nn, nb, Dinv, R32,
                                                     nv, nrhs, c.bad, c.done));
            k_refine_add<<<blocks(cnt, 256), 256, 0, ctx->stream>>>(X, R32, nv, cnt, c.done, c.bad);
            // R = RHS - op(D) X, then the residual ratio and the marks
            MH_CUDA_TRY(ctx, launch_gemv(ctx, conj_trans, D64, n, nb, X, RHS, R, nrhs, -1.0, 1.0, c.done, c.bad));
            k_rel_residual<<<nb, 256, 0, ctx->stream>>>(R, RHS, n, nrhs, c.res, tol, c.done, c.bad, c.sweeps, it);
            ctx->launches += 3;
            MH_CUDA_TRY(ctx, cudaGetLastError());
        }
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(host.data(), c.res, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        const auto* hr = (const double*)host.data();
        const auto* hi = (const int*)(hr + nb);
        bool active = false;
        for (int z = 0; z < nb; ++z) {
            h.bad[z] = hi[z];
            h.done[z] = hi[nb + z];
            h.sweeps[z] = hi[2 * nb + z];
            h.res[z] = h.sweeps[z] ? hr[z] : INFINITY;
            active = active || (!h.bad[z] && !h.done[z]);
        }
        if (!active) break;
    }
    int most = 0;
    for (int z = 0; z < nb; ++z)
        if (h.ok(z)) most = std::max(most, h.sweeps[z]);
    if (most > 0) ctx->refine_ahead[dir] = std::min(most, 8);
    return MH_OK;
}

int mixed_refine_solve(mh_ctx* ctx, int64_t n, int nb, int nrhs, const double2* D64, const float2* Dlo,
                       const float2* Dinv, const double2* RHS, double2* X, double2* R, float2* R32, void* ctl_block,
                       bool conj_trans, double tol, int max_iter, FallbackStore& fb, mh_batch_info* info)
{
    const int64_t nn = n * n, nv = n * nrhs;
    int rc;
    const RefineCtl c = refine_ctl(ctl_block, nb);
    // problems whose forward solve fell back to FP64 are not refined
    std::vector<int> used(nb, 0);
    for (int z = 0; z < nb; ++z) used[z] = fb.used[z] ? 1 : 0;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(c.bad, used.data(), sizeof(int) * (size_t)nb, cudaMemcpyHostToDevice,
                                     ctx->stream));
    RefineState h;
    if ((rc = refine_sweeps(ctx, conj_trans, n, nb, nrhs, D64, Dlo, Dinv, RHS, X, R, R32, c, tol, max_iter, h)))
        return rc;
    info->refine_iterations = std::max(info->refine_iterations, h.most_sweeps());
    for (int z = 0; z < nb; ++z) {
        if (!fb.used[z] && h.ok(z)) {
            info->max_rel_residual = std::max(info->max_rel_residual, h.res[z]);
            continue;
        }
        if (!fb.used[z]) {
            info->n_fallback += 1;
            if ((rc = fallback_factor(ctx, &fb, n, nb, z, D64 + (int64_t)z * nn))) return rc;
        }
        double2* Xz = X + (int64_t)z * nv;
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(Xz, RHS + (int64_t)z * nv, sizeof(double2) * nv, cudaMemcpyDeviceToDevice,
                                         ctx->stream));
        if ((rc = fp64_getrs(ctx, conj_trans, n, fb.lu + (int64_t)z * nn, fb.piv + (int64_t)z * n, Xz, nrhs)))
            return rc;
    }
    return MH_OK;
}

int fallback_factor(mh_ctx* ctx, FallbackStore* fb, int64_t n, int nb, int z, const double2* D)
{
    const int64_t nn = n * n;
    if (!fb->lu) {
        fb->lu = (double2*)ws_get(ctx, WS_FB, sizeof(double2) * nn * nb + sizeof(int) * n * nb);
        if (!fb->lu) return MH_ERR_OOM;
        fb->piv = (int*)(fb->lu + nn * nb);
    }
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(fb->lu + (int64_t)z * nn, D, sizeof(double2) * nn,
                                     cudaMemcpyDeviceToDevice, ctx->stream));
    fb->used[z] = 1;
    return fp64_lu_factor(ctx, n, fb->lu + (int64_t)z * nn, fb->piv + (int64_t)z * n);
}

int rankine_real(const Batch& bt, double* SR, double* DR)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    phase_begin(ctx, PH_RANKINE);
    k_rankine_real<<<dim3(blocks(n, kRows), blocks(n, kCols)), kRows, 0, ctx->stream>>>(
        bt.m->geom, n, bt.mask & (MH_GF_RANKINE | MH_GF_RANKINE_REFLECTED |
                                  MH_GF_RANKINE_REFLECTED_NEGATIVE), bt.direct, SR, DR);
    ctx->launches += 1;
    phase_end(ctx, PH_RANKINE);
    MH_CUDA_TRY(ctx, cudaGetLastError());
    return MH_OK;
}

cudaError_t launch_bc_batch(const Batch& bt, const double* d_omegas, int nb, double2* BC)
{
    k_bc_batch<<<dim3(blocks(bt.n, 256), (unsigned)nb), 256, 0, bt.ctx->stream>>>(
        bt.m->geom, bt.n, bt.d_dofs, bt.ndof, bt.d_betas, bt.nbeta, d_omegas, bt.g, BC);
    bt.ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_forces_batch(const Batch& bt, const double* d_omegas, int nb, const double2* PHI,
                                double2* d_F, double2* d_FK)
{
    k_forces_batch<<<nb * bt.nrhs, 256, 0, bt.ctx->stream>>>(bt.m->geom, bt.n, bt.d_dofs, bt.ndof,
                                                             bt.d_betas, bt.nbeta, d_omegas, bt.rho,
                                                             bt.g, PHI, d_F, d_FK);
    bt.ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_to_f32(mh_ctx* ctx, const double2* a, float2* b, int64_t count)
{
    k_to_f32<<<blocks(count, 256), 256, 0, ctx->stream>>>(a, b, count);
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_add_f32(mh_ctx* ctx, double2* x, const float2* d, int64_t count)
{
    k_add_f32<<<blocks(count, 256), 256, 0, ctx->stream>>>(x, d, count);
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_gemv(mh_ctx* ctx, bool conj_trans, const double2* A, int64_t n, int nb, const double2* X,
                        const double2* B, double2* R, int nrhs, double alpha, double beta, const int* done,
                        const int* bad, cudaStream_t stream)
{
    cudaStream_t strm = stream ? stream : ctx->stream;
    if (nrhs < 1 || nrhs > kMaxRhs) return cudaErrorInvalidValue;
    if (beta == 0.0) B = nullptr;
    const dim3 gn(blocks(n, 256), (unsigned)nb);
    if (conj_trans) {  // 8 warps per CTA, JW columns per warp
        const dim3 g4(blocks(n, 32), (unsigned)nb);
        if (nrhs == 1) k_resid_c<1, 4><<<g4, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
        else if (nrhs == 2) k_resid_c<2, 4><<<g4, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
        else if (nrhs == 3) k_resid_c<3, 4><<<g4, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
        else if (nrhs == 4) k_resid_c<4, 4><<<g4, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
        else if (nrhs <= 8)
            k_resid_c<8, 2><<<dim3(blocks(n, 16), (unsigned)nb), 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha,
                                                                                      beta, done, bad);
        else
            k_resid_c<kMaxRhs, 1><<<dim3(blocks(n, 8), (unsigned)nb), 256, 0, strm>>>(A, X, B, R, n, nrhs,
                                                                                           alpha, beta, done, bad);
    } else {
        if (nrhs <= 4) k_resid_n<4><<<gn, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
        else if (nrhs <= 8) k_resid_n<8><<<gn, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
        else k_resid_n<kMaxRhs><<<gn, 256, 0, strm>>>(A, X, B, R, n, nrhs, alpha, beta, done, bad);
    }
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_residual(mh_ctx* ctx, bool conj_trans, const double2* A, int64_t n, int nb, const double2* X,
                            const double2* B, double2* R, int nrhs)
{
    return launch_gemv(ctx, conj_trans, A, n, nb, X, B, R, nrhs, -1.0, 1.0);
}

cudaError_t launch_rel_residual(mh_ctx* ctx, const double2* r, const double2* b, int64_t n, int nrhs,
                                int nb, double* out)
{
    k_rel_residual<<<nb, 256, 0, ctx->stream>>>(r, b, n, nrhs, out, 0.0, nullptr, nullptr, nullptr, 0);
    ctx->launches += 1;
    return cudaGetLastError();
}

void unpack_outputs(const double2* h, int64_t nomega, const double* omegas, int64_t ndof, int64_t nbeta,
                    double* added_mass, double* damping, double* diffraction, double* froude_krylov)
{
    const int64_t nrhs = ndof + nbeta;
    // outputs in the reference's layout (src/problems_and_results.jl:137-165):
    // added_mass[i, j, w] (i influenced, j radiating), diffraction[i, w, b]
    for (int64_t z = 0; z < nomega; ++z) {
        const double w = omegas[z];
        for (int64_t jq = 0; jq < ndof; ++jq)
            for (int64_t i = 0; i < ndof; ++i) {
                double2 F = h[((size_t)z * nrhs + jq) * ndof + i];
                size_t o = (size_t)i + (size_t)ndof * ((size_t)jq + (size_t)ndof * (size_t)z);
                if (added_mass) added_mass[o] = F.x / (w * w);
                if (damping) damping[o] = F.y / w;
            }
        for (int64_t b = 0; b < nbeta; ++b)
            for (int64_t i = 0; i < ndof; ++i) {
                double2 F = h[((size_t)z * nrhs + ndof + b) * ndof + i];
                double2 K = h[(size_t)nomega * nrhs * ndof + ((size_t)z * nbeta + b) * ndof + i];
                size_t o = (size_t)i + (size_t)ndof * ((size_t)z + (size_t)nomega * (size_t)b);
                if (diffraction) {
                    diffraction[2 * o] = F.x;
                    diffraction[2 * o + 1] = F.y;
                }
                if (froude_krylov) {
                    froude_krylov[2 * o] = K.x;
                    froude_krylov[2 * o + 1] = K.y;
                }
            }
    }
}

int hydro_batch(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                const double* dofs, int64_t nbeta, const double* betas, double rho, double g,
                uint32_t mask, int direct, int precision, double tol, int max_iter,
                double* added_mass, double* damping, double* diffraction, double* froude_krylov,
                mh_batch_info* info)
{
    const int64_t n = m->n;
    const int nrhs = (int)(ndof + nbeta);
    mh_batch_info local{};
    // inputs to the device
    const size_t dof_bytes = sizeof(double) * 3 * (size_t)n * (size_t)ndof;
    const size_t in_bytes = dof_bytes + sizeof(double) * (size_t)(2 * nomega + nbeta) + 64;
    auto* in = (char*)ws_get(ctx, WS_DOF, in_bytes);
    const size_t out_count = (size_t)nomega * (size_t)(nrhs * ndof + nbeta * ndof);
    auto* d_out = (double2*)ws_get(ctx, WS_OUT, sizeof(double2) * out_count + 16);
    if (!in || !d_out) return MH_ERR_OOM;
    auto* d_dofs = (double*)in;
    auto* d_omegas = (double*)(in + dof_bytes);
    auto* d_k = d_omegas + nomega;
    auto* d_betas = d_k + nomega;
    std::vector<double> hk(nomega);
    for (int64_t z = 0; z < nomega; ++z) hk[z] = omegas[z] * omegas[z] / g;
    if (ndof) MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_dofs, dofs, dof_bytes, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_omegas, omegas, sizeof(double) * nomega, cudaMemcpyHostToDevice,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_k, hk.data(), sizeof(double) * nomega, cudaMemcpyHostToDevice,
                                     ctx->stream));
    if (nbeta)
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_betas, betas, sizeof(double) * nbeta, cudaMemcpyHostToDevice,
                                         ctx->stream));
    double2* d_F = d_out;
    double2* d_FK = d_out + (size_t)nomega * nrhs * ndof;
    Batch bt{ctx, m, n, (int)ndof, (int)nbeta, nrhs, d_dofs, d_betas, rho, g, mask, direct};
    int rc = MH_OK;
    if (precision == MH_PRECISION_FP64) {
        rc = run_fp64(bt, d_omegas, (int)nomega, d_F, d_FK);
    } else {
        const size_t nn = (size_t)n * (size_t)n;
        auto* SR = (double*)ws_get(ctx, WS_SR, sizeof(double) * nn * 2);
        if (!SR) return MH_ERR_OOM;
        double* DR = SR + nn;
        if ((rc = rankine_real(bt, SR, DR))) return rc;
        const size_t per = nn * (2 * sizeof(double2) + sizeof(float2)) +
                           (size_t)n * nrhs * (5 * sizeof(double2) + sizeof(float2));
        const int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(nomega, kBatchBytes / per));
        for (int64_t z0 = 0; z0 < nomega && rc == MH_OK; z0 += chunk) {
            const int nb = (int)std::min<int64_t>(chunk, nomega - z0);
            if (precision == MH_PRECISION_FP64_BATCHED)
                rc = run_fp64_chunk(bt, d_omegas + z0, d_k + z0, nb, SR, DR, d_F + z0 * nrhs * ndof,
                                    d_FK + z0 * nbeta * ndof);
            else
                rc = run_mixed_chunk(bt, d_omegas + z0, d_k + z0, nb, SR, DR, tol, max_iter,
                                     d_F + z0 * nrhs * ndof, d_FK + z0 * nbeta * ndof, &local, nullptr);
        }
    }
    if (rc) return rc;
    phase_collect(ctx);
    std::vector<double2> h(out_count);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), d_out, sizeof(double2) * out_count,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    unpack_outputs(h.data(), nomega, omegas, ndof, nbeta, added_mass, damping, diffraction,
                   froude_krylov);
    if (info) *info = local;
    return MH_OK;
}

}  // namespace mh
