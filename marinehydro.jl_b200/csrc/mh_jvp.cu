// Forward-mode (tangent) derivatives of the batched hydrodynamic
// coefficients along one direction of the inputs.
//
// Replaces the reference's ForwardDiff branch: `assemble_matrices` with Dual
// element types (src/matrix_assembly.jl:7-11) and `solve` with Duals
// (:108-114), as used through `compute_hydrodynamic_coefficients` by
// test/outputs_differentiation.jl:133-151.  Given the tangent of every mesh
// field (vertices, centres, normals, areas), of the frequencies and of the
// dof fields, it returns the outputs and their tangents dA, dB, dF, dFK.
//
// Per frequency, direct: D phi = S b gives
//   dphi = D^-1 (dS b + S db - dD phi);
// indirect: K sigma = b, phi = S sigma gives
//   dsigma = K^-1 (db - dK sigma), dphi = dS sigma + S dsigma.
// dS and dD are formed per frequency (same layout as S and D): the Rankine
// part is frequency independent and is differentiated once per call through
// the templated `rankine_pair` with 1-way dual numbers; the wave part per pair
// and frequency from the r, z derivatives of the dimensionless term (Wu by
// dual numbers, Delhommeau by its identities, frequency batched like the
// forward pass).  The products with b, phi use the batched bandwidth-bound
// GEMV (launch_gemv), the solve reuses the forward factors (FP64 zgetrs, or
// the low-precision factors with FP64 refinement).
#include <cuComplex.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mh_device.cuh"
#include "mh_internal.h"

namespace mh {
namespace {

constexpr int kJR = 128;  // rows (threads) per CTA of the pair kernels
constexpr double kI4P = 1.0 / (4.0 * kPi);
constexpr int kJvpAllwMinFreqs = 4;

using d1 = dualn<1>;

unsigned nblk(int64_t count, int threads) { return (unsigned)((count + threads - 1) / threads); }

#include "mh_grad.cuh"

// Tangent panel (the same fields as a Panel).
__device__ __forceinline__ void stage_t(Panel* tp, const double* __restrict__ tgeom, int64_t n, int64_t j0)
{
    stage(tp, tgeom, n, j0);
}

__device__ __forceinline__ PanelT<d1> dual_panel(const Panel& p, const Panel& t)
{
    PanelT<d1> q;
    for (int a = 0; a < 3; ++a) {
        q.c[a].v = p.c[a];
        q.c[a].d[0] = t.c[a];
        q.n[a].v = p.n[a];
        q.n[a].d[0] = t.n[a];
    }
    for (int k = 0; k < 12; ++k) {
        q.v[k].v = p.v[k];
        q.v[k].d[0] = t.v[k];
    }
    q.area.v = p.area;
    q.area.d[0] = t.area;
    q.radius.v = p.radius;
    q.radius.d[0] = 0.0;  // radii only select branches
    return q;
}

// Tangent of the frequency-independent Rankine terms (rankine.jl,
// rankine_reflected*.jl) along tgeom: dSR = -d(sum integral)/4pi,
// dDR = -d(nD . sum gradient)/4pi, stored as complex with zero imaginary part.
__global__ void __launch_bounds__(kJR)
k_rankine_tangent(const double* __restrict__ geom, const double* __restrict__ tgeom, int64_t n, uint32_t mask,
                  int direct, double2* __restrict__ dSR, double2* __restrict__ dDR)
{
    __shared__ Panel sp[kGradCols], tp[kGradCols];
    const int64_t j0 = (int64_t)blockIdx.y * kGradCols;
    stage(sp, geom, n, j0);
    stage_t(tp, tgeom, n, j0);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kJR + threadIdx.x;
    if (i >= n) return;
    d1 x[3], ni[3];
    for (int c = 0; c < 3; ++c) {
        x[c].v = geom[(G_CX + c) * n + i];
        x[c].d[0] = tgeom[(G_CX + c) * n + i];
        ni[c].v = geom[(G_NX + c) * n + i];
        ni[c].d[0] = tgeom[(G_NX + c) * n + i];
    }
    const int jend = (int)min((int64_t)kGradCols, n - j0);
    const uint32_t rmask = mask & (MH_GF_RANKINE | MH_GF_RANKINE_REFLECTED | MH_GF_RANKINE_REFLECTED_NEGATIVE);
    for (int jj = 0; jj < jend; ++jj) {
        const PanelT<d1> q = dual_panel(sp[jj], tp[jj]);
        const int64_t j = j0 + jj;
        cx<d1> s, g[3];
        pair_integrals(x, q, tconst<d1>(0.0), rmask, !direct, nullptr, s, g);
        const d1* nD = direct ? q.n : ni;
        const d1 dn = nD[0] * g[0].re + nD[1] * g[1].re + nD[2] * g[2].re;
        const int64_t o = j * n + i;
        dSR[o] = make_double2(-kI4P * s.re.d[0], 0.0);
        dDR[o] = make_double2(-kI4P * dn.d[0], 0.0);
    }
}

// Pair tangents of the wave term (abstract_greens_function.jl:88-155 with
// the one-point rule): s = k A G, g = (sg k^2 A u_x G_r, sg k^2 A u_y G_r,
// k^2 A G_z); returns ds and d(nD . g) along (tdx, tdy, tzs, tA, dk, tnD).
struct WaveTan {
    double tdx, tdy, tzs, tA, dk;
    double tn[3];
};

__device__ __forceinline__ void wave_tangent(const GDer& o, const WaveGeom& w, double k, double A, bool wrt_first,
                                             const double nD[3], const WaveTan& t, cplx& ds, cplx& dDn)
{
    const bool rad = fabs(k * w.dis) > 1e-6;
    const double sg = wrt_first ? 1.0 : -1.0;
    const double k2 = k * k;
    const double ddis = w.u0 * t.tdx + w.u1 * t.tdy;
    const double dr = t.dk * w.dis + k * ddis, dz = t.dk * w.zs + k * t.tzs;
    cplx dG[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) dG[m] = o.Gr[m] * dr + o.Gz[m] * dz;
    const double dkA = t.dk * A + k * t.tA;            // d(k A)
    const double dk2A = 2.0 * k * t.dk * A + k2 * t.tA;  // d(k^2 A)
    ds = dkA * o.G[0] + (k * A) * dG[0];
    cplx g[3], dg[3];
    if (rad) {
        const double du0 = ((1.0 - w.u0 * w.u0) * t.tdx - w.u0 * w.u1 * t.tdy) * w.invd;
        const double du1 = ((1.0 - w.u1 * w.u1) * t.tdy - w.u0 * w.u1 * t.tdx) * w.invd;
        g[0] = (sg * k2 * A * w.u0) * o.G[1];
        g[1] = (sg * k2 * A * w.u1) * o.G[1];
        dg[0] = (sg * (dk2A * w.u0 + k2 * A * du0)) * o.G[1] + (sg * k2 * A * w.u0) * dG[1];
        dg[1] = (sg * (dk2A * w.u1 + k2 * A * du1)) * o.G[1] + (sg * k2 * A * w.u1) * dG[1];
    } else {
        g[0] = g[1] = dg[0] = dg[1] = mk(0.0, 0.0);
    }
    g[2] = (k2 * A) * o.G[2];
    dg[2] = dk2A * o.G[2] + (k2 * A) * dG[2];
    dDn = t.tn[0] * g[0] + t.tn[1] * g[1] + t.tn[2] * g[2] + nD[0] * dg[0] + nD[1] * dg[1] + nD[2] * dg[2];
}

__device__ __forceinline__ WaveTan pair_tan(const double tx[3], const double tni[3], const Panel& tp, bool direct,
                                            double dk)
{
    WaveTan t;
    t.tdx = tx[0] - tp.c[0];
    t.tdy = tx[1] - tp.c[1];
    t.tzs = tx[2] + tp.c[2];
    t.tA = tp.area;
    t.dk = dk;
    for (int a = 0; a < 3; ++a) t.tn[a] = direct ? tp.n[a] : tni[a];
    return t;
}

// Per-frequency tangent matrices (grid z = frequency), any wave term:
// dS = dSR - ds/4pi, dD = dDR - d(nD . g)/4pi.
__global__ void __launch_bounds__(kJR)
k_wave_tangent(int kind, const double* __restrict__ geom, const double* __restrict__ tgeom, int64_t n, int direct,
               const double* __restrict__ tab, const double* __restrict__ kvec, const double* __restrict__ dkvec,
               const double2* __restrict__ dSR, const double2* __restrict__ dDR, double2* __restrict__ dS,
               double2* __restrict__ dD)
{
    __shared__ Panel sp[kGradCols], tp[kGradCols];
    const int64_t j0 = (int64_t)blockIdx.y * kGradCols;
    stage(sp, geom, n, j0);
    stage_t(tp, tgeom, n, j0);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kJR + threadIdx.x;
    if (i >= n) return;
    const int z = blockIdx.z;
    const double k = kvec[z], dk = dkvec[z];
    const int64_t mat = (int64_t)z * n * n;
    double x[3], ni[3], tx[3], tni[3];
    for (int c = 0; c < 3; ++c) {
        x[c] = geom[(G_CX + c) * n + i];
        ni[c] = geom[(G_NX + c) * n + i];
        tx[c] = tgeom[(G_CX + c) * n + i];
        tni[c] = tgeom[(G_NX + c) * n + i];
    }
    const int jend = (int)min((int64_t)kGradCols, n - j0);
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t o = (j0 + jj) * n + i;
        double2 s = dSR[o], d = dDR[o];
        if (kind) {
            const WaveGeom w = wave_geom(x, p);
            GDer g;
            wave_dimless_grad(kind, tab, k * w.dis, k * w.zs, g);
            cplx ds, dDn;
            wave_tangent(g, w, k, p.area, !direct, direct ? p.n : ni, pair_tan(tx, tni, tp[jj], direct, dk), ds, dDn);
            s.x -= kI4P * ds.re;
            s.y -= kI4P * ds.im;
            d.x -= kI4P * dDn.re;
            d.y -= kI4P * dDn.im;
        }
        dS[mat + o] = s;
        dD[mat + o] = d;
    }
}

// Frequency-batched tangent of the tabulated Delhommeau term (the tangent of
// the forward's frequency-batched pass): the alpha contraction of the four
// polar tables once per pair, 1-D Clenshaw in R per frequency, derivatives
// from the identities.
constexpr int kTW = 64;  // rows (threads) per CTA
constexpr int kTS = 4;   // series: B, C, E0, E1

// contracted series of every row, then k, 1/k, log k and dk/d(direction) per frequency
size_t tan_allw_smem(int nb) { return sizeof(double) * ((size_t)kTS * kTabNU * kTW + 4 * (size_t)nb); }

// The four polar functions' Chebyshev coefficients in constant memory (every
// lane of the alpha contraction reads the same one); copied from the
// context's table before each launch (every context builds the same table).
__constant__ double c_polar_cheb[kTS * kTabPolarFn];

__global__ void __launch_bounds__(kTW, 5)
k_wave_tangent_allw(const double* __restrict__ geom, const double* __restrict__ tgeom, int64_t n, int direct,
                    const double* __restrict__ kvec,
                    const double* __restrict__ dkvec, int nb, const double2* __restrict__ dSR,
                    const double2* __restrict__ dDR, double2* __restrict__ dS, double2* __restrict__ dD,
                    int* __restrict__ fall)
{
    extern __shared__ double dsm[];
    double* w = dsm;                        // [kTS * kTabNU][kTW]
    double* ksh = w + kTS * kTabNU * kTW;   // [nb] k
    double* iksh = ksh + nb;                // [nb] 1/k
    double* logk = iksh + nb;               // [nb] log k
    double* dksh = logk + nb;               // [nb] dk
    __shared__ Panel sp[kGradCols], tp[kGradCols];
    const int64_t j0 = (int64_t)blockIdx.y * kGradCols;
    stage(sp, geom, n, j0);
    stage_t(tp, tgeom, n, j0);
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        ksh[t] = kvec[t];
        iksh[t] = 1.0 / kvec[t];
        logk[t] = log(kvec[t]);
        dksh[t] = dkvec[t];
    }
    __syncthreads();
    const int tid = threadIdx.x;
    const int64_t i = (int64_t)blockIdx.x * kTW + tid;
    if (i >= n) return;  // no block-level synchronisation below
    double x[3], ni[3], tx[3], tni[3];
    for (int c = 0; c < 3; ++c) {
        x[c] = geom[(G_CX + c) * n + i];
        ni[c] = geom[(G_NX + c) * n + i];
        tx[c] = tgeom[(G_CX + c) * n + i];
        tni[c] = tgeom[(G_NX + c) * n + i];
    }
    const int jend = (int)min((int64_t)kGradCols, n - j0);
    const int64_t nn = n * n;
    double* wt = w + tid;
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t o = (j0 + jj) * n + i;
        const double* nD = direct ? p.n : ni;
        const WaveGeom wg = wave_geom(x, p);
        const double az1 = -wg.zs;
        const double rho = hypot(wg.dis, wg.zs);
        const bool polar_ok = az1 >= 0.0 && rho > 0.0;
        const double lp = log(0.5 * (rho + az1));
        const double gp = wg.dis / (rho * (rho + az1));
        const double2 sR = dSR[o], dR_ = dDR[o];
        if (polar_ok) {  // the four functions' recurrences interleaved
            const double v = 4.0 * atan2(wg.dis, az1) / kPi - 1.0, v2 = 2.0 * v;
#pragma unroll 1
            for (int row = 0; row < kTabNU; ++row) {
                const double* cr = c_polar_cheb + row * kTabNV;
                double b1[kTS] = {0.0, 0.0, 0.0, 0.0}, b2[kTS] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int col = kTabNV - 1; col >= 1; --col) {
#pragma unroll
                    for (int q = 0; q < kTS; ++q) {
                        const double t = fma(v2, b1[q], cr[q * kTabPolarFn + col] - b2[q]);
                        b2[q] = b1[q];
                        b1[q] = t;
                    }
                }
#pragma unroll
                for (int q = 0; q < kTS; ++q) wt[(q * kTabNU + row) * kTW] = fma(v, b1[q], cr[q * kTabPolarFn] - b2[q]);
            }
        }
        bool nfall = false;
        for (int z = 0; z < nb; ++z) {
            const double k = ksh[z];
            const double R = k * rho;
            if (!(polar_ok && R < kTabRPolar)) {  // left to k_wave_tangent_allw_rest
                nfall = true;
                continue;
            }
            const WaveTan t = pair_tan(tx, tni, tp[jj], direct, dksh[z]);
            GDer o3;
            {
                const double u = 2.0 * R / kTabRPolar - 1.0, u2 = 2.0 * u;
                double b1[kTS], b2[kTS];
#pragma unroll
                for (int q = 0; q < kTS; ++q) b1[q] = b2[q] = 0.0;
#pragma unroll 4
                for (int row = kTabNU - 1; row >= 1; --row)
#pragma unroll
                    for (int q = 0; q < kTS; ++q) {
                        const double nt = fma(u2, b1[q], wt[(q * kTabNU + row) * kTW] - b2[q]);
                        b2[q] = b1[q];
                        b1[q] = nt;
                    }
                double sv[kTS];
#pragma unroll
                for (int q = 0; q < kTS; ++q) sv[q] = fma(u, b1[q], wt[q * kTabNU * kTW] - b2[q]);
                const double L = logk[z] + lp;
                cplx G[3];
                const double G_re = -2.0 * sv[2] * L + sv[0], G_im = 2.0 * kPi * sv[2];
                G[0] = mk(G_re, G_im);
                G[1] = mk(2.0 * sv[3] * L - 2.0 * sv[2] * gp * iksh[z] + sv[1], -2.0 * kPi * sv[3]);
                G[2] = mk(G_re + 2.0 / R, G_im);
                gder_identities(G, k * wg.dis, k * wg.zs, R, o3);
            }
            cplx ds, dDn;
            wave_tangent(o3, wg, k, p.area, !direct, nD, t, ds, dDn);
            dS[(int64_t)z * nn + o] = make_double2(sR.x - kI4P * ds.re, sR.y - kI4P * ds.im);
            dD[(int64_t)z * nn + o] = make_double2(dR_.x - kI4P * dDn.re, dR_.y - kI4P * dDn.im);
        }
        if (nfall) *fall = 1;
    }
}

// The (pair, frequency) tangents k_wave_tangent_allw left to the full table
// (pairs above the free surface or at R = k d >= 2); exits at once when it
// flagged none.  The test takes a margin of 1e-12 in R, so a pair on the
// patch edge is written by one kernel at least (by this one last when both).
__global__ void __launch_bounds__(kTW)
k_wave_tangent_allw_rest(const int* __restrict__ fall, const double* __restrict__ geom,
                         const double* __restrict__ tgeom, int64_t n, int direct, const double* __restrict__ tab,
                         const double* __restrict__ kvec, const double* __restrict__ dkvec, int nb,
                         const double2* __restrict__ dSR, const double2* __restrict__ dDR, double2* __restrict__ dS,
                         double2* __restrict__ dD)
{
    if (*fall == 0) return;
    __shared__ Panel sp[kGradCols], tp[kGradCols];
    const int64_t j0 = (int64_t)blockIdx.y * kGradCols;
    stage(sp, geom, n, j0);
    stage_t(tp, tgeom, n, j0);
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kTW + threadIdx.x;
    if (i >= n) return;
    double x[3], ni[3], tx[3], tni[3];
    for (int c = 0; c < 3; ++c) {
        x[c] = geom[(G_CX + c) * n + i];
        ni[c] = geom[(G_NX + c) * n + i];
        tx[c] = tgeom[(G_CX + c) * n + i];
        tni[c] = tgeom[(G_NX + c) * n + i];
    }
    const int jend = (int)min((int64_t)kGradCols, n - j0);
    const int64_t nn = n * n;
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t o = (j0 + jj) * n + i;
        const double* nD = direct ? p.n : ni;
        const WaveGeom wg = wave_geom(x, p);
        const double rho = hypot(wg.dis, wg.zs);
        const bool polar_ok = -wg.zs >= 0.0 && rho > 0.0;
        const double2 sR = dSR[o], dR_ = dDR[o];
#pragma unroll 1
        for (int z = 0; z < nb; ++z) {
            const double k = kvec[z];
            if (polar_ok && k * rho < kTabRPolar * (1.0 - 1e-12)) continue;
            const WaveTan t = pair_tan(tx, tni, tp[jj], direct, dkvec[z]);
            GDer o3;
            delh_point_grad(tab, k * wg.dis, k * wg.zs, &o3);
            cplx ds, dDn;
            wave_tangent(o3, wg, k, p.area, !direct, nD, t, ds, dDn);
            dS[(int64_t)z * nn + o] = make_double2(sR.x - kI4P * ds.re, sR.y - kI4P * ds.im);
            dD[(int64_t)z * nn + o] = make_double2(dR_.x - kI4P * dDn.re, dR_.y - kI4P * dDn.im);
        }
    }
}

// Tangents of the boundary conditions (src/waves.jl:89-101, 121-142):
// radiation b = -i w (n . dof); diffraction b = -(g k / w) e^{kz} e^{i k wbar}
// (n_x cos + n_y sin - i n_z).
__global__ void k_bc_tangent(const double* __restrict__ geom, const double* __restrict__ tgeom, int64_t n,
                             const double* __restrict__ dofs, const double* __restrict__ tdofs, int ndof,
                             const double* __restrict__ betas, int nbeta, const double* __restrict__ omegas,
                             const double* __restrict__ domegas, double gacc, double2* __restrict__ dBC)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nrhs = ndof + nbeta;
    const int z = blockIdx.y;
    const double w = omegas[z], dw = domegas[z];
    const double k = w * w / gacc, dk = 2.0 * w * dw / gacc;
    double2* out = dBC + (int64_t)z * n * nrhs;
    double nv[3], tn[3];
    for (int c = 0; c < 3; ++c) {
        nv[c] = geom[(G_NX + c) * n + i];
        tn[c] = tgeom[(G_NX + c) * n + i];
    }
    for (int q = 0; q < ndof; ++q) {
        const double* d = dofs + (int64_t)q * 3 * n;
        const double* td = tdofs + (int64_t)q * 3 * n;
        double nd = 0.0, dnd = 0.0;
        for (int c = 0; c < 3; ++c) {
            nd += nv[c] * d[c * n + i];
            dnd += tn[c] * d[c * n + i] + nv[c] * td[c * n + i];
        }
        out[(int64_t)q * n + i] = make_double2(0.0, -(dw * nd + w * dnd));
    }
    const double x = geom[G_CX * n + i], y = geom[G_CY * n + i], zc = geom[G_CZ * n + i];
    const double tx = tgeom[G_CX * n + i], ty = tgeom[G_CY * n + i], tz = tgeom[G_CZ * n + i];
    const double f = gacc * k / w, df = gacc * dk / w - gacc * k * dw / (w * w);
    const double ez = exp(k * zc);
    for (int b = 0; b < nbeta; ++b) {
        double sb, cb, sw, cw;
        sincos(betas[b], &sb, &cb);
        const double wv = x * cb + y * sb, dwv = tx * cb + ty * sb;
        sincos(k * wv, &sw, &cw);
        const cplx E = mk(ez * cw, ez * sw);
        const cplx dE = E * mk(dk * zc + k * tz, dk * wv + k * dwv);
        const cplx h = mk(nv[0] * cb + nv[1] * sb, -nv[2]);
        const cplx dh = mk(tn[0] * cb + tn[1] * sb, -tn[2]);
        const cplx db = -((df * E) * h + (f * dE) * h + (f * E) * dh);
        out[(int64_t)(ndof + b) * n + i] = make_double2(db.re, db.im);
    }
}

// Tangents of the forces (src/waves.jl:72-85, 157-163) for right-hand side
// q of frequency z (blockIdx.x = z * nrhs + q):
// F_d = i rho w sum phi m_d, m_d = -(n . dof_d) area; FK_d = sum p m_d.
__global__ void __launch_bounds__(256)
k_forces_tangent(const double* __restrict__ geom, const double* __restrict__ tgeom, int64_t n,
                 const double* __restrict__ dofs, const double* __restrict__ tdofs, int ndof,
                 const double* __restrict__ betas, int nbeta, const double* __restrict__ omegas,
                 const double* __restrict__ domegas, double rho, double gacc, const double2* __restrict__ phi,
                 const double2* __restrict__ dphi, double2* __restrict__ dF, double2* __restrict__ dFK)
{
    const int nrhs = ndof + nbeta;
    const int z = blockIdx.x / nrhs, q = blockIdx.x % nrhs;
    const double w = omegas[z], dw = domegas[z];
    const double k = w * w / gacc, dk = 2.0 * w * dw / gacc;
    const int64_t off = ((int64_t)z * nrhs + q) * n;
    const bool diff = q >= ndof;
    double cb = 1.0, sb = 0.0;
    if (diff) sincos(betas[q - ndof], &sb, &cb);
    double acc[4 * kMaxRhs];
    for (int t = 0; t < 4 * ndof; ++t) acc[t] = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        double nv[3], tn[3];
        for (int c = 0; c < 3; ++c) {
            nv[c] = geom[(G_NX + c) * n + j];
            tn[c] = tgeom[(G_NX + c) * n + j];
        }
        const double a = geom[G_AREA * n + j], ta = tgeom[G_AREA * n + j];
        const double2 ph = phi[off + j], dph = dphi[off + j];
        // i rho w phi and its tangent
        const cplx P = mk(-rho * w * ph.y, rho * w * ph.x);
        const cplx dP = mk(-rho * (dw * ph.y + w * dph.y), rho * (dw * ph.x + w * dph.x));
        cplx pin = mk(0.0, 0.0), dpin = mk(0.0, 0.0);
        if (diff) {
            const double x = geom[G_CX * n + j], y = geom[G_CY * n + j], zz = geom[G_CZ * n + j];
            const double tx = tgeom[G_CX * n + j], ty = tgeom[G_CY * n + j], tz = tgeom[G_CZ * n + j];
            const double wv = x * cb + y * sb, dwv = tx * cb + ty * sb;
            double sw, cw;
            sincos(k * wv, &sw, &cw);
            const double m = rho * gacc * exp(k * zz);
            pin = mk(m * cw, m * sw);
            dpin = pin * mk(dk * zz + k * tz, dk * wv + k * dwv);
        }
        for (int d = 0; d < ndof; ++d) {
            const double* dd = dofs + (int64_t)d * 3 * n;
            const double* td = tdofs + (int64_t)d * 3 * n;
            double nd = 0.0, dnd = 0.0;
            for (int c = 0; c < 3; ++c) {
                nd += nv[c] * dd[c * n + j];
                dnd += tn[c] * dd[c * n + j] + nv[c] * td[c * n + j];
            }
            const double m = -nd * a, dm = -(dnd * a + nd * ta);
            const cplx f = dP * m + P * dm, g = dpin * m + pin * dm;
            acc[4 * d] += f.re;
            acc[4 * d + 1] += f.im;
            acc[4 * d + 2] += g.re;
            acc[4 * d + 3] += g.im;
        }
    }
    __shared__ double red[8][4 * kMaxRhs];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = 0; t < 4 * ndof; ++t) {
        double v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][t] = v;
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
        dF[((int64_t)z * nrhs + q) * ndof + d] = make_double2(red[0][4 * d], red[0][4 * d + 1]);
        if (diff)
            dFK[((int64_t)z * nbeta + (q - ndof)) * ndof + d] = make_double2(red[0][4 * d + 2], red[0][4 * d + 3]);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct Jvp {
    const double* tgeom;
    const double* tdofs;
    const double* d_domegas;
    const double* d_dk;
    double2* dSR;  // n x n (null without Rankine terms)
    double2* dDR;
    int wave_kind;  // 0 none, 1 Wu, 2 Delhommeau
};

// dS, dD for nb frequencies into dS, dD (nb matrices each).
int tangent_matrices(const Batch& bt, const Jvp& jv, const double* d_k, const double* d_dk, int nb,
                     const double* tab, double2* dS, double2* dD)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    if (jv.wave_kind == 2 && tab && nb >= kJvpAllwMinFreqs) {
        const size_t smem = tan_allw_smem(nb);
        auto* fall = (int*)ws_get(ctx, WS_FALL, sizeof(int));
        if (!fall) return MH_ERR_OOM;
        MH_CUDA_TRY(ctx, raise_smem_cap((const void*)k_wave_tangent_allw, smem));
        MH_CUDA_TRY(ctx, cudaMemcpyToSymbolAsync(c_polar_cheb, tab, sizeof(c_polar_cheb), 0, cudaMemcpyDeviceToDevice,
                                                 ctx->stream));
        MH_CUDA_TRY(ctx, cudaMemsetAsync(fall, 0, sizeof(int), ctx->stream));
        const dim3 g2(nblk(n, kTW), nblk(n, kGradCols));
        k_wave_tangent_allw<<<g2, kTW, smem, ctx->stream>>>(bt.m->geom, jv.tgeom, n, bt.direct, d_k, d_dk, nb,
                                                            jv.dSR, jv.dDR, dS, dD, fall);
        k_wave_tangent_allw_rest<<<g2, kTW, 0, ctx->stream>>>(fall, bt.m->geom, jv.tgeom, n, bt.direct, tab, d_k,
                                                             d_dk, nb, jv.dSR, jv.dDR, dS, dD);
        ctx->launches += 1;
    } else {
        k_wave_tangent<<<dim3(nblk(n, kJR), nblk(n, kGradCols), (unsigned)nb), kJR, 0, ctx->stream>>>(
            jv.wave_kind, bt.m->geom, jv.tgeom, n, bt.direct, jv.wave_kind == 2 ? tab : nullptr, d_k, d_dk, jv.dSR,
            jv.dDR, dS, dD);
    }
    ctx->launches += 1;
    MH_CUDA_TRY(ctx, cudaGetLastError());
    return MH_OK;
}

// Tangent solve and forces for nb frequencies whose forward state is
// (S, D factors, BC, X = phi or sigma, PHI).  solve(rhs, x): the forward
// factors' solve into x.
template <class Solve>
int tangent_chunk(const Batch& bt, const Jvp& jv, const double* d_om, const double* d_dom, const double* d_k,
                  const double* d_dk, int nb, const double* tab, const double2* S64, const double2* BC,
                  const double2* X, const double2* PHI, double2* dS, double2* dD, double2* dBC, double2* T,
                  double2* DX, double2* DPHI, double2* dF, double2* dFK, Solve solve)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const int nrhs = bt.nrhs;
    int rc;
    if ((rc = tangent_matrices(bt, jv, d_k, d_dk, nb, tab, dS, dD))) return rc;
    k_bc_tangent<<<dim3(nblk(n, 256), (unsigned)nb), 256, 0, ctx->stream>>>(
        bt.m->geom, jv.tgeom, n, bt.d_dofs, jv.tdofs, bt.ndof, bt.d_betas, bt.nbeta, d_om, d_dom, bt.g, dBC);
    ctx->launches += 1;
    MH_CUDA_TRY(ctx, cudaGetLastError());
    if (bt.direct) {  // T = dS b + S db - dD phi; dphi = D^-1 T
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, dS, n, nb, BC, nullptr, T, nrhs, 1.0, 0.0));
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, S64, n, nb, dBC, T, T, nrhs, 1.0, 1.0));
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, dD, n, nb, X, T, T, nrhs, -1.0, 1.0));
        if ((rc = solve(T, DPHI))) return rc;
    } else {  // T = db - dK sigma; dsigma = K^-1 T; dphi = dS sigma + S dsigma
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, dD, n, nb, X, dBC, T, nrhs, -1.0, 1.0));
        if ((rc = solve(T, DX))) return rc;
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, dS, n, nb, X, nullptr, DPHI, nrhs, 1.0, 0.0));
        MH_CUDA_TRY(ctx, launch_gemv(ctx, false, S64, n, nb, DX, DPHI, DPHI, nrhs, 1.0, 1.0));
    }
    k_forces_tangent<<<nb * nrhs, 256, 0, ctx->stream>>>(bt.m->geom, jv.tgeom, n, bt.d_dofs, jv.tdofs, bt.ndof,
                                                        bt.d_betas, bt.nbeta, d_om, d_dom, bt.rho, bt.g, PHI, DPHI,
                                                        dF, dFK);
    ctx->launches += 1;
    MH_CUDA_TRY(ctx, cudaGetLastError());
    return MH_OK;
}

}  // namespace

int hydro_batch_jvp(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                    const double* dofs, int64_t nbeta, const double* betas, double rho, double g, uint32_t mask,
                    int direct, int precision, double tol, int max_iter, const double* t_vertices,
                    const double* t_centers, const double* t_normals, const double* t_areas, const double* t_omegas,
                    const double* t_dofs, double* added_mass, double* damping, double* diffraction,
                    double* froude_krylov, double* d_added_mass, double* d_damping, double* d_diffraction,
                    double* d_froude_krylov, mh_batch_info* info)
{
    const int64_t n = m->n;
    const int nrhs = (int)(ndof + nbeta);
    const size_t nn = (size_t)n * (size_t)n;
    mh_batch_info local{};
    // ---- inputs, tangents ----
    const size_t dof_bytes = sizeof(double) * 3 * (size_t)n * (size_t)ndof;
    const size_t tg_words = (size_t)G_NFIELDS * n;
    const size_t in_bytes = 2 * dof_bytes + sizeof(double) * (4 * (size_t)nomega + nbeta + tg_words) + 64;
    auto* in = (char*)ws_get(ctx, WS_DOF, in_bytes);
    const size_t out_count = (size_t)nomega * (size_t)(nrhs * ndof + nbeta * ndof);
    auto* d_out = (double2*)ws_get(ctx, WS_OUT, sizeof(double2) * out_count * 2 + 16);
    if (!in || !d_out) return MH_ERR_OOM;
    auto* d_dofs = (double*)in;
    auto* d_tdofs = (double*)(in + dof_bytes);
    auto* d_om = (double*)(in + 2 * dof_bytes);
    auto* d_k = d_om + nomega;
    auto* d_dom = d_k + nomega;
    auto* d_dk = d_dom + nomega;
    auto* d_betas = d_dk + nomega;
    auto* d_tgeom = d_betas + nbeta;
    std::vector<double> hk(nomega), hdw(nomega), hdk(nomega);
    for (int64_t z = 0; z < nomega; ++z) {
        hk[z] = omegas[z] * omegas[z] / g;
        hdw[z] = t_omegas ? t_omegas[z] : 0.0;
        hdk[z] = 2.0 * omegas[z] * hdw[z] / g;
    }
    std::vector<double> htg(tg_words, 0.0);
    for (int64_t i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) {
            if (t_centers) htg[(G_CX + c) * n + i] = t_centers[c * n + i];
            if (t_normals) htg[(G_NX + c) * n + i] = t_normals[c * n + i];
        }
        if (t_areas) htg[G_AREA * n + i] = t_areas[i];
        if (t_vertices)
            for (int a = 0; a < 4; ++a) {
                const int64_t v = m->faces[(size_t)a * n + i];
                for (int c = 0; c < 3; ++c) htg[(G_V + 3 * a + c) * n + i] = t_vertices[c * m->nv + v];
            }
    }
    if (ndof) {
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_dofs, dofs, dof_bytes, cudaMemcpyHostToDevice, ctx->stream));
        if (t_dofs) MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_tdofs, t_dofs, dof_bytes, cudaMemcpyHostToDevice, ctx->stream));
        else MH_CUDA_TRY(ctx, cudaMemsetAsync(d_tdofs, 0, dof_bytes, ctx->stream));
    }
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_om, omegas, sizeof(double) * nomega, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_k, hk.data(), sizeof(double) * nomega, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_dom, hdw.data(), sizeof(double) * nomega, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_dk, hdk.data(), sizeof(double) * nomega, cudaMemcpyHostToDevice, ctx->stream));
    if (nbeta)
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_betas, betas, sizeof(double) * nbeta, cudaMemcpyHostToDevice,
                                         ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_tgeom, htg.data(), sizeof(double) * tg_words, cudaMemcpyHostToDevice,
                                     ctx->stream));
    double2* d_F = d_out;
    double2* d_FK = d_out + (size_t)nomega * nrhs * ndof;
    double2* d_dF = d_out + out_count;
    double2* d_dFK = d_dF + (size_t)nomega * nrhs * ndof;
    Batch bt{ctx, m, n, (int)ndof, (int)nbeta, nrhs, d_dofs, d_betas, rho, g, mask, direct};
    Jvp jv{};
    jv.tgeom = d_tgeom;
    jv.tdofs = d_tdofs;
    jv.d_domegas = d_dom;
    jv.d_dk = d_dk;
    jv.wave_kind = (mask & MH_GF_DELHOMMEAU) ? 2 : ((mask & MH_GF_WU) ? 1 : 0);
    if ((mask & MH_GF_WU) && (mask & MH_GF_DELHOMMEAU))
        return set_err(ctx, MH_ERR_ARG, "the tangent path takes one wave term (GFWu or Delhommeau)");
    // Rankine tangent once per call
    jv.dSR = (double2*)ws_get(ctx, WS_WSD, sizeof(double2) * nn * 2);
    if (!jv.dSR) return MH_ERR_OOM;
    jv.dDR = jv.dSR + nn;
    k_rankine_tangent<<<dim3(nblk(n, kJR), nblk(n, kGradCols)), kJR, 0, ctx->stream>>>(m->geom, d_tgeom, n, mask,
                                                                                     direct, jv.dSR, jv.dDR);
    ctx->launches += 1;
    MH_CUDA_TRY(ctx, cudaGetLastError());
    int rc;
    const double* tab = delh_table_for(ctx, mask, &rc);
    if (rc) return rc;
    const int64_t nv = n * nrhs;
    if (precision == MH_PRECISION_FP64) {
        const size_t mat = sizeof(double2) * nn;
        auto* S = (double2*)ws_get(ctx, WS_S, mat);
        auto* D = (double2*)ws_get(ctx, WS_D, mat);
        auto* BC = (double2*)ws_get(ctx, WS_RHS, sizeof(double2) * nv);
        auto* X = (double2*)ws_get(ctx, WS_PHI, sizeof(double2) * nv);
        auto* piv = (int*)ws_get(ctx, WS_PIV, sizeof(int) * (size_t)n);
        auto* dmat = (double2*)ws_get(ctx, WS_FB, mat * 2);
        auto* vec = (double2*)ws_get(ctx, WS_ADJ, sizeof(double2) * nv * 6);
        if (!S || !D || !BC || !X || !piv || !dmat || !vec) return MH_ERR_OOM;
        double2 *PHI = vec, *dBC = vec + nv, *T = vec + 2 * nv, *DX = vec + 3 * nv, *DPHI = vec + 4 * nv;
        for (int64_t z = 0; z < nomega; ++z) {
            phase_begin(ctx, PH_FP64_ASSEMBLY);
            MH_CUDA_TRY(ctx, launch_assemble_f64(ctx, m, hk[z], mask, direct, tab, S, D));
            phase_end(ctx, PH_FP64_ASSEMBLY);
            MH_CUDA_TRY(ctx, launch_bc_batch(bt, d_om + z, 1, BC));
            phase_begin(ctx, PH_FP64_LU);
            if ((rc = fp64_lu_factor(ctx, n, D, piv))) return rc;
            if (direct) {
                if ((rc = zgemm_strided(ctx, n, nrhs, S, BC, X, 1, 1.0, 0.0))) return rc;
                if ((rc = fp64_getrs(ctx, false, n, D, piv, X, nrhs))) return rc;
                MH_CUDA_TRY(ctx, cudaMemcpyAsync(PHI, X, sizeof(double2) * nv, cudaMemcpyDeviceToDevice,
                                                 ctx->stream));
            } else {
                MH_CUDA_TRY(ctx, cudaMemcpyAsync(X, BC, sizeof(double2) * nv, cudaMemcpyDeviceToDevice, ctx->stream));
                if ((rc = fp64_getrs(ctx, false, n, D, piv, X, nrhs))) return rc;
                if ((rc = zgemm_strided(ctx, n, nrhs, S, X, PHI, 1, 1.0, 0.0))) return rc;
            }
            phase_end(ctx, PH_FP64_LU);
            MH_CUDA_TRY(ctx, launch_forces_batch(bt, d_om + z, 1, PHI, d_F + z * nrhs * ndof,
                                                 d_FK + z * nbeta * ndof));
            auto solve = [&](double2* rhs, double2* out) -> int {
                if (out != rhs)
                    MH_CUDA_TRY(ctx, cudaMemcpyAsync(out, rhs, sizeof(double2) * nv, cudaMemcpyDeviceToDevice,
                                                     ctx->stream));
                return fp64_getrs(ctx, false, n, D, piv, out, nrhs);
            };
            if ((rc = tangent_chunk(bt, jv, d_om + z, d_dom + z, d_k + z, d_dk + z, 1, tab, S, BC, X, PHI, dmat,
                                    dmat + nn, dBC, T, DX, DPHI, d_dF + z * nrhs * ndof, d_dFK + z * nbeta * ndof,
                                    solve)))
                return rc;
        }
    } else {
        auto* SR = (double*)ws_get(ctx, WS_SR, sizeof(double) * nn * 2);
        if (!SR) return MH_ERR_OOM;
        double* DR = SR + nn;
        if ((rc = rankine_real(bt, SR, DR))) return rc;
        const size_t per = nn * (4 * sizeof(double2) + sizeof(float2)) +
                           (size_t)n * nrhs * (12 * sizeof(double2) + 2 * sizeof(float2));
        constexpr size_t kJvpBatchBytes = 32ull << 30;
        const int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(nomega, (int64_t)(kJvpBatchBytes / per)));
        FallbackStore fb;
        for (int64_t z0 = 0; z0 < nomega && rc == MH_OK; z0 += chunk) {
            const int nb = (int)std::min<int64_t>(chunk, nomega - z0);
            fb.lu = nullptr;
            fb.piv = nullptr;
            fb.used.assign(nb, 0);
            rc = run_mixed_chunk(bt, d_om + z0, d_k + z0, nb, SR, DR, tol, max_iter, d_F + z0 * nrhs * ndof,
                                 d_FK + z0 * nbeta * ndof, &local, &fb);
            if (rc) break;
            const int64_t cnt = nv * nb;
            auto* dmat = (double2*)ws_get(ctx, WS_PART, sizeof(double2) * nn * nb * 2);
            auto* vec = (double2*)ws_get(ctx, WS_ADJ, sizeof(double2) * cnt * 6);
            auto* R32 = (float2*)ws_get(ctx, WS_TMP32, sizeof(float2) * cnt);
            auto* misc = ws_get(ctx, WS_MISC, refine_ctl_bytes(nb) + 64);
            if (!dmat || !vec || !R32 || !misc) return MH_ERR_OOM;
            auto* S64 = (double2*)ctx->ws[WS_S];
            auto* D64 = (double2*)ctx->ws[WS_D];
            auto* Dlo = (float2*)ctx->ws[WS_LO];
            auto* Dinv = (float2*)ctx->ws[WS_DINV];
            auto* BC = (double2*)ctx->ws[WS_RHS];
            auto* X = (double2*)ctx->ws[WS_PHI];
            const double2* PHI = direct ? X : (double2*)ctx->ws[WS_TMP];
            double2 *dBC = vec, *T = vec + cnt, *DX = vec + 2 * cnt, *DPHI = vec + 3 * cnt, *R = vec + 4 * cnt;
            auto solve = [&](double2* rhs, double2* out) -> int {
                return mixed_refine_solve(ctx, n, nb, nrhs, D64, Dlo, Dinv, rhs, out, R, R32, misc, false, tol,
                                          max_iter, fb, &local);
            };
            rc = tangent_chunk(bt, jv, d_om + z0, d_dom + z0, d_k + z0, d_dk + z0, nb, tab, S64, BC, X, PHI, dmat,
                               dmat + nn * nb, dBC, T, DX, DPHI, d_dF + z0 * nrhs * ndof, d_dFK + z0 * nbeta * ndof,
                               solve);
        }
    }
    if (rc) return rc;
    std::vector<double2> h(2 * out_count);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), d_out, sizeof(double2) * 2 * out_count, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    unpack_outputs(h.data(), nomega, omegas, ndof, nbeta, added_mass, damping, diffraction, froude_krylov);
    // tangents: dA = Re dF / w^2 - 2 Re F dw / w^3, dB = Im dF / w - Im F dw / w^2
    const double2* hF = h.data();
    const double2* hdF = h.data() + out_count;
    for (int64_t z = 0; z < nomega; ++z) {
        const double w = omegas[z], dw = hdw[z];
        for (int64_t q = 0; q < ndof; ++q)
            for (int64_t i = 0; i < ndof; ++i) {
                const size_t src = ((size_t)z * nrhs + q) * ndof + i;
                const size_t o = (size_t)i + (size_t)ndof * ((size_t)q + (size_t)ndof * (size_t)z);
                const double2 F = hF[src], dF = hdF[src];
                if (d_added_mass) d_added_mass[o] = dF.x / (w * w) - 2.0 * F.x * dw / (w * w * w);
                if (d_damping) d_damping[o] = dF.y / w - F.y * dw / (w * w);
            }
        for (int64_t b = 0; b < nbeta; ++b)
            for (int64_t i = 0; i < ndof; ++i) {
                const size_t o = (size_t)i + (size_t)ndof * ((size_t)z + (size_t)nomega * (size_t)b);
                const double2 dF = hdF[((size_t)z * nrhs + ndof + b) * ndof + i];
                const double2 dK = hdF[(size_t)nomega * nrhs * ndof + ((size_t)z * nbeta + b) * ndof + i];
                if (d_diffraction) {
                    d_diffraction[2 * o] = dF.x;
                    d_diffraction[2 * o + 1] = dF.y;
                }
                if (d_froude_krylov) {
                    d_froude_krylov[2 * o] = dK.x;
                    d_froude_krylov[2 * o + 1] = dK.y;
                }
            }
    }
    if (info) *info = local;
    return MH_OK;
}

}  // namespace mh
