// Adjoint (reverse-mode) gradients of the batched hydrodynamic coefficients.
//
// Replaces the reference's differentiation of this path: Zygote through the
// assembly, ImplicitAD's implicit_linear for the solve
// (src/matrix_assembly.jl:105-133) and the ForwardDiff branch (:108-114).
// For output cotangents (of added mass, damping, diffraction and
// Froude-Krylov forces) it returns the cotangents of every mesh field
// (vertices, centres, normals, areas, radii), of every frequency and of the
// dof arrays, i.e. the Tangent{Mesh} plus omega-bar of an rrule.
//
// Per frequency, with S, D (K when indirect), boundary conditions b and
// output cotangent phi-bar (from the force sums):
//   direct   D phi = S b:    lambda = D^-H phi-bar, b-bar = S^H lambda,
//            S-bar = lambda b^H, D-bar = -lambda phi^H;
//   indirect K sigma = b, phi = S sigma: mu = K^-H S^H phi-bar, b-bar = mu,
//            S-bar = phi-bar sigma^H, K-bar = -mu sigma^H.
// The adjoint solve reuses the forward factors: FP64 (zgetrs with
// conjugate transpose) or the low-precision factors with FP64 refinement of
// D^H x = r.  S-bar and D-bar are never formed: the pair kernels form
// sum_q a_iq conj(b_jq) on the fly.  The Rankine terms are frequency
// independent, so their contraction runs once per call against
// Re sum_w S-bar(w) and Re sum_w D-bar(w), accumulated by ZGEMM; the wave
// term runs per frequency, with exact derivatives of the table or Wu
// formulas (dual numbers in (r, z)) chained by hand to the panel geometry
// and k.  The near-field Rankine integral is differentiated with 6-way dual
// numbers (three passes over centre+normal and the four vertices).
#include <cuComplex.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mh_device.cuh"
#include "mh_internal.h"

namespace mh {
namespace {

constexpr int kAR = 128;  // rows (threads) per CTA of the pair kernels
constexpr int kAC = 16;   // columns (panels in shared memory) per CTA (kGradCols)
constexpr double kI4P = 1.0 / (4.0 * kPi);

// Per-panel cotangent fields (device array gbar[GB_NF][n]).
enum GbarField : int { GB_C = 0, GB_N = 3, GB_A = 6, GB_V = 7, GB_NF = 19 };
constexpr int kRowF = 6;   // row partials: centre (3), normal (3)
constexpr int kWaveF = 7;  // wave column partials: centre, normal, area
constexpr int kAdjAllwMinFreqs = 4;  // chunks this large use the frequency-batched Delhommeau adjoint

unsigned nblk(int64_t count, int threads) { return (unsigned)((count + threads - 1) / threads); }

#include "mh_grad.cuh"
static_assert(kAC == kGradCols, "pair kernels stage kGradCols panels");

struct WaveBar {
    double dx, dy, zs, area, k;
    double n[3];
};

// Reverse of wave_pair for one pair and one k, given the dimensionless term
// and its derivatives at (r, z) = k (dis, zs): L = Re(cs s + cw (nD . g)),
// s = k A G, g = (sg k^2 A u_x G_r, sg k^2 A u_y G_r, k^2 A G_z),
// sg = +1 for the gradient with respect to the first variable.  Returns
// dL/d(dx, dy, zs, area, k) and dL/dnD.
__device__ __forceinline__ void wave_chain(const GDer& o, const WaveGeom& w, double k, double A, bool wrt_first,
                                           cplx cs, cplx cw, const double nD[3], WaveBar& wb)
{
    const bool rad = fabs(k * w.dis) > 1e-6;
    const double sg = wrt_first ? 1.0 : -1.0;
    const double k2 = k * k;
    const cplx c0 = cw * nD[0], c1 = cw * nD[1], c2 = cw * nD[2];  // conj of the g cotangents
    const cplx P1 = rad ? sg * (c0 * w.u0 + c1 * w.u1) : mk(0.0, 0.0);
    const cplx a0 = cs * k, a1 = P1 * k2, a2 = c2 * k2;
    const double Lr = A * (re_mul(a0, o.Gr[0]) + re_mul(a1, o.Gr[1]) + re_mul(a2, o.Gr[2]));
    const double Lz = A * (re_mul(a0, o.Gz[0]) + re_mul(a1, o.Gz[1]) + re_mul(a2, o.Gz[2]));
    const double U0 = rad ? sg * k2 * A * re_mul(c0, o.G[1]) : 0.0;
    const double U1 = rad ? sg * k2 * A * re_mul(c1, o.G[1]) : 0.0;
    wb.dx = Lr * k * w.u0 + (U0 * (1.0 - w.u0 * w.u0) - U1 * w.u0 * w.u1) * w.invd;
    wb.dy = Lr * k * w.u1 + (U1 * (1.0 - w.u1 * w.u1) - U0 * w.u0 * w.u1) * w.invd;
    wb.zs = Lz * k;
    const double e0 = re_mul(cs, o.G[0]), e12 = re_mul(P1, o.G[1]) + re_mul(c2, o.G[2]);
    wb.area = k * e0 + k2 * e12;
    wb.k = Lr * w.dis + Lz * w.zs + A * e0 + 2.0 * k * A * e12;
    const double gr = rad ? sg * k2 * A : 0.0;
    const cplx g0 = (gr * w.u0) * o.G[1], g1 = (gr * w.u1) * o.G[1], g2 = (k2 * A) * o.G[2];
    wb.n[0] = re_mul(cw, g0);
    wb.n[1] = re_mul(cw, g1);
    wb.n[2] = re_mul(cw, g2);
}

__device__ __forceinline__ void wave_pair_vjp(int kind, const double x[3], const Panel& p, double k,
                                              bool wrt_first, const double* __restrict__ tab, cplx cs,
                                              cplx cw, const double nD[3], WaveBar& wb)
{
    const WaveGeom w = wave_geom(x, p);
    GDer o;
    wave_dimless_grad(kind, tab, k * w.dis, k * w.zs, o);
    wave_chain(o, w, k, p.area, wrt_first, cs, cw, nD, wb);
}

// Wave-term contraction over the pairs of a 128-row x 16-column tile for
// every frequency of the chunk.  S-bar_ij(z) = sum_q VA_iq conj(VB_jq),
// D-bar_ij(z) = -sum_q VC_iq conj(VD_jq) (vectors [z][q][n]).
// rowpart[colblock][kRowF][n], colpart[rowblock][kWaveF][n],
// kpart[z][block]: deterministic partial sums.
__global__ void __launch_bounds__(kAR)
k_adj_wave(int kind, const double* __restrict__ geom, int64_t n, int direct, const double* __restrict__ tab,
           const double* __restrict__ kvec, int nb, int nrhs, const double2* __restrict__ VA,
           const double2* __restrict__ VB, const double2* __restrict__ VC, const double2* __restrict__ VD,
           double* __restrict__ rowpart, double* __restrict__ colpart, double* __restrict__ kpart)
{
    extern __shared__ double ksm[];  // [4 warps][nb]
    __shared__ Panel sp[kAC];
    __shared__ double csm[kAR / 32][kAC][kWaveF];
    const int64_t j0 = (int64_t)blockIdx.y * kAC;
    stage(sp, geom, n, j0);
    for (int t = threadIdx.x; t < (kAR / 32) * nb; t += blockDim.x) ksm[t] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * kAR + threadIdx.x;
    const bool live = i < n;
    const int64_t ii = live ? i : 0;
    const double x[3] = {geom[G_CX * n + ii], geom[G_CY * n + ii], geom[G_CZ * n + ii]};
    const double ni[3] = {geom[G_NX * n + ii], geom[G_NY * n + ii], geom[G_NZ * n + ii]};
    const int jend = (int)min((int64_t)kAC, n - j0);
    const int64_t nv = n * nrhs;
    double xb[3] = {0.0, 0.0, 0.0}, nbi[3] = {0.0, 0.0, 0.0};
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        const double* nD = direct ? p.n : ni;
        double cacc[kWaveF] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int z = 0; z < nb; ++z) {
            const int64_t base = (int64_t)z * nv;
            double sr = 0.0, si = 0.0, dr = 0.0, di = 0.0;
            for (int q = 0; q < nrhs; ++q) {
                const double2 a = VA[base + q * n + ii], b = VB[base + q * n + j];
                const double2 c = VC[base + q * n + ii], d = VD[base + q * n + j];
                sr += a.x * b.x + a.y * b.y;
                si += a.y * b.x - a.x * b.y;
                dr -= c.x * d.x + c.y * d.y;
                di -= c.y * d.x - c.x * d.y;
            }
            // cs = conj(-S-bar / 4pi), cw = conj(-D-bar / 4pi)
            const cplx cs = mk(-kI4P * sr, kI4P * si), cw = mk(-kI4P * dr, kI4P * di);
            double bk = 0.0;
            if (live) {
                WaveBar wb;
                wave_pair_vjp(kind, x, p, kvec[z], !direct, tab, cs, cw, nD, wb);
                xb[0] += wb.dx;
                xb[1] += wb.dy;
                xb[2] += wb.zs;
                cacc[0] -= wb.dx;
                cacc[1] -= wb.dy;
                cacc[2] += wb.zs;
                if (direct) {
                    cacc[3] += wb.n[0];
                    cacc[4] += wb.n[1];
                    cacc[5] += wb.n[2];
                } else {
                    nbi[0] += wb.n[0];
                    nbi[1] += wb.n[1];
                    nbi[2] += wb.n[2];
                }
                cacc[6] += wb.area;
                bk = wb.k;
            }
            bk = warp_sum(bk);
            if (lane == 0) ksm[warp * nb + z] += bk;
        }
#pragma unroll
        for (int f = 0; f < kWaveF; ++f) {
            const double v = warp_sum(cacc[f]);
            if (lane == 0) csm[warp][jj][f] = v;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < jend * kWaveF; t += blockDim.x) {
        const int jj = t / kWaveF, f = t % kWaveF;
        double s = 0.0;
        for (int w = 0; w < kAR / 32; ++w) s += csm[w][jj][f];
        colpart[((int64_t)blockIdx.x * kWaveF + f) * n + j0 + jj] = s;
    }
    if (live) {
        for (int c = 0; c < 3; ++c) {
            rowpart[((int64_t)blockIdx.y * kRowF + c) * n + i] = xb[c];
            rowpart[((int64_t)blockIdx.y * kRowF + 3 + c) * n + i] = nbi[c];
        }
    }
    const int64_t P = (int64_t)gridDim.x * gridDim.y;
    const int64_t blk = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    for (int z = threadIdx.x; z < nb; z += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kAR / 32; ++w) s += ksm[w * nb + z];
        kpart[(int64_t)z * P + blk] = s;
    }
}

// Delhommeau contraction from the forward's tape: the forward pass of the
// same call stored the dimensionless (G, G_r) of every pair and frequency
// (S layout, 32 B each), so no table is evaluated here; G_z = G + 2/R and
// the second derivatives come from the identities.  Otherwise as k_adj_wave:
// S-bar_ij(z) = sum_q VA_iq conj(VB_jq), D-bar_ij(z) = -sum_q VC_iq conj(VD_jq)
// (vectors [z][q][n]).  Each sweep over the frequencies takes kTJ columns
// at once, so the row vectors VA, VC are read once per kTJ pairs and the
// k partial sums are reduced across the warp once per kTJ pairs.
// The kernel is bound by load latency, so every load of an iteration
// (sweep, z) is issued one iteration ahead by cp.async into a two-slot ring
// in shared memory, in flight without holding registers:
//   - per thread: its 2 kTJ tape entries (G, G_r of each pair) and, when the
//     right-hand-side count NQ is a compile-time constant (1 to 3), its row
//     vectors VA, VC of every right-hand side;
//   - per warp: the column vectors VB, VD of the iteration (the same for
//     every lane), one entry per lane.
// Each thread waits on its own copies, then a __syncwarp publishes the
// warp's VB/VD slot and retires the slot that the next copies overwrite;
// there is no CTA barrier in the loop.  NQ = 0 takes any count up to
// kMaxRhs and loads VA, VC directly.
// rowpart[colblock][kRowF][n], colpart[rowblock][kWaveF][n],
// kpart[z][block]: deterministic partial sums.
constexpr int kTJ = 2;
constexpr int kTapeStages = 2;
static_assert(kAC % kTJ == 0, "column blocks split into sweeps of kTJ pairs");

template <int NQ>
struct TapeRing {
    static constexpr int kThread = 2 * kTJ + 2 * NQ;                // double2 per thread and slot
    static constexpr int kWarp = 2 * kTJ * (NQ > 0 ? NQ : kMaxRhs);  // double2 per warp and slot
    static constexpr size_t kBytes = sizeof(double2) * kTapeStages * (kThread * kAR + kWarp * (kAR / 32));
};

template <int NQ>
size_t tape_smem(int nb)
{
    return TapeRing<NQ>::kBytes + sizeof(double) * (kAR / 32 + 2) * nb;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

template <int NQ>
__global__ void __launch_bounds__(kAR, 4)
k_adj_delh_tape(const double* __restrict__ geom, int64_t n, int direct, const double2* __restrict__ tape,
                const double* __restrict__ kvec, int nb, int nrhs, const double2* __restrict__ VA,
                const double2* __restrict__ VB, const double2* __restrict__ VC, const double2* __restrict__ VD,
                double* __restrict__ rowpart, double* __restrict__ colpart, double* __restrict__ kpart)
{
    using Ring = TapeRing<NQ>;
    extern __shared__ __align__(16) unsigned char tsm[];
    double2* ring = (double2*)tsm;                                                // [slot][Ring::kThread][kAR]
    double2* wring = ring + kTapeStages * Ring::kThread * kAR;                    // [slot][warp][Ring::kWarp]
    double* ksm = (double*)(wring + kTapeStages * Ring::kWarp * (kAR / 32));      // [4 warps][nb]
    double* ksh = ksm + (kAR / 32) * nb;                                          // k [nb]
    double* iksh = ksh + nb;                                                      // 1/k [nb]
    __shared__ Panel sp[kAC];
    __shared__ double csm[kAR / 32][kAC][kWaveF];
    const int64_t j0 = (int64_t)blockIdx.y * kAC;
    stage(sp, geom, n, j0);
    for (int t = threadIdx.x; t < (kAR / 32) * nb; t += blockDim.x) ksm[t] = 0.0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) {
        ksh[t] = kvec[t];
        iksh[t] = 1.0 / kvec[t];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t i = (int64_t)blockIdx.x * kAR + threadIdx.x;
    const bool live = i < n;
    const int64_t ii = live ? i : 0;
    const double x[3] = {geom[G_CX * n + ii], geom[G_CY * n + ii], geom[G_CZ * n + ii]};
    const double ni[3] = {geom[G_NX * n + ii], geom[G_NY * n + ii], geom[G_NZ * n + ii]};
    const int jend = (int)min((int64_t)kAC, n - j0);
    const int64_t nv = n * nrhs, nn = n * n;
    double xb[3] = {0.0, 0.0, 0.0}, nbi[3] = {0.0, 0.0, 0.0};
    const double sg = direct ? -1.0 : 1.0;  // +1 for the gradient with respect to the first variable
    // ring fill: iterations (sweep, z) in loop order, slot = iteration & 1.
    // Out-of-range rows copy row 0 and a short last sweep its last pair (in
    // bounds, unused), so every lane copies the same pattern.
    const int went = 2 * kTJ * (NQ > 0 ? NQ : nrhs);  // VB/VD entries per iteration: (q * kTJ + u) * 2 + {B, D}
    const int nsweep = (jend + kTJ - 1) / kTJ;
    int pf_s = 0, pf_z = 0, pf_slot = 0;
    auto ring_issue = [&]() {
        if (pf_s < nsweep) {
            double2* mine = ring + (size_t)pf_slot * Ring::kThread * kAR + threadIdx.x;
            const int64_t zo = (int64_t)pf_z * nv;
#pragma unroll
            for (int u = 0; u < kTJ; ++u) {
                const int64_t j = j0 + min(pf_s * kTJ + u, jend - 1);
                const double2* src = tape + 2 * ((int64_t)pf_z * nn + j * n + ii);
                cp_async16(mine + (2 * u) * kAR, src);
                cp_async16(mine + (2 * u + 1) * kAR, src + 1);
            }
            if constexpr (NQ > 0) {
#pragma unroll
                for (int q = 0; q < NQ; ++q) {
                    cp_async16(mine + (2 * kTJ + 2 * q) * kAR, VA + zo + (int64_t)q * n + ii);
                    cp_async16(mine + (2 * kTJ + 2 * q + 1) * kAR, VC + zo + (int64_t)q * n + ii);
                }
            }
            double2* wslot = wring + ((size_t)pf_slot * (kAR / 32) + warp) * Ring::kWarp;
            for (int e = lane; e < went; e += 32) {
                const int q = e / (2 * kTJ), u = (e >> 1) % kTJ;
                const int64_t j = j0 + min(pf_s * kTJ + u, jend - 1);
                cp_async16(wslot + e, ((e & 1) ? VD : VB) + zo + (int64_t)q * n + j);
            }
            if (++pf_z == nb) {
                pf_z = 0;
                ++pf_s;
            }
        }
        cp_async_commit();
        pf_slot ^= 1;
    };
    ring_issue();
    int rd_slot = 0;
    for (int jb = 0; jb < jend; jb += kTJ) {
        WaveGeom wg[kTJ];
        double irho[kTJ], s01[kTJ];
        // frequency moments of the chain: sums over z of k^p re(c G') (see below)
        double Sa2[kTJ], Sb3r[kTJ], Sc3[kTJ], Sc3r[kTJ], Sd2r[kTJ], Se2[kTJ], Sf3[kTJ], Sg1[kTJ], Sh2[kTJ];
#pragma unroll
        for (int u = 0; u < kTJ; ++u) {
            const int jj = min(jb + u, jend - 1);  // a short last sweep repeats its last pair, masked below
            wg[u] = wave_geom(x, sp[jj]);
            irho[u] = 1.0 / hypot(wg[u].dis, wg[u].zs);
            const double* nD = direct ? sp[jj].n : ni;
            s01[u] = sg * (nD[0] * wg[u].u0 + nD[1] * wg[u].u1);
            Sa2[u] = Sb3r[u] = Sc3[u] = Sc3r[u] = Sd2r[u] = Se2[u] = Sf3[u] = Sg1[u] = Sh2[u] = 0.0;
        }
        for (int z = 0; z < nb; ++z) {
            const double k = ksh[z], ik = iksh[z], k2 = k * k, k3 = k2 * k;
            cp_async_wait_all();  // this thread's copies of iteration (jb, z)
            __syncwarp();         // the warp's VB/VD copies; every lane is done with the other slot
            ring_issue();         // iteration (jb, z) + 1 into the other slot
            const double2* mine = ring + (size_t)rd_slot * Ring::kThread * kAR + threadIdx.x;
            const double2* vcol = wring + ((size_t)rd_slot * (kAR / 32) + warp) * Ring::kWarp;
            rd_slot ^= 1;
            double bk = 0.0;
            double sr[kTJ], si[kTJ], dr[kTJ], di[kTJ];
#pragma unroll
            for (int u = 0; u < kTJ; ++u) sr[u] = si[u] = dr[u] = di[u] = 0.0;
            auto rhs_term = [&](int q, double2 a, double2 c) {
#pragma unroll
                for (int u = 0; u < kTJ; ++u) {
                    const double2 b = vcol[(q * kTJ + u) * 2], d = vcol[(q * kTJ + u) * 2 + 1];
                    sr[u] += a.x * b.x + a.y * b.y;
                    si[u] += a.y * b.x - a.x * b.y;
                    dr[u] -= c.x * d.x + c.y * d.y;
                    di[u] -= c.y * d.x - c.x * d.y;
                }
            };
            if constexpr (NQ > 0) {
#pragma unroll
                for (int q = 0; q < NQ; ++q)
                    rhs_term(q, mine[(2 * kTJ + 2 * q) * kAR], mine[(2 * kTJ + 2 * q + 1) * kAR]);
            } else {
                const int64_t base = (int64_t)z * nv;
                for (int q = 0; q < nrhs; ++q) rhs_term(q, VA[base + q * n + ii], VC[base + q * n + ii]);
            }
#pragma unroll
            for (int u = 0; u < kTJ; ++u) {
                const int jj = jb + u;
                if (jj >= jend) break;
                if (!live) continue;
                const Panel& p = sp[jj];
                const double* nD = direct ? p.n : ni;
                // cs = conj(-S-bar / 4pi), cw = conj(-D-bar / 4pi)
                const double csr = -kI4P * sr[u], csi = kI4P * si[u];
                const double cwr = -kI4P * dr[u], cwi = kI4P * di[u];
                // dimensionless G, G_r from the tape; G_z = G + 2/R, second
                // derivatives from the identities (as gder_identities)
                const double iR = ik * irho[u], iR3 = iR * iR * iR;  // 1 / R, R = k rho
                const double r = k * wg[u].dis, zz = k * wg[u].zs;
                const double2 g0 = mine[(2 * u) * kAR], g1 = mine[(2 * u + 1) * kAR];
                const double G2r = g0.x + 2.0 * iR, G2i = g0.y;
                const double Gzzr = G2r - 2.0 * zz * iR3, Gzzi = G2i;
                const double Grzr = g1.x - 2.0 * r * iR3, Grzi = g1.y;
                double Grrr, Grri;
                if (r > 1e-3) {
                    const double ir = ik * wg[u].invd;
                    Grrr = -g1.x * ir - Gzzr;
                    Grri = -g1.y * ir - Gzzi;
                } else {
                    Grrr = -0.5 * Gzzr;
                    Grri = -0.5 * Gzzi;
                }
                const double va = csr * g1.x - csi * g1.y;  // re(cs G_r)
                const double vb = cwr * Grrr - cwi * Grri;  // re(cw G_rr)
                const double vc = cwr * Grzr - cwi * Grzi;  // re(cw G_rz)
                const double vd = cwr * g1.x - cwi * g1.y;  // re(cw G_r)
                const double ve = csr * G2r - csi * G2i;    // re(cs G_z)
                const double vf = cwr * Gzzr - cwi * Gzzi;  // re(cw G_zz)
                const double vg = csr * g0.x - csi * g0.y;  // re(cs G)
                const double vh = cwr * G2r - cwi * G2i;    // re(cw G_z)
                const bool rad = fabs(r) > 1e-6;
                Sa2[u] += k2 * va;
                Sc3[u] += k3 * vc;
                Se2[u] += k2 * ve;
                Sf3[u] += k3 * vf;
                Sg1[u] += k * vg;
                Sh2[u] += k2 * vh;
                if (rad) {
                    Sb3r[u] += k3 * vb;
                    Sc3r[u] += k3 * vc;
                    Sd2r[u] += k2 * vd;
                }
                // dL/dk of this pair and frequency (wave_chain's k term)
                const double A = p.area, rs = rad ? s01[u] : 0.0;
                const double Lr = A * (k * va + rs * k2 * vb + nD[2] * k2 * vc);
                const double Lz = A * (k * ve + rs * k2 * vc + nD[2] * k2 * vf);
                bk += Lr * wg[u].dis + Lz * wg[u].zs + A * vg + 2.0 * k * A * (rs * vd + nD[2] * vh);
            }
            bk = warp_sum(bk);
            if (lane == 0) ksm[warp * nb + z] += bk;
        }
        // the chain of wave_chain summed over the frequencies: per pair
        // dx, dy, z, area and the normal, from the moments
#pragma unroll
        for (int u = 0; u < kTJ; ++u) {
            if (jb + u >= jend) break;
            double col[kWaveF] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            if (live) {
                const Panel& p = sp[jb + u];
                const double* nD = direct ? p.n : ni;
                const double A = p.area, u0 = wg[u].u0, u1 = wg[u].u1, invd = wg[u].invd;
                const double lin = Sa2[u] + s01[u] * Sb3r[u] + nD[2] * Sc3[u];
                const double dx = A * u0 * lin + sg * A * invd * (nD[0] * (1.0 - u0 * u0) - nD[1] * u0 * u1) * Sd2r[u];
                const double dy = A * u1 * lin + sg * A * invd * (nD[1] * (1.0 - u1 * u1) - nD[0] * u0 * u1) * Sd2r[u];
                const double zs = A * (Se2[u] + s01[u] * Sc3r[u] + nD[2] * Sf3[u]);
                const double area = Sg1[u] + s01[u] * Sd2r[u] + nD[2] * Sh2[u];
                const double nb0 = sg * A * u0 * Sd2r[u], nb1 = sg * A * u1 * Sd2r[u], nb2 = A * Sh2[u];
                xb[0] += dx;
                xb[1] += dy;
                xb[2] += zs;
                col[0] = -dx;
                col[1] = -dy;
                col[2] = zs;
                if (direct) {
                    col[3] = nb0;
                    col[4] = nb1;
                    col[5] = nb2;
                } else {
                    nbi[0] += nb0;
                    nbi[1] += nb1;
                    nbi[2] += nb2;
                }
                col[6] = area;
            }
#pragma unroll
            for (int f = 0; f < kWaveF; ++f) {
                const double v = warp_sum(col[f]);
                if (lane == 0) csm[warp][jb + u][f] = v;
            }
        }
    }
    cp_async_wait_all();  // only an empty group remains
    __syncthreads();
    for (int t = threadIdx.x; t < jend * kWaveF; t += blockDim.x) {
        const int jj = t / kWaveF, f = t % kWaveF;
        double s = 0.0;
        for (int w = 0; w < kAR / 32; ++w) s += csm[w][jj][f];
        colpart[((int64_t)blockIdx.x * kWaveF + f) * n + j0 + jj] = s;
    }
    if (live) {
        for (int c = 0; c < 3; ++c) {
            rowpart[((int64_t)blockIdx.y * kRowF + c) * n + i] = xb[c];
            rowpart[((int64_t)blockIdx.y * kRowF + 3 + c) * n + i] = nbi[c];
        }
    }
    const int64_t P = (int64_t)gridDim.x * gridDim.y;
    const int64_t blk = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    for (int z = threadIdx.x; z < nb; z += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kAR / 32; ++w) s += ksm[w * nb + z];
        kpart[(int64_t)z * P + blk] = s;
    }
}

// One (pair, frequency) of the Delhommeau adjoint off the polar patch: the
// per-point table gradient and the chain (out of line, so the polar path
// keeps its state in registers).
__device__ __noinline__ void delh_pair_vjp_point(const double* __restrict__ tab, const WaveGeom* wg, double k,
                                                 double A, bool wrt_first, cplx cs, cplx cw, const double* nD,
                                                 WaveBar* wb)
{
    GDer o;
    delh_point_grad(tab, k * wg->dis, k * wg->zs, &o);
    wave_chain(o, *wg, k, A, wrt_first, cs, cw, nD, *wb);
}

// Frequency-batched adjoint of the tabulated Delhommeau term (the reverse
// of the forward's frequency-batched pass, same arithmetic for the values).
// A pair keeps its polar angle alpha at every frequency, so the alpha
// direction of the four polar tables (B, C, E0 = e^z J0(r), E1 = e^z J1(r))
// is contracted once per pair into series in R (shared memory, one column
// per thread); each frequency runs 1-D Clenshaw recurrences in u(R), two
// frequencies at a time, forms (G, G_r, G_z) as the forward does and takes
// the derivatives from the identities.  Frequencies at which the pair
// leaves the polar patch use the per-point table.  Partial sums as
// k_adj_wave.
constexpr int kAW = 64;  // rows (threads) per CTA
constexpr int kZC = 2;   // frequencies per Clenshaw pass
constexpr int kNS = 4;   // series: B, C, E0, E1

size_t adj_allw_smem(int nb)
{
    return sizeof(double) * ((size_t)kNS * kTabNU * kAW + (size_t)(kAW / 32) * nb + nb);
}

__global__ void __launch_bounds__(kAW, 5)
k_adj_delh_allw(const double* __restrict__ geom, int64_t n, int direct, const double* __restrict__ tab,
                const double* __restrict__ kvec, int nb, int nrhs, const double2* __restrict__ VA,
                const double2* __restrict__ VB, const double2* __restrict__ VC, const double2* __restrict__ VD,
                double* __restrict__ rowpart, double* __restrict__ colpart, double* __restrict__ kpart)
{
    extern __shared__ double dsm[];
    double* w = dsm;                              // [kNS * kTabNU][kAW]
    double* ksm = w + kNS * kTabNU * kAW;         // [kAW / 32][nb]
    double* logk = ksm + (kAW / 32) * nb;         // [nb]
    __shared__ Panel sp[kAC];
    __shared__ double csm[kAW / 32][kAC][kWaveF];
    const int64_t j0 = (int64_t)blockIdx.y * kAC;
    stage(sp, geom, n, j0);
    for (int t = threadIdx.x; t < (kAW / 32) * nb; t += blockDim.x) ksm[t] = 0.0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) logk[t] = log(kvec[t]);
    __syncthreads();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t i = (int64_t)blockIdx.x * kAW + tid;
    const bool live = i < n;
    const int64_t ii = live ? i : 0;
    const double x[3] = {geom[G_CX * n + ii], geom[G_CY * n + ii], geom[G_CZ * n + ii]};
    const double ni[3] = {geom[G_NX * n + ii], geom[G_NY * n + ii], geom[G_NZ * n + ii]};
    const int jend = (int)min((int64_t)kAC, n - j0);
    const int64_t nv = n * nrhs;
    double* wt = w + tid;
    double xb[3] = {0.0, 0.0, 0.0}, nbi[3] = {0.0, 0.0, 0.0};
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        const double* nD = direct ? p.n : ni;
        const WaveGeom wg = wave_geom(x, p);
        const double az1 = -wg.zs;
        const double rho = hypot(wg.dis, wg.zs);
        const bool polar_ok = az1 >= 0.0 && rho > 0.0;
        const double lp = log(0.5 * (rho + az1));
        const double gp = wg.dis / (rho * (rho + az1));  // r / (R (R + |z|)) at k = 1
        if (polar_ok) {  // contract alpha: w_q[row] = sum_col c_q[row][col] T_col(v)
            const double v = 4.0 * atan2(wg.dis, az1) / kPi - 1.0;
#pragma unroll 1
            for (int q = 0; q < kNS; ++q) {
                const double* c = tab + q * kTabPolarFn;
#pragma unroll 1
                for (int row = 0; row < kTabNU; ++row) {
                    const double* cr = c + row * kTabNV;
                    double b1 = 0.0, b2 = 0.0;
#pragma unroll
                    for (int col = kTabNV - 1; col >= 1; --col) {
                        const double t = fma(2.0 * v, b1, __ldg(cr + col) - b2);
                        b2 = b1;
                        b1 = t;
                    }
                    wt[(q * kTabNU + row) * kAW] = fma(v, b1, __ldg(cr) - b2);
                }
            }
        }
        double cacc[kWaveF] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        for (int zc = 0; zc < nb; zc += kZC) {
            double kk[kZC], uu[kZC];
            bool pol[kZC];
            cplx csz[kZC], cwz[kZC];  // weights first: their loads overlap the recurrences
#pragma unroll
            for (int t = 0; t < kZC; ++t) {
                const int z = min(zc + t, nb - 1);
                const int64_t base = (int64_t)z * nv;
                double sr_ = 0.0, si_ = 0.0, dr_ = 0.0, di_ = 0.0;
                for (int q = 0; q < nrhs; ++q) {
                    const double2 a = VA[base + q * n + ii], b = VB[base + q * n + j];
                    const double2 c = VC[base + q * n + ii], d = VD[base + q * n + j];
                    sr_ += a.x * b.x + a.y * b.y;
                    si_ += a.y * b.x - a.x * b.y;
                    dr_ -= c.x * d.x + c.y * d.y;
                    di_ -= c.y * d.x - c.x * d.y;
                }
                csz[t] = mk(-kI4P * sr_, kI4P * si_);
                cwz[t] = mk(-kI4P * dr_, kI4P * di_);
                kk[t] = kvec[z];
                const double R = kk[t] * rho;
                pol[t] = polar_ok && (zc + t < nb) && R < kTabRPolar;
                uu[t] = 2.0 * R / kTabRPolar - 1.0;
            }
            double sv[kZC][kNS];
            if (pol[0] || pol[kZC - 1]) {
                double b1[kZC][kNS], b2[kZC][kNS];
#pragma unroll
                for (int t = 0; t < kZC; ++t)
#pragma unroll
                    for (int q = 0; q < kNS; ++q) b1[t][q] = b2[t][q] = 0.0;
#pragma unroll 2
                for (int row = kTabNU - 1; row >= 1; --row) {
                    double cq[kNS];
#pragma unroll
                    for (int q = 0; q < kNS; ++q) cq[q] = wt[(q * kTabNU + row) * kAW];
#pragma unroll
                    for (int t = 0; t < kZC; ++t) {
                        const double u2 = 2.0 * uu[t];
#pragma unroll
                        for (int q = 0; q < kNS; ++q) {
                            const double nt = fma(u2, b1[t][q], cq[q] - b2[t][q]);
                            b2[t][q] = b1[t][q];
                            b1[t][q] = nt;
                        }
                    }
                }
#pragma unroll
                for (int t = 0; t < kZC; ++t)
#pragma unroll
                    for (int q = 0; q < kNS; ++q) sv[t][q] = fma(uu[t], b1[t][q], wt[q * kTabNU * kAW] - b2[t][q]);
            }
#pragma unroll
            for (int t = 0; t < kZC; ++t) {
                const int z = zc + t;
                if (z >= nb) break;
                const double k = kk[t];
                double bk = 0.0;
                if (live) {
                    WaveBar wb;
                    if (pol[t]) {
                        const double R = k * rho;
                        const double B = sv[t][0], C = sv[t][1], E0 = sv[t][2], E1 = sv[t][3];
                        const double L = logk[z] + lp;
                        cplx G[3];
                        const double G_re = -2.0 * E0 * L + B, G_im = 2.0 * kPi * E0;
                        G[0] = mk(G_re, G_im);
                        G[1] = mk(2.0 * E1 * L - 2.0 * E0 * gp / k + C, -2.0 * kPi * E1);
                        G[2] = mk(G_re + 2.0 / R, G_im);
                        GDer o;
                        gder_identities(G, k * wg.dis, k * wg.zs, R, o);
                        wave_chain(o, wg, k, p.area, !direct, csz[t], cwz[t], nD, wb);
                    } else {
                        delh_pair_vjp_point(tab, &wg, k, p.area, !direct, csz[t], cwz[t], nD, &wb);
                    }
                    xb[0] += wb.dx;
                    xb[1] += wb.dy;
                    xb[2] += wb.zs;
                    cacc[0] -= wb.dx;
                    cacc[1] -= wb.dy;
                    cacc[2] += wb.zs;
                    if (direct) {
                        cacc[3] += wb.n[0];
                        cacc[4] += wb.n[1];
                        cacc[5] += wb.n[2];
                    } else {
                        nbi[0] += wb.n[0];
                        nbi[1] += wb.n[1];
                        nbi[2] += wb.n[2];
                    }
                    cacc[6] += wb.area;
                    bk = wb.k;
                }
                bk = warp_sum(bk);
                if (lane == 0) ksm[warp * nb + z] += bk;
            }
        }
#pragma unroll
        for (int f = 0; f < kWaveF; ++f) {
            const double v = warp_sum(cacc[f]);
            if (lane == 0) csm[warp][jj][f] = v;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < jend * kWaveF; t += blockDim.x) {
        const int jj = t / kWaveF, f = t % kWaveF;
        double s = 0.0;
        for (int w2 = 0; w2 < kAW / 32; ++w2) s += csm[w2][jj][f];
        colpart[((int64_t)blockIdx.x * kWaveF + f) * n + j0 + jj] = s;
    }
    if (live) {
        for (int c = 0; c < 3; ++c) {
            rowpart[((int64_t)blockIdx.y * kRowF + c) * n + i] = xb[c];
            rowpart[((int64_t)blockIdx.y * kRowF + 3 + c) * n + i] = nbi[c];
        }
    }
    const int64_t P = (int64_t)gridDim.x * gridDim.y;
    const int64_t blk = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    for (int z = threadIdx.x; z < nb; z += blockDim.x) {
        double s = 0.0;
        for (int w2 = 0; w2 < kAW / 32; ++w2) s += ksm[w2 * nb + z];
        kpart[(int64_t)z * P + blk] = s;
    }
}

// ---------------------------------------------------------------------------
// Rankine terms
// ---------------------------------------------------------------------------

// Far field reverse (rankine.jl:33-34): I = A/r, grad = A rb / r^3,
// L = ibar I + gb . grad; returns dL/dy (= -dL/dc) and adds dL/dA.
__device__ __forceinline__ void rankine_far_vjp(const double rb[3], double r, double A, double ibar,
                                                const double gb[3], double yb[3], double& ab, double gr[3])
{
    const double ir = 1.0 / r, ir3 = ir * ir * ir, ir5 = ir3 * ir * ir;
    const double gdr = gb[0] * rb[0] + gb[1] * rb[1] + gb[2] * rb[2];
    for (int a = 0; a < 3; ++a) {
        gr[a] = rb[a] * ir3 * A;
        yb[a] = A * (-ibar * rb[a] * ir3 + gb[a] * ir3 - 3.0 * gdr * rb[a] * ir5);
    }
    ab += ibar * ir + gdr * ir3;
}

// Reverse of rankine_pair for L = ibar I + gb . grad in one pass: out[0..2]
// dL/dc, out[3..5] dL/dn, out[6 + 3 a + k] dL/dv_a,k, and gr the forward
// gradient.  The forward sweep is rankine_pair's (rankine.jl:36-61, 65-123:
// same branches and guards); the reverse walks each edge's terms back to
// the edge vector, the normal, the point-to-vertex vectors and the vertex
// distances, then GZ = (y - c) . n.  |GZ| is differentiated as the dual
// numbers do (slope +1 at 0), sign(GZ) and the guards are constants.  One
// thread per entry replaces eighteen forward passes (one per direction).
__device__ __forceinline__ void rankine_pair_vjp(const double y[3], const Panel& p, double ibar, const double gb[3],
                                                 double out[18], double gr[3])
{
#pragma unroll
    for (int k = 0; k < 18; ++k) out[k] = 0.0;
    const double rb[3] = {y[0] - p.c[0], y[1] - p.c[1], y[2] - p.c[2]};
    const double r = sqrt(rb[0] * rb[0] + rb[1] * rb[1] + rb[2] * rb[2]);
    if (r > 7.0 * p.radius) {  // far field: only the centre moves it (the area is not a direction here)
        double yb[3], ab = 0.0;
        rankine_far_vjp(rb, r, p.area, ibar, gb, yb, ab, gr);
        for (int a = 0; a < 3; ++a) out[a] = -yb[a];
        return;
    }
    const double GZ = rb[0] * p.n[0] + rb[1] * p.n[1] + rb[2] * p.n[2];
    const double aGZ = fabs(GZ);
    const double sg = signd(GZ);
    const bool use_at = aGZ >= 1e-4 * p.radius;
    double RR[4], DRX[4][3];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double d0 = y[0] - p.v[3 * a], d1 = y[1] - p.v[3 * a + 1], d2 = y[2] - p.v[3 * a + 2];
        RR[a] = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
        DRX[a][0] = d0 / RR[a];
        DRX[a][1] = d1 / RR[a];
        DRX[a][2] = d2 / RR[a];
    }
    double RRb[4] = {0.0, 0.0, 0.0, 0.0}, DRXb[4][3] = {};
    double aGZb = 0.0, nb[3] = {0.0, 0.0, 0.0};
    double* vb = out + 6;
    double g[3] = {0.0, 0.0, 0.0};
    const double w[3] = {-gb[0], -gb[1], -gb[2]};  // dL/dgg: grad = -sum over edges of gg
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int b = (a + 1) & 3;
        const double e[3] = {p.v[3 * b] - p.v[3 * a], p.v[3 * b + 1] - p.v[3 * a + 1], p.v[3 * b + 2] - p.v[3 * a + 2]};
        const double L = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        if (!(L >= 1e-3 * p.radius)) continue;
        // ---- forward ----
        const double u[3] = {e[0] / L, e[1] / L, e[2] / L};
        const double GYX[3] = {p.n[1] * u[2] - p.n[2] * u[1], p.n[2] * u[0] - p.n[0] * u[2],
                               p.n[0] * u[1] - p.n[1] * u[0]};
        const double pa[3] = {y[0] - p.v[3 * a], y[1] - p.v[3 * a + 1], y[2] - p.v[3 * a + 2]};
        const double GY = pa[0] * GYX[0] + pa[1] * GYX[1] + pa[2] * GYX[2];
        const double sE = RR[b] + RR[a];
        const double ANT = 2.0 * GY * L;
        const double DNT = sE * sE - L * L + 2.0 * aGZ * sE;
        const double ANL = sE + L, DNL = sE - L;
        const double ALDEN = log(ANL / DNL);
        const double AT = use_at ? atan2(ANT, DNT) : 0.0;
        const double q = GY * (DNL - ANL) / (ANL * DNL);
        const double den = ANT * ANT + DNT * DNT;
        double ANLX[3], ANTX[3], DNTX[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ANLX[c] = DRX[b][c] + DRX[a][c];
            ANTX[c] = 2.0 * L * GYX[c];
            DNTX[c] = 2.0 * (sE + aGZ) * ANLX[c] + (2.0 * sg) * sE * p.n[c];
            g[c] -= ALDEN * GYX[c] - (2.0 * sg) * AT * p.n[c] + q * ANLX[c]
                    - 2.0 * aGZ * (ANTX[c] * DNT - DNTX[c] * ANT) / den;
        }
        // ---- reverse of gg[c] (weights w[c]) ----
        const double K = -2.0 * aGZ / den;
        double ALDENb = 0.0, ATb = 0.0, qb = 0.0, denb = 0.0, DNTb = 0.0, ANTb = 0.0, sb = 0.0, Lb = 0.0;
        double GYXb[3], ANLXb[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double term = ANTX[c] * DNT - DNTX[c] * ANT;
            ALDENb += w[c] * GYX[c];
            GYXb[c] = w[c] * ALDEN;
            ATb += w[c] * (-2.0 * sg * p.n[c]);
            nb[c] += w[c] * (-2.0 * sg * AT);
            qb += w[c] * ANLX[c];
            ANLXb[c] = w[c] * q;
            aGZb += w[c] * (-2.0 * term / den);
            denb += w[c] * (2.0 * aGZ * term / (den * den));
            const double ANTXb = w[c] * K * DNT;
            DNTb += w[c] * K * ANTX[c];
            const double DNTXb = -w[c] * K * ANT;
            ANTb += -w[c] * K * DNTX[c];
            // DNTX = 2 (s + aGZ) ANLX + 2 sg s n
            sb += DNTXb * (2.0 * ANLX[c] + 2.0 * sg * p.n[c]);
            aGZb += DNTXb * 2.0 * ANLX[c];
            ANLXb[c] += DNTXb * 2.0 * (sE + aGZ);
            nb[c] += DNTXb * 2.0 * sg * sE;
            // ANTX = 2 L GYX
            Lb += ANTXb * 2.0 * GYX[c];
            GYXb[c] += ANTXb * 2.0 * L;
            // ANLX = DRX_b + DRX_a
            DRXb[b][c] += ANLXb[c];
            DRXb[a][c] += ANLXb[c];
        }
        // den = ANT^2 + DNT^2
        ANTb += denb * 2.0 * ANT;
        DNTb += denb * 2.0 * DNT;
        // q = GY (1/ANL - 1/DNL)
        double GYb = qb * (1.0 / ANL - 1.0 / DNL);
        double ANLb = -qb * GY / (ANL * ANL), DNLb = qb * GY / (DNL * DNL);
        // integral: -2 aGZ AT (use_at) + GY ALDEN (|GY| > 1e-5)
        if (use_at) {
            aGZb += ibar * (-2.0 * AT);
            ATb += ibar * (-2.0 * aGZ);
        }
        if (fabs(GY) > 1e-5) {
            GYb += ibar * ALDEN;
            ALDENb += ibar * GY;
        }
        if (use_at) {  // AT = atan2(ANT, DNT)
            ANTb += ATb * DNT / den;
            DNTb += -ATb * ANT / den;
        }
        // ALDEN = log(ANL) - log(DNL)
        ANLb += ALDENb / ANL;
        DNLb -= ALDENb / DNL;
        // ANL = s + L, DNL = s - L
        sb += ANLb + DNLb;
        Lb += ANLb - DNLb;
        // DNT = s^2 - L^2 + 2 aGZ s
        sb += DNTb * (2.0 * sE + 2.0 * aGZ);
        Lb += DNTb * (-2.0 * L);
        aGZb += DNTb * 2.0 * sE;
        // ANT = 2 GY L
        GYb += ANTb * 2.0 * L;
        Lb += ANTb * 2.0 * GY;
        // s = RR_b + RR_a
        RRb[b] += sb;
        RRb[a] += sb;
        // GY = pa . GYX, pa = y - v_a
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            GYXb[c] += GYb * pa[c];
            vb[3 * a + c] -= GYb * GYX[c];
        }
        // GYX = n x u: n-bar += u x GYX-bar, u-bar = GYX-bar x n
        nb[0] += u[1] * GYXb[2] - u[2] * GYXb[1];
        nb[1] += u[2] * GYXb[0] - u[0] * GYXb[2];
        nb[2] += u[0] * GYXb[1] - u[1] * GYXb[0];
        const double ub[3] = {GYXb[1] * p.n[2] - GYXb[2] * p.n[1], GYXb[2] * p.n[0] - GYXb[0] * p.n[2],
                              GYXb[0] * p.n[1] - GYXb[1] * p.n[0]};
        // u = e / L, L = |e|
        const double udot = ub[0] * u[0] + ub[1] * u[1] + ub[2] * u[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double eb = (ub[c] - udot * u[c]) / L + Lb * u[c];
            vb[3 * b + c] += eb;
            vb[3 * a + c] -= eb;
        }
    }
    // RR_a = |y - v_a|, DRX_a = (y - v_a) / RR_a
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const double dd = DRXb[a][0] * DRX[a][0] + DRXb[a][1] * DRX[a][1] + DRXb[a][2] * DRX[a][2];
#pragma unroll
        for (int c = 0; c < 3; ++c) vb[3 * a + c] -= (DRXb[a][c] - dd * DRX[a][c]) / RR[a] + RRb[a] * DRX[a][c];
    }
    // aGZ = |GZ| (slope +1 at 0, as the dual numbers), GZ = (y - c) . n
    const double GZb = aGZb * (GZ < 0.0 ? -1.0 : 1.0);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        out[c] = -GZb * p.n[c];
        out[3 + c] = nb[c] + GZb * rb[c];
        gr[c] = g[c];
    }
}

// Rankine-term contraction against the frequency sums WS = Re sum_w S-bar(w),
// WD = Re sum_w D-bar(w) (only the real parts enter), 128 rows x 16 columns per CTA, in
// three kernels: k_adj_rankine reverses the far-field terms in place and
// lists the near-field (row, column, term) entries of its CTA in row-major
// order (global list, kNearCap codes per CTA); k_adj_near reverses every
// listed entry by rankine_pair_vjp (cotangents of the centre, normal and
// four vertices in one pass), one entry per thread over the whole matrix, so
// the uneven near-field counts of the CTAs do not matter; k_adj_near_accum
// then adds each CTA's entries to its row and column partials in list order
// (fixed order: bitwise reproducible).  Partials as k_adj_wave with GB_NF
// column fields.
constexpr int kNearF = 21;  // per entry: centre, normal, vertex cotangents (18), D-term normal cotangent (3)
constexpr int kNearCap = kAR * kAC * 2;  // entries a CTA can list

__global__ void __launch_bounds__(kAR)
k_adj_rankine(const double* __restrict__ geom, int64_t n, uint32_t mask, int direct,
              const double* __restrict__ WS, const double* __restrict__ WD, double* __restrict__ rowpart,
              double* __restrict__ colpart, unsigned short* __restrict__ ncode, int* __restrict__ ncount,
              int* __restrict__ nrow, int* __restrict__ ncol, unsigned short* __restrict__ ccode)
{
    __shared__ Panel sp[kAC];
    __shared__ int cpre[kAC][kAR + 1];  // per column: entries of the rows before each row
    __shared__ int cbase[kAC + 1];
    __shared__ double csm[kAR / 32][kAC][GB_NF];
    __shared__ int offs[kAR + 1];
    const int64_t j0 = (int64_t)blockIdx.y * kAC;
    stage(sp, geom, n, j0);
    __syncthreads();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t i0 = (int64_t)blockIdx.x * kAR;
    const int64_t i = i0 + tid;
    const bool live = i < n;
    const int64_t ii = live ? i : 0;
    const double x[3] = {geom[G_CX * n + ii], geom[G_CY * n + ii], geom[G_CZ * n + ii]};
    const double ni[3] = {geom[G_NX * n + ii], geom[G_NY * n + ii], geom[G_NZ * n + ii]};
    const int jend = (int)min((int64_t)kAC, n - j0);
    const bool wrt_first = !direct;
    const double sg = wrt_first ? -1.0 : 1.0, sz = wrt_first ? -1.0 : 1.0;
    const uint32_t refl = mask & (MH_GF_RANKINE_REFLECTED | MH_GF_RANKINE_REFLECTED_NEGATIVE);
    const bool has_refl = refl == MH_GF_RANKINE_REFLECTED || refl == MH_GF_RANKINE_REFLECTED_NEGATIVE;
    const bool has_dir = (mask & MH_GF_RANKINE) != 0;
    const double sgn = (refl == MH_GF_RANKINE_REFLECTED) ? 1.0 : -1.0;
    const double mref[3] = {sgn * sg, sgn * sg, sgn * sg * sz};
    double xb[3] = {0.0, 0.0, 0.0}, nbi[3] = {0.0, 0.0, 0.0};
    uint32_t near = 0;
    // ---- far field in place; near entries marked (bit 2 jj + term) ----
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        const double* nD = direct ? p.n : ni;
        double pb[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // centre, normal, area
        if (live) {
            const double ws = WS[j * n + i], wd = WD[j * n + i];
            const double ibar = -kI4P * ws;
            const double gbar[3] = {-kI4P * wd * nD[0], -kI4P * wd * nD[1], -kI4P * wd * nD[2]};
            double gt[3] = {0.0, 0.0, 0.0};
            for (int term = 0; term < 2; ++term) {
                if (term == 0 ? !has_dir : !has_refl) continue;
                const double y[3] = {x[0], x[1], term ? -x[2] : x[2]};
                const double f[3] = {term ? mref[0] : sg, term ? mref[1] : sg, term ? mref[2] : sg};
                const double rb[3] = {y[0] - p.c[0], y[1] - p.c[1], y[2] - p.c[2]};
                const double r = sqrt(rb[0] * rb[0] + rb[1] * rb[1] + rb[2] * rb[2]);
                if (!(r > 7.0 * p.radius)) {
                    near |= 1u << (2 * jj + term);
                    continue;
                }
                const double gb[3] = {f[0] * gbar[0], f[1] * gbar[1], f[2] * gbar[2]};
                double yb[3], gr[3];
                rankine_far_vjp(rb, r, p.area, term ? sgn * ibar : ibar, gb, yb, pb[6], gr);
                for (int a = 0; a < 3; ++a) {
                    pb[a] -= yb[a];
                    gt[a] += f[a] * gr[a];
                }
                xb[0] += yb[0];
                xb[1] += yb[1];
                xb[2] += term ? -yb[2] : yb[2];
            }
            for (int a = 0; a < 3; ++a) {
                const double nb_a = -kI4P * wd * gt[a];
                if (direct) pb[3 + a] += nb_a;
                else nbi[a] += nb_a;
            }
        }
#pragma unroll
        for (int f = 0; f < 7; ++f) {
            const double v = warp_sum(pb[f]);
            if (lane == 0) csm[warp][jj][f] = v;
        }
    }
    // ---- near-field list (row-major: thread, then column, then term) ----
    offs[tid + 1] = __popc(near);
    if (tid == 0) offs[0] = 0;
    __syncthreads();
    if (tid == 0)
        for (int t = 1; t <= kAR; ++t) offs[t] += offs[t - 1];
    __syncthreads();
    const int64_t cta = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    // the same entries in column order (column, then row, then term): per
    // column an exclusive count over the rows, then the column bases
    for (int jj = 0; jj < kAC; ++jj) cpre[jj][tid + 1] = __popc((near >> (2 * jj)) & 3u);
    if (tid < kAC) cpre[tid][0] = 0;
    __syncthreads();
    if (tid < kAC)
        for (int t = 1; t <= kAR; ++t) cpre[tid][t] += cpre[tid][t - 1];
    __syncthreads();
    if (tid == 0) {
        cbase[0] = 0;
        for (int jj = 0; jj < kAC; ++jj) cbase[jj + 1] = cbase[jj] + cpre[jj][kAR];
    }
    __syncthreads();
    {
        unsigned short* list = ncode + cta * kNearCap;
        unsigned short* clist = ccode + cta * kNearCap;
        int o = offs[tid];
        for (uint32_t m = near; m; m &= m - 1) {
            const int bit = __ffs(m) - 1, jj = bit >> 1;
            const int sub = (bit & 1) && (near & (1u << (2 * jj))) ? 1 : 0;  // term 1 after term 0
            clist[cbase[jj] + cpre[jj][tid] + sub] = (unsigned short)o;
            list[o++] = (unsigned short)((tid << 5) | bit);
        }
    }
    nrow[cta * (kAR + 1) + tid] = offs[tid];
    if (tid == 0) {
        nrow[cta * (kAR + 1) + kAR] = offs[kAR];
        ncount[cta] = offs[kAR];
    }
    if (tid < kAC) ncol[cta * kAC + tid] = cpre[tid][kAR];
    for (int t = threadIdx.x; t < jend * GB_NF; t += blockDim.x) {
        const int jj = t / GB_NF, f = t % GB_NF;
        double s = 0.0;
        if (f < 7)
            for (int w = 0; w < kAR / 32; ++w) s += csm[w][jj][f];
        colpart[((int64_t)blockIdx.x * GB_NF + f) * n + j0 + jj] = s;
    }
    if (live) {
        for (int c = 0; c < 3; ++c) {
            rowpart[((int64_t)blockIdx.y * kRowF + c) * n + i] = xb[c];
            rowpart[((int64_t)blockIdx.y * kRowF + 3 + c) * n + i] = nbi[c];
        }
    }
}

// Exclusive prefix sum of the per-CTA near-field counts (one CTA of 1024
// threads); noff[ncta] = total.
__global__ void __launch_bounds__(1024) k_near_scan(const int* __restrict__ ncount, int64_t ncta,
                                                     int64_t* __restrict__ noff)
{
    __shared__ int64_t part[1024];
    const int t = threadIdx.x;
    const int64_t per = (ncta + 1023) / 1024, b0 = t * per, b1 = min(ncta, b0 + per);
    int64_t s = 0;
    for (int64_t c = b0; c < b1; ++c) s += ncount[c];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        int64_t acc = 0;
        for (int u = 0; u < 1024; ++u) {
            const int64_t v = part[u];
            part[u] = acc;
            acc += v;
        }
        noff[ncta] = acc;
    }
    __syncthreads();
    int64_t acc = part[t];
    for (int64_t c = b0; c < b1; ++c) {
        noff[c] = acc;
        acc += ncount[c];
    }
}

__device__ __forceinline__ void load_panel(const double* __restrict__ geom, int64_t n, int64_t j, Panel& p)
{
    for (int a = 0; a < 3; ++a) {
        p.c[a] = geom[(G_CX + a) * n + j];
        p.n[a] = geom[(G_NX + a) * n + j];
    }
    for (int t = 0; t < 12; ++t) p.v[t] = geom[(G_V + t) * n + j];
    p.area = geom[G_AREA * n + j];
    p.radius = geom[G_RADIUS * n + j];
}

// Reverse of every listed near-field entry, one entry per thread (entries
// numbered CTA by CTA in list order, noff): res[e][0..17] the cotangents of
// the panel's centre, normal and four vertices, res[e][18..20] the normal
// cotangent of the D term.
__global__ void __launch_bounds__(128, 2)
k_adj_near(const double* __restrict__ geom, int64_t n, uint32_t mask, int direct, const double* __restrict__ WS,
           const double* __restrict__ WD, const unsigned short* __restrict__ ncode,
           const int64_t* __restrict__ noff, int64_t ncta, int rb, double* __restrict__ res)
{
    const int64_t total = noff[ncta];
    const bool wrt_first = !direct;
    const double sg = wrt_first ? -1.0 : 1.0, sz = wrt_first ? -1.0 : 1.0;
    const uint32_t refl = mask & (MH_GF_RANKINE_REFLECTED | MH_GF_RANKINE_REFLECTED_NEGATIVE);
    const double sgn = (refl == MH_GF_RANKINE_REFLECTED) ? 1.0 : -1.0;
    const double mref[3] = {sgn * sg, sgn * sg, sgn * sg * sz};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = ncta - 1;  // the last CTA whose first entry is <= e
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) >> 1;
            if (noff[mid] <= e) lo = mid;
            else hi = mid - 1;
        }
        const int code = ncode[lo * kNearCap + (e - noff[lo])];
        const int r = code >> 5, bit = code & 31, jj = bit >> 1, term = bit & 1;
        const int64_t ie = (lo % rb) * kAR + r, j = (lo / rb) * kAC + jj;
        Panel p;
        load_panel(geom, n, j, p);
        const double xe[3] = {geom[G_CX * n + ie], geom[G_CY * n + ie], geom[G_CZ * n + ie]};
        double nD[3];
        for (int a = 0; a < 3; ++a) nD[a] = direct ? p.n[a] : geom[(G_NX + a) * n + ie];
        const double ws = WS[j * n + ie], wd = WD[j * n + ie];
        const double f[3] = {term ? mref[0] : sg, term ? mref[1] : sg, term ? mref[2] : sg};
        const double gb[3] = {-kI4P * wd * nD[0] * f[0], -kI4P * wd * nD[1] * f[1], -kI4P * wd * nD[2] * f[2]};
        const double y[3] = {xe[0], xe[1], term ? -xe[2] : xe[2]};
        double out[18], gr[3];
        rankine_pair_vjp(y, p, (term ? sgn : 1.0) * (-kI4P * ws), gb, out, gr);
        for (int k = 0; k < 18; ++k) res[e * kNearF + k] = out[k];
        for (int a = 0; a < 3; ++a) res[e * kNearF + 18 + a] = -kI4P * wd * f[a] * gr[a];
    }
}

// Each CTA (grid as k_adj_rankine) adds its near-field entries to its row
// and column partials in list order: every row sums its own contiguous
// segment of the row-major list (nrow), and every (column, field) sum has a
// thread that walks the column's entries through the column-order index
// (ccode: column, row, term), so no thread scans the whole list.  Each sum
// runs in the same order as a walk of the row-major list would.
constexpr int kNearColF = 18;  // column fields: centre 3, normal 3, vertices 12
__global__ void __launch_bounds__(kAR)
k_adj_near_accum(int64_t n, int direct, const unsigned short* __restrict__ ncode,
                 const unsigned short* __restrict__ ccode, const int* __restrict__ nrow,
                 const int* __restrict__ ncol, const int64_t* __restrict__ noff, const double* __restrict__ resg,
                 double* __restrict__ rowpart, double* __restrict__ colpart)
{
    __shared__ int cstart[kAC + 1];
    const int tid = threadIdx.x;
    const int64_t cta = (int64_t)blockIdx.y * gridDim.x + blockIdx.x;
    const int64_t base = noff[cta];
    if (noff[cta + 1] == base) return;
    const int64_t i = (int64_t)blockIdx.x * kAR + tid;
    const int64_t j0 = (int64_t)blockIdx.y * kAC;
    if (tid == 0) {
        cstart[0] = 0;
        for (int jj = 0; jj < kAC; ++jj) cstart[jj + 1] = cstart[jj] + ncol[cta * kAC + jj];
    }
    // rows: y-bar = -(c-bar + sum of vertex bars), mirrored back for the image
    {
        double xb[3] = {0.0, 0.0, 0.0}, nbi[3] = {0.0, 0.0, 0.0};
        const int e1 = nrow[cta * (kAR + 1) + tid + 1];
        for (int e = nrow[cta * (kAR + 1) + tid]; e < e1; ++e) {
            const int term = ncode[cta * kNearCap + e] & 1;
            const double* q = resg + (base + e) * kNearF;
            double yb[3];
            for (int a = 0; a < 3; ++a) yb[a] = -(q[a] + q[6 + a] + q[9 + a] + q[12 + a] + q[15 + a]);
            xb[0] += yb[0];
            xb[1] += yb[1];
            xb[2] += term ? -yb[2] : yb[2];
            if (!direct)
                for (int a = 0; a < 3; ++a) nbi[a] += q[18 + a];
        }
        if (i < n) {
            for (int c = 0; c < 3; ++c) {
                rowpart[((int64_t)blockIdx.y * kRowF + c) * n + i] += xb[c];
                rowpart[((int64_t)blockIdx.y * kRowF + 3 + c) * n + i] += nbi[c];
            }
        }
    }
    __syncthreads();
    // columns: centre, normal (+ the D term's normal cotangent when direct), vertices
    for (int task = tid; task < kAC * kNearColF; task += blockDim.x) {
        const int jj = task / kNearColF, f = task % kNearColF;
        if (j0 + jj >= n) continue;
        double sum = 0.0;
        for (int k = cstart[jj]; k < cstart[jj + 1]; ++k) {
            const double* q = resg + (base + ccode[cta * kNearCap + k]) * kNearF;
            sum += (f >= 3 && f < 6) ? q[f] + (direct ? q[15 + f] : 0.0) : q[f];
        }
        const int gf = f < 3 ? GB_C + f : f < 6 ? GB_N + (f - 3) : GB_V + (f - 6);
        colpart[((int64_t)blockIdx.x * GB_NF + gf) * n + j0 + jj] += sum;
    }
}

// gbar[f][i] += sum over row partials (fields 0..kRowF), then += sum over
// column partials (fields 0..colF), each in a fixed order; field f =
// blockIdx.y (launch max(kRowF, colF) of them), so every (panel, field) sum
// has its own thread.
__global__ void k_adj_reduce(int64_t n, const double* __restrict__ rowpart, int nrow, const double* __restrict__ colpart,
                             int ncol, int colF, double* __restrict__ gbar)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int f = (int)blockIdx.y;
    if (i >= n) return;
    if (f < kRowF) {
        double s = 0.0;
        for (int p = 0; p < nrow; ++p) s += rowpart[((int64_t)p * kRowF + f) * n + i];
        gbar[(int64_t)f * n + i] += s;
    }
    if (f < colF) {
        double s = 0.0;
        for (int p = 0; p < ncol; ++p) s += colpart[((int64_t)p * colF + f) * n + i];
        gbar[(int64_t)f * n + i] += s;
    }
}

// out[z] += sum_p part[z][p] (one CTA per z, fixed-order tree).
__global__ void __launch_bounds__(256) k_sum_parts(const double* __restrict__ part, int64_t P, double* __restrict__ out)
{
    __shared__ double red[256];
    const int z = blockIdx.x;
    double s = 0.0;
    for (int64_t p = threadIdx.x; p < P; p += blockDim.x) s += part[(int64_t)z * P + p];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[z] += red[0];
}

// ---------------------------------------------------------------------------
// O(n) terms: forces, Froude-Krylov, boundary conditions
// ---------------------------------------------------------------------------

// The frequency loops of k_adj_forces and k_adj_bc run in chunks of zper
// frequencies (blockIdx.y), so a launch has nblk(n) x chunks CTAs instead of
// nblk(n).  Each chunk stores its per-panel sums as lin_fields(ndof) rows
// of cpart[chunk][field][n] (field: centre 0-2, normal 3-5, area 6, then
// dof d component c at 7 + 3 d + c); k_adj_lin_reduce adds the chunks in
// order into gbar and dofbar.
__host__ __device__ inline int lin_fields(int ndof) { return 7 + 3 * ndof; }

__device__ __forceinline__ void lin_chunk_store(double* __restrict__ cpart, int64_t n, int64_t i, int ndof,
                                                const double* gc, const double* gn, double ga,
                                                const double (*zb)[3])
{
    double* p = cpart + (int64_t)blockIdx.y * lin_fields(ndof) * n + i;
    for (int c = 0; c < 3; ++c) {
        p[c * n] = gc[c];
        p[(3 + c) * n] = gn[c];
    }
    p[6 * n] = ga;
    for (int d = 0; d < ndof; ++d)
        for (int c = 0; c < 3; ++c) p[(7 + 3 * d + c) * n] = zb[d][c];
}

__global__ void __launch_bounds__(256)
k_adj_lin_reduce(const double* __restrict__ cpart, int nchunk, int ndof, int64_t n, double* __restrict__ gbar,
                 double* __restrict__ dofbar)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int F = lin_fields(ndof);
    for (int f = 0; f < F; ++f) {
        double s = 0.0;
        for (int c = 0; c < nchunk; ++c) s += cpart[((int64_t)c * F + f) * n + i];
        double* dst = f < 3 ? gbar + (GB_C + f) * n : f < 6 ? gbar + (GB_N + f - 3) * n
                    : f == 6 ? gbar + GB_A * n : dofbar + (int64_t)(f - 7) * n;
        dst[i] += s;
    }
}

// Reverse of the force sums (src/waves.jl:72-85, 157-163) for the nb
// frequencies of a chunk; thread = panel.  CF[z][q][d]: complex cotangent of
// F_dq; CK[z][b][d]: of the Froude-Krylov force.  Writes phi-bar
// PB[z][q][n] and accumulates panel and dof cotangents; kpart[z][block]
// gets the k cotangents of the incident pressure.
__global__ void __launch_bounds__(256)
k_adj_forces(const double* __restrict__ geom, int64_t n, const double* __restrict__ dofs, int ndof,
             const double* __restrict__ betas, int nbeta, const double* __restrict__ omegas, int nb,
             double rho, double gacc, const double2* __restrict__ PHI, const double2* __restrict__ CF,
             const double2* __restrict__ CK, double2* __restrict__ PB, int zper, double* __restrict__ cpart,
             double* __restrict__ kpart)
{
    __shared__ double red[8];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const int64_t ii = live ? i : 0;
    const int nrhs = ndof + nbeta;
    const double x = geom[G_CX * n + ii], y = geom[G_CY * n + ii], zc = geom[G_CZ * n + ii];
    const double nx = geom[G_NX * n + ii], ny = geom[G_NY * n + ii], nz = geom[G_NZ * n + ii];
    const double a = geom[G_AREA * n + ii];
    double gc[3] = {0.0, 0.0, 0.0}, gn[3] = {0.0, 0.0, 0.0}, ga = 0.0;
    double zb[kMaxRhs][3];
    double nzd[kMaxRhs], md[kMaxRhs];
    for (int d = 0; d < ndof; ++d) {
        const double* dd = dofs + (int64_t)d * 3 * n;
        zb[d][0] = zb[d][1] = zb[d][2] = 0.0;
        nzd[d] = nx * dd[ii] + ny * dd[n + ii] + nz * dd[2 * n + ii];
        md[d] = -nzd[d] * a;
    }
    const int zlo = (int)blockIdx.y * zper, zhi = min(nb, zlo + zper);
    for (int z = zlo; z < zhi; ++z) {
        const double w = omegas[z], k = w * w / gacc;
        const double2* cf = CF + (int64_t)z * nrhs * ndof;
        double mb[kMaxRhs];
        for (int d = 0; d < ndof; ++d) mb[d] = 0.0;
        for (int q = 0; q < nrhs; ++q) {
            double ar = 0.0, ai = 0.0;
            for (int d = 0; d < ndof; ++d) {
                ar += md[d] * cf[q * ndof + d].x;
                ai += md[d] * cf[q * ndof + d].y;
            }
            const double2 ph = PHI[((int64_t)z * nrhs + q) * n + ii];
            if (live) PB[((int64_t)z * nrhs + q) * n + i] = make_double2(rho * w * ai, -rho * w * ar);
            // m-bar_d += Re(conj(c) i rho w phi) = -rho w Im(conj(c) phi)
            for (int d = 0; d < ndof; ++d) {
                const double2 c = cf[q * ndof + d];
                mb[d] -= rho * w * (c.x * ph.y - c.y * ph.x);
            }
        }
        double kb = 0.0;
        for (int b = 0; b < nbeta; ++b) {
            double sb, cb, sw, cw;
            sincos(betas[b], &sb, &cb);
            const double wv = x * cb + y * sb;
            sincos(k * wv, &sw, &cw);
            const double m = rho * gacc * exp(k * zc);
            const double pr = m * cw, pi = m * sw;
            const double2* ck = CK + ((int64_t)z * nbeta + b) * ndof;
            double pbr = 0.0, pbi = 0.0;
            for (int d = 0; d < ndof; ++d) {
                mb[d] += ck[d].x * pr + ck[d].y * pi;
                pbr += ck[d].x * md[d];
                pbi += ck[d].y * md[d];
            }
            // cpp = conj(p-bar) p
            const double cr = pbr * pr + pbi * pi, ci = pbr * pi - pbi * pr;
            gc[2] += cr * k;
            gc[0] -= ci * k * cb;
            gc[1] -= ci * k * sb;
            kb += cr * zc - ci * wv;
        }
        for (int d = 0; d < ndof; ++d) {
            const double* dd = dofs + (int64_t)d * 3 * n;
            const double zeta[3] = {dd[ii], dd[n + ii], dd[2 * n + ii]};
            gn[0] -= mb[d] * zeta[0] * a;
            gn[1] -= mb[d] * zeta[1] * a;
            gn[2] -= mb[d] * zeta[2] * a;
            ga -= mb[d] * nzd[d];
            zb[d][0] -= mb[d] * nx * a;
            zb[d][1] -= mb[d] * ny * a;
            zb[d][2] -= mb[d] * nz * a;
        }
        const double s = block_sum(live ? kb : 0.0, red);
        if (threadIdx.x == 0) kpart[(int64_t)z * gridDim.x + blockIdx.x] = s;
    }
    if (!live) return;
    lin_chunk_store(cpart, n, i, ndof, gc, gn, ga, zb);
}

// Reverse of the boundary conditions (src/waves.jl:89-101, 121-142) for
// b-bar BB[z][q][n]: radiation -i w (n . dof_q); diffraction
// -(g k / w) e^{k z} e^{i k (x cos b + y sin b)} (n_x cos b + n_y sin b - i n_z).
// kpart/wpart[z][block]: k and explicit omega cotangents.
__global__ void __launch_bounds__(256)
k_adj_bc(const double* __restrict__ geom, int64_t n, const double* __restrict__ dofs, int ndof,
         const double* __restrict__ betas, int nbeta, const double* __restrict__ omegas, int nb, double gacc,
         const double2* __restrict__ BB, int zper, double* __restrict__ cpart, double* __restrict__ kpart,
         double* __restrict__ wpart)
{
    __shared__ double red[8];
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const int64_t ii = live ? i : 0;
    const int nrhs = ndof + nbeta;
    const double x = geom[G_CX * n + ii], y = geom[G_CY * n + ii], zc = geom[G_CZ * n + ii];
    const double nv[3] = {geom[G_NX * n + ii], geom[G_NY * n + ii], geom[G_NZ * n + ii]};
    double gc[3] = {0.0, 0.0, 0.0}, gn[3] = {0.0, 0.0, 0.0};
    double zb[kMaxRhs][3];
    for (int q = 0; q < ndof; ++q) zb[q][0] = zb[q][1] = zb[q][2] = 0.0;
    const int zlo = (int)blockIdx.y * zper, zhi = min(nb, zlo + zper);
    for (int z = zlo; z < zhi; ++z) {
        const double w = omegas[z], k = w * w / gacc;
        double kb = 0.0, wb = 0.0;
        for (int q = 0; q < ndof; ++q) {
            const double* dd = dofs + (int64_t)q * 3 * n;
            const double zeta[3] = {dd[ii], dd[n + ii], dd[2 * n + ii]};
            const double s = -BB[((int64_t)z * nrhs + q) * n + ii].y;  // Re(conj(b-bar) (-i))
            for (int c = 0; c < 3; ++c) {
                gn[c] += w * s * zeta[c];
                zb[q][c] += w * s * nv[c];
            }
            wb += s * (nv[0] * zeta[0] + nv[1] * zeta[1] + nv[2] * zeta[2]);
        }
        const double f = gacc * k / w, ez = exp(k * zc);
        for (int b = 0; b < nbeta; ++b) {
            double sb, cb, sw, cw;
            sincos(betas[b], &sb, &cb);
            const double wv = x * cb + y * sb;
            sincos(k * wv, &sw, &cw);
            const cplx E = mk(f * ez * cw, f * ez * sw);
            const cplx h = mk(nv[0] * cb + nv[1] * sb, -nv[2]);
            const cplx bv = -(E * h);
            const double2 bbar = BB[((int64_t)z * nrhs + ndof + b) * n + ii];
            const cplx cbb = mk(bbar.x, -bbar.y);  // conj(b-bar)
            const cplx cb_ = cbb * bv;
            gc[2] += cb_.re * k;
            gc[0] -= cb_.im * k * cb;
            gc[1] -= cb_.im * k * sb;
            kb += cb_.re * zc - cb_.im * wv + cb_.re / k;
            wb -= cb_.re / w;
            const cplx Ep = cbb * (-E);
            gn[0] += Ep.re * cb;
            gn[1] += Ep.re * sb;
            gn[2] += Ep.im;
        }
        double s = block_sum(live ? kb : 0.0, red);
        if (threadIdx.x == 0) kpart[(int64_t)z * gridDim.x + blockIdx.x] = s;
        s = block_sum(live ? wb : 0.0, red);
        if (threadIdx.x == 0) wpart[(int64_t)z * gridDim.x + blockIdx.x] = s;
    }
    if (!live) return;
    lin_chunk_store(cpart, n, i, ndof, gc, gn, 0.0, zb);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// C = alpha A^H B + beta C for nb strided n x n by n x nrhs products.
int zgemm_ct_strided(mh_ctx* ctx, int64_t n, int nrhs, const double2* A, const double2* B, double2* C, int nb,
                     double alpha_re, double beta_re)
{
    const cuDoubleComplex alpha = make_cuDoubleComplex(alpha_re, 0.0);
    const cuDoubleComplex beta = make_cuDoubleComplex(beta_re, 0.0);
    cublasStatus_t st = cublasZgemmStridedBatched(
        ctx->cublas, CUBLAS_OP_C, CUBLAS_OP_N, (int)n, nrhs, (int)n, &alpha, (const cuDoubleComplex*)A,
        (int)n, n * n, (const cuDoubleComplex*)B, (int)n, n * nrhs, &beta, (cuDoubleComplex*)C, (int)n,
        n * nrhs, nb);
    if (st != CUBLAS_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cublasZgemmStridedBatched (conjugate transpose) failed (%d)", (int)st);
    return MH_OK;
}

// out[k][i] = in[k][i].x, out[K + k][i] = in[k][i].y: K complex columns of
// length n as 2K real ones.
__global__ void k_split_re_im(const double2* __restrict__ in, int64_t n, int64_t K, double* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * K) return;
    const double2 v = in[t];
    out[t] = v.x;
    out[n * K + t] = v.y;
}

// W += alpha Re(U V^H) = alpha (Re U Re V^T + Im U Im V^T), U and V n x K
// complex, W n x n real: one real product over the stacked 2K columns (half
// the flops and half the output of the complex product, whose imaginary
// part the contraction does not use).
int dgemm_outer_re(mh_ctx* ctx, int64_t n, int64_t K, const double2* U, const double2* V, double* W,
                   double alpha)
{
    auto* U2 = (double*)ws_get(ctx, WS_REPACK, sizeof(double) * 4 * (size_t)n * K);
    if (!U2) return MH_ERR_OOM;
    double* V2 = U2 + 2 * n * K;
    const unsigned g = (unsigned)((n * K + 255) / 256);
    k_split_re_im<<<g, 256, 0, ctx->stream>>>(U, n, K, U2);
    k_split_re_im<<<g, 256, 0, ctx->stream>>>(V, n, K, V2);
    ctx->launches += 2;
    const double beta = 1.0;
    cublasStatus_t st = cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_T, (int)n, (int)n, (int)(2 * K), &alpha,
                                    U2, (int)n, V2, (int)n, &beta, W, (int)n);
    if (st != CUBLAS_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cublasDgemm (outer product) failed (%d)", (int)st);
    return MH_OK;
}

// Device state of one vjp call.
struct Vjp {
    double* gbar;    // [GB_NF][n]
    double* dofbar;  // [ndof][3][n]
    double* kbar;    // [nomega]
    double* wbar;    // [nomega] explicit omega cotangent
    double* WS;      // n x n, real part of the sum over frequencies of S-bar (Rankine contraction)
    double* WD;
    double2* CF;     // [nomega][nrhs][ndof]
    double2* CK;     // [nomega][nbeta][ndof]
    double* part;    // partial sums
    size_t part_words;
    double2* tape;   // forward (G, G_r) per pair and frequency of the chunk, or null
    bool rankine;
    int wave_kinds[2];
    int nwave;
};

constexpr int kLinChunks = 16;  // frequency chunks of k_adj_forces / k_adj_bc

size_t part_words_needed(int64_t n, int nb)
{
    const int64_t rb = nblk(n, std::min(kAR, kAW)), cb = nblk(n, kAC);
    const size_t pairs = (size_t)cb * kRowF * n + (size_t)rb * GB_NF * n + (size_t)nb * rb * cb;
    const size_t lin = (size_t)2 * nb * nblk(n, 256) + (size_t)kLinChunks * lin_fields(kMaxRhs) * n;
    return std::max(pairs, lin);
}

// Contraction of the pair kernels for the vectors of nb frequencies.
int contract_pairs_wave(const Batch& bt, Vjp& vj, const double* d_k, int nb, int z0, const double* tab,
                        const double2* VA, const double2* VB, const double2* VC, const double2* VD)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const unsigned cb = nblk(n, kAC);
    phase_begin(ctx, PH_ADJ_WAVE);
    for (int w = 0; w < vj.nwave; ++w) {
        const int kind = vj.wave_kinds[w];
        const bool use_tape = kind == 2 && vj.tape;
        const bool allw = !use_tape && kind == 2 && tab && nb >= kAdjAllwMinFreqs;
        const unsigned nrb = allw ? nblk(n, kAW) : nblk(n, kAR);
        const unsigned ncb = cb;
        double* rowpart = vj.part;
        double* colpart = rowpart + (size_t)ncb * kRowF * n;
        double* kpart = colpart + (size_t)nrb * kWaveF * n;
        if (use_tape) {
            if (bt.nrhs < 1 || bt.nrhs > kMaxRhs) return MH_ERR_ARG;  // the VB/VD ring holds kMaxRhs at most
            auto* kern = bt.nrhs == 1   ? k_adj_delh_tape<1>
                         : bt.nrhs == 2 ? k_adj_delh_tape<2>
                         : bt.nrhs == 3 ? k_adj_delh_tape<3>
                                        : k_adj_delh_tape<0>;
            const size_t smem = bt.nrhs == 1   ? tape_smem<1>(nb)
                                : bt.nrhs == 2 ? tape_smem<2>(nb)
                                : bt.nrhs == 3 ? tape_smem<3>(nb)
                                               : tape_smem<0>(nb);
            MH_CUDA_TRY(ctx, raise_smem_cap((const void*)kern, smem));
            kern<<<dim3(nrb, cb), kAR, smem, ctx->stream>>>(bt.m->geom, n, bt.direct, vj.tape, d_k, nb, bt.nrhs, VA,
                                                            VB, VC, VD, rowpart, colpart, kpart);
        } else if (allw) {
            const size_t smem = adj_allw_smem(nb);
            MH_CUDA_TRY(ctx, raise_smem_cap((const void*)k_adj_delh_allw, smem));
            k_adj_delh_allw<<<dim3(nrb, ncb), kAW, smem, ctx->stream>>>(bt.m->geom, n, bt.direct, tab, d_k, nb,
                                                                        bt.nrhs, VA, VB, VC, VD, rowpart, colpart,
                                                                        kpart);
        } else {
            const size_t smem = sizeof(double) * (kAR / 32) * nb;
            k_adj_wave<<<dim3(nrb, cb), kAR, smem, ctx->stream>>>(kind, bt.m->geom, n, bt.direct,
                                                                 kind == 2 ? tab : nullptr, d_k, nb, bt.nrhs,
                                                                 VA, VB, VC, VD, rowpart, colpart, kpart);
        }
        const dim3 gr(nblk(n, 256), std::max(kRowF, kWaveF));
        k_adj_reduce<<<gr, 256, 0, ctx->stream>>>(n, rowpart, (int)ncb, colpart, (int)nrb, kWaveF, vj.gbar);
        k_sum_parts<<<nb, 256, 0, ctx->stream>>>(kpart, (int64_t)nrb * ncb, vj.kbar + z0);
        ctx->launches += 3;
        MH_CUDA_TRY(ctx, cudaGetLastError());
    }
    phase_end(ctx, PH_ADJ_WAVE);
    return MH_OK;
}

// Everything after the adjoint solve for nb frequencies: Rankine sums,
// wave contraction, boundary-condition reverse.
int adjoint_tail(const Batch& bt, Vjp& vj, const double* d_omegas, const double* d_k, int nb, int z0,
                 const double* tab, const double2* VA, const double2* VB, const double2* VC,
                 const double2* VD, const double2* BB)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    int rc;
    if (vj.rankine) {
        phase_begin(ctx, PH_ADJ_RANKINE);
        const int64_t K = (int64_t)nb * bt.nrhs;
        if ((rc = dgemm_outer_re(ctx, n, K, VA, VB, vj.WS, 1.0))) return rc;
        if ((rc = dgemm_outer_re(ctx, n, K, VC, VD, vj.WD, -1.0))) return rc;
        phase_end(ctx, PH_ADJ_RANKINE);
    }
    if ((rc = contract_pairs_wave(bt, vj, d_k, nb, z0, tab, VA, VB, VC, VD))) return rc;
    phase_begin(ctx, PH_ADJ_LINEAR);
    const unsigned lb = nblk(n, 256);
    double* kpart = vj.part;
    double* wpart = kpart + (size_t)nb * lb;
    double* cpart = wpart + (size_t)nb * lb;
    const int zper = (nb + kLinChunks - 1) / kLinChunks, nch = (nb + zper - 1) / zper;
    k_adj_bc<<<dim3(lb, nch), 256, 0, ctx->stream>>>(bt.m->geom, n, bt.d_dofs, bt.ndof, bt.d_betas, bt.nbeta,
                                                     d_omegas, nb, bt.g, BB, zper, cpart, kpart, wpart);
    k_adj_lin_reduce<<<lb, 256, 0, ctx->stream>>>(cpart, nch, bt.ndof, n, vj.gbar, vj.dofbar);
    k_sum_parts<<<nb, 256, 0, ctx->stream>>>(kpart, lb, vj.kbar + z0);
    k_sum_parts<<<nb, 256, 0, ctx->stream>>>(wpart, lb, vj.wbar + z0);
    ctx->launches += 4;
    phase_end(ctx, PH_ADJ_LINEAR);
    MH_CUDA_TRY(ctx, cudaGetLastError());
    return MH_OK;
}

int seed_forces(const Batch& bt, Vjp& vj, const double* d_omegas, int nb, int z0, const double2* PHI,
                double2* PB)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const unsigned lb = nblk(n, 256);
    double* kpart = vj.part;
    double* cpart = kpart + (size_t)2 * nb * lb;
    const int zper = (nb + kLinChunks - 1) / kLinChunks, nch = (nb + zper - 1) / zper;
    phase_begin(ctx, PH_ADJ_LINEAR);
    k_adj_forces<<<dim3(lb, nch), 256, 0, ctx->stream>>>(bt.m->geom, n, bt.d_dofs, bt.ndof, bt.d_betas,
                                                         bt.nbeta, d_omegas, nb, bt.rho, bt.g, PHI,
                                                         vj.CF + (int64_t)z0 * bt.nrhs * bt.ndof,
                                                         vj.CK + (int64_t)z0 * bt.nbeta * bt.ndof, PB, zper,
                                                         cpart, kpart);
    k_adj_lin_reduce<<<lb, 256, 0, ctx->stream>>>(cpart, nch, bt.ndof, n, vj.gbar, vj.dofbar);
    k_sum_parts<<<nb, 256, 0, ctx->stream>>>(kpart, lb, vj.kbar + z0);
    ctx->launches += 3;
    phase_end(ctx, PH_ADJ_LINEAR);
    MH_CUDA_TRY(ctx, cudaGetLastError());
    return MH_OK;
}

// Mixed adjoint of one chunk: the forward state of run_mixed_chunk is in
// the workspace.  Solves D^H x = rhs with the low-precision factors and FP64
// refinement; problems that left the mixed path in the forward solve, or
// whose adjoint refinement does not converge, use FP64 factors.
int adjoint_mixed_chunk(const Batch& bt, Vjp& vj, const double* d_omegas, const double* d_k, int nb, int z0,
                        double tol, int max_iter, FallbackStore& fb, mh_batch_info* info)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const int nrhs = bt.nrhs;
    const int64_t nv = n * nrhs, cnt = nv * nb;
    auto* S64 = (double2*)ctx->ws[WS_S];
    auto* D64 = (double2*)ctx->ws[WS_D];
    auto* Dlo = (float2*)ctx->ws[WS_LO];
    auto* Dinv = (float2*)ctx->ws[WS_DINV];
    auto* BC = (double2*)ctx->ws[WS_RHS];
    auto* X = (double2*)ctx->ws[WS_PHI];
    auto* PHIi = (double2*)ctx->ws[WS_TMP];  // phi = S sigma (indirect)
    auto* adj = (double2*)ws_get(ctx, WS_ADJ, sizeof(double2) * cnt * 5);
    auto* R32 = (float2*)ws_get(ctx, WS_TMP32, sizeof(float2) * cnt);
    auto* misc = ws_get(ctx, WS_MISC, refine_ctl_bytes(nb) + 64);
    if (!adj || !R32 || !misc) return MH_ERR_OOM;
    double2* PB = adj;
    double2* LAM = adj + cnt;
    double2* BB = adj + 2 * cnt;
    double2* RHS = adj + 3 * cnt;
    double2* R = adj + 4 * cnt;
    int rc;
    const double* tab = delh_table_for(ctx, bt.mask, &rc);
    if (rc) return rc;
    if ((rc = seed_forces(bt, vj, d_omegas, nb, z0, bt.direct ? X : PHIi, PB))) return rc;
    phase_begin(ctx, PH_ADJ_SOLVE);
    if (bt.direct) {
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(RHS, PB, sizeof(double2) * cnt, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        MH_CUDA_TRY(ctx, launch_gemv(ctx, true, S64, n, nb, PB, nullptr, RHS, nrhs, 1.0, 0.0));
    }
    // D^H lam = RHS: low-precision factors + FP64 refinement, FP64 fallback
    if ((rc = mixed_refine_solve(ctx, n, nb, nrhs, D64, Dlo, Dinv, RHS, LAM, R, R32, misc, true, tol, max_iter,
                                 fb, info)))
        return rc;
    if (bt.direct) MH_CUDA_TRY(ctx, launch_gemv(ctx, true, S64, n, nb, LAM, nullptr, BB, nrhs, 1.0, 0.0));
    phase_end(ctx, PH_ADJ_SOLVE);
    if (bt.direct) return adjoint_tail(bt, vj, d_omegas, d_k, nb, z0, tab, LAM, BC, LAM, X, BB);
    return adjoint_tail(bt, vj, d_omegas, d_k, nb, z0, tab, PB, X, LAM, X, LAM);
}

// Adjoint of one chunk of the batched FP64 path: the forward state of
// run_fp64_chunk is in the workspace; D^H lam = rhs with its pivoted FP64
// factors (cuSOLVER zgetrs, conjugate transpose), then the same tail as the
// mixed adjoint.
int adjoint_fp64_batched_chunk(const Batch& bt, Vjp& vj, const double* d_omegas, const double* d_k, int nb,
                               int z0)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const int nrhs = bt.nrhs;
    const int64_t nv = n * nrhs, cnt = nv * nb;
    auto* S64 = (double2*)ctx->ws[WS_S];
    auto* BC = (double2*)ctx->ws[WS_RHS];
    auto* X = (double2*)ctx->ws[WS_PHI];
    auto* PHIi = (double2*)ctx->ws[WS_TMP];  // phi = S sigma (indirect)
    auto* adj = (double2*)ws_get(ctx, WS_ADJ, sizeof(double2) * cnt * 5);
    if (!adj) return MH_ERR_OOM;
    double2* PB = adj;
    double2* LAM = adj + cnt;
    double2* BB = adj + 2 * cnt;
    int rc;
    const double* tab = delh_table_for(ctx, bt.mask, &rc);
    if (rc) return rc;
    if ((rc = seed_forces(bt, vj, d_omegas, nb, z0, bt.direct ? X : PHIi, PB))) return rc;
    phase_begin(ctx, PH_ADJ_SOLVE);
    if (bt.direct) {
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(LAM, PB, sizeof(double2) * cnt, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        MH_CUDA_TRY(ctx, launch_gemv(ctx, true, S64, n, nb, PB, nullptr, LAM, nrhs, 1.0, 0.0));
    }
    if ((rc = fp64_batched_getrs(ctx, true, n, nb, nrhs, LAM))) return rc;
    if (bt.direct) MH_CUDA_TRY(ctx, launch_gemv(ctx, true, S64, n, nb, LAM, nullptr, BB, nrhs, 1.0, 0.0));
    phase_end(ctx, PH_ADJ_SOLVE);
    if (bt.direct) return adjoint_tail(bt, vj, d_omegas, d_k, nb, z0, tab, LAM, BC, LAM, X, BB);
    return adjoint_tail(bt, vj, d_omegas, d_k, nb, z0, tab, PB, X, LAM, X, LAM);
}

// FP64 forward + adjoint of one frequency (pivoted cuSOLVER LU, kept for
// the conjugate-transposed solve).
int fp64_vjp_one(const Batch& bt, Vjp& vj, const double* d_omega, const double* d_k, double k, int z,
                 double2* d_F, double2* d_FK)
{
    mh_ctx* ctx = bt.ctx;
    const int64_t n = bt.n;
    const int nrhs = bt.nrhs;
    const int64_t nv = n * nrhs;
    const size_t mat = sizeof(double2) * (size_t)n * (size_t)n;
    auto* S = (double2*)ws_get(ctx, WS_S, mat);
    auto* D = (double2*)ws_get(ctx, WS_D, mat);
    auto* BC = (double2*)ws_get(ctx, WS_RHS, sizeof(double2) * nv);
    auto* X = (double2*)ws_get(ctx, WS_PHI, sizeof(double2) * nv);
    auto* piv = (int*)ws_get(ctx, WS_PIV, sizeof(int) * (size_t)n);
    auto* adj = (double2*)ws_get(ctx, WS_ADJ, sizeof(double2) * nv * 5);
    if (!S || !D || !BC || !X || !piv || !adj) return MH_ERR_OOM;
    double2* PB = adj;
    double2* LAM = adj + nv;
    double2* BB = adj + 2 * nv;
    double2* PHI = adj + 3 * nv;
    int rc;
    const double* tab = delh_table_for(ctx, bt.mask, &rc);
    if (rc) return rc;
    phase_begin(ctx, PH_FP64_ASSEMBLY);
    MH_CUDA_TRY(ctx, launch_assemble_f64(ctx, bt.m, k, bt.mask, bt.direct, tab, S, D));
    phase_end(ctx, PH_FP64_ASSEMBLY);
    MH_CUDA_TRY(ctx, launch_bc_batch(bt, d_omega, 1, BC));
    phase_begin(ctx, PH_FP64_LU);
    if ((rc = fp64_lu_factor(ctx, n, D, piv))) return rc;
    if (bt.direct) {
        if ((rc = zgemm_strided(ctx, n, nrhs, S, BC, X, 1, 1.0, 0.0))) return rc;
        if ((rc = fp64_getrs(ctx, false, n, D, piv, X, nrhs))) return rc;
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(PHI, X, sizeof(double2) * nv, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(X, BC, sizeof(double2) * nv, cudaMemcpyDeviceToDevice, ctx->stream));
        if ((rc = fp64_getrs(ctx, false, n, D, piv, X, nrhs))) return rc;
        if ((rc = zgemm_strided(ctx, n, nrhs, S, X, PHI, 1, 1.0, 0.0))) return rc;
    }
    phase_end(ctx, PH_FP64_LU);
    MH_CUDA_TRY(ctx, launch_forces_batch(bt, d_omega, 1, PHI, d_F, d_FK));
    if ((rc = seed_forces(bt, vj, d_omega, 1, z, PHI, PB))) return rc;
    phase_begin(ctx, PH_ADJ_SOLVE);
    if (bt.direct) {
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(LAM, PB, sizeof(double2) * nv, cudaMemcpyDeviceToDevice, ctx->stream));
    } else if ((rc = zgemm_ct_strided(ctx, n, nrhs, S, PB, LAM, 1, 1.0, 0.0))) {
        return rc;
    }
    if ((rc = fp64_getrs(ctx, true, n, D, piv, LAM, nrhs))) return rc;
    if (bt.direct && (rc = zgemm_ct_strided(ctx, n, nrhs, S, LAM, BB, 1, 1.0, 0.0))) return rc;
    phase_end(ctx, PH_ADJ_SOLVE);
    if (bt.direct) return adjoint_tail(bt, vj, d_omega, d_k, 1, z, tab, LAM, BC, LAM, X, BB);
    return adjoint_tail(bt, vj, d_omega, d_k, 1, z, tab, PB, X, LAM, X, LAM);
}

}  // namespace

int hydro_batch_vjp(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                    const double* dofs, int64_t nbeta, const double* betas, double rho, double g,
                    uint32_t mask, int direct, int precision, double tol, int max_iter,
                    const double* bar_added_mass, const double* bar_damping, const double* bar_diffraction,
                    const double* bar_froude_krylov, double* added_mass, double* damping,
                    double* diffraction, double* froude_krylov, double* d_vertices, double* d_centers,
                    double* d_normals, double* d_areas, double* d_radii, double* d_omegas_out,
                    double* d_dofs_out, mh_batch_info* info)
{
    const int64_t n = m->n;
    const int nrhs = (int)(ndof + nbeta);
    mh_batch_info local{};
    // ---- inputs and cotangents to the device ----
    const size_t dof_bytes = sizeof(double) * 3 * (size_t)n * (size_t)ndof;
    const size_t in_bytes = dof_bytes + sizeof(double) * (size_t)(2 * nomega + nbeta) + 64;
    auto* in = (char*)ws_get(ctx, WS_DOF, in_bytes);
    const size_t out_count = (size_t)nomega * (size_t)(nrhs * ndof + nbeta * ndof);
    auto* d_out = (double2*)ws_get(ctx, WS_OUT, sizeof(double2) * out_count * 2 + 16);
    const size_t gb_words = (size_t)GB_NF * n + 3 * (size_t)n * ndof + 2 * (size_t)nomega;
    auto* gb = (double*)ws_get(ctx, WS_GBAR, sizeof(double) * gb_words);
    if (!in || !d_out || !gb) return MH_ERR_OOM;
    auto* d_dofs = (double*)in;
    auto* d_om = (double*)(in + dof_bytes);
    auto* d_k = d_om + nomega;
    auto* d_betas = d_k + nomega;
    std::vector<double> hk(nomega);
    for (int64_t z = 0; z < nomega; ++z) hk[z] = omegas[z] * omegas[z] / g;
    if (ndof) MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_dofs, dofs, dof_bytes, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_om, omegas, sizeof(double) * nomega, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_k, hk.data(), sizeof(double) * nomega, cudaMemcpyHostToDevice, ctx->stream));
    if (nbeta)
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_betas, betas, sizeof(double) * nbeta, cudaMemcpyHostToDevice,
                                         ctx->stream));
    // complex force cotangents: c = A-bar / w^2 + i B-bar / w (radiation), F-bar (diffraction)
    std::vector<double2> hcf((size_t)nomega * nrhs * ndof), hck((size_t)nomega * nbeta * ndof);
    for (int64_t z = 0; z < nomega; ++z) {
        const double w = omegas[z];
        for (int64_t q = 0; q < ndof; ++q)
            for (int64_t i = 0; i < ndof; ++i) {
                const size_t o = (size_t)i + (size_t)ndof * ((size_t)q + (size_t)ndof * (size_t)z);
                const double ab = bar_added_mass ? bar_added_mass[o] : 0.0;
                const double bb = bar_damping ? bar_damping[o] : 0.0;
                hcf[((size_t)z * nrhs + q) * ndof + i] = make_double2(ab / (w * w), bb / w);
            }
        for (int64_t b = 0; b < nbeta; ++b)
            for (int64_t i = 0; i < ndof; ++i) {
                const size_t o = (size_t)i + (size_t)ndof * ((size_t)z + (size_t)nomega * (size_t)b);
                hcf[((size_t)z * nrhs + ndof + b) * ndof + i] =
                    bar_diffraction ? make_double2(bar_diffraction[2 * o], bar_diffraction[2 * o + 1])
                                    : make_double2(0.0, 0.0);
                hck[((size_t)z * nbeta + b) * ndof + i] =
                    bar_froude_krylov ? make_double2(bar_froude_krylov[2 * o], bar_froude_krylov[2 * o + 1])
                                      : make_double2(0.0, 0.0);
            }
    }
    double2* d_F = d_out;
    double2* d_FK = d_out + (size_t)nomega * nrhs * ndof;
    double2* d_CF = d_out + out_count;
    double2* d_CK = d_CF + (size_t)nomega * nrhs * ndof;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_CF, hcf.data(), sizeof(double2) * hcf.size(), cudaMemcpyHostToDevice,
                                     ctx->stream));
    if (!hck.empty())
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(d_CK, hck.data(), sizeof(double2) * hck.size(), cudaMemcpyHostToDevice,
                                         ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(gb, 0, sizeof(double) * gb_words, ctx->stream));
    Vjp vj{};
    vj.gbar = gb;
    vj.dofbar = gb + (size_t)GB_NF * n;
    vj.kbar = vj.dofbar + 3 * (size_t)n * ndof;
    vj.wbar = vj.kbar + nomega;
    vj.CF = d_CF;
    vj.CK = d_CK;
    vj.rankine = (mask & (MH_GF_RANKINE | MH_GF_RANKINE_REFLECTED | MH_GF_RANKINE_REFLECTED_NEGATIVE)) != 0;
    vj.nwave = 0;
    if (mask & MH_GF_WU) vj.wave_kinds[vj.nwave++] = 1;
    if (mask & MH_GF_DELHOMMEAU) vj.wave_kinds[vj.nwave++] = 2;
    const size_t nn = (size_t)n * (size_t)n;
    if (vj.rankine) {
        vj.WS = (double*)ws_get(ctx, WS_WSD, sizeof(double) * nn * 2);
        if (!vj.WS) return MH_ERR_OOM;
        vj.WD = vj.WS + nn;
        MH_CUDA_TRY(ctx, cudaMemsetAsync(vj.WS, 0, sizeof(double) * nn * 2, ctx->stream));
    }
    Batch bt{ctx, m, n, (int)ndof, (int)nbeta, nrhs, d_dofs, d_betas, rho, g, mask, direct};
    int rc = MH_OK;
    if (precision == MH_PRECISION_FP64) {
        vj.part_words = part_words_needed(n, 1);
        vj.part = (double*)ws_get(ctx, WS_PART, sizeof(double) * vj.part_words);
        if (!vj.part) return MH_ERR_OOM;
        for (int64_t z = 0; z < nomega && rc == MH_OK; ++z)
            rc = fp64_vjp_one(bt, vj, d_om + z, d_k + z, hk[z], (int)z, d_F + z * nrhs * ndof,
                              d_FK + z * nbeta * ndof);
    } else {
        auto* SR = (double*)ws_get(ctx, WS_SR, sizeof(double) * nn * 2);
        if (!SR) return MH_ERR_OOM;
        double* DR = SR + nn;
        if ((rc = rankine_real(bt, SR, DR))) return rc;
        // the Delhommeau table term keeps a tape of (G, G_r) per pair and frequency
        int trc = MH_OK;
        const bool tape = (mask & MH_GF_DELHOMMEAU) && delh_table_for(ctx, mask, &trc) != nullptr;
        if (trc) return trc;
        const size_t per = nn * (2 * sizeof(double2) + sizeof(float2) + (tape ? 2 * sizeof(double2) : 0)) +
                           (size_t)n * nrhs * (10 * sizeof(double2) + 2 * sizeof(float2));
        constexpr size_t kVjpBatchBytes = 32ull << 30;
        const int64_t fit = std::min<int64_t>(1024, (int64_t)(kVjpBatchBytes / per));
        const int chunk = (int)std::max<int64_t>(1, std::min<int64_t>(nomega, fit));
        vj.part_words = part_words_needed(n, chunk);
        vj.part = (double*)ws_get(ctx, WS_PART, sizeof(double) * vj.part_words);
        if (!vj.part) return MH_ERR_OOM;
        if (tape) {
            vj.tape = (double2*)ws_get(ctx, WS_TAPE, sizeof(double2) * 2 * nn * (size_t)chunk);
            if (!vj.tape) return MH_ERR_OOM;
            bt.tape = vj.tape;
        }
        FallbackStore fb;
        for (int64_t z0 = 0; z0 < nomega && rc == MH_OK; z0 += chunk) {
            const int nb = (int)std::min<int64_t>(chunk, nomega - z0);
            fb.lu = nullptr;
            fb.piv = nullptr;
            fb.used.assign(nb, 0);
            if (precision == MH_PRECISION_FP64_BATCHED) {
                rc = run_fp64_chunk(bt, d_om + z0, d_k + z0, nb, SR, DR, d_F + z0 * nrhs * ndof,
                                    d_FK + z0 * nbeta * ndof);
                if (rc == MH_OK) rc = adjoint_fp64_batched_chunk(bt, vj, d_om + z0, d_k + z0, nb, (int)z0);
                continue;
            }
            rc = run_mixed_chunk(bt, d_om + z0, d_k + z0, nb, SR, DR, tol, max_iter, d_F + z0 * nrhs * ndof,
                                 d_FK + z0 * nbeta * ndof, &local, &fb);
            if (rc == MH_OK)
                rc = adjoint_mixed_chunk(bt, vj, d_om + z0, d_k + z0, nb, (int)z0, tol, max_iter, fb, &local);
        }
    }
    if (rc) return rc;
    if (vj.rankine) {
        phase_begin(ctx, PH_ADJ_RANKINE);
        const unsigned rb = nblk(n, kAR), cb = nblk(n, kAC);
        double* rowpart = vj.part;
        double* colpart = rowpart + (size_t)cb * kRowF * n;
        const int64_t ncta = (int64_t)rb * cb;
        auto* nbuf = (char*)ws_get(ctx, WS_NEAR, sizeof(int64_t) * (ncta + 1) +
                                                     sizeof(int) * ncta * (1 + (kAR + 1) + kAC) +
                                                     2 * sizeof(unsigned short) * kNearCap * ncta);
        if (!nbuf) return MH_ERR_OOM;
        auto* noff = (int64_t*)nbuf;
        auto* ncount = (int*)(noff + ncta + 1);
        auto* nrow = ncount + ncta;                           // [cta][kAR + 1] row offsets
        auto* ncol = nrow + ncta * (kAR + 1);                 // [cta][kAC] entries per column
        auto* ncode = (unsigned short*)(ncol + ncta * kAC);   // [cta][kNearCap] row-major list
        auto* ccode = ncode + ncta * kNearCap;                // [cta][kNearCap] column-order index
        k_adj_rankine<<<dim3(rb, cb), kAR, 0, ctx->stream>>>(m->geom, n, mask, direct, vj.WS, vj.WD, rowpart,
                                                             colpart, ncode, ncount, nrow, ncol, ccode);
        k_near_scan<<<1, 1024, 0, ctx->stream>>>(ncount, ncta, noff);
        ctx->launches += 2;
        int64_t total = 0;
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(&total, noff + ncta, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                         ctx->stream));
        MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
        if (total > 0) {
            auto* nres = (double*)ws_get(ctx, WS_NEARRES, sizeof(double) * kNearF * (size_t)total);
            if (!nres) return MH_ERR_OOM;
            const unsigned gn = (unsigned)std::min<int64_t>((total + 127) / 128, 148 * 64);
            k_adj_near<<<gn, 128, 0, ctx->stream>>>(m->geom, n, mask, direct, vj.WS, vj.WD, ncode, noff, ncta,
                                                    (int)rb, nres);
            k_adj_near_accum<<<dim3(rb, cb), kAR, 0, ctx->stream>>>(n, direct, ncode, ccode, nrow, ncol, noff,
                                                                    nres, rowpart, colpart);
            ctx->launches += 2;
        }
        const dim3 gr(nblk(n, 256), std::max(kRowF, (int)GB_NF));
        k_adj_reduce<<<gr, 256, 0, ctx->stream>>>(n, rowpart, (int)cb, colpart, (int)rb, GB_NF, vj.gbar);
        ctx->launches += 1;
        phase_end(ctx, PH_ADJ_RANKINE);
        MH_CUDA_TRY(ctx, cudaGetLastError());
    }
    phase_collect(ctx);
    // ---- results to the host ----
    std::vector<double2> h(out_count);
    std::vector<double> hg(gb_words);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h.data(), d_out, sizeof(double2) * out_count, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(hg.data(), gb, sizeof(double) * gb_words, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    unpack_outputs(h.data(), nomega, omegas, ndof, nbeta, added_mass, damping, diffraction, froude_krylov);
    const double* G = hg.data();
    if (d_centers)
        for (int c = 0; c < 3; ++c)
            for (int64_t i = 0; i < n; ++i) d_centers[c * n + i] = G[(GB_C + c) * n + i];
    if (d_normals)
        for (int c = 0; c < 3; ++c)
            for (int64_t i = 0; i < n; ++i) d_normals[c * n + i] = G[(GB_N + c) * n + i];
    if (d_areas)
        for (int64_t i = 0; i < n; ++i) d_areas[i] = G[GB_A * n + i];
    if (d_radii)
        for (int64_t i = 0; i < n; ++i) d_radii[i] = 0.0;  // radii only select branches
    if (d_vertices) {
        const int64_t nvtx = m->nv;
        std::fill(d_vertices, d_vertices + 3 * nvtx, 0.0);
        for (int64_t i = 0; i < n; ++i)
            for (int a = 0; a < 4; ++a) {
                const int64_t v = m->faces[(size_t)a * n + i];
                for (int c = 0; c < 3; ++c) d_vertices[c * nvtx + v] += G[(GB_V + 3 * a + c) * n + i];
            }
    }
    if (d_dofs_out)
        for (int64_t t = 0; t < 3 * n * ndof; ++t) d_dofs_out[t] = G[GB_NF * n + t];
    if (d_omegas_out) {
        const double* kb = G + (size_t)GB_NF * n + 3 * (size_t)n * ndof;
        const double* wb = kb + nomega;
        for (int64_t z = 0; z < nomega; ++z) {
            const double w = omegas[z];
            double s = wb[z] + kb[z] * 2.0 * w / g;
            // explicit omega of the outputs: A = Re F / w^2, B = Im F / w, F = i rho w sum(...)
            for (int64_t q = 0; q < nrhs; ++q)
                for (int64_t i = 0; i < ndof; ++i) {
                    const double2 F = h[((size_t)z * nrhs + q) * ndof + i];
                    const double2 c = hcf[((size_t)z * nrhs + q) * ndof + i];
                    s += (c.x * F.x + c.y * F.y) / w;
                    if (q < ndof) {
                        const size_t o = (size_t)i + (size_t)ndof * ((size_t)q + (size_t)ndof * (size_t)z);
                        const double ab = bar_added_mass ? bar_added_mass[o] : 0.0;
                        const double bb = bar_damping ? bar_damping[o] : 0.0;
                        s += ab * (-2.0 * F.x / (w * w * w)) + bb * (-F.y / (w * w));
                    }
                }
            d_omegas_out[z] = s;
        }
    }
    if (info) *info = local;
    return MH_OK;
}

}  // namespace mh
