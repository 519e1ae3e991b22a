// FP64 kernels: influence-matrix assembly, boundary conditions and the
// pressure -> force reduction.
//
// Assembly (src/matrix_assembly.jl:4-42): one CTA owns a tile of 128
// collocation rows x 16 source columns.  The 16 source panels are staged in
// shared memory (20 doubles each: centre, normal, area, radius, 4 vertices)
// and broadcast to all threads; each thread keeps its collocation point in
// registers and walks the 16 columns.  For a fixed column the 128 threads
// write 128 consecutive complex128 entries of the column-major matrix, so every
// store is a fully coalesced 2 KiB run.
#include <cuda_runtime.h>

#include "mh_device.cuh"
#include "mh_internal.h"

namespace mh {

namespace {

constexpr int kRows = 128;
constexpr int kCols = 16;
constexpr double kInv4Pi = 1.0 / (4.0 * kPi);  // -1/(2 tau), tau = 2 pi (MarineHydro.jl:11)

__device__ __forceinline__ void load_panel_field(Panel& p, int f, double v)
{
    // geometry field order -> Panel layout
    if (f < 3) p.c[f] = v;
    else if (f < 6) p.n[f - 3] = v;
    else if (f == G_AREA) p.area = v;
    else if (f == G_RADIUS) p.radius = v;
    else p.v[f - G_V] = v;
}

__global__ void __launch_bounds__(kRows)
k_assemble_f64(const double* __restrict__ geom, int64_t n, double k, uint32_t mask, int direct,
               const double* __restrict__ tab, double2* __restrict__ S, double2* __restrict__ D)
{
    __shared__ Panel sp[kCols];
    const int64_t j0 = (int64_t)blockIdx.y * kCols;
    for (int t = threadIdx.x; t < kCols * G_NFIELDS; t += blockDim.x) {
        int f = t / kCols, jj = t % kCols;
        int64_t j = j0 + jj;
        double v = (j < n) ? geom[(int64_t)f * n + j] : 0.0;
        load_panel_field(sp[jj], f, v);
    }
    __syncthreads();
    const int64_t i = (int64_t)blockIdx.x * kRows + threadIdx.x;
    if (i >= n) return;
    const double x[3] = {geom[G_CX * n + i], geom[G_CY * n + i], geom[G_CZ * n + i]};
    const double ni[3] = {geom[G_NX * n + i], geom[G_NY * n + i], geom[G_NZ * n + i]};
    const bool wrt_first = !direct;
    const int jend = (int)min((int64_t)kCols, n - j0);
    for (int jj = 0; jj < jend; ++jj) {
        const Panel& p = sp[jj];
        const int64_t j = j0 + jj;
        cplx s, g[3];
        pair_integrals(x, p, k, mask, wrt_first, tab, s, g);
        const int64_t o = j * n + i;
        if (S) S[o] = make_double2(-kInv4Pi * s.re, -kInv4Pi * s.im);
        if (D) {
            const double* nn = direct ? p.n : ni;
            double dre = nn[0] * g[0].re + nn[1] * g[1].re + nn[2] * g[2].re;
            double dim = nn[0] * g[0].im + nn[1] * g[1].im + nn[2] * g[2].im;
            D[o] = make_double2((i == j ? 0.5 : 0.0) - kInv4Pi * dre, -kInv4Pi * dim);
        }
    }
}

__device__ __forceinline__ void dof_at(const double* dof, int64_t dof_rows, int64_t n, int64_t i,
                                       double d[3])
{
    if (dof_rows == 1) {
        d[0] = dof[0];
        d[1] = dof[1];
        d[2] = dof[2];
    } else {
        d[0] = dof[i];
        d[1] = dof[n + i];
        d[2] = dof[2 * n + i];
    }
}

// src/waves.jl:4-18, :89-101
__global__ void k_radiation_bc(const double* __restrict__ geom, int64_t n,
                               const double* __restrict__ dof, int64_t dof_rows, double omega,
                               double2* __restrict__ bc)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d[3];
    dof_at(dof, dof_rows, n, i, d);
    double nd = geom[G_NX * n + i] * d[0] + geom[G_NY * n + i] * d[1] + geom[G_NZ * n + i] * d[2];
    bc[i] = make_double2(0.0, -omega * nd);  // -i omega (n . dof)
}

// src/waves.jl:121-142: v = (g k / omega) e^{i k wbar} (cos b e^{kz}, sin b e^{kz}, -i e^{kz})
__global__ void k_airy_bc(const double* __restrict__ geom, int64_t n, double omega, double beta,
                          double gacc, double2* __restrict__ bc)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double k = omega * omega / gacc;
    double cb, sb;
    sincos(beta, &sb, &cb);
    double x = geom[G_CX * n + i], y = geom[G_CY * n + i], z = geom[G_CZ * n + i];
    double wbar = x * cb + y * sb;
    double cih = exp(k * z);
    double sw, cw;
    sincos(k * wbar, &sw, &cw);
    double f = gacc * k / omega;
    cplx e = mk(f * cw, f * sw);
    cplx v0 = e * (cb * cih), v1 = e * (sb * cih), v2 = e * mk(0.0, -cih);
    double nx = geom[G_NX * n + i], ny = geom[G_NY * n + i], nz = geom[G_NZ * n + i];
    cplx vn = v0 * nx + v1 * ny + v2 * nz;
    bc[i] = make_double2(-vn.re, -vn.im);
}

// src/waves.jl:21-25 with p = i rho omega phi (src/waves.jl:34, :56).
// One CTA; a fixed-order tree reduction, so the result is deterministic.
__global__ void __launch_bounds__(1024)
k_force(const double* __restrict__ geom, int64_t n, const double2* __restrict__ phi,
        const double* __restrict__ dof, int64_t dof_rows, double rho, double omega,
        double2* __restrict__ F_out)
{
    __shared__ double sr[1024], si[1024];
    double ar = 0.0, ai = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        double d[3];
        dof_at(dof, dof_rows, n, i, d);
        double amp = -(geom[G_NX * n + i] * d[0] + geom[G_NY * n + i] * d[1] +
                       geom[G_NZ * n + i] * d[2]);
        double w = amp * geom[G_AREA * n + i];
        double2 ph = phi[i];
        // i rho omega phi = rho omega (-phi.im, phi.re)
        ar += rho * omega * (-ph.y) * w;
        ai += rho * omega * (ph.x) * w;
    }
    sr[threadIdx.x] = ar;
    si[threadIdx.x] = ai;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sr[threadIdx.x] += sr[threadIdx.x + s];
            si[threadIdx.x] += si[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) F_out[0] = make_double2(sr[0], si[0]);
}

}  // namespace

cudaError_t launch_assemble_f64(mh_ctx* ctx, const mh_mesh* m, double k, uint32_t mask, int direct,
                                const double* tab, double2* S, double2* D)
{
    const int64_t n = m->n;
    dim3 grid((unsigned)((n + kRows - 1) / kRows), (unsigned)((n + kCols - 1) / kCols));
    k_assemble_f64<<<grid, kRows, 0, ctx->stream>>>(m->geom, n, k, mask, direct, tab, S, D);
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_radiation_bc(mh_ctx* ctx, const mh_mesh* m, const double* dof, int64_t dof_rows,
                                double omega, double2* bc)
{
    const int64_t n = m->n;
    k_radiation_bc<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(m->geom, n, dof, dof_rows,
                                                                         omega, bc);
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_airy_bc(mh_ctx* ctx, const mh_mesh* m, double omega, double beta, double g,
                           double2* bc)
{
    const int64_t n = m->n;
    k_airy_bc<<<(unsigned)((n + 255) / 256), 256, 0, ctx->stream>>>(m->geom, n, omega, beta, g, bc);
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_force(mh_ctx* ctx, const mh_mesh* m, const double2* phi, const double* dof,
                         int64_t dof_rows, double rho, double omega, double2* F_out)
{
    k_force<<<1, 1024, 0, ctx->stream>>>(m->geom, m->n, phi, dof, dof_rows, rho, omega, F_out);
    ctx->launches += 1;
    return cudaGetLastError();
}


}  // namespace mh
