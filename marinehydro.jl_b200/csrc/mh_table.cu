// Construction of the tabulated Guevel-Delhommeau wave term (see mh_table.cuh)
// and the point-evaluation hook mh_wave_term.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "mh_internal.h"
#include "mh_device.cuh"

namespace mh {
namespace {

// B and C at the table nodes, from the FP64 adaptive quadrature.
__global__ void k_table_nodes(const double* __restrict__ rr, const double* __restrict__ zz, int n,
                              double* __restrict__ B, double* __restrict__ C,
                              double* __restrict__ E0, double* __restrict__ E1)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double r = rr[t], z = zz[t];
    cplx o[3];
    delh_dimless(r, z, o);
    double az = -z, R = hypot(r, z);
    double e = exp(z), J0 = j0(r), J1 = j1(r);
    double L = log(0.5 * (R + az));
    B[t] = o[0].re + 2.0 * e * J0 * L;
    C[t] = o[1].re - (2.0 * e * J1 * L - 2.0 * e * J0 * r / (R * (R + az)));
    E0[t] = e * J0;
    E1[t] = e * J1;
}

// Dimensionless (G, dG/dr, dG/dz) at arbitrary points.
__global__ void k_wave_term(const double* __restrict__ tab, uint32_t which, int64_t n,
                            const double* __restrict__ rr, const double* __restrict__ zz,
                            double* __restrict__ out)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    cplx o[3];
    if (which == MH_GF_WU) wu_dimless(rr[t], zz[t], o);
    else if (tab) delh_dimless_table(tab, rr[t], zz[t], o);
    else delh_dimless(rr[t], zz[t], o);
    for (int q = 0; q < 3; ++q) {
        out[6 * t + 2 * q] = o[q].re;
        out[6 * t + 2 * q + 1] = o[q].im;
    }
}

void cheb_nodes(int n, double a, double b, std::vector<double>& x)
{
    x.resize(n);
    for (int k = 0; k < n; ++k)
        x[k] = 0.5 * (a + b) + 0.5 * (b - a) * std::cos(M_PI * (k + 0.5) / n);
}

// Chebyshev coefficients of an n x n block of node values (row = first coord).
void cheb_coeffs(int n, const double* vals, double* coef)
{
    std::vector<double> T((size_t)n * n), tmp((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
            T[i * n + k] = (i == 0 ? 1.0 : 2.0) / n * std::cos(M_PI * i * (k + 0.5) / n);
    for (int i = 0; i < n; ++i)
        for (int l = 0; l < n; ++l) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += T[i * n + k] * vals[k * n + l];
            tmp[i * n + l] = s;
        }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            double s = 0.0;
            for (int l = 0; l < n; ++l) s += tmp[i * n + l] * T[j * n + l];
            coef[i * n + j] = s;
        }
}

}  // namespace

int ensure_delh_table(mh_ctx* ctx)
{
    if (ctx->delh_table) return MH_OK;
    // node coordinates: polar patch, then cells
    std::vector<double> r, z;
    std::vector<double> xa, xb;
    cheb_nodes(kTabNP, 0.0, kTabRPolar, xa);
    cheb_nodes(kTabNP, 0.0, 0.5 * M_PI, xb);
    for (int k = 0; k < kTabNP; ++k)
        for (int l = 0; l < kTabNP; ++l) {
            r.push_back(xa[k] * std::sin(xb[l]));
            z.push_back(-xa[k] * std::cos(xb[l]));
        }
    for (int iz = 0; iz < kTabNCell; ++iz)
        for (int ir = 0; ir < kTabNCell; ++ir) {
            cheb_nodes(kTabNC, ir * kTabH, (ir + 1) * kTabH, xa);
            cheb_nodes(kTabNC, iz * kTabH, (iz + 1) * kTabH, xb);
            for (int k = 0; k < kTabNC; ++k)
                for (int l = 0; l < kTabNC; ++l) {
                    r.push_back(xa[k]);
                    z.push_back(-xb[l]);
                }
        }
    const int n = (int)r.size();
    double *d_r = nullptr, *d_z = nullptr, *d_B = nullptr, *d_C = nullptr, *d_E0 = nullptr,
           *d_E1 = nullptr, *d_tab = nullptr;
    auto cleanup = [&]() {
        cudaFree(d_r);
        cudaFree(d_z);
        cudaFree(d_B);
        cudaFree(d_C);
        cudaFree(d_E0);
        cudaFree(d_E1);
    };
    size_t bytes = sizeof(double) * (size_t)n;
    if (cudaMalloc(&d_r, bytes) != cudaSuccess || cudaMalloc(&d_z, bytes) != cudaSuccess ||
        cudaMalloc(&d_B, bytes) != cudaSuccess || cudaMalloc(&d_C, bytes) != cudaSuccess ||
        cudaMalloc(&d_E0, bytes) != cudaSuccess || cudaMalloc(&d_E1, bytes) != cudaSuccess ||
        cudaMalloc(&d_tab, sizeof(double) * kTabWords) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        cudaFree(d_tab);
        return set_err(ctx, MH_ERR_OOM, "allocation of the Delhommeau table failed");
    }
    std::vector<double> hB(n), hC(n), hE0(n), hE1(n), tab(kTabWords);
    cudaError_t e = cudaMemcpyAsync(d_r, r.data(), bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_z, z.data(), bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        k_table_nodes<<<(n + 127) / 128, 128, 0, ctx->stream>>>(d_r, d_z, n, d_B, d_C, d_E0, d_E1);
        ctx->launches += 1;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(hB.data(), d_B, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hC.data(), d_C, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hE0.data(), d_E0, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hE1.data(), d_E1, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cleanup();
        cudaFree(d_tab);
        return set_err(ctx, MH_ERR_CUDA, "Delhommeau table nodes: %s", cudaGetErrorString(e));
    }
    // polar block: B, C, E0, E1, fitted on kTabNP x kTabNP nodes; the first
    // kTabNU rows (degrees in R) are kept, and again with the rows in the
    // monomial basis of u: T_i(u) = sum_m P[i][m] u^m
    {
        std::vector<double> full((size_t)kTabNP * kTabNP);
        std::vector<double> P((size_t)kTabNU * kTabNU, 0.0);  // P[i][m]
        P[0] = 1.0;
        if (kTabNU > 1) P[1 * kTabNU + 1] = 1.0;
        for (int i = 2; i < kTabNU; ++i)  // T_i = 2 u T_{i-1} - T_{i-2}
            for (int m = 0; m < kTabNU; ++m)
                P[(size_t)i * kTabNU + m] = (m > 0 ? 2.0 * P[(size_t)(i - 1) * kTabNU + m - 1] : 0.0) -
                                            P[(size_t)(i - 2) * kTabNU + m];
        const double* src[4] = {hB.data(), hC.data(), hE0.data(), hE1.data()};
        for (int q = 0; q < 4; ++q) {
            cheb_coeffs(kTabNP, src[q], full.data());
            for (int i = 0; i < kTabNU; ++i)
                for (int j = 0; j < kTabNV; ++j)
                    tab[(size_t)q * kTabPolarFn + i * kTabNV + j] = full[(size_t)i * kTabNP + j];
            for (int m = 0; m < kTabNU; ++m)
                for (int j = 0; j < kTabNV; ++j) {
                    double a = 0.0;
                    for (int i = m; i < kTabNU; ++i) a += P[(size_t)i * kTabNU + m] * full[(size_t)i * kTabNP + j];
                    tab[kTabMonoOff + (size_t)q * kTabPolarFn + m * kTabNV + j] = a;
                }
        }
    }
    // cells
    const int np = kTabNP * kTabNP, nc = kTabNC * kTabNC;
    for (int c = 0; c < kTabNCell * kTabNCell; ++c) {
        double* dst = tab.data() + kTabPolarWords + (size_t)c * kTabCellWords;
        cheb_coeffs(kTabNC, hB.data() + np + (size_t)c * nc, dst);
        cheb_coeffs(kTabNC, hC.data() + np + (size_t)c * nc, dst + nc);
    }
    e = cudaMemcpyAsync(d_tab, tab.data(), sizeof(double) * kTabWords, cudaMemcpyHostToDevice,
                        ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cleanup();
    if (e != cudaSuccess) {
        cudaFree(d_tab);
        return set_err(ctx, MH_ERR_CUDA, "Delhommeau table upload: %s", cudaGetErrorString(e));
    }
    ctx->delh_table = d_tab;
    return MH_OK;
}

const double* delh_table_for(mh_ctx* ctx, uint32_t mask, int* status)
{
    *status = MH_OK;
    if (!(mask & MH_GF_DELHOMMEAU) || ctx->delh_method == MH_DELHOMMEAU_EXACT) return nullptr;
    *status = ensure_delh_table(ctx);
    return ctx->delh_table;
}

cudaError_t launch_wave_term(mh_ctx* ctx, const double* tab, uint32_t which, int64_t n,
                             const double* r, const double* z, double* out)
{
    k_wave_term<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(tab, which, n, r, z, out);
    ctx->launches += 1;
    return cudaGetLastError();
}

}  // namespace mh
