// Batched pivot-free blocked LU and triangular solves in complex FP32.
//
// The low-precision half of the mixed-precision solve: the LU is a
// preconditioner for FP64 iterative refinement, so it only needs to be a
// good approximation of the FP64 matrix.  The BEM matrices D (direct) and K
// (indirect) are well conditioned (kappa ~ 2-3 on the hemisphere meshes) and
// LAPACK's partial pivoting leaves their rows in place, so the factorisation
// runs without row exchanges; a zero or non-finite pivot sets a per-matrix
// flag and the host re-solves that problem with the pivoted FP64 LU.
//
// Layout: B matrices, each n x n column-major float2 (re, im), `stride`
// elements apart.  Right-looking blocked algorithm, block size NB:
//   k_lu_diag    factor the NB x NB diagonal block in shared memory;
//   k_lu_trsm    L21 = A21 U11^-1 (one thread per row) and
//                U12 = L11^-1 A12 (one thread per column);
//   k_lu_update  A22 -= L21 U12 (64 x 64 output tile per CTA).
#include <cuda_runtime.h>

#include "mh_internal.h"
#include "mh_lu_kernels.cuh"

namespace mh {
namespace {

constexpr int NB = 32;

// A22 -= L21 U12 over rows/cols [k0+NB, n); 64 x 64 tile per CTA, 256 threads,
// 4 x 4 complex outputs per thread.
__global__ void __launch_bounds__(256)
k_lu_update(float2* __restrict__ A, int64_t n, int64_t stride, int64_t k0)
{
    __shared__ float2 sL[NB][64 + 1];  // sL[k][row]
    __shared__ float2 sU[NB][64 + 1];  // sU[k][col]
    float2* M = A + (int64_t)blockIdx.z * stride;
    const int64_t base = k0 + NB;
    const int64_t r0 = base + (int64_t)blockIdx.x * 64;
    const int64_t c0 = base + (int64_t)blockIdx.y * 64;
    for (int t = threadIdx.x; t < NB * 64; t += blockDim.x) {
        int rr = t % 64, k = t / 64;
        int64_t gr = r0 + rr;
        sL[k][rr] = (gr < n) ? M[(k0 + k) * n + gr] : make_float2(0.f, 0.f);
        int cc = t / NB, kk = t % NB;
        int64_t gc = c0 + cc;
        sU[kk][cc] = (gc < n) ? M[gc * n + k0 + kk] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int tr = threadIdx.x % 16, tc = threadIdx.x / 16;
    float2 acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = make_float2(0.f, 0.f);
#pragma unroll 8
    for (int k = 0; k < NB; ++k) {
        float2 l[4], u[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) l[a] = sL[k][tr + 16 * a];
#pragma unroll
        for (int c = 0; c < 4; ++c) u[c] = sU[k][tc + 16 * c];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                acc[a][c].x = fmaf(l[a].x, u[c].x, fmaf(-l[a].y, u[c].y, acc[a][c].x));
                acc[a][c].y = fmaf(l[a].x, u[c].y, fmaf(l[a].y, u[c].x, acc[a][c].y));
            }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        int64_t gc = c0 + tc + 16 * c;
        if (gc >= n) continue;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            int64_t gr = r0 + tr + 16 * a;
            if (gr < n) {
                float2 v = M[gc * n + gr];
                M[gc * n + gr] = csubf(v, acc[a][c]);
            }
        }
    }
}

// Solve (L U) X = B in place for X (n x nrhs float2 per matrix, column-major,
// ld n), one CTA per matrix, all right-hand sides together so the factors
// are read once.  Blocks of NB rows: the diagonal block is applied through
// its stored inverse, the rows below (forward) or above (backward) are
// updated in parallel.
template <int MAXRHS>
__global__ void __launch_bounds__(256)
k_lu_solve(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
           int64_t dstride, float2* __restrict__ X, int64_t xstride, int nrhs)
{
    const int b = blockIdx.x;
    const float2* M = A + (int64_t)b * stride;
    const float2* inv = Dinv + (int64_t)b * dstride;
    float2* x = X + (int64_t)b * xstride;
    __shared__ float2 xs[MAXRHS][NB];
    const int nblk = (int)((n + NB - 1) / NB);
    // forward: L y = b
    for (int blk = 0; blk < nblk; ++blk) {
        const int64_t k0 = (int64_t)blk * NB;
        const int kb = (int)min((int64_t)NB, n - k0);
        const float2* Li = inv + (int64_t)blk * 2 * NB * NB;
        for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
            int r = t % NB, q = t / NB;
            float2 acc = make_float2(0.f, 0.f);
            if (r < kb)
                for (int c = 0; c <= r; ++c) {
                    float2 v = x[(int64_t)q * n + k0 + c];
                    float2 l = Li[c * NB + r];
                    acc.x += l.x * v.x - l.y * v.y;
                    acc.y += l.x * v.y + l.y * v.x;
                }
            xs[q][r] = acc;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
            int r = t % kb, q = t / kb;
            x[(int64_t)q * n + k0 + r] = xs[q][r];
        }
        for (int64_t i = k0 + kb + threadIdx.x; i < n; i += blockDim.x) {
            float2 acc[MAXRHS];
            for (int q = 0; q < nrhs; ++q) acc[q] = x[(int64_t)q * n + i];
            for (int t = 0; t < kb; ++t) {
                float2 l = M[(k0 + t) * n + i];
                for (int q = 0; q < nrhs; ++q) acc[q] = cfms(acc[q], l, xs[q][t]);
            }
            for (int q = 0; q < nrhs; ++q) x[(int64_t)q * n + i] = acc[q];
        }
        __syncthreads();
    }
    // backward: U x = y
    for (int blk = nblk - 1; blk >= 0; --blk) {
        const int64_t k0 = (int64_t)blk * NB;
        const int kb = (int)min((int64_t)NB, n - k0);
        const float2* Ui = inv + (int64_t)blk * 2 * NB * NB + NB * NB;
        for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
            int r = t % NB, q = t / NB;
            float2 acc = make_float2(0.f, 0.f);
            if (r < kb)
                for (int c = r; c < kb; ++c) {
                    float2 v = x[(int64_t)q * n + k0 + c];
                    float2 u = Ui[c * NB + r];
                    acc.x += u.x * v.x - u.y * v.y;
                    acc.y += u.x * v.y + u.y * v.x;
                }
            xs[q][r] = acc;
        }
        __syncthreads();
        for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
            int r = t % kb, q = t / kb;
            x[(int64_t)q * n + k0 + r] = xs[q][r];
        }
        for (int64_t i = threadIdx.x; i < k0; i += blockDim.x) {
            float2 acc[MAXRHS];
            for (int q = 0; q < nrhs; ++q) acc[q] = x[(int64_t)q * n + i];
            for (int t = 0; t < kb; ++t) {
                float2 u = M[(k0 + t) * n + i];
                for (int q = 0; q < nrhs; ++q) acc[q] = cfms(acc[q], u, xs[q][t]);
            }
            for (int q = 0; q < nrhs; ++q) x[(int64_t)q * n + i] = acc[q];
        }
        __syncthreads();
    }
}

}  // namespace

int64_t lu_dinv_stride(int64_t n) { return ((n + NB - 1) / NB) * 2 * NB * NB; }

cudaError_t launch_lu_f32(mh_ctx* ctx, float2* A, int64_t n, int64_t stride, int nbatch,
                          float2* Dinv, int* bad)
{
    const int64_t dstride = lu_dinv_stride(n);
    for (int64_t k0 = 0; k0 < n; k0 += NB) {
        k_lu_diag<NB><<<nbatch, 256, lu_diag_smem_bytes<NB>(), ctx->stream>>>(A, n, stride, k0, Dinv,
                                                                               dstride, bad);
        ctx->launches += 1;
        const int64_t rest = n - k0 - NB;
        if (rest > 0) {
            dim3 g1((unsigned)((rest + 127) / 128), 2, (unsigned)nbatch);
            k_lu_trsm<NB><<<g1, 128, 0, ctx->stream>>>(A, n, stride, k0);
            dim3 g2((unsigned)((rest + 63) / 64), (unsigned)((rest + 63) / 64), (unsigned)nbatch);
            k_lu_update<<<g2, 256, 0, ctx->stream>>>(A, n, stride, k0);
            ctx->launches += 2;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_lu_solve_f32(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                                const float2* Dinv, float2* X, int64_t xstride, int nrhs)
{
    if (nrhs > kMaxRhs) return cudaErrorInvalidValue;
    k_lu_solve<kMaxRhs><<<nbatch, 256, 0, ctx->stream>>>(A, n, stride, Dinv, lu_dinv_stride(n), X,
                                                         xstride, nrhs);
    ctx->launches += 1;
    return cudaGetLastError();
}

}  // namespace mh
