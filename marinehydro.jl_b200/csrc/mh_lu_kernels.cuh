// Shared device code of the batched complex FP32 LU (pivot-free, blocked):
// the diagonal-block factorisation with inverse diagonal blocks and the
// panel triangular solves, templated on the block size NB.
//
// Layout: matrices n x n column-major float2, `stride` elements apart;
// Dinv holds, per matrix and diagonal block, inv(L11) then inv(U11), each
// NB x NB column-major.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mh {
namespace {

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 csubf(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// a - b*c
__device__ __forceinline__ float2 cfms(float2 a, float2 b, float2 c)
{
    return make_float2(a.x - (b.x * c.x - b.y * c.y), a.y - (b.x * c.y + b.y * c.x));
}
__device__ __forceinline__ float2 cdivf(float2 a, float2 b)
{
    float d = b.x * b.x + b.y * b.y;
    return make_float2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// Factor the diagonal block [k0, k0+kb) of every matrix in place, and store
// inv(L11) (unit lower) and inv(U11) in Dinv (per matrix: n/NB blocks of
// 2 x NB x NB, column-major) for the triangular solves.
template <int NB, int THREADS = 256>
__global__ void __launch_bounds__(THREADS)
k_lu_diag(float2* __restrict__ A, int64_t n, int64_t stride, int64_t k0, float2* __restrict__ Dinv,
          int64_t dstride, int* __restrict__ bad)
{
    extern __shared__ float2 lu_diag_smem[];
    auto s = reinterpret_cast<float2 (*)[NB + 1]>(lu_diag_smem);            // s[row][col]
    auto w = reinterpret_cast<float2 (*)[NB + 1]>(lu_diag_smem + NB * (NB + 1));  // inverse
    const int64_t b = blockIdx.x;
    float2* M = A + b * stride;
    const int kb = (int)min((int64_t)NB, n - k0);
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        int r = t % NB, c = t / NB;
        s[r][c] = (r < kb && c < kb) ? M[(k0 + c) * n + k0 + r]
                                     : make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
    for (int c = 0; c < kb; ++c) {
        float2 piv = s[c][c];
        float mag = piv.x * piv.x + piv.y * piv.y;
        if (threadIdx.x == 0 && !(mag > 1e-30f && mag < 3e38f)) atomicExch(bad + b, 1);
        for (int r = c + 1 + threadIdx.x; r < kb; r += blockDim.x) s[r][c] = cdivf(s[r][c], piv);
        __syncthreads();
        int m = kb - c - 1;
        for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
            int r = c + 1 + t % m, q = c + 1 + t / m;
            s[r][q] = cfms(s[r][q], s[r][c], s[c][q]);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < kb * kb; t += blockDim.x) {
        int r = t % kb, c = t / kb;
        M[(k0 + c) * n + k0 + r] = s[r][c];
    }
    float2* out = Dinv + b * dstride + (k0 / NB) * 2 * NB * NB;
    // inv(L11), unit lower: W = I, then for t ascending the rows below t
    // subtract L[r][t] W[t][:] (row t is final at step t); all threads per sweep.
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t % NB, c = t / NB;
        w[r][c] = make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
    for (int t = 0; t + 1 < kb; ++t) {
        const int wdt = t + 1, cnt = (kb - 1 - t) * wdt;
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
            const int r = t + 1 + e / wdt, c = e % wdt;
            w[r][c] = cfms(w[r][c], s[r][t], w[t][c]);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) out[t] = w[t % NB][t / NB];
    __syncthreads();
    // inv(U11): W = I, then for t descending the rows above t subtract
    // U[r][t] / U[t][t] W[t][:], and finally row r is scaled by 1 / U[r][r].
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t % NB, c = t / NB;
        w[r][c] = make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
    if (threadIdx.x < NB) {  // the padding column of w holds 1 / U[r][r]
        const int r = threadIdx.x;
        w[r][NB] = r < kb ? cdivf(make_float2(1.f, 0.f), s[r][r]) : make_float2(1.f, 0.f);
    }
    __syncthreads();
    for (int t = kb - 1; t >= 1; --t) {
        const int wdt = kb - t, cnt = t * wdt;
        const float2 f = w[t][NB];
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
            const int r = e / wdt, c = t + e % wdt;
            w[r][c] = cfms(w[r][c], cmulf(s[r][t], f), w[t][c]);
        }
        __syncthreads();
    }
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        const int r = t % NB, c = t / NB;
        out[NB * NB + t] = (r < kb) ? cmulf(w[r][NB], w[r][c]) : w[r][c];
    }
}

// The B operands of the tensor-core panel TRSMs of a diagonal block, packed
// once here instead of by every TRSM CTA: 128 x 128 FP16 K-major no-swizzle
// images (8-row x 16-byte core matrices), rows R < 64 = [Re v | -Im v],
// rows 64 + R = [Im v | Re v] of the complex row v = column R of inv(U11)
// (image 0, for L21 = A21 inv(U11)) or row R of inv(L11) (image 1, for
// U12^T = A12^T inv(L11)^T).  x holds inv(L) strictly below the diagonal
// (unit diagonal implicit) and inv(U) on and above it.
constexpr int kTrsmBImage = 128 * 128 * 2;  // bytes per image

template <int LD>
__device__ __forceinline__ void pack_trsm_b(const float2 (*x)[LD], unsigned char* img)
{
    for (int e = threadIdx.x; e < 2 * 128 * 16; e += blockDim.x) {
        const int im = e / (128 * 16), R = (e / 16) % 128, cc = e % 16;
        const int r = R & 63, t0 = (cc & 7) * 8;
        float v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int t = t0 + q;
            float2 z;
            if (im == 0) z = t <= r ? x[t][r] : make_float2(0.f, 0.f);  // inv(U)[t][r]
            else z = t == r ? make_float2(1.f, 0.f) : (r > t ? x[r][t] : make_float2(0.f, 0.f));  // inv(L)[r][t]
            const bool im_row = R >= 64, second = cc >= 8;
            v[q] = im_row ? (second ? z.x : z.y) : (second ? -z.y : z.x);
        }
        uint4 w;
        __half2 h0 = __floats2half2_rn(v[0], v[1]), h1 = __floats2half2_rn(v[2], v[3]);
        __half2 h2 = __floats2half2_rn(v[4], v[5]), h3 = __floats2half2_rn(v[6], v[7]);
        w.x = *reinterpret_cast<uint32_t*>(&h0);
        w.y = *reinterpret_cast<uint32_t*>(&h1);
        w.z = *reinterpret_cast<uint32_t*>(&h2);
        w.w = *reinterpret_cast<uint32_t*>(&h3);
        const uint32_t off = (uint32_t)((cc * 16 + R / 8) * 128 + (R % 8) * 16);
        *reinterpret_cast<uint4*>(img + (size_t)im * kTrsmBImage + off) = w;
    }
}

// k_lu_diag for NB = 64, blocked by eight columns in shared memory: for each
// panel P of columns 8P .. 8P+7, (1) one warp factors the panel (rows 8P ..
// 63, two rows per lane, the pivot row passed by warp shuffles: no CTA
// barrier inside the panel), (2) the panel's block row of U right of it is
// solved with the panel's unit-lower 8 x 8 L, one column per thread, (3)
// every thread applies the rank-8 update to its part of the trailing block:
// three barriers per panel, 24 in all instead of one per column.  The
// two triangular inverses are then built by recursive doubling from the
// factored block in shared memory: with the inverses of the diagonal blocks
// A and C of size s known, [A 0; B C]^-1 has the off-diagonal block
// -inv(C) B inv(A) (and [A B; 0 C]^-1 has -inv(A) B inv(C)), two small
// products per level, s = 1, 2, ..., 32: twelve barriers instead of one per
// row.  The block is padded with the identity, so all 64 steps run for any
// kb <= 64 and the padding stays the identity.  Same outputs as k_lu_diag.
constexpr int kDiag64Threads = 512;
// dynamic shared memory: the factored block, the inverses (inv(L) strictly
// below the diagonal, inv(U) on and above), two product buffers
constexpr int kDiagLd = 65;
constexpr size_t kDiag64Smem = sizeof(float2) * (2 * 64 * kDiagLd + 2 * 32 * 32 * 2);

__global__ void __launch_bounds__(kDiag64Threads)
k_lu_diag64(float2* __restrict__ A, int64_t n, int64_t stride, int64_t k0, float2* __restrict__ Dinv,
            int64_t dstride, int* __restrict__ bad, unsigned char* __restrict__ bimg, int64_t bstride)
{
    constexpr int NB = 64;
    extern __shared__ float2 diag_smem[];
    auto f = reinterpret_cast<float2 (*)[kDiagLd]>(diag_smem);                 // factored block
    auto x = reinterpret_cast<float2 (*)[kDiagLd]>(diag_smem + NB * kDiagLd);  // the two inverses
    float2* tl_buf = diag_smem + 2 * NB * kDiagLd;                               // products
    float2* tu_buf = tl_buf + 2 * 32 * 32;
    const int64_t b = blockIdx.x;
    float2* M = A + b * stride;
    const int kb = (int)min((int64_t)NB, n - k0);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    // the block, padded with the identity past kb, column by column (coalesced)
    for (int e = t; e < NB * NB; e += blockDim.x) {
        const int c = e / NB, r = e % NB;
        f[r][c] = (r < kb && c < kb) ? M[(k0 + c) * n + k0 + r] : make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 1
    for (int P = 0; P < NB / 8; ++P) {
        const int p0 = 8 * P;
        // (1) panel: lane l holds rows p0 + l and p0 + l + 32 (when < 64)
        if (warp == 0) {
            const int ra = p0 + lane, rb = ra + 32;
            const bool has_a = ra < NB, has_b = rb < NB;
            float2 va[8], vb[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                va[j] = has_a ? f[ra][p0 + j] : make_float2(0.f, 0.f);
                vb[j] = has_b ? f[rb][p0 + j] : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                // pivot row p0 + c is lane c's first row
                float2 pr[8];
#pragma unroll
                for (int j = c; j < 8; ++j)
                    pr[j] = make_float2(__shfl_sync(0xffffffffu, va[j].x, c), __shfl_sync(0xffffffffu, va[j].y, c));
                const float2 piv = pr[c];
                if (lane == c && p0 + c < kb) {
                    const float mag = piv.x * piv.x + piv.y * piv.y;
                    if (!(mag > 1e-30f && mag < 3e38f)) atomicExch(bad + b, 1);
                }
                // 1 / piv once per step (one division), then products
                const float im2 = 1.f / (piv.x * piv.x + piv.y * piv.y);
                const float2 ip = make_float2(piv.x * im2, -piv.y * im2);
                if (has_a && ra > p0 + c) {
                    const float2 l = make_float2(va[c].x * ip.x - va[c].y * ip.y, va[c].x * ip.y + va[c].y * ip.x);
                    va[c] = l;
#pragma unroll
                    for (int j = c + 1; j < 8; ++j) va[j] = cfms(va[j], l, pr[j]);
                }
                if (has_b) {  // rb >= 32 > p0 + c for every panel with rows past 32
                    const float2 l = make_float2(vb[c].x * ip.x - vb[c].y * ip.y, vb[c].x * ip.y + vb[c].y * ip.x);
                    vb[c] = l;
#pragma unroll
                    for (int j = c + 1; j < 8; ++j) vb[j] = cfms(vb[j], l, pr[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (has_a) f[ra][p0 + j] = va[j];
                if (has_b) f[rb][p0 + j] = vb[j];
            }
        }
        __syncthreads();
        const int q0 = p0 + 8;  // first column (and row) past the panel
        if (q0 >= NB) break;
        // (2) U block row: rows p0 .. p0+7, columns q0 .. 63, by the panel's unit-lower L
        if (t < NB - q0) {
            const int cq = q0 + t;
            float2 u[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) u[i] = f[p0 + i][cq];
#pragma unroll
            for (int i = 1; i < 8; ++i)
#pragma unroll
                for (int k2 = 0; k2 < i; ++k2) u[i] = cfms(u[i], f[p0 + i][p0 + k2], u[k2]);
#pragma unroll
            for (int i = 1; i < 8; ++i) f[p0 + i][cq] = u[i];
        }
        __syncthreads();
        // (3) rank-8 update of rows and columns q0 .. 63: thread t takes row
        // q0 + t / 8 and the columns q0 + t % 8 + 8 j
        {
            const int r = q0 + (t >> 3), g = t & 7;
            if (r < NB) {
                float2 lr[8];
#pragma unroll
                for (int k2 = 0; k2 < 8; ++k2) lr[k2] = f[r][p0 + k2];
                for (int cq = q0 + g; cq < NB; cq += 8) {
                    float2 acc = f[r][cq];
#pragma unroll
                    for (int k2 = 0; k2 < 8; ++k2) acc = cfms(acc, lr[k2], f[p0 + k2][cq]);
                    f[r][cq] = acc;
                }
            }
        }
        __syncthreads();
    }
    // the factors back over the block (coalesced)
    for (int e = t; e < NB * NB; e += blockDim.x) {
        const int c = e / NB, r = e % NB;
        if (r < kb && c < kb) M[(k0 + c) * n + k0 + r] = f[r][c];
    }
    __syncthreads();
    // inverses by recursive doubling; x starts as the inverse diagonal of U
    for (int e = t; e < NB * NB; e += blockDim.x) {
        const int i = e / NB, j = e % NB;
        x[i][j] = i == j ? cdivf(make_float2(1.f, 0.f), f[i][i]) : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 1
    for (int lsz = 0; (1 << lsz) < NB; ++lsz) {  // block size sz = 2^lsz: index arithmetic by shifts
        const int sz = 1 << lsz;
        const int items = (NB / (2 * sz)) * sz * sz;  // outputs per triangle and phase
        // phase 1: -L[C,A] inv(L)[A,A] and -U[A,C] inv(U)[C,C]
        for (int e = t; e < 2 * items; e += blockDim.x) {
            const bool up = e >= items;
            const int ee = up ? e - items : e;
            const int pr = ee >> (2 * lsz), i = (ee >> lsz) & (sz - 1), j = ee & (sz - 1);
            const int a0 = 2 * sz * pr, c0 = a0 + sz;
            float2 acc = make_float2(0.f, 0.f);
            if (!up) {  // row c0 + i, column a0 + j; inv(L) is 1 on the diagonal
                for (int u = j; u < sz; ++u) {
                    const float2 xl = u == j ? make_float2(1.f, 0.f) : x[a0 + u][a0 + j];
                    acc = cfms(acc, f[c0 + i][a0 + u], xl);
                }
                tl_buf[ee] = acc;
            } else {  // row a0 + i, column c0 + j; inv(U)[u][j] for u <= j
                for (int u = 0; u <= j; ++u) acc = cfms(acc, f[a0 + i][c0 + u], x[c0 + u][c0 + j]);
                tu_buf[ee] = acc;
            }
        }
        __syncthreads();
        // phase 2: inv(L)[C,A] = inv(L)[C,C] (phase 1), inv(U)[A,C] = inv(U)[A,A] (phase 1)
        for (int e = t; e < 2 * items; e += blockDim.x) {
            const bool up = e >= items;
            const int ee = up ? e - items : e;
            const int pr = ee >> (2 * lsz), i = (ee >> lsz) & (sz - 1), j = ee & (sz - 1);
            const int a0 = 2 * sz * pr, c0 = a0 + sz;
            const float2* T = (up ? tu_buf : tl_buf) + pr * sz * sz;
            float2 acc = make_float2(0.f, 0.f);
            if (!up) {  // inv(L)[c0+i][c0+u] for u <= i (1 on the diagonal)
                for (int u = 0; u <= i; ++u) {
                    const float2 xl = u == i ? make_float2(1.f, 0.f) : x[c0 + i][c0 + u];
                    const float2 tv = T[u * sz + j];
                    acc.x += xl.x * tv.x - xl.y * tv.y;
                    acc.y += xl.x * tv.y + xl.y * tv.x;
                }
                x[c0 + i][a0 + j] = acc;
            } else {  // inv(U)[a0+i][a0+u] for u >= i
                for (int u = i; u < sz; ++u) {
                    const float2 xu = x[a0 + i][a0 + u];
                    const float2 tv = T[u * sz + j];
                    acc.x += xu.x * tv.x - xu.y * tv.y;
                    acc.y += xu.x * tv.y + xu.y * tv.x;
                }
                x[a0 + i][c0 + j] = acc;
            }
        }
        __syncthreads();
    }
    float2* out = Dinv + b * dstride + (k0 / NB) * 2 * NB * NB;
    for (int e = t; e < NB * NB; e += blockDim.x) {
        const int c = e / NB, rr = e % NB;
        out[e] = rr == c ? make_float2(1.f, 0.f) : (rr > c ? x[rr][c] : make_float2(0.f, 0.f));
        out[NB * NB + e] = rr <= c ? x[rr][c] : make_float2(0.f, 0.f);
    }
    if (bimg) pack_trsm_b<kDiagLd>(x, bimg + b * bstride + (k0 / NB) * 2 * kTrsmBImage);
}

// blockIdx.y == 0: rows of L21 = A21 U11^-1; blockIdx.y == 1: columns of
// U12 = L11^-1 A12.  blockIdx.z = matrix.
template <int NB>
__global__ void __launch_bounds__(128)
k_lu_trsm(float2* __restrict__ A, int64_t n, int64_t stride, int64_t k0)
{
    __shared__ float2 s[NB][NB + 1];
    float2* M = A + (int64_t)blockIdx.z * stride;
    const int kb = (int)min((int64_t)NB, n - k0);
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) {
        int r = t % NB, c = t / NB;
        s[r][c] = (r < kb && c < kb) ? M[(k0 + c) * n + k0 + r] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int64_t idx = k0 + kb + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    float2 v[NB];
    if (blockIdx.y == 0) {
        // row idx: x U11 = a  ->  x_c = (a_c - sum_{t<c} x_t u_tc) / u_cc
#pragma unroll
        for (int c = 0; c < NB; ++c) v[c] = (c < kb) ? M[(k0 + c) * n + idx] : make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < NB; ++c) {
            if (c < kb) {
                float2 acc = v[c];
#pragma unroll
                for (int t = 0; t < c; ++t) acc = cfms(acc, v[t], s[t][c]);
                v[c] = cdivf(acc, s[c][c]);
            }
        }
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if (c < kb) M[(k0 + c) * n + idx] = v[c];
    } else {
        // column idx: L11 y = a (unit lower)  ->  y_r = a_r - sum_{t<r} l_rt y_t
        const float2* col = M + idx * n + k0;
#pragma unroll
        for (int r = 0; r < NB; ++r) v[r] = (r < kb) ? col[r] : make_float2(0.f, 0.f);
#pragma unroll
        for (int r = 0; r < NB; ++r) {
            if (r < kb) {
                float2 acc = v[r];
#pragma unroll
                for (int t = 0; t < r; ++t) acc = cfms(acc, s[r][t], v[t]);
                v[r] = acc;
            }
        }
        float2* colw = M + idx * n + k0;
#pragma unroll
        for (int r = 0; r < NB; ++r)
            if (r < kb) colw[r] = v[r];
    }
}


// Dynamic shared memory of k_lu_diag<NB>.
template <int NB>
constexpr size_t lu_diag_smem_bytes() { return sizeof(float2) * 2 * NB * (NB + 1); }

}  // namespace
}  // namespace mh
