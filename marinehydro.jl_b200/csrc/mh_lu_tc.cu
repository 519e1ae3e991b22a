// Batched pivot-free complex LU with the trailing update on the 5th-generation
// tensor cores (tcgen05), and block-parallel triangular solves.
//
// Panels of NB = 64 complex columns, trailing updates every two panels (one
// 128-wide tile).  Per panel k0:
//   k_lu_diag64        factor the 64 x 64 diagonal block (registers, one
//                      barrier per elimination step), store inv(L11), inv(U11);
//   k_lu_trsm_tc       L21 = A21 inv(U11) and U12^T = A12^T inv(L11)^T as
//                      tcgen05 GEMMs (M=128, N=128, K=128); writes the FP32
//                      factors into the matrix and the FP16 operand panels of
//                      the update, pre-packed as their shared-memory images
//                      at absolute 128-row (column) tile slots;
//   k_lu_update_tc     A22 -= sum_p L21_p U12_p over panel pairs: the
//                      packed panels arrive by cp.async.bulk (no register
//                      staging), sixteen MMAs per pair accumulate in TMEM.
//
// The trailing update of a 128 x 128 complex tile of A22 is two real GEMMs
// over the FP16 images A = [Re L21 | Im L21] and B = [Re U12^T | Im U12^T]
// (128 rows each, K = 128: the 64 complex K entries' real parts, then their
// imaginary parts): Re(L21 U12) = A_re B_re - A_im B_im into tensor-memory
// columns 0..127 (the K steps of the imaginary half with A negated by the
// instruction descriptor) and Im(L21 U12) = A_re B_im + A_im B_re into
// columns 128..255 (B's K halves swapped through the descriptors' start
// addresses).  Each operand holds each real and imaginary part once: 64 KB
// per panel pair.  Operands are rounded to FP16 and staged in shared memory
// in the UMMA K-major no-swizzle layout (8-row x 16-byte core matrices; SBO =
// 128 B between 8-row groups, LBO = one K chunk of 8 elements); one thread
// issues sixteen tcgen05.mma.kind::f16 (M=128, N=128, K=16) per panel pair
// and commits them to an mbarrier; the four warps read their 32 TMEM lanes
// back with tcgen05.ld and subtract from A22 in FP32.  Every wait is bounded: a timeout marks the
// matrix bad (the host then re-solves it with the FP64 pivoted LU) instead
// of spinning.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "mh_internal.h"
#include "mh_lu_kernels.cuh"

namespace mh {
namespace {

constexpr int TC_NB = 64;                 // complex K of the trailing update
constexpr int TC_TM = 128;                // C rows per CTA (UMMA M)
constexpr int TC_TN = 128;                // C complex columns per CTA (UMMA N = 256)
constexpr int TC_KR = 2 * TC_NB;          // real K = 128 (8 UMMA K-steps of 16)
constexpr uint32_t kSmemA = TC_TM * TC_KR * 2;          // 32 KiB of FP16
constexpr uint32_t kSmemB = 2 * TC_TN * TC_KR * 2;      // 64 KiB: the B operand (32 KiB) and room after it
constexpr uint32_t kTmemCols = 2 * TC_TN;               // 256 FP32 columns
constexpr uint32_t kLboA = (TC_TM / 8) * 128;           // bytes between K chunks of A
constexpr uint32_t kSbo = 128;                          // bytes between 8-row groups
// Instruction descriptor: F32 accumulator (bits 4-5 = 1), A and B F16
// (bits 7-9, 10-12 = 0), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
constexpr uint32_t kIdescN128 = (1u << 4) | (128u >> 3 << 17) | ((uint32_t)TC_TM >> 4 << 24);
constexpr uint32_t kLboB128 = (128 / 8) * 128;          // B of the TRSM GEMM: 128 rows
constexpr uint32_t kPanelL = kSmemA;                    // packed L21 tile (A image), bytes
constexpr uint32_t kPanelU = kSmemA;                    // packed U12 tile (B image, 128 rows), bytes
constexpr int kWaitPolls = 4096;          // bounded mbarrier polls ...
constexpr uint32_t kWaitHintNs = 1000;    // ... each suspending at most ~1 us

// Dynamic shared memory of k_lu_update_tc: the two operand tiles (64 KiB) and
// the room the epilogue's three 32 KiB chunks of C need (96 KiB in all), so
// two CTAs share an SM and its 512 TMEM columns.
constexpr uint32_t kTcSmemBytes = kSmemA + kSmemB;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, no swizzle, Blackwell version field = 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Byte offset of (row, K chunk kc) in a K-major no-swizzle tile with `rows` rows.
__device__ __forceinline__ uint32_t core_off(int row, int kc, int rows)
{
    return (uint32_t)((kc * (rows / 8) + row / 8) * 128 + (row % 8) * 16);
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b)
{
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase)
{
    for (int it = 0; it < kWaitPolls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(phase), "r"(kWaitHintNs)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16};"
        :: "r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
           "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(slot)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Eight K=16 MMAs over a K=128 (real) operand pair, then commit to `bar`;
// the first one overwrites the accumulator unless `accumulate`.
__device__ __forceinline__ void mma_k128(uint32_t tmem, uint32_t a0, uint32_t lbo_a, uint32_t b0,
                                        uint32_t lbo_b, uint32_t idesc, uint32_t bar, bool accumulate = false)
{
#pragma unroll
    for (int s = 0; s < TC_KR / 16; ++s) {
        const uint64_t da = umma_desc(a0 + 2 * s * lbo_a, lbo_a, kSbo);
        const uint64_t db = umma_desc(b0 + 2 * s * lbo_b, lbo_b, kSbo);
        const uint32_t acc = (s > 0 || accumulate) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(bar) : "memory");
}

// The complex product of one panel pair, C += L21 U12, from the FP16 images
// A = [Re L21 | Im L21] (128 rows, K = 128) and B = [Re U12^T | Im U12^T]
// (128 rows, K = 128): sixteen K=16 MMAs of N = 128, the real part into
// tensor-memory columns 0..127 as A_s B_s over the K steps s (A negated by
// the instruction descriptor for s >= 4: - Im L Im U), the imaginary part into
// columns 128..255 as A_s B_(s+4 mod 8) (Re L Im U + Im L Re U); then commit
// to `bar`.  The first MMAs overwrite the accumulator unless `accumulate`.
// B holds each of Re U12, Im U12 once: 32 KB per pair instead of the 64 KB
// of a [Re -Im; Im Re] image.
__device__ __forceinline__ void mma_cplx(uint32_t tmem, uint32_t a0, uint32_t b0, uint32_t bar, bool accumulate)
{
    constexpr uint32_t kNegA = 1u << 13;
#pragma unroll
    for (int s = 0; s < TC_KR / 16; ++s) {
        const uint64_t da = umma_desc(a0 + 2 * s * kLboA, kLboA, kSbo);
        const uint64_t dre = umma_desc(b0 + 2 * s * kLboB128, kLboB128, kSbo);
        const uint64_t dim = umma_desc(b0 + 2 * ((s + 4) & 7) * kLboB128, kLboB128, kSbo);
        const uint32_t acc = (s > 0 || accumulate) ? 1u : 0u;
        const uint32_t idre = kIdescN128 | (s >= 4 ? kNegA : 0u);
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            :: "r"(tmem), "l"(da), "l"(dre), "r"(idre), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
            :: "r"(tmem + (uint32_t)TC_TN), "l"(da), "l"(dim), "r"(kIdescN128), "r"(acc), "r"(0u), "r"(0u),
               "r"(0u), "r"(0u));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(bar) : "memory");
}

// Eight consecutive FP32 words of a TMEM read-back (x[o .. o + 7], o a
// compile-time offset after unrolling) as FP16, times sign.
__device__ __forceinline__ uint4 pack8u(const uint32_t (&x)[32], int o, float sign)
{
    return make_uint4(pack_h2(sign * __uint_as_float(x[o]), sign * __uint_as_float(x[o + 1])),
                      pack_h2(sign * __uint_as_float(x[o + 2]), sign * __uint_as_float(x[o + 3])),
                      pack_h2(sign * __uint_as_float(x[o + 4]), sign * __uint_as_float(x[o + 5])),
                      pack_h2(sign * __uint_as_float(x[o + 6]), sign * __uint_as_float(x[o + 7])));
}

__device__ __forceinline__ uint4 pack8(const float2* v, bool imag, float sign)
{
    if (imag)
        return make_uint4(pack_h2(sign * v[0].y, sign * v[1].y), pack_h2(sign * v[2].y, sign * v[3].y),
                          pack_h2(sign * v[4].y, sign * v[5].y), pack_h2(sign * v[6].y, sign * v[7].y));
    return make_uint4(pack_h2(sign * v[0].x, sign * v[1].x), pack_h2(sign * v[2].x, sign * v[3].x),
                      pack_h2(sign * v[4].x, sign * v[5].x), pack_h2(sign * v[6].x, sign * v[7].x));
}

// Panel TRSMs of step k0 on the tensor cores.  blockIdx.x < ntile: a 128-row
// tile of L21 = A21 inv(U11); otherwise a 128-column tile of U12 = inv(L11)
// A12, computed as U12^T = A12^T inv(L11)^T.  blockIdx.y = matrix.  Tiles are
// absolute (tile T holds rows, or columns, 128 T .. 128 T + 127), starting
// at the tile of row k0 + 64; the rows (columns) of that tile above k0 + 64
// are zero in the images and are not written back.  Writes the FP32 factors
// back and the packed FP16 panels Lp (A image of the update: rows i =
// [Re L21(i, :) | Im]) and Up (B image: rows j = [Re U12(:, j) | Im]), each at
// its absolute tile slot.
__global__ void __launch_bounds__(128, 2)
k_lu_trsm_tc(float2* __restrict__ Ab, int64_t n, int64_t stride, int64_t k0,
             const unsigned char* __restrict__ bimg, int64_t bstride, unsigned char* __restrict__ Lp,
             unsigned char* __restrict__ Up, int64_t pstride, int ntile, int* __restrict__ bad)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ uint64_t mbar, mbar_ld;
    __shared__ uint32_t tmem_slot;
    unsigned char* sA = tc_smem;             // 128 x 128 FP16 (32 KiB)
    unsigned char* sB = tc_smem + kSmemA;    // 128 x 128 FP16 (32 KiB)
    const int b = blockIdx.y;
    float2* M = Ab + (int64_t)b * stride;
    const int64_t blk = k0 / TC_NB;
    const bool lower = (int)blockIdx.x < ntile;
    const int64_t lo = k0 + TC_NB;  // first row of L21 / column of U12
    const int tile = (int)(lo / TC_TM) + (lower ? (int)blockIdx.x : (int)blockIdx.x - ntile);
    const int64_t g = (int64_t)tile * TC_TM + threadIdx.x;  // row of L21 or column of U12
    const bool ok = g >= lo && g < n;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tmem_alloc(&tmem_slot, 128);
    const uint32_t bar_ld = smem_u32(&mbar_ld);
    if (tid == 0) {
        mbar_init(&mbar);
        mbar_init(&mbar_ld);
        // B operand: the image the diagonal kernel packed (inv(U11) columns for
        // L21, inv(L11) rows for U12), by bulk copy while the threads stage A
        const unsigned char* src = bimg + (int64_t)b * bstride + (blk * 2 + (lower ? 0 : 1)) * kTrsmBImage;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(bar_ld), "r"((uint32_t)kTrsmBImage) : "memory");
        constexpr uint32_t kChunk = 16384;
#pragma unroll 1
        for (uint32_t off = 0; off < (uint32_t)kTrsmBImage; off += kChunk)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"(smem_u32(sB + off)), "l"(src + off), "r"(kChunk), "r"(bar_ld) : "memory");
    }
    // A operand: row tid = A21(g, :) or A12(:, g)^T, 64 complex -> Re chunks 0..7, Im 8..15
    if (lower) {  // A21 is column-major: consecutive rows g are consecutive lanes
#pragma unroll 2
        for (int c = 0; c < 8; ++c) {
            float2 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int64_t t = k0 + 8 * c + q;
                v[q] = ok ? M[t * n + g] : make_float2(0.f, 0.f);
            }
            *reinterpret_cast<uint4*>(sA + core_off(tid, c, TC_TM)) = pack8(v, false, 1.f);
            *reinterpret_cast<uint4*>(sA + core_off(tid, 8 + c, TC_TM)) = pack8(v, true, 1.f);
        }
    } else {  // a column of A12 is contiguous: one warp reads it, lane l holds t = 2l, 2l + 1
        const int cpos = (2 * lane) & 7, cc = (2 * lane) >> 3;
#pragma unroll 4
        for (int i = 0; i < 32; ++i) {
            const int row = warp * 32 + i;
            const int64_t gc = (int64_t)tile * TC_TM + row;
            float2 v0 = make_float2(0.f, 0.f), v1 = v0;
            if (gc >= lo && gc < n) {
                v0 = M[gc * n + k0 + 2 * lane];
                v1 = M[gc * n + k0 + 2 * lane + 1];
            }
            *reinterpret_cast<uint32_t*>(sA + core_off(row, cc, TC_TM) + 2 * cpos) = pack_h2(v0.x, v1.x);
            *reinterpret_cast<uint32_t*>(sA + core_off(row, 8 + cc, TC_TM) + 2 * cpos) = pack_h2(v0.y, v1.y);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t bar = smem_u32(&mbar);
    const bool loaded = __syncthreads_and(mbar_wait(bar_ld, 0)) != 0;
    if (loaded && tid == 0) mma_k128(tmem, smem_u32(sA), kLboA, smem_u32(sB), kLboB128, kIdescN128, bar);
    const bool done = loaded && __syncthreads_and(mbar_wait(bar, 0)) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (done) {
        const int row = warp * 32 + lane;  // TMEM lane = A row = tid of the loader above
        const int64_t gg = (int64_t)tile * TC_TM + row;
        const bool okr = gg >= lo && gg < n;
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
        unsigned char* panel = lower ? Lp + (int64_t)b * pstride + (int64_t)tile * kPanelL
                                     : Up + (int64_t)b * pstride + (int64_t)tile * kPanelU;
#pragma unroll 1
        for (int half = 0; half < 2; ++half) {
            uint32_t re[32], im[32];
            tmem_ld32(lane_base + (uint32_t)(half * 32), re);
            tmem_ld32(lane_base + (uint32_t)(64 + half * 32), im);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (!okr) {
#pragma unroll
                for (int q = 0; q < 32; ++q) re[q] = im[q] = 0u;
            }
            if (lower) {  // rows gg of L21: consecutive lanes, coalesced per column t
                if (okr) {
#pragma unroll
                    for (int q = 0; q < 32; ++q)  // unrolled: re and im stay in registers
                        M[(k0 + half * 32 + q) * n + gg] = make_float2(__uint_as_float(re[q]), __uint_as_float(im[q]));
                }
            } else {  // columns gg of U12: transposed through shared memory (the operands are
                      // consumed), then one warp writes 32 contiguous entries of a column
                auto st = reinterpret_cast<float2 (*)[33]>(tc_smem);
#pragma unroll
                for (int q = 0; q < 32; ++q) st[row][q] = make_float2(__uint_as_float(re[q]), __uint_as_float(im[q]));
                __syncthreads();
#pragma unroll 4
                for (int i = 0; i < 32; ++i) {
                    const int rr = warp * 32 + i;
                    const int64_t gc = (int64_t)tile * TC_TM + rr;
                    if (gc >= lo && gc < n) M[gc * n + k0 + half * 32 + lane] = st[rr][lane];
                }
                __syncthreads();
            }
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const int c = half * 4 + c4;
                // both images [Re | Im] by rows (L21 rows; U12 columns = U12^T rows)
                *reinterpret_cast<uint4*>(panel + core_off(row, c, TC_TM)) = pack8u(re, 8 * c4, 1.f);
                *reinterpret_cast<uint4*>(panel + core_off(row, 8 + c, TC_TM)) = pack8u(im, 8 * c4, 1.f);
            }
        }
    } else {
        if (lane == 0) atomicExch(bad + b, 2);
        // bounded: the image copy or the MMAs may still be in flight
        if (!loaded) mbar_wait(bar_ld, 0);
        else mbar_wait(bar, 0);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 128);
}

// Packed panel pairs of one update (one per 64-column panel).
constexpr int kMaxPairs = 16;  // an outer step's panels (8 at most) and the previous step's deferred ones
struct PanelPairs {
    const unsigned char* L[kMaxPairs];
    const unsigned char* U[kMaxPairs];
};

// Epilogue of a full interior tile through shared memory: C -= P (P the
// product in TMEM) in kCChunks chunks of 32 complex columns (32 KB, one
// column = 128 rows = 1 KB contiguous), kCBufs chunk buffers in the freed
// operand space.  Chunks 0..kCBufs-1 are fetched at once by cp.async.bulk;
// each chunk is updated in place by the thread of its row, made visible to
// the async proxy, stored by cp.async.bulk and, once that store has read
// its buffer, the buffer takes chunk + kCBufs.  Every wait is bounded:
// false when one ran out (after waiting, bounded, for what is in flight).
constexpr int kCCols = 32;                      // complex columns per chunk
constexpr int kCChunks = TC_TN / kCCols;        // 4
constexpr int kCBufs = 3;                       // chunk buffers
constexpr uint32_t kCBytes = kCCols * TC_TM * sizeof(float2);  // 32 KB
static_assert(kCBufs * kCBytes <= kSmemA + kSmemB, "the chunk buffers fit in the operand space");

__device__ __forceinline__ void bulk_load_chunk(const float2* M, int64_t n, int64_t r0, int64_t col0,
                                                unsigned char* buf, uint32_t bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(kCBytes) : "memory");
    for (int q = 0; q < kCCols; ++q)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     :: "r"(smem_u32(buf + q * TC_TM * sizeof(float2))), "l"(M + (col0 + q) * n + r0),
                        "r"((uint32_t)(TC_TM * sizeof(float2))), "r"(bar) : "memory");
}

__device__ __forceinline__ bool epilogue_bulk(float2* M, int64_t n, int64_t r0, int64_t c0, unsigned char* smem,
                                              uint64_t* cbar, uint32_t tmem, int warp, int lane, int tid)
{
    const int row = warp * 32 + lane;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    if (tid == 0)
        for (int k = 0; k < kCBufs; ++k)
            bulk_load_chunk(M, n, r0, c0 + k * kCCols, smem + k * kCBytes, smem_u32(&cbar[k]));
    // thread 0 issues chunk k + kCBufs at the end of iteration k, so before
    // iteration k the loads of chunks 0 .. min(kCChunks, kCBufs + k) - 1 are issued
    bool ok = true;
    int k = 0;
    for (; k < kCChunks; ++k) {
        const int bi = k % kCBufs;
        ok = __syncthreads_and(mbar_wait(smem_u32(&cbar[bi]), (uint32_t)((k / kCBufs) & 1))) != 0;
        if (!ok) break;
        float2* cs = reinterpret_cast<float2*>(smem + bi * kCBytes);
#pragma unroll
        for (int cc = 0; cc < kCCols / 16; ++cc) {
            uint32_t re[16], im[16];
            tmem_ld16(lane_base + (uint32_t)(k * kCCols + cc * 16), re);
            tmem_ld16(lane_base + (uint32_t)(TC_TN + k * kCCols + cc * 16), im);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                float2& v = cs[(cc * 16 + q) * TC_TM + row];
                v = make_float2(v.x - __uint_as_float(re[q]), v.y - __uint_as_float(im[q]));
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            for (int q = 0; q < kCCols; ++q)
                asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                             :: "l"(M + (c0 + k * kCCols + q) * n + r0),
                                "r"(smem_u32(cs + q * TC_TM)), "r"((uint32_t)(TC_TM * sizeof(float2)))
                             : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            if (k + kCBufs < kCChunks) {  // this buffer takes chunk k + kCBufs once the store has read it
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                bulk_load_chunk(M, n, r0, c0 + (k + kCBufs) * kCCols, smem + bi * kCBytes, smem_u32(&cbar[bi]));
            }
        }
    }
    if (!ok) {  // loads of chunks k .. issued - 1 may still land: wait for them (bounded)
        const int issued = min(kCChunks, kCBufs + k);
        for (int j = k; j < issued; ++j) mbar_wait(smem_u32(&cbar[j % kCBufs]), (uint32_t)((j / kCBufs) & 1));
    }
    if (tid == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    return ok;
}

// A22 -= sum_p L21_p U12_p for one 128 x 128 complex tile (absolute tiles
// ti, tj); the operands are the packed panels of k_lu_trsm_tc (npair <= 16
// panel pairs, K = 64 complex each), fetched by cp.async.bulk into shared
// memory one pair at a time and accumulated in tensor memory.  Only rows and
// columns >= lo are written.  Tiles, relative to t0 (ntile of them per side):
// mode 1: the first w tile rows and tile columns (an L of width w; w (2 ntile
// - w) tiles, the part the next panels depend on; tile x of the L is
// blockIdx.x + xoff, tile 0 being the diagonal tile (t0, t0)); mode 2: the
// tiles past them (grid (ntile - w)^2).
__global__ void __launch_bounds__(128, 2)
k_lu_update_tc(float2* __restrict__ Ab, int64_t n, int64_t stride, int t0, int ntile, int mode, int w,
               PanelPairs pp, int npair, int64_t pstride, int64_t lo, int* __restrict__ bad,
               int xoff)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ uint64_t mbar[2 + kCBufs];
    __shared__ uint32_t tmem_slot;
    unsigned char* sA = tc_smem;
    unsigned char* sB = tc_smem + kSmemA;
    const int b = blockIdx.z;
    float2* M = Ab + (int64_t)b * stride;
    int ti, tj;
    if (mode == 1) {
        const int x = (int)blockIdx.x + xoff;
        if (x < w * ntile) {
            ti = t0 + x / ntile;
            tj = t0 + x % ntile;
        } else {
            const int y = x - w * ntile, rest = ntile - w;
            tj = t0 + y / rest;
            ti = t0 + w + y % rest;
        }
    } else {
        ti = t0 + w + (int)blockIdx.x;
        tj = t0 + w + (int)blockIdx.y;
    }
    const int64_t r0 = (int64_t)ti * TC_TM;
    const int64_t c0 = (int64_t)tj * TC_TN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tmem_alloc(&tmem_slot, kTmemCols);
    const uint32_t bar_ld = smem_u32(&mbar[0]), bar_mma = smem_u32(&mbar[1]);
    if (tid == 0)
        for (int q = 0; q < 2 + kCBufs; ++q) mbar_init(&mbar[q]);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    // a tile wholly inside the trailing matrix (and n even, so every column
    // of it starts on a 16-byte boundary) goes through shared memory by bulk
    // copies after the MMAs; other tiles use per-thread loads and stores
    const bool full = r0 >= lo && c0 >= lo && r0 + TC_TM <= n && c0 + TC_TN <= n && (n & 1) == 0;
    // this thread's row of C does not depend on the products: its first 16
    // columns are loaded while the panel copies and the MMAs run
    const int64_t gi = r0 + warp * 32 + lane;
    const bool row_ok = gi >= lo && gi < n;
    constexpr int kEc = 16;  // columns per epilogue chunk
    float2 cv[kEc];
    if (!full) {
        const float2* pc = M + c0 * n + gi;
#pragma unroll
        for (int q = 0; q < kEc; ++q, pc += n) {
            const int64_t gj = c0 + q;
            cv[q] = (row_ok && gj >= lo && gj < n) ? *pc : make_float2(0.f, 0.f);
        }
    }
    bool ok = true;     // every wait so far completed
    int pend_ld = -1;   // pair whose copies were issued and not seen complete
    int pend_mma = -1;  // pair whose MMAs were issued and not seen complete
#pragma unroll 1
    for (int p = 0; p < npair && ok; ++p) {
        if (tid == 0) {
            const unsigned char* srcA = pp.L[p] + (int64_t)b * pstride + (int64_t)ti * kPanelL;
            const unsigned char* srcB = pp.U[p] + (int64_t)b * pstride + (int64_t)tj * kPanelU;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         :: "r"(bar_ld), "r"(kPanelL + kPanelU) : "memory");
            constexpr uint32_t kChunk = 16384;
#pragma unroll 1
            for (uint32_t off = 0; off < kPanelL; off += kChunk)
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             :: "r"(smem_u32(sA + off)), "l"(srcA + off), "r"(kChunk), "r"(bar_ld) : "memory");
#pragma unroll 1
            for (uint32_t off = 0; off < kPanelU; off += kChunk)
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             :: "r"(smem_u32(sB + off)), "l"(srcB + off), "r"(kChunk), "r"(bar_ld) : "memory");
        }
        pend_ld = p;
        ok = __syncthreads_and(mbar_wait(bar_ld, (uint32_t)(p & 1))) != 0;
        if (!ok) break;
        pend_ld = -1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) mma_cplx(tmem, smem_u32(sA), smem_u32(sB), bar_mma, p > 0);
        // the next pair's copies overwrite the operands: wait for these MMAs
        pend_mma = p;
        ok = __syncthreads_and(mbar_wait(bar_mma, (uint32_t)(p & 1))) != 0;
        if (ok) pend_mma = -1;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && full) {
        ok = epilogue_bulk(M, n, r0, c0, tc_smem, mbar + 2, tmem, warp, lane, tid);
        if (!ok && lane == 0) atomicExch(bad + b, 2);
    } else if (ok) {
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
        // chunk cc + 1 of C is loaded before chunk cc is stored
#pragma unroll
        for (int cc = 0; cc < TC_TN / kEc; ++cc) {
            uint32_t re[kEc], im[kEc];
            tmem_ld16(lane_base + (uint32_t)(cc * kEc), re);
            tmem_ld16(lane_base + (uint32_t)(TC_TN + cc * kEc), im);
            float2 nv[kEc];
            if (cc + 1 < TC_TN / kEc) {
                const float2* pc = M + (c0 + (cc + 1) * kEc) * n + gi;
#pragma unroll
                for (int q = 0; q < kEc; ++q, pc += n) {
                    const int64_t gj = c0 + (cc + 1) * kEc + q;
                    nv[q] = (row_ok && gj >= lo && gj < n) ? *pc : make_float2(0.f, 0.f);
                }
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row_ok) {
                float2* pc = M + (c0 + cc * kEc) * n + gi;
#pragma unroll
                for (int q = 0; q < kEc; ++q, pc += n) {
                    const int64_t gj = c0 + cc * kEc + q;
                    if (gj >= lo && gj < n)
                        *pc = make_float2(cv[q].x - __uint_as_float(re[q]), cv[q].y - __uint_as_float(im[q]));
                }
            }
            if (cc + 1 < TC_TN / kEc) {
#pragma unroll
                for (int q = 0; q < kEc; ++q) cv[q] = nv[q];
            }
        }
    } else {
        if (lane == 0) atomicExch(bad + b, 2);
        // bounded: copies or MMAs of the failed pair may still be in flight
        if (pend_ld >= 0) mbar_wait(bar_ld, (uint32_t)(pend_ld & 1));
        if (pend_mma >= 0) mbar_wait(bar_mma, (uint32_t)(pend_mma & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// The same update with C staged in tensor memory first: every thread loads
// its row of the C tile (negated) into the accumulator's TMEM columns while
// the first panel pair is copied, the MMAs accumulate L21 U12 onto it, and
// the epilogue only reads the accumulator back and stores C - L21 U12 (the
// negation undone).  The C read thus overlaps the operand copies instead of
// following the MMAs.  Grid, tiles and operands as k_lu_update_tc.
__global__ void __launch_bounds__(128, 2)
k_lu_update_tc_acc(float2* __restrict__ Ab, int64_t n, int64_t stride, int t0, int ntile, int mode, int w,
                   PanelPairs pp, int npair, int64_t pstride, int64_t lo, int* __restrict__ bad,
               int xoff)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    __shared__ uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    unsigned char* sA = tc_smem;
    unsigned char* sB = tc_smem + kSmemA;
    const int b = blockIdx.z;
    float2* M = Ab + (int64_t)b * stride;
    int ti, tj;
    if (mode == 1) {
        const int x = (int)blockIdx.x + xoff;
        if (x < w * ntile) {
            ti = t0 + x / ntile;
            tj = t0 + x % ntile;
        } else {
            const int y = x - w * ntile, rest = ntile - w;
            tj = t0 + y / rest;
            ti = t0 + w + y % rest;
        }
    } else {
        ti = t0 + w + (int)blockIdx.x;
        tj = t0 + w + (int)blockIdx.y;
    }
    const int64_t r0 = (int64_t)ti * TC_TM;
    const int64_t c0 = (int64_t)tj * TC_TN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tmem_alloc(&tmem_slot, kTmemCols);
    const uint32_t bar_ld = smem_u32(&mbar[0]), bar_mma = smem_u32(&mbar[1]);
    if (tid == 0) {
        mbar_init(&mbar[0]);
        mbar_init(&mbar[1]);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    auto copy_pair = [&](int p) {
        const unsigned char* srcA = pp.L[p] + (int64_t)b * pstride + (int64_t)ti * kPanelL;
        const unsigned char* srcB = pp.U[p] + (int64_t)b * pstride + (int64_t)tj * kPanelU;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     :: "r"(bar_ld), "r"(kPanelL + kPanelU) : "memory");
        constexpr uint32_t kChunk = 16384;
#pragma unroll 1
        for (uint32_t off = 0; off < kPanelL; off += kChunk)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"(smem_u32(sA + off)), "l"(srcA + off), "r"(kChunk), "r"(bar_ld) : "memory");
#pragma unroll 1
        for (uint32_t off = 0; off < kPanelU; off += kChunk)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                         :: "r"(smem_u32(sB + off)), "l"(srcB + off), "r"(kChunk), "r"(bar_ld) : "memory");
    };
    if (tid == 0) copy_pair(0);
    // -C into the accumulator, 16 columns at a time (rows or columns outside
    // [lo, n) as zeros; they are not stored back)
    const int64_t gi = r0 + warp * 32 + lane;
    const bool row_ok = gi >= lo && gi < n;
    constexpr int kEc = 16;
#pragma unroll 2
    for (int cc = 0; cc < TC_TN / kEc; ++cc) {
        uint32_t re[kEc], im[kEc];
        const float2* pc = M + (c0 + cc * kEc) * n + gi;
#pragma unroll
        for (int q = 0; q < kEc; ++q) {
            const int64_t gj = c0 + cc * kEc + q;
            const float2 v = (row_ok && gj >= lo && gj < n) ? pc[(int64_t)q * n] : make_float2(0.f, 0.f);
            re[q] = __float_as_uint(-v.x);
            im[q] = __float_as_uint(-v.y);
        }
        tmem_st16(lane_base + (uint32_t)(cc * kEc), re);
        tmem_st16(lane_base + (uint32_t)(TC_TN + cc * kEc), im);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    bool ok = true;     // every wait so far completed
    int pend_ld = -1;   // pair whose copies were issued and not seen complete
    int pend_mma = -1;  // pair whose MMAs were issued and not seen complete
#pragma unroll 1
    for (int p = 0; p < npair && ok; ++p) {
        if (tid == 0 && p > 0) copy_pair(p);
        pend_ld = p;
        // also orders every thread's TMEM stores of C before the first MMAs
        ok = __syncthreads_and(mbar_wait(bar_ld, (uint32_t)(p & 1))) != 0;
        if (!ok) break;
        pend_ld = -1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) mma_cplx(tmem, smem_u32(sA), smem_u32(sB), bar_mma, true);
        // the next pair's copies overwrite the operands: wait for these MMAs
        pend_mma = p;
        ok = __syncthreads_and(mbar_wait(bar_mma, (uint32_t)(p & 1))) != 0;
        if (ok) pend_mma = -1;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok) {
#pragma unroll 2
        for (int cc = 0; cc < TC_TN / kEc; ++cc) {
            uint32_t re[kEc], im[kEc];
            tmem_ld16(lane_base + (uint32_t)(cc * kEc), re);
            tmem_ld16(lane_base + (uint32_t)(TC_TN + cc * kEc), im);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row_ok) {
                float2* pc = M + (c0 + cc * kEc) * n + gi;
#pragma unroll
                for (int q = 0; q < kEc; ++q) {
                    const int64_t gj = c0 + cc * kEc + q;
                    if (gj >= lo && gj < n)
                        pc[(int64_t)q * n] = make_float2(-__uint_as_float(re[q]), -__uint_as_float(im[q]));
                }
            }
        }
    } else {
        if (lane == 0) atomicExch(bad + b, 2);
        // bounded: copies or MMAs of the failed pair may still be in flight
        if (pend_ld >= 0) mbar_wait(bar_ld, (uint32_t)(pend_ld & 1));
        if (pend_mma >= 0) mbar_wait(bar_mma, (uint32_t)(pend_mma & 1));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// ---------------------------------------------------------------------------
// block-parallel triangular solves, one launch per diagonal block
// ---------------------------------------------------------------------------

// Forward step of L y = x for diagonal block `blk`: y_blk = inv(L11) x_blk
// (written to Y by CTA 0), then x_i -= L_i,blk y_blk for the rows below,
// 128 rows per CTA.
template <int NB>
__global__ void __launch_bounds__(128)
k_trsv_fwd(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
           int64_t dstride, float2* __restrict__ X, float2* __restrict__ Y, int64_t xstride, int nrhs,
           int blk)
{
    __shared__ float2 ys[kMaxRhs * NB];
    const int b = blockIdx.y;
    const float2* M = A + (int64_t)b * stride;
    const float2* Li = Dinv + (int64_t)b * dstride + (int64_t)blk * 2 * NB * NB;
    float2* x = X + (int64_t)b * xstride;
    float2* y = Y + (int64_t)b * xstride;
    const int64_t k0 = (int64_t)blk * NB;
    const int kb = (int)min((int64_t)NB, n - k0);
    for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
        const int r = t % NB, q = t / NB;
        float2 acc = make_float2(0.f, 0.f);
        if (r < kb)
            for (int c = 0; c <= r; ++c) {
                const float2 l = Li[c * NB + r], v = x[(int64_t)q * n + k0 + c];
                acc.x += l.x * v.x - l.y * v.y;
                acc.y += l.x * v.y + l.y * v.x;
            }
        ys[q * NB + r] = acc;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
            const int r = t % kb, q = t / kb;
            y[(int64_t)q * n + k0 + r] = ys[q * NB + r];
        }
    const int64_t i = k0 + kb + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int q = 0; q < nrhs; ++q) {
        float2 acc = x[(int64_t)q * n + i];
        for (int t = 0; t < kb; ++t) acc = cfms(acc, M[(k0 + t) * n + i], ys[q * NB + t]);
        x[(int64_t)q * n + i] = acc;
    }
}

// Backward step of U z = y for block `blk`: z_blk = inv(U11) y_blk (written
// to Z by CTA 0), then y_i -= U_i,blk z_blk for the rows above.
template <int NB>
__global__ void __launch_bounds__(128)
k_trsv_bwd(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
           int64_t dstride, float2* __restrict__ Y, float2* __restrict__ Z, int64_t xstride, int nrhs,
           int blk)
{
    __shared__ float2 zs[kMaxRhs * NB];
    const int b = blockIdx.y;
    const float2* M = A + (int64_t)b * stride;
    const float2* Ui = Dinv + (int64_t)b * dstride + (int64_t)blk * 2 * NB * NB + NB * NB;
    float2* y = Y + (int64_t)b * xstride;
    float2* z = Z + (int64_t)b * xstride;
    const int64_t k0 = (int64_t)blk * NB;
    const int kb = (int)min((int64_t)NB, n - k0);
    for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
        const int r = t % NB, q = t / NB;
        float2 acc = make_float2(0.f, 0.f);
        if (r < kb)
            for (int c = r; c < kb; ++c) {
                const float2 u = Ui[c * NB + r], v = y[(int64_t)q * n + k0 + c];
                acc.x += u.x * v.x - u.y * v.y;
                acc.y += u.x * v.y + u.y * v.x;
            }
        zs[q * NB + r] = acc;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
            const int r = t % kb, q = t / kb;
            z[(int64_t)q * n + k0 + r] = zs[q * NB + r];
        }
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k0) return;
    for (int q = 0; q < nrhs; ++q) {
        float2 acc = y[(int64_t)q * n + i];
        for (int t = 0; t < kb; ++t) acc = cfms(acc, M[(k0 + t) * n + i], zs[q * NB + t]);
        y[(int64_t)q * n + i] = acc;
    }
}

// Conjugate-transposed solves with the same factors, D^H x = r = U^H L^H x:
// U^H y = r by blocks in increasing order, then L^H x = y in decreasing
// order.  Row i of U^H (or L^H) is column i of the stored factor, so the
// update of row i reads NB consecutive entries of column i: 8 lanes per
// row, each lane every 8th entry, reduced with three shuffles.
__device__ __forceinline__ float2 cconjmul(float2 a, float2 b)  // conj(a) * b
{
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

template <int NB>
__global__ void __launch_bounds__(128)
k_trsv_ct_fwd(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
              int64_t dstride, float2* __restrict__ X, float2* __restrict__ Y, int64_t xstride, int nrhs,
              int blk)
{
    __shared__ float2 ys[kMaxRhs * NB];
    const int b = blockIdx.y;
    const float2* M = A + (int64_t)b * stride;
    const float2* Ui = Dinv + (int64_t)b * dstride + (int64_t)blk * 2 * NB * NB + NB * NB;
    float2* x = X + (int64_t)b * xstride;
    float2* y = Y + (int64_t)b * xstride;
    const int64_t k0 = (int64_t)blk * NB;
    const int kb = (int)min((int64_t)NB, n - k0);
    // y_blk = inv(U11)^H x_blk; inv(U11)^H[r][c] = conj(inv(U11)[c][r]), c <= r
    for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
        const int r = t % NB, q = t / NB;
        float2 acc = make_float2(0.f, 0.f);
        if (r < kb)
            for (int c = 0; c <= r; ++c) {
                const float2 v = cconjmul(Ui[r * NB + c], x[(int64_t)q * n + k0 + c]);
                acc.x += v.x;
                acc.y += v.y;
            }
        ys[q * NB + r] = acc;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
            const int r = t % kb, q = t / kb;
            y[(int64_t)q * n + k0 + r] = ys[q * NB + r];
        }
    // x_i -= sum_t conj(U[k0+t][i]) y_t for the rows below, 16 rows per CTA
    const int sub = threadIdx.x & 7;
    const int64_t i = k0 + kb + (int64_t)blockIdx.x * 16 + (threadIdx.x >> 3);
    const bool live = i < n;
    const float2* col = M + (live ? i : 0) * n + k0;
    for (int q = 0; q < nrhs; ++q) {
        float ax = 0.f, ay = 0.f;
        if (live)
            for (int t = sub; t < kb; t += 8) {
                const float2 v = cconjmul(col[t], ys[q * NB + t]);
                ax += v.x;
                ay += v.y;
            }
        for (int off = 4; off > 0; off >>= 1) {
            ax += __shfl_down_sync(0xffffffffu, ax, off, 8);
            ay += __shfl_down_sync(0xffffffffu, ay, off, 8);
        }
        if (live && sub == 0) {
            float2 v = x[(int64_t)q * n + i];
            x[(int64_t)q * n + i] = make_float2(v.x - ax, v.y - ay);
        }
    }
}

template <int NB>
__global__ void __launch_bounds__(128)
k_trsv_ct_bwd(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
              int64_t dstride, float2* __restrict__ Y, float2* __restrict__ Z, int64_t xstride, int nrhs,
              int blk)
{
    __shared__ float2 zs[kMaxRhs * NB];
    const int b = blockIdx.y;
    const float2* M = A + (int64_t)b * stride;
    const float2* Li = Dinv + (int64_t)b * dstride + (int64_t)blk * 2 * NB * NB;
    float2* y = Y + (int64_t)b * xstride;
    float2* z = Z + (int64_t)b * xstride;
    const int64_t k0 = (int64_t)blk * NB;
    const int kb = (int)min((int64_t)NB, n - k0);
    // z_blk = inv(L11)^H y_blk; inv(L11)^H[r][c] = conj(inv(L11)[c][r]), c >= r
    for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
        const int r = t % NB, q = t / NB;
        float2 acc = make_float2(0.f, 0.f);
        if (r < kb)
            for (int c = r; c < kb; ++c) {
                const float2 v = cconjmul(Li[r * NB + c], y[(int64_t)q * n + k0 + c]);
                acc.x += v.x;
                acc.y += v.y;
            }
        zs[q * NB + r] = acc;
    }
    __syncthreads();
    if (blockIdx.x == 0)
        for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
            const int r = t % kb, q = t / kb;
            z[(int64_t)q * n + k0 + r] = zs[q * NB + r];
        }
    // y_i -= sum_t conj(L[k0+t][i]) z_t for the rows above
    const int sub = threadIdx.x & 7;
    const int64_t i = (int64_t)blockIdx.x * 16 + (threadIdx.x >> 3);
    const bool live = i < k0;
    const float2* col = M + (live ? i : 0) * n + k0;
    for (int q = 0; q < nrhs; ++q) {
        float ax = 0.f, ay = 0.f;
        if (live)
            for (int t = sub; t < kb; t += 8) {
                const float2 v = cconjmul(col[t], zs[q * NB + t]);
                ax += v.x;
                ay += v.y;
            }
        for (int off = 4; off > 0; off >>= 1) {
            ax += __shfl_down_sync(0xffffffffu, ax, off, 8);
            ay += __shfl_down_sync(0xffffffffu, ay, off, 8);
        }
        if (live && sub == 0) {
            float2 v = y[(int64_t)q * n + i];
            y[(int64_t)q * n + i] = make_float2(v.x - ax, v.y - ay);
        }
    }
}

// Persistent substitution: one thread-block cluster of kSolveCluster CTAs
// per matrix runs every block step of both triangles in one launch,
// streaming each triangle of the factors once.  Rows are owned block-
// cyclically (row block rb by CTA rb % kSolveCluster); at each step every
// CTA forms the diagonal block's solution redundantly from x (global), the
// owner writes it back, each CTA updates the rows it owns, and one cluster
// barrier (release/acquire) orders the steps.
// kCT = false: L U x = b (L unit lower, right-looking).  kCT = true:
// U^H L^H x = b (row i of U^H is column i of U).  The diagonal blocks use
// the stored inverses.  Right-hand sides in groups of 4.
constexpr int kSolveThreads = 512;
constexpr int kSolveCluster = 4;

template <int NB>
constexpr size_t persist_smem_bytes()
{
    return sizeof(float2) * (3 * kMaxRhs * NB + NB * (NB + 1));
}

// ys = op(T11^-1) x_blk with T11^-1 (column-major NB x NB, op = identity or
// conjugate transpose; staged with a padded leading dimension NB + 1) and
// x_blk staged in shared memory first.
template <int NB, bool kCT>
__device__ __forceinline__ void persist_diag(const float2* __restrict__ Ti, bool lower, const float2* __restrict__ x,
                                             int64_t n, int64_t k0, int kb, int nrhs, float2* ys, float2* ts,
                                             float2* xs)
{
    for (int t = threadIdx.x; t < NB * NB; t += blockDim.x) ts[(t / NB) * (NB + 1) + t % NB] = Ti[t];
    for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
        const int r = t % NB, q = t / NB;
        xs[t] = r < kb ? x[(int64_t)q * n + k0 + r] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NB * nrhs; t += blockDim.x) {
        const int r = t % NB, q = t / NB;
        float2 acc = make_float2(0.f, 0.f);
        if (r < kb) {
            const int c0 = lower ? 0 : r, c1 = lower ? r : kb - 1;
            const float2* xq = xs + q * NB;
            for (int c = c0; c <= c1; ++c) {
                const float2 v = xq[c];
                if (!kCT) {
                    const float2 l = ts[c * (NB + 1) + r];
                    acc.x += l.x * v.x - l.y * v.y;
                    acc.y += l.x * v.y + l.y * v.x;
                } else {
                    const float2 l = ts[r * (NB + 1) + c];  // conj(T[c][r])
                    acc.x += l.x * v.x + l.y * v.y;
                    acc.y += l.x * v.y - l.y * v.x;
                }
            }
        }
        ys[q * NB + r] = acc;
    }
    __syncthreads();
}

// x_blk = ys, by the block's owner one step later: every CTA of the cluster
// reads x_blk during the step that solves it.
template <int NB>
__device__ __forceinline__ void persist_writeback(float2* __restrict__ x, int64_t n, int64_t k0, int kb, int nrhs,
                                                  const float2* ys)
{
    for (int t = threadIdx.x; t < kb * nrhs; t += blockDim.x) {
        const int r = t % kb, q = t / kb;
        x[(int64_t)q * n + k0 + r] = ys[q * NB + r];
    }
}

// Rows [r0, r1) owned by this CTA: x_i -= sum_t op(M)[i][k0 + t] ys_t.
// Four lanes per row, each loading its NB/4 entries of the row's panel
// segment at once (entries t = lane + 4 s: M[i][k0 + t] down column k0 + t,
// or for the conjugate transpose the NB-long piece of column i), then a
// 2-step shuffle reduction.
template <int NB, bool kCT>
__device__ __forceinline__ void persist_update(const float2* __restrict__ M, float2* __restrict__ x, int64_t n,
                                               int64_t k0, int kb, int nrhs, const float2* ys, int64_t r0,
                                               int64_t r1, int rank)
{
    if (r1 <= r0) return;
    // owned row blocks intersecting [r0, r1): rb = rb0, rb0 + C, ...
    const int64_t first = r0 / NB;
    const int64_t rb0 = first + ((rank - first % kSolveCluster) + kSolveCluster) % kSolveCluster;
    const int64_t nown = rb0 * NB < r1 ? ((r1 - 1) / NB - rb0) / kSolveCluster + 1 : 0;
    constexpr int CQ = NB / 4;
    const int sub = threadIdx.x & 3;
    const int per = blockDim.x >> 2;
    for (int64_t ib = 0; ib < nown * NB; ib += per) {  // uniform trip count (shuffles below)
        const int64_t it = ib + (threadIdx.x >> 2);
        const int64_t i = (rb0 + (it / NB) * kSolveCluster) * NB + it % NB;
        const bool live = it < nown * NB && i >= r0 && i < r1;
        float2 m[CQ];
#pragma unroll
        for (int s = 0; s < CQ; ++s) {
            const int t = sub + 4 * s;
            m[s] = make_float2(0.f, 0.f);
            if (live && t < kb) m[s] = kCT ? M[i * n + k0 + t] : M[(k0 + t) * n + i];
        }
        for (int q0 = 0; q0 < nrhs; q0 += 4) {
            const int nq = min(4, nrhs - q0);
            float ax[4] = {0.f, 0.f, 0.f, 0.f}, ay[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int s = 0; s < CQ; ++s) {
                const int t = sub + 4 * s;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float2 y = ys[(q0 + (q < nq ? q : 0)) * NB + t];
                    if (!kCT) {
                        ax[q] += m[s].x * y.x - m[s].y * y.y;
                        ay[q] += m[s].x * y.y + m[s].y * y.x;
                    } else {  // conj(m) * y
                        ax[q] += m[s].x * y.x + m[s].y * y.y;
                        ay[q] += m[s].x * y.y - m[s].y * y.x;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                ax[q] += __shfl_xor_sync(0xffffffffu, ax[q], 1);
                ay[q] += __shfl_xor_sync(0xffffffffu, ay[q], 1);
                ax[q] += __shfl_xor_sync(0xffffffffu, ax[q], 2);
                ay[q] += __shfl_xor_sync(0xffffffffu, ay[q], 2);
            }
            if (live && sub == 0)
                for (int q = 0; q < nq; ++q) {
                    const float2 v = x[(int64_t)(q0 + q) * n + i];
                    x[(int64_t)(q0 + q) * n + i] = make_float2(v.x - ax[q], v.y - ay[q]);
                }
        }
    }
}

__device__ __forceinline__ void cluster_sync_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

template <int NB, bool kCT>
__global__ void __cluster_dims__(kSolveCluster, 1, 1) __launch_bounds__(kSolveThreads, 2)
k_lu_solve_persist(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
                   int64_t dstride, float2* __restrict__ X, int64_t xstride, int nrhs, const int* done,
                   const int* bad)
{
    extern __shared__ float2 psm[];
    float2* ys[2] = {psm, psm + kMaxRhs * NB};
    float2* xs = psm + 2 * kMaxRhs * NB;
    float2* ts = psm + 3 * kMaxRhs * NB;  // NB x (NB + 1)
    const int64_t b = blockIdx.x / kSolveCluster;
    if (done && (done[b] || bad[b])) return;  // the whole cluster, before any cluster barrier
    const int rank = (int)cluster_rank();
    const float2* M = A + b * stride;
    const float2* Dv = Dinv + b * dstride;
    float2* x = X + b * xstride;
    const int nblk = (int)((n + NB - 1) / NB);
    // first triangle, blocks ascending: L (unit lower) or U^H (lower)
    for (int blk = 0; blk < nblk; ++blk) {
        const int64_t k0 = (int64_t)blk * NB;
        const int kb = (int)min((int64_t)NB, n - k0);
        const float2* Ti = Dv + (int64_t)blk * 2 * NB * NB + (kCT ? NB * NB : 0);
        float2* cur = ys[blk & 1];
        persist_diag<NB, kCT>(Ti, true, x, n, k0, kb, nrhs, cur, ts, xs);
        if (blk > 0 && (blk - 1) % kSolveCluster == rank)  // rows above: untouched this step
            persist_writeback<NB>(x, n, k0 - NB, NB, nrhs, ys[(blk - 1) & 1]);
        persist_update<NB, kCT>(M, x, n, k0, kb, nrhs, cur, k0 + kb, n, rank);
        cluster_sync_all();
    }
    {
        const int blk = nblk - 1;
        const int64_t k0 = (int64_t)blk * NB;
        if (blk % kSolveCluster == rank)
            persist_writeback<NB>(x, n, k0, (int)min((int64_t)NB, n - k0), nrhs, ys[blk & 1]);
        cluster_sync_all();
    }
    // second triangle, blocks descending: U (upper) or L^H (unit upper)
    for (int blk = nblk - 1; blk >= 0; --blk) {
        const int64_t k0 = (int64_t)blk * NB;
        const int kb = (int)min((int64_t)NB, n - k0);
        const float2* Ti = Dv + (int64_t)blk * 2 * NB * NB + (kCT ? 0 : NB * NB);
        const int par = (nblk - 1 - blk) & 1;
        persist_diag<NB, kCT>(Ti, false, x, n, k0, kb, nrhs, ys[par], ts, xs);
        if (blk < nblk - 1 && (blk + 1) % kSolveCluster == rank)  // rows below: untouched this step
            persist_writeback<NB>(x, n, k0 + NB, (int)min((int64_t)NB, n - k0 - NB), nrhs, ys[par ^ 1]);
        persist_update<NB, kCT>(M, x, n, k0, kb, nrhs, ys[par], 0, k0, rank);
        cluster_sync_all();
    }
    if (0 % kSolveCluster == rank) persist_writeback<NB>(x, n, 0, (int)min((int64_t)NB, n), nrhs, ys[(nblk - 1) & 1]);
}

unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// triangular solves with the block-64 factors: flag-synchronised substitution
// ---------------------------------------------------------------------------
//
// One cluster of kFsCluster CTAs per matrix; row block i belongs to CTA
// i mod kFsCluster, which applies to x_i every off-diagonal tile product
// T_ik y_k, in the triangle's order of k, and solves y_i = inv(T_ii) x_i.
// Instead of a barrier after every block, each solved block is published:
// its owner writes y_i over x_i in global memory and then releases a flag
// (per matrix, triangle and block; zeroed before the launch), and the other
// CTAs acquire the flag before reading y_i (from L2, bypassing L1).  The
// owner of the next block in the triangle's order applies the new y_k to
// its block first, solves and publishes it, and only then applies y_k to
// its other blocks, so the sequential chain per block is one 64 x 64 tile
// product, one 64 x 64 inverse product and one flag hand-off, while the
// bulk of the tile products of every CTA overlaps with it.  The blocks of
// one matrix only wait on blocks of the same matrix (same cluster, whose
// CTAs are co-scheduled), and every wait is bounded: a wait that runs out
// records the matrix in `bad`, and the CTA stops waiting (its result is
// then garbage, which the FP64 residual of the refinement rejects).
//
// Tile products: thread (r = tid / 4, tq = tid % 4) holds the 16 entries
// (r, t = 4 j + tq) of a tile in registers, and the four threads of a row
// reduce by shuffles.  kCT selects the
// conjugate-transposed factors: triangle 0 is U^H (tile (i, k) =
// conj(U_ki)^T), triangle 1 is L^H.
constexpr int kFsThreads = 256;
constexpr int kFsCluster = 4;
constexpr int kFsLanes = 4;              // threads per tile row
constexpr int kFsPer = 64 / kFsLanes;    // tile entries per thread
constexpr int kFsPolls = 1 << 15;        // bounded wait for a published block ...
constexpr unsigned kFsSleepNs = 256;     // ... sleeping between polls (~10 ms in all)
constexpr int kFsInjectPolls = 64;       // limit of an injected wait on a flag nothing sets

__device__ __forceinline__ int fs_ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fs_st_release(int* p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ float2 fs_conj(float2 a) { return make_float2(a.x, -a.y); }

// Column t of a tile held by entry j of the thread with lane tq of its row:
// each thread holds the adjacent pairs (t, t + 1), t = 8 (j / 2) + 2 tq, so
// one 16-byte shared load brings the two y entries a pair multiplies.
__device__ __forceinline__ int fs_t(int j, int tq) { return 8 * (j >> 1) + 2 * tq + (j & 1); }

// Entries (r, fs_t(j, tq)), j < kFsPer, of tile (i, k) of the triangle (zero outside the matrix).
template <bool kCT>
__device__ __forceinline__ void fs_load(const float2* __restrict__ M, int64_t n, int i, int k,
                                        float2 (&m)[kFsPer])
{
    constexpr int NB = 64;
    const int r = threadIdx.x / kFsLanes, tq = threadIdx.x % kFsLanes;
    const int64_t i0 = (int64_t)i * NB, k0 = (int64_t)k * NB;
    if (i0 + NB <= n && k0 + NB <= n) {  // the whole tile inside: no checks, one row or column pointer
        if (kCT) {
            const float2* p = M + (i0 + r) * n + k0 + 2 * tq;
#pragma unroll
            for (int j = 0; j < kFsPer; ++j) m[j] = fs_conj(p[8 * (j >> 1) + (j & 1)]);
        } else {
            const float2* p = M + (k0 + 2 * tq) * n + i0 + r;
#pragma unroll
            for (int j = 0; j < kFsPer; ++j) m[j] = p[(int64_t)(8 * (j >> 1) + (j & 1)) * n];
        }
        return;
    }
    const bool rok = i0 + r < n;
#pragma unroll
    for (int j = 0; j < kFsPer; ++j) {
        const int t = fs_t(j, tq);
        m[j] = make_float2(0.f, 0.f);
        if (rok && k0 + t < n) m[j] = kCT ? fs_conj(M[(i0 + r) * n + k0 + t]) : M[(k0 + t) * n + i0 + r];
    }
}

// The same entries of the inverse diagonal block (column-major; conjugate-transposed for kCT).
template <bool kCT>
__device__ __forceinline__ void fs_load_inv(const float2* __restrict__ Inv, float2 (&iv)[kFsPer])
{
    constexpr int NB = 64;
    const int r = threadIdx.x / kFsLanes, tq = threadIdx.x % kFsLanes;
#pragma unroll
    for (int j = 0; j < kFsPer; ++j) {
        const int t = fs_t(j, tq);
        iv[j] = kCT ? fs_conj(Inv[r * NB + t]) : Inv[t * NB + r];
    }
}

// A staged 64 x 64 block: column-major, columns padded to kFsLd entries (an
// unpadded column would put the four lanes of a row on one bank).
constexpr int kFsLd = 68;
constexpr size_t kFsStageBytes = sizeof(float2) * 64 * kFsLd;

// Rows row0 .. row0 + 63, columns col0 .. col0 + 63 of the column-major
// matrix src (leading dimension ld, both extents lim) into dst by 8-byte
// cp.async (8 bytes keep any ld aligned); entries outside are zero-filled
// (source size 0, with the in-range address src).
__device__ __forceinline__ void fs_stage(float2* dst, const float2* __restrict__ src, int64_t ld, int64_t row0,
                                         int64_t col0, int64_t lim)
{
    for (int e = threadIdx.x; e < 64 * 64; e += kFsThreads) {
        const int c = e / 64, rr = e % 64;
        const bool ok = row0 + rr < lim && col0 + c < lim;
        const float2* g = ok ? src + (col0 + c) * ld + row0 + rr : src;
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;"
                     :: "r"(smem_u32(dst + c * kFsLd + rr)), "l"(g), "r"(ok ? 8 : 0) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void fs_stage_wait() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The entries fs_load / fs_load_inv give, from a block staged by fs_stage
// (at (i0, k0) of the factors, or (k0, i0) for kCT; the inverse at (0, 0)),
// columns LD entries apart.
template <bool kCT, int LD = kFsLd>
__device__ __forceinline__ void fs_from_stage(const float2* s, float2 (&m)[kFsPer])
{
    const int r = threadIdx.x / kFsLanes, tq = threadIdx.x % kFsLanes;
#pragma unroll
    for (int j = 0; j < kFsPer; ++j) {
        const int t = fs_t(j, tq);
        m[j] = kCT ? fs_conj(s[r * LD + t]) : s[t * LD + r];
    }
}

// Two adjacent y entries (16 bytes of shared memory).  Volatile, so that it
// stays inside the tile loop: held in registers across tiles, a thread's 16
// entries of up to four right-hand sides would not fit beside the tiles.
__device__ __forceinline__ float4 fs_lds4(const float2* p)
{
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(smem_u32(p)) : "memory");
    return v;
}

// Row r of (tile m) (src columns q0 .. q0 + nq), summed over the row's lanes
// (every lane of the row ends with the sum).  src: shared memory, rows
// 16-byte aligned.
__device__ __forceinline__ void fs_rowdot(const float2 (&m)[kFsPer], const float2 (*src)[64], int q0, int nq,
                                          float (&ax)[4], float (&ay)[4])
{
    const int tq = threadIdx.x % kFsLanes;
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) ax[qq] = ay[qq] = 0.f;
#pragma unroll
    for (int j = 0; j < kFsPer; j += 2) {
#pragma unroll
        for (int qq = 0; qq < 4; ++qq) {
            if (qq < nq) {
                const float4 v = fs_lds4(&src[q0 + qq][fs_t(j, tq)]);
                const float2 a = m[j], b = m[j + 1];
                ax[qq] += a.x * v.x - a.y * v.y;
                ay[qq] += a.x * v.y + a.y * v.x;
                ax[qq] += b.x * v.z - b.y * v.w;
                ay[qq] += b.x * v.w + b.y * v.z;
            }
        }
    }
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) {
#pragma unroll
        for (int o = 1; o < kFsLanes; o <<= 1) {
            ax[qq] += __shfl_xor_sync(0xffffffffu, ax[qq], o);
            ay[qq] += __shfl_xor_sync(0xffffffffu, ay[qq], o);
        }
    }
}

// x_i -= T_ik y for the tile held in m; entry (q, r) of block i at
// xb[q * xq + r] (global memory or the CTA's shared copy).  NQ > 0: exactly
// NQ (<= 4) right-hand sides, known at compile time; 0: nrhs of them.
template <int NQ>
__device__ __forceinline__ void fs_apply(const float2 (&m)[kFsPer], int64_t n, int i, float2* xb, int64_t xq,
                                         const float2 (*y)[64], int nrhs)
{
    const int r = threadIdx.x / kFsLanes, tq = threadIdx.x % kFsLanes;
    const int64_t row = (int64_t)i * 64 + r;
    const int nr = NQ ? NQ : nrhs;
    for (int q0 = 0; q0 < nr; q0 += 4) {
        const int nq = NQ ? NQ : min(4, nrhs - q0);
        float ax[4], ay[4];
        fs_rowdot(m, y, q0, nq, ax, ay);
        if (tq == 0 && row < n)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                if (qq < nq) {
                    float2* p = xb + (q0 + qq) * xq + r;
                    const float2 v = *p;
                    *p = make_float2(v.x - ax[qq], v.y - ay[qq]);
                }
            }
    }
}

// y_i = inv(T_ii) v (v complete in vs, inverse entries in iv), into ynext and
// over x_i; then publish.  vs may be the CTA's shared copy of block i.
template <int NQ>
__device__ __forceinline__ void fs_solve_publish(const float2 (&iv)[kFsPer], int64_t n, int i, float2* x,
                                                 const float2 (*vs)[64], float2 (*ynext)[64], int nrhs, int* flag)
{
    const int r = threadIdx.x / kFsLanes, tq = threadIdx.x % kFsLanes;
    const int64_t i0 = (int64_t)i * 64;
    const bool rok = i0 + r < n;
    const int nr = NQ ? NQ : nrhs;
    for (int q0 = 0; q0 < nr; q0 += 4) {
        const int nq = NQ ? NQ : min(4, nrhs - q0);
        float ax[4], ay[4];
        fs_rowdot(iv, vs, q0, nq, ax, ay);
        if (tq == 0)
#pragma unroll
            for (int qq = 0; qq < 4; ++qq) {
                if (qq < nq) {
                    const float2 v = rok ? make_float2(ax[qq], ay[qq]) : make_float2(0.f, 0.f);
                    ynext[q0 + qq][r] = v;
                    if (rok) x[(int64_t)(q0 + qq) * n + i0 + r] = v;
                }
            }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        fs_st_release(flag, 1);
    }
}

// kXS: the x entries of the CTA's own blocks live in shared memory (dynamic,
// ceil(nblk / kFsCluster) * nrhs * 64 entries) from the start to the end of
// the kernel, so the tile products update them without global round trips;
// each solved block is still written to global memory when published.
// NQ > 0: exactly NQ right-hand sides (<= 4), known at compile time; 0: nrhs.
template <bool kCT, bool kXS, int NQ>
__global__ void __cluster_dims__(kFsCluster, 1, 1) __launch_bounds__(kFsThreads, 2)
k_lu_solve_flags(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
                 int64_t dstride, float2* X, int64_t xstride, int nrhs, int* flags, int* bad, int stage,
                 const int* done, const int* unset_flag)
{
    constexpr int NB = 64;
    __shared__ __align__(16) float2 ys[2][kMaxRhs][NB];  // y of the block being applied and of the next one
    __shared__ __align__(16) float2 vs[kMaxRhs][NB];     // x of the block being solved (global x)
    __shared__ int s_fail;
    extern __shared__ __align__(16) float2 xs_smem[];  // kXS: [own block][nrhs][NB]; then, if stage, two staged blocks
    const int64_t b = blockIdx.x / kFsCluster;
    // a matrix whose refinement converged, or that is marked bad, is left
    // alone (every CTA of its cluster returns here, before any barrier)
    if (done && (done[b] || bad[b])) return;
    const int rank = (int)cluster_rank();
    const float2* M = A + b * stride;
    const float2* Dv = Dinv + b * dstride;
    float2* x = X + b * xstride;
    const int nblk = (int)((n + NB - 1) / NB);
    int* fl = flags + b * 2 * nblk;
    const int tid = threadIdx.x;
    if (NQ) nrhs = NQ;
    // block i's entries (q, r) at xblk(i)[q * xq + r]
    const int64_t xq = kXS ? NB : n;
    auto xblk = [&](int i) -> float2* {
        return kXS ? xs_smem + (int64_t)(i / kFsCluster) * nrhs * NB : x + (int64_t)i * NB;
    };
    // the next block's tile and inverse diagonal block, staged during the wait for y_k
    float2* st_tile = xs_smem + (kXS ? (int64_t)((nblk + kFsCluster - 1) / kFsCluster) * nrhs * NB : 0);
    float2* st_inv = st_tile + NB * kFsLd;
    if (tid == 0) s_fail = 0;
    if (kXS) {
        for (int i = rank; i < nblk; i += kFsCluster) {
            float2* xb = xblk(i);
            const int64_t i0 = (int64_t)i * NB;
            for (int e = tid; e < nrhs * NB; e += blockDim.x) {
                const int q = e / NB, rr = e % NB;
                xb[q * NB + rr] = i0 + rr < n ? x[(int64_t)q * n + i0 + rr] : make_float2(0.f, 0.f);
            }
        }
    }
    __syncthreads();
    for (int tri = 0; tri < 2; ++tri) {
        const bool fwd = tri == 0;
        // inverse diagonal blocks: inv(L11) at offset 0, inv(U11) at NB * NB
        const int inv_off = (fwd != kCT) ? 0 : NB * NB;
        int* tfl = fl + tri * nblk;
        const int k_first = fwd ? 0 : nblk - 1;
        // solve block i from its complete x (shared copy or staged) with its
        // inverse diagonal block iv, publish, keep y in ynext
        auto solve_own = [&](int i, float2 (*ynext)[NB], const float2 (&iv)[kFsPer]) {
            const float2 (*src)[NB] = vs;
            if (kXS) {
                src = reinterpret_cast<const float2 (*)[NB]>(xblk(i));
            } else {
                const int64_t f0 = (int64_t)i * NB;
                for (int e = tid; e < nrhs * NB; e += blockDim.x) {
                    const int q = e / NB, rr = e % NB;
                    vs[q][rr] = f0 + rr < n ? x[(int64_t)q * n + f0 + rr] : make_float2(0.f, 0.f);
                }
            }
            __syncthreads();
            fs_solve_publish<NQ>(iv, n, i, x, src, ynext, nrhs, tfl + i);
            if (kXS) {  // the solved block becomes the next triangle's right-hand side
                float2* xb = xblk(i);
                for (int e = tid; e < nrhs * NB; e += blockDim.x) xb[e] = ynext[e / NB][e % NB];
            }
        };
        if (k_first % kFsCluster == rank) {
            float2 iv[kFsPer];
            fs_load_inv<kCT>(Dv + (int64_t)k_first * 2 * NB * NB + inv_off, iv);
            solve_own(k_first, ys[0], iv);
        }
        for (int p = 0; p < nblk; ++p) {
            const int k = fwd ? p : nblk - 1 - p;
            const int kn = fwd ? k + 1 : k - 1;
            const bool next_mine = p + 1 < nblk && kn % kFsCluster == rank;
            float2 (*y)[NB] = ys[p & 1];
            // the next block's tile (kn, k) and inverse diagonal block do not
            // depend on y_k: with stage, they are copied into shared memory
            // during the wait for it, so the hand-off chain holds no
            // global-memory round trip but y_k's
            if (next_mine && stage) {
                const int64_t a0 = (int64_t)(kCT ? k : kn) * NB, b0 = (int64_t)(kCT ? kn : k) * NB;
                fs_stage(st_tile, M, n, a0, b0, n);
                fs_stage(st_inv, Dv + (int64_t)kn * 2 * NB * NB + inv_off, NB, 0, 0, NB);
            }
            if (k % kFsCluster != rank) {
                if (tid == 0 && !s_fail) {
                    // failure injection: wait on a flag that nothing publishes,
                    // with a short limit, so the wait expires
                    const int* wf = unset_flag ? unset_flag : tfl + k;
                    const int limit = unset_flag ? kFsInjectPolls : kFsPolls;
                    int it = 0;
                    while (fs_ld_acquire(wf) == 0 && ++it < limit) __nanosleep(kFsSleepNs);
                    if (it >= limit) {
                        s_fail = 1;
                        atomicExch(bad + b, 3);
                    }
                }
                __syncthreads();
                const int64_t k0 = (int64_t)k * NB;
                for (int e = tid; e < nrhs * NB; e += blockDim.x) {
                    const int q = e / NB, rr = e % NB;
                    y[q][rr] = k0 + rr < n ? __ldcg(x + (int64_t)q * n + k0 + rr) : make_float2(0.f, 0.f);
                }
            }
            if (next_mine && stage) fs_stage_wait();
            __syncthreads();
            if (next_mine) {  // the next block first: apply y_k to it, solve, publish
                float2 m[kFsPer];
                if (stage) fs_from_stage<kCT>(st_tile, m);
                else fs_load<kCT>(M, n, kn, k, m);
                fs_apply<NQ>(m, n, kn, xblk(kn), xq, y, nrhs);
                float2 iv[kFsPer];
                if (stage) fs_from_stage<kCT>(st_inv, iv);
                else fs_load_inv<kCT>(Dv + (int64_t)kn * 2 * NB * NB + inv_off, iv);
                solve_own(kn, ys[(p + 1) & 1], iv);
            }
            // the rest of this CTA's blocks after kn in the triangle's order, two tiles in flight
            int q = p + 2;
            while (q < nblk && (fwd ? q : nblk - 1 - q) % kFsCluster != rank) ++q;
            for (; q < nblk; q += 2 * kFsCluster) {
                const int i1 = fwd ? q : nblk - 1 - q;
                const int q2 = q + kFsCluster;
                const int i2 = fwd ? q2 : nblk - 1 - q2;
                float2 m1[kFsPer], m2[kFsPer];
                fs_load<kCT>(M, n, i1, k, m1);
                if (q2 < nblk) fs_load<kCT>(M, n, i2, k, m2);
                fs_apply<NQ>(m1, n, i1, xblk(i1), xq, y, nrhs);
                if (q2 < nblk) fs_apply<NQ>(m2, n, i2, xblk(i2), xq, y, nrhs);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// streamed triangular solves: left-looking, operands streamed ahead
// ---------------------------------------------------------------------------
//
// The triangles, block ownership (block i to CTA i mod kFsCluster of the
// matrix's cluster) and published flags of k_lu_solve_flags, with the work
// of each block gathered on its owner (left-looking): x_i = b_i - sum_j
// T_ij y_j accumulates in registers over the blocks j before i in the
// triangle's order, then y_i = inv(T_ii) x_i is written over x_i and
// published.  Every operand a CTA reads is known in advance (its blocks'
// tiles in order, each block followed by its inverse diagonal block), so
// two producer warps stream them through a ring of kSsStages shared-memory
// stages while eight consumer warps multiply: the tile warp copies each tile
// (64 columns of up to 512 bytes, one column per warp instruction of 16-byte
// cp.async) as soon as its stage is free, one lane of the y warp adds the
// y_j the tile multiplies (cp.async.bulk) once y_j's flag is published
// (separate warps: a lane spinning on a flag would hold up the tile copies
// of its warp; 16-byte copies: 64 bulk copies of 512 bytes per tile kept
// the SM's bulk-copy unit from streaming at the memory's rate).  The tile
// stream thus runs ahead of the flag chain, whose step is one copy of a
// published y_j, one tile product and one inverse product.
// Needs n even (16-byte aligned columns) and one to four right-hand sides;
// the launcher uses k_lu_solve_flags otherwise.  Stage waits and flag waits
// are bounded: a flag wait that runs out marks the matrix (3) and the
// kernel finishes with garbage for it; a stage wait that runs out marks it
// (2).  Failure injection (unset_flag) as k_lu_solve_flags.
constexpr int kSsStages = 3;
constexpr int kSsLd = 66;  // staged column stride in float2: the consumers' reads are bank-conflict-free
constexpr uint32_t kSsTileBytes = 64 * kSsLd * sizeof(float2);
constexpr uint32_t kSsYBytes = 4 * 64 * sizeof(float2);  // y_j of up to four right-hand sides
constexpr uint32_t kSsStageBytes = kSsTileBytes + kSsYBytes;
constexpr int kSsConsumers = 256;
constexpr int kSsThreads = kSsConsumers + 64;  // eight consumer warps, the tile warp and the y warp
constexpr size_t kSsSmemBytes = (size_t)kSsStages * kSsStageBytes + kSsYBytes;  // + x_i of the block being solved
constexpr uint32_t kSsWaitNs = 50000000;   // bounded stage waits: 50 ms of the global timer (a poll may
constexpr uint32_t kSsWaitHintNs = 1000;    // return before its suspend hint, so the bound is in time) ...
constexpr int kSsFlagPolls = 1 << 17;     // ... and flag waits (> 8 ms), as long as k_lu_solve_flags' flag waits

__device__ __forceinline__ void ss_bar_init(uint64_t* bar, int count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool ss_wait(uint64_t* bar, uint32_t phase)
{
    const uint32_t a = smem_u32(bar);
    uint32_t t0;  // the timer's low word: differences are exact across its 4.3 s wrap
    asm volatile("mov.u32 %0, %%globaltimer_lo;" : "=r"(t0));
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(phase), "r"(kSsWaitHintNs)
            : "memory");
        if (ok) return true;
        uint32_t t;
        asm volatile("mov.u32 %0, %%globaltimer_lo;" : "=r"(t));
        if (t - t0 > kSsWaitNs) return false;
    }
}

__device__ __forceinline__ void ss_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void ss_arrive_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void ss_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void ss_consumer_sync()
{
    asm volatile("bar.sync 1, %0;" :: "r"(kSsConsumers) : "memory");
}

// The blocks of CTA `rank` in the order of triangle `tri` (0: ascending,
// 1: descending): count and the bi-th one.
__device__ __forceinline__ int ss_nown(int nblk, int rank)
{
    return rank < nblk ? (nblk - 1 - rank) / kFsCluster + 1 : 0;
}

__device__ __forceinline__ int ss_own(int tri, int nblk, int rank, int bi)
{
    return tri == 0 ? rank + kFsCluster * bi : rank + kFsCluster * (ss_nown(nblk, rank) - 1 - bi);
}

// Tiles of block i (the blocks before it in the triangle's order) and the jj-th of them.
__device__ __forceinline__ int ss_ntiles(int tri, int nblk, int i) { return tri == 0 ? i : nblk - 1 - i; }
__device__ __forceinline__ int ss_tile_j(int tri, int nblk, int jj) { return tri == 0 ? jj : nblk - 1 - jj; }

// x_i -= T_ij y_j for one staged tile, as partial sums of row r over the
// thread's 16 columns (reduced over the row's lanes once per block).  kMask:
// a tile at the matrix's edge, whose rows past the end (!rok) and columns
// from jlim on are stale shared memory and count as zero (n even: columns c
// and c + 1 are valid together).
template <bool kCT, int NQ, bool kMask>
__device__ inline void ss_tile(const float2* __restrict__ st, const float2 (*__restrict__ ys)[64], int r,
                                        int tq, bool rok, int jlim, float (&ax)[4], float (&ay)[4])
{
    // one pair of tile entries at a time (columns c, c + 1): few registers
    // live, so the consumer warps fit the two-CTA register budget unspilled
#pragma unroll
    for (int e = 0; e < kFsPer; e += 2) {
        const int c = fs_t(e, tq);
        float2 a = kCT ? fs_conj(st[r * kSsLd + c]) : st[c * kSsLd + r];
        float2 a2 = kCT ? fs_conj(st[r * kSsLd + c + 1]) : st[(c + 1) * kSsLd + r];
        if (kMask && !(rok && c < jlim)) a = a2 = make_float2(0.f, 0.f);  // n even: c, c + 1 together
#pragma unroll
        for (int qq = 0; qq < NQ; ++qq) {
            float4 v = fs_lds4(&ys[qq][c]);  // volatile: the loads stay in the loop, beside their FMAs
            if (kMask && c >= jlim) v = make_float4(0.f, 0.f, 0.f, 0.f);
            ax[qq] = fmaf(a.x, v.x, ax[qq]);
            ax[qq] = fmaf(-a.y, v.y, ax[qq]);
            ay[qq] = fmaf(a.x, v.y, ay[qq]);
            ay[qq] = fmaf(a.y, v.x, ay[qq]);
            ax[qq] = fmaf(a2.x, v.z, ax[qq]);
            ax[qq] = fmaf(-a2.y, v.w, ax[qq]);
            ay[qq] = fmaf(a2.x, v.w, ay[qq]);
            ay[qq] = fmaf(a2.y, v.z, ay[qq]);
        }
    }
}

template <bool kCT, int NQ>
__global__ void __cluster_dims__(kFsCluster, 1, 1) __launch_bounds__(kSsThreads, 2)
k_lu_solve_stream(const float2* __restrict__ A, int64_t n, int64_t stride, const float2* __restrict__ Dinv,
                  int64_t dstride, float2* X, int64_t xstride, int* flags, int* bad, const int* done,
                  const int* unset_flag)
{
    constexpr int NB = 64;
    extern __shared__ __align__(128) unsigned char ss_smem[];
    __shared__ uint64_t full[kSsStages], empty[kSsStages];
    const int64_t b = blockIdx.x / kFsCluster;
    // a matrix whose refinement converged, or that is marked bad, is left
    // alone (every CTA of its cluster returns here, before any barrier)
    if (done && (done[b] || bad[b])) return;
    const int rank = (int)cluster_rank();
    const float2* M = A + b * stride;
    const float2* Dv = Dinv + b * dstride;
    float2* x = X + b * xstride;
    const int nblk = (int)((n + NB - 1) / NB);
    int* fl = flags + b * 2 * nblk;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nown = ss_nown(nblk, rank);
    auto stage = [&](int s) { return reinterpret_cast<float2*>(ss_smem + (size_t)s * kSsStageBytes); };
    auto ystage = [&](int s) {
        return reinterpret_cast<float2(*)[NB]>(ss_smem + (size_t)s * kSsStageBytes + kSsTileBytes);
    };
    auto xs = reinterpret_cast<float2(*)[NB]>(ss_smem + (size_t)kSsStages * kSsStageBytes);
    if (tid == 0) {
        for (int s = 0; s < kSsStages; ++s) {
            ss_bar_init(&full[s], 33);                      // the tile warp's lanes and the y lane
            ss_bar_init(&empty[s], kSsConsumers / 32);      // every consumer warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp >= kSsConsumers / 32) {  // producer warps
        if (warp == kSsConsumers / 32) {  // tiles
            int t = 0;
            for (int tri = 0; tri < 2; ++tri) {
                const int inv_off = ((tri == 0) != kCT) ? 0 : NB * NB;
                for (int bi = 0; bi < nown; ++bi) {
                    const int i = ss_own(tri, nblk, rank, bi);
                    const int nt = ss_ntiles(tri, nblk, i);
                    for (int jj = 0; jj <= nt; ++jj, ++t) {
                        const int s = t % kSsStages;
                        // lane 0 waits for the stage; the other lanes write into it after
                        if (t >= kSsStages && lane == 0 && !ss_wait(&empty[s], (uint32_t)((t / kSsStages - 1) & 1)))
                            atomicExch(bad + b, 2);
                        __syncwarp();
                        const float2* src;
                        int64_t ld;
                        int ncol, nrow;
                        if (jj < nt) {  // tile (i, j): rows of block i and columns of block j (kCT: transposed)
                            const int64_t i0 = (int64_t)i * NB, j0 = (int64_t)ss_tile_j(tri, nblk, jj) * NB;
                            const int64_t r0 = kCT ? j0 : i0, c0 = kCT ? i0 : j0;
                            src = M + c0 * n + r0;
                            ld = n;
                            ncol = (int)min((int64_t)NB, n - c0);
                            nrow = (int)min((int64_t)NB, n - r0);
                        } else {  // inverse diagonal block of i (full 64 x 64, column-major)
                            src = Dv + (int64_t)i * 2 * NB * NB + inv_off;
                            ld = NB;
                            ncol = NB;
                            nrow = NB;
                        }
                        // one 16-byte cp.async per lane and column: a column (512 bytes)
                        // per warp instruction; each lane's arrival on the stage's
                        // barrier fires when its copies have landed
                        if (2 * lane < nrow) {
                            const float2* sp = src + 2 * lane;
                            const uint32_t dp = smem_u32(stage(s) + 2 * lane);
#pragma unroll 8
                            for (int c = 0; c < ncol; ++c)
                                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;"
                                             :: "r"(dp + (uint32_t)(c * kSsLd * sizeof(float2))), "l"(sp + c * ld)
                                             : "memory");
                        }
                        asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];"
                                     :: "r"(smem_u32(&full[s])) : "memory");
                    }
                }
            }
        } else if (lane == 0) {  // y
            int t = 0;
            bool gave_up = false;
            // flags already acquired: the blocks of a triangle are needed in its
            // order (block i takes j = 0 .. i - 1, or nblk - 1 .. i + 1), so the
            // acquired ones form a prefix (seen_f) or a suffix (seen_b)
            int seen_f = 0, seen_b = nblk;
            for (int tri = 0; tri < 2; ++tri) {
                for (int bi = 0; bi < nown; ++bi) {
                    const int i = ss_own(tri, nblk, rank, bi);
                    const int nt = ss_ntiles(tri, nblk, i);
                    for (int jj = 0; jj <= nt; ++jj, ++t) {
                        const int s = t % kSsStages;
                        if (t >= kSsStages && !ss_wait(&empty[s], (uint32_t)((t / kSsStages - 1) & 1)))
                            atomicExch(bad + b, 2);
                        if (jj == nt) {  // the inverse item carries no y
                            ss_arrive(&full[s]);
                            continue;
                        }
                        const int j = ss_tile_j(tri, nblk, jj);
                        const bool known = tri == 0 ? j < seen_f : j >= seen_b;
                        if (!known && !gave_up) {
                            // failure injection: a wait on another CTA's block waits
                            // on a flag that nothing publishes, with a short limit
                            const bool inject = unset_flag && j % kFsCluster != rank;
                            const int* wf = inject ? unset_flag : fl + tri * nblk + j;
                            const int limit = inject ? kFsInjectPolls : kSsFlagPolls;
                            int it = 0;
                            while (fs_ld_acquire(wf) == 0 && ++it < limit) __nanosleep(64);
                            if (it >= limit) {
                                gave_up = true;  // later flags are not waited for: the matrix is garbage now
                                atomicExch(bad + b, 3);
                            }
                            if (tri == 0 && j == seen_f) ++seen_f;
                            if (tri == 1 && j == seen_b - 1) --seen_b;
                            // the y_j just acquired was written by generic stores:
                            // order the bulk copies that read it after the acquire
                            asm volatile("fence.proxy.async.global;" ::: "memory");
                        }
                        const int64_t j0 = (int64_t)j * NB;
                        const int nrow = (int)min((int64_t)NB, n - j0);
                        ss_arrive_tx(&full[s], (uint32_t)(NQ * nrow * sizeof(float2)));
#pragma unroll
                        for (int q = 0; q < NQ; ++q)
                            ss_copy(ystage(s)[q], x + (int64_t)q * n + j0, (uint32_t)(nrow * sizeof(float2)),
                                    &full[s]);
                    }
                }
            }
        }
        return;
    }
    // consumer warps: thread (r, tq) holds entries (r, fs_t(jj, tq)) of each tile
    const int r = tid / kFsLanes, tq = tid % kFsLanes;
    int t = 0;
    bool ok = true;
    auto take = [&](int s) {
        if (!ss_wait(&full[s], (uint32_t)((t / kSsStages) & 1)) && ok) {
            ok = false;
            if (lane == 0) atomicExch(bad + b, 2);
        }
    };
    auto give = [&](int s) {
        __syncwarp();
        if (lane == 0) ss_arrive(&empty[s]);
        ++t;
    };
    for (int tri = 0; tri < 2; ++tri) {
        for (int bi = 0; bi < nown; ++bi) {
            const int i = ss_own(tri, nblk, rank, bi);
            const int nt = ss_ntiles(tri, nblk, i);
            const int64_t i0 = (int64_t)i * NB;
            const bool rok = i0 + r < n;
            float ax[4] = {0.f, 0.f, 0.f, 0.f}, ay[4] = {0.f, 0.f, 0.f, 0.f};
            for (int jj = 0; jj < nt; ++jj) {
                const int s = t % kSsStages;
                const int64_t j0 = (int64_t)ss_tile_j(tri, nblk, jj) * NB;
                take(s);
                if (i0 + NB <= n && j0 + NB <= n)  // the whole tile inside the matrix: no masks
                    ss_tile<kCT, NQ, false>(stage(s), ystage(s), r, tq, true, NB, ax, ay);
                else
                    ss_tile<kCT, NQ, true>(stage(s), ystage(s), r, tq, rok, (int)min((int64_t)NB, n - j0), ax, ay);
                give(s);
            }
#pragma unroll
            for (int qq = 0; qq < NQ; ++qq) {
#pragma unroll
                for (int o = 1; o < kFsLanes; o <<= 1) {
                    ax[qq] += __shfl_xor_sync(0xffffffffu, ax[qq], o);
                    ay[qq] += __shfl_xor_sync(0xffffffffu, ay[qq], o);
                }
            }
            // x_i = b_i - sum_j T_ij y_j, rows outside the matrix zero
            if (tq == 0) {
#pragma unroll
                for (int qq = 0; qq < NQ; ++qq) {
                    float2 v = make_float2(0.f, 0.f);
                    if (rok) {
                        const float2 bv = __ldcg(x + (int64_t)qq * n + i0 + r);
                        v = make_float2(bv.x - ax[qq], bv.y - ay[qq]);
                    }
                    xs[qq][r] = v;
                }
            }
            ss_consumer_sync();
            // y_i = inv(T_ii) x_i, over x_i; then publish
            const int s = t % kSsStages;
            take(s);
            float bx[4] = {0.f, 0.f, 0.f, 0.f}, by[4] = {0.f, 0.f, 0.f, 0.f};
            ss_tile<kCT, NQ, false>(stage(s), xs, r, tq, true, NB, bx, by);  // the inverse block: a whole tile
            give(s);
#pragma unroll
            for (int qq = 0; qq < NQ; ++qq) {
#pragma unroll
                for (int o = 1; o < kFsLanes; o <<= 1) {
                    bx[qq] += __shfl_xor_sync(0xffffffffu, bx[qq], o);
                    by[qq] += __shfl_xor_sync(0xffffffffu, by[qq], o);
                }
            }
            if (tq == 0 && rok) {
#pragma unroll
                for (int qq = 0; qq < NQ; ++qq) x[(int64_t)qq * n + i0 + r] = make_float2(bx[qq], by[qq]);
            }
            ss_consumer_sync();
            if (tid == 0) {
                __threadfence();
                fs_st_release(fl + tri * nblk + i, 1);
            }
        }
    }
}

}  // namespace

int64_t lu_dinv_stride_tc(int64_t n) { return ((n + TC_NB - 1) / TC_NB) * 2 * TC_NB * TC_NB; }

namespace {
// Test matrices of the LU autotuner: 1/2 on the diagonal plus off-diagonal
// entries of modulus <= 0.3 / n from a hash of (matrix, row, column), so
// every matrix is strictly diagonally dominant (no pivoting needed).
__global__ void k_fill_lu_test(float2* __restrict__ A, int64_t n, int64_t count)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int64_t e = t % (n * n);
    const int64_t i = e % n, j = e / n;
    uint64_t h = (uint64_t)t * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    const float u = (float)(h & 0xFFFFFF) / 16777216.f - 0.5f;
    const float v = (float)((h >> 24) & 0xFFFFFF) / 16777216.f - 0.5f;
    const float s = 0.4f / (float)n;
    A[t] = i == j ? make_float2(0.5f, 0.f) : make_float2(s * u, s * v);
}
}  // namespace

cudaError_t launch_fill_lu_test(mh_ctx* ctx, float2* A, int64_t n, int nbatch)
{
    const int64_t count = n * n * nbatch;
    k_fill_lu_test<<<(unsigned)((count + 255) / 256), 256, 0, ctx->stream>>>(A, n, count);
    ctx->launches += 1;
    return cudaGetLastError();
}

// Panel buffers per matrix: the panel pairs of an outer step stay live while
// its interior update runs, and the next outer step writes the other set
// (2 x the outer step's panels, sized for the widest schedule).
constexpr int kOuterMax = 8;  // 64-column panels per outer step, at most (512 columns)
// After them, the packed TRSM B operands of every diagonal block (two images each).
int64_t lu_panel_bytes_tc(int64_t n)
{
    return 2 * kOuterMax * ((n + TC_TM - 1) / TC_TM) * (int64_t)(kPanelL + kPanelU) +
           ((n + TC_NB - 1) / TC_NB) * 2 * (int64_t)kTrsmBImage;
}

// Blocked LU in outer steps of op 64-column panels (op even: 2 to 8, i.e.
// 128 to 512 columns; op = 4 by default), with look-ahead.  Outer step K0
// (tile T0 = K0 / 128), on the main
// (high-priority) stream: for each panel k = K0 + 64 s, its TRSM, then (but
// for the last) the update of the tile row and column holding the next
// panel (an L of width 1, rows and columns >= k + 64) -- with this panel
// when the next one is in the same tile, else with all the outer step's
// panels so far (the next tile's first update in this outer step) -- and
// the next diagonal block; then the
// trailing tiles (>= T0 + op/2) are updated once with all op panel pairs
// accumulated in TMEM (K = 64 op complex): their first op/2 tile rows and
// columns on the main stream, the interior concurrently on the side
// (low-priority) stream, then the next diagonal block.  The trailing matrix
// is read and written once per outer step.  An outer step's trailing
// update waits for the previous interior; everything before it only touches
// tile rows and columns T0 .. T0 + op/2 - 1, which that interior does not.
namespace {
// The schedule above for nbatch matrices on one (main, side) stream pair;
// panels: lu_panel_bytes_tc(n) * nbatch bytes for these matrices.
cudaError_t lu_tc_group(mh_ctx* ctx, float2* A, int64_t n, int64_t stride, int nbatch, float2* Dinv,
                        unsigned char* panels, int* bad, const LuStreams& st, const int op, const int update)
{
    auto* upd = update ? k_lu_update_tc_acc : k_lu_update_tc;
    cudaError_t e;
    cudaStream_t main_s = st.main, side_s = st.side, strip_s = st.strip;
    const int64_t dstride = lu_dinv_stride_tc(n);
    const int64_t pstride = (int64_t)((n + TC_TM - 1) / TC_TM) * (kPanelL + kPanelU);  // one buffer, per matrix
    const int64_t bstride = ((n + TC_NB - 1) / TC_NB) * 2 * (int64_t)kTrsmBImage;       // B images, per matrix
    unsigned char* bimg = panels + 2 * kOuterMax * pstride * nbatch;
    const int ntiles = (int)((n + TC_TM - 1) / TC_TM);
    const unsigned nbz = (unsigned)nbatch;
    const int kW = op / 2;  // tiles per outer step
    if ((e = cudaEventRecord(st.ev_side, side_s)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(st.ev_strip_done, strip_s)) != cudaSuccess) return e;
    // An L of the trailing matrix (mode 1 at tile t0, width w) updated with
    // the panel pairs q: its diagonal tile (t0, t0), which holds the next
    // diagonal block, on the main stream; the rest on the strip stream,
    // concurrently with the next diagonal-block factorisation; the next panel
    // solve waits for it (strip_join).
    auto strip = [&](int t0, int nt, int w, const PanelPairs& q, int np, int64_t lo) -> cudaError_t {
        cudaError_t e2;
        upd<<<dim3(1, 1, nbz), 128, kTcSmemBytes, main_s>>>(A, n, stride, t0, nt, 1, w, q, np, pstride, lo, bad, 0);
        ctx->launches += 1;
        const int rest = w * (2 * nt - w) - 1;
        if (rest > 0) {
            if ((e2 = cudaEventRecord(st.ev_strip_go, main_s)) != cudaSuccess) return e2;
            if ((e2 = cudaStreamWaitEvent(strip_s, st.ev_strip_go, 0)) != cudaSuccess) return e2;
            upd<<<dim3(rest, 1, nbz), 128, kTcSmemBytes, strip_s>>>(A, n, stride, t0, nt, 1, w, q, np, pstride, lo,
                                                                    bad, 1);
            ctx->launches += 1;
            if ((e2 = cudaEventRecord(st.ev_strip_done, strip_s)) != cudaSuccess) return e2;
        }
        return cudaGetLastError();
    };
    auto strip_join = [&]() { return cudaStreamWaitEvent(main_s, st.ev_strip_done, 0); };
    k_lu_diag64<<<nbatch, kDiag64Threads, kDiag64Smem, main_s>>>(A, n, stride, 0, Dinv, dstride, bad, bimg,
                                                                   bstride);
    ctx->launches += 1;
    int outer = 0;
    PanelPairs prev;  // the previous outer step's panels (their update of this step's tiles past the first is deferred)
    int nprev = 0;
    for (int64_t K0 = 0; K0 < n; K0 += op * TC_NB, ++outer) {
        const int T0 = (int)(K0 / TC_TM);
        PanelPairs pp;
        for (int s = 0; s < op; ++s) {
            pp.L[s] = panels + (int64_t)(op * (outer & 1) + s) * pstride * nbatch;
            pp.U[s] = pp.L[s] + (int64_t)ntiles * kPanelL;
        }
        bool done = false;
        for (int s = 0; s < op; ++s) {
            const int64_t k = K0 + (int64_t)s * TC_NB;
            if (n - k - TC_NB <= 0) {
                done = true;
                break;
            }
            const int t0 = (int)((k + TC_NB) / TC_TM), nt = ntiles - t0;
            // the panel's column and row blocks carry every earlier update
            if ((e = strip_join()) != cudaSuccess) return e;
            k_lu_trsm_tc<<<dim3(2 * nt, nbz), 128, kSmemA + kSmemA, main_s>>>(
                A, n, stride, k, bimg, bstride, (unsigned char*)pp.L[s], (unsigned char*)pp.U[s], pstride, nt, bad);
            ctx->launches += 1;
            if (s + 1 < op) {
                // only the tile holding the next panel (t0) is brought up to
                // date, left-looking: after the first panel of a tile (s
                // even), that tile's L with this panel; after the second (s
                // odd), the next tile's L, untouched since the previous outer
                // step's first tile update, with the previous step's panels
                // and all of this step's panels 0 .. s at once (one pass over
                // it instead of one per outer step and panel); then the next
                // diagonal block
                PanelPairs q;
                int np = 0;
                if (s & 1)
                    for (int r = 0; r < nprev; ++r, ++np) {
                        q.L[np] = prev.L[r];
                        q.U[np] = prev.U[r];
                    }
                for (int r = (s & 1) ? 0 : s; r <= s; ++r, ++np) {
                    q.L[np] = pp.L[r];
                    q.U[np] = pp.U[r];
                }
                if ((e = strip(t0, nt, 1, q, np, k + TC_NB)) != cudaSuccess) return e;
                k_lu_diag64<<<nbatch, kDiag64Threads, kDiag64Smem, main_s>>>(A, n, stride, k + TC_NB, Dinv, dstride,
                                                                           bad, bimg, bstride);
                ctx->launches += 1;
            }
        }
        if (done) break;
        // trailing tiles >= T0 + kW with all the outer step's panel pairs
        const int64_t lo = K0 + (int64_t)op * TC_NB;
        const int t0 = T0 + kW, nt = ntiles - t0;
        if (nt <= 0) break;
        // the previous interior update and the in-block strips are done
        // before this trailing update
        if ((e = cudaStreamWaitEvent(main_s, st.ev_side, 0)) != cudaSuccess) return e;
        if ((e = strip_join()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(st.ev_panel, main_s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(side_s, st.ev_panel, 0)) != cudaSuccess) return e;
        // the interior: tiles past the next outer step's tiles, on the side
        // stream; the next outer step's first tile row and column now (its
        // first panel needs them), its other tiles' rows and columns with
        // these panels when that step reaches them (deferred, above)
        const int w = std::min(kW, nt);
        if (nt > w) {
            upd<<<dim3(nt - w, nt - w, nbz), 128, kTcSmemBytes, side_s>>>(
                A, n, stride, t0, nt, 2, w, pp, op, pstride, lo, bad, 0);
            ctx->launches += 1;
        }
        if ((e = cudaEventRecord(st.ev_side, side_s)) != cudaSuccess) return e;
        if ((e = strip(t0, nt, 1, pp, op, lo)) != cudaSuccess) return e;
        prev = pp;
        nprev = op;
        if (lo < n) {
            k_lu_diag64<<<nbatch, kDiag64Threads, kDiag64Smem, main_s>>>(A, n, stride, lo, Dinv, dstride, bad,
                                                                         bimg, bstride);
            ctx->launches += 1;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // join: everything of the side and strip streams is done before the main stream goes on
    if ((e = cudaStreamWaitEvent(main_s, st.ev_side, 0)) != cudaSuccess) return e;
    if ((e = strip_join()) != cudaSuccess) return e;
    return cudaSuccess;
}
}  // namespace

// The matrices in groups (the ctx's schedule for n: 1 to kLuGroups groups,
// contiguous, sizes differing by one at most), each on its own (main, side) stream pair: group 0 on the context's
// streams, the others forked from its stream and joined back, so the
// diagonal-block factorisations and panel solves of one group (one CTA per
// matrix, latency bound) run beside the trailing updates of another.
cudaError_t launch_lu_tc(mh_ctx* ctx, float2* A, int64_t n, int64_t stride, int nbatch, float2* Dinv,
                         unsigned char* panels, int* bad)
{
    cudaError_t e;
    static_assert(TC_NB == 64, "the diagonal blocks are factored by k_lu_diag64");
    static_assert(TC_TM == 2 * TC_NB && TC_TN == TC_TM, "two panels per 128-wide tile");
    const LuSchedule sched = ctx->lu_schedule(n);
    if (sched.groups < 1 || sched.groups > kLuGroups || sched.outer < 2 || sched.outer > kOuterMax ||
        (sched.outer & 1) || sched.update < 0 || sched.update > 1)
        return cudaErrorInvalidValue;
    if ((e = cudaFuncSetAttribute(k_lu_update_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kTcSmemBytes)) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_lu_update_tc_acc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kSmemA + kSmemB))) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_lu_trsm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(kSmemA + kSmemA))) != cudaSuccess)
        return e;
    if ((e = cudaFuncSetAttribute(k_lu_diag64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kDiag64Smem)) != cudaSuccess)
        return e;
    const int groups = std::min(sched.groups, nbatch);
    const int64_t dstride = lu_dinv_stride_tc(n);
    const int64_t pbytes = lu_panel_bytes_tc(n);
    if (groups > 1) {
        if ((e = cudaEventRecord(ctx->ev_fork, ctx->stream)) != cudaSuccess) return e;
        for (int g = 1; g < groups; ++g)
            if ((e = cudaStreamWaitEvent(ctx->grp_main[g - 1], ctx->ev_fork, 0)) != cudaSuccess) return e;
    }
    int b0 = 0;
    for (int g = 0; g < groups; ++g) {
        const int nbg = nbatch / groups + (g < nbatch % groups ? 1 : 0);
        LuStreams st;
        st.main = g ? ctx->grp_main[g - 1] : ctx->stream;
        st.side = g ? ctx->grp_side[g - 1] : ctx->side;
        st.strip = ctx->lu_strip[g];
        st.ev_side = g ? ctx->grp_ev_side[g - 1] : ctx->ev_side;
        st.ev_panel = g ? ctx->grp_ev_panel[g - 1] : ctx->ev_panel;
        st.ev_strip_go = ctx->lu_ev_strip_go[g];
        st.ev_strip_done = ctx->lu_ev_strip_done[g];
        if ((e = lu_tc_group(ctx, A + (int64_t)b0 * stride, n, stride, nbg, Dinv + (int64_t)b0 * dstride,
                             panels + (int64_t)b0 * pbytes, bad + b0, st, sched.outer, sched.update)) != cudaSuccess)
            return e;
        b0 += nbg;
    }
    for (int g = 1; g < groups; ++g) {
        if ((e = cudaEventRecord(ctx->grp_ev_join[g - 1], ctx->grp_main[g - 1])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(ctx->stream, ctx->grp_ev_join[g - 1], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

namespace {
template <int NB>
cudaError_t solve_blocks(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                         const float2* Dinv, int64_t dstride, float2* X, float2* T, int64_t xstride,
                         int nrhs)
{
    if (nrhs < 1 || nrhs > kMaxRhs) return cudaErrorInvalidValue;
    const int nblk = (int)((n + NB - 1) / NB);
    for (int blk = 0; blk < nblk; ++blk) {
        const int64_t below = n - (int64_t)(blk + 1) * NB;
        dim3 g(below > 0 ? cdiv(below, 128) : 1u, (unsigned)nbatch);
        k_trsv_fwd<NB><<<g, 128, 0, ctx->stream>>>(A, n, stride, Dinv, dstride, X, T, xstride, nrhs, blk);
    }
    for (int blk = nblk - 1; blk >= 0; --blk) {
        const int64_t above = (int64_t)blk * NB;
        dim3 g(above > 0 ? cdiv(above, 128) : 1u, (unsigned)nbatch);
        k_trsv_bwd<NB><<<g, 128, 0, ctx->stream>>>(A, n, stride, Dinv, dstride, T, X, xstride, nrhs, blk);
    }
    ctx->launches += 2 * nblk;
    return cudaGetLastError();
}

template <int NB>
cudaError_t solve_blocks_ct(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                            const float2* Dinv, int64_t dstride, float2* X, float2* T, int64_t xstride,
                            int nrhs)
{
    if (nrhs < 1 || nrhs > kMaxRhs) return cudaErrorInvalidValue;
    const int nblk = (int)((n + NB - 1) / NB);
    for (int blk = 0; blk < nblk; ++blk) {
        const int64_t below = n - (int64_t)(blk + 1) * NB;
        dim3 g(below > 0 ? cdiv(below, 16) : 1u, (unsigned)nbatch);
        k_trsv_ct_fwd<NB><<<g, 128, 0, ctx->stream>>>(A, n, stride, Dinv, dstride, X, T, xstride, nrhs,
                                                       blk);
    }
    for (int blk = nblk - 1; blk >= 0; --blk) {
        const int64_t above = (int64_t)blk * NB;
        dim3 g(above > 0 ? cdiv(above, 16) : 1u, (unsigned)nbatch);
        k_trsv_ct_bwd<NB><<<g, 128, 0, ctx->stream>>>(A, n, stride, Dinv, dstride, T, X, xstride, nrhs,
                                                       blk);
    }
    ctx->launches += 2 * nblk;
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_lu_solve_persist(mh_ctx* ctx, int backend, bool conj_trans, const float2* A, int64_t n,
                                    int64_t stride, int nbatch, const float2* Dinv, float2* X, int64_t xstride,
                                    int nrhs, int* bad, const int* done, cudaStream_t stream, int flags_slot)
{
    cudaStream_t strm = stream ? stream : ctx->stream;
    if (nrhs < 1 || nrhs > kMaxRhs) return cudaErrorInvalidValue;
    if (done && !bad) return cudaErrorInvalidValue;
    const dim3 g((unsigned)nbatch * kSolveCluster);
    cudaError_t e;
    if (backend == MH_LU_TCGEN05_F16) {
        const int64_t ds = lu_dinv_stride_tc(n);
        const int64_t nblk = (n + TC_NB - 1) / TC_NB;
        // flags of every block and triangle, then (when the caller gives no
        // per-matrix array) the timeout marks, then one flag nothing publishes
        const size_t fbytes = sizeof(int) * (size_t)(2 * nblk * nbatch + nbatch + 1);
        auto* flags = (int*)ws_get(ctx, flags_slot, fbytes);
        if (!flags) return cudaErrorMemoryAllocation;
        int* fbad = bad ? bad : flags + 2 * nblk * nbatch;
        const int* unset = ctx->inject_wait_timeout ? flags + 2 * nblk * nbatch + nbatch : nullptr;
        if ((e = cudaMemsetAsync(flags, 0, fbytes, strm)) != cudaSuccess) return e;
        const dim3 gf((unsigned)nbatch * kFsCluster);
        // n even (every column and block of y starts on 16 bytes) and one to
        // four right-hand sides: the streamed left-looking solve
        auto a16 = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
        if (n % 2 == 0 && nrhs <= 4 && stride % 2 == 0 && xstride % 2 == 0 && a16(A) && a16(Dinv) && a16(X)) {
            auto run = [&](auto kern) -> cudaError_t {
                cudaError_t e2;
                if ((e2 = raise_smem_cap((const void*)kern, kSsSmemBytes)) != cudaSuccess) return e2;
                // two CTAs per SM need the largest shared-memory carveout
                if ((e2 = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                               100)) != cudaSuccess)
                    return e2;
                kern<<<gf, kSsThreads, kSsSmemBytes, strm>>>(A, n, stride, Dinv, ds, X, xstride, flags, fbad, done,
                                                             unset);
                return cudaSuccess;
            };
            switch (nrhs * 2 + (conj_trans ? 1 : 0)) {
            case 2: e = run(k_lu_solve_stream<false, 1>); break;
            case 3: e = run(k_lu_solve_stream<true, 1>); break;
            case 4: e = run(k_lu_solve_stream<false, 2>); break;
            case 5: e = run(k_lu_solve_stream<true, 2>); break;
            case 6: e = run(k_lu_solve_stream<false, 3>); break;
            case 7: e = run(k_lu_solve_stream<true, 3>); break;
            case 8: e = run(k_lu_solve_stream<false, 4>); break;
            default: e = run(k_lu_solve_stream<true, 4>); break;
            }
            if (e != cudaSuccess) return e;
            ctx->launches += 1;
            return cudaGetLastError();
        }
        const size_t xsb = sizeof(float2) * (size_t)((nblk + kFsCluster - 1) / kFsCluster) * nrhs * TC_NB;
        const bool shared_x = xsb <= 96 * 1024;
        // staging of the next block (two more 34 KB blocks) only while two
        // CTAs still fit on an SM
        int dev = 0, sm_bytes = 0, reserved = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
            return e;
        if ((e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess)
            return e;
        auto go = [&](auto kern, size_t xs) -> cudaError_t {
            cudaError_t e2;
            cudaFuncAttributes fa;
            if ((e2 = cudaFuncGetAttributes(&fa, (const void*)kern)) != cudaSuccess) return e2;
            const bool stage = 2 * (fa.sharedSizeBytes + xs + 2 * kFsStageBytes + (size_t)reserved) <= (size_t)sm_bytes;
            const size_t smem = xs + (stage ? 2 * kFsStageBytes : 0);
            if (smem && (e2 = raise_smem_cap((const void*)kern, smem)) != cudaSuccess) return e2;
            kern<<<gf, kFsThreads, smem, strm>>>(A, n, stride, Dinv, ds, X, xstride, nrhs, flags, fbad,
                                                        stage ? 1 : 0, done, unset);
            return cudaSuccess;
        };
        // right-hand-side counts 1 to 4 (radiation dofs and headings of one
        // body) by their own compile-time variants
        const int nq = shared_x && nrhs <= 4 ? nrhs : 0;
        if (conj_trans) {
            switch (nq) {
            case 1: e = go(k_lu_solve_flags<true, true, 1>, xsb); break;
            case 2: e = go(k_lu_solve_flags<true, true, 2>, xsb); break;
            case 3: e = go(k_lu_solve_flags<true, true, 3>, xsb); break;
            case 4: e = go(k_lu_solve_flags<true, true, 4>, xsb); break;
            default: e = shared_x ? go(k_lu_solve_flags<true, true, 0>, xsb) : go(k_lu_solve_flags<true, false, 0>, 0);
            }
        } else {
            switch (nq) {
            case 1: e = go(k_lu_solve_flags<false, true, 1>, xsb); break;
            case 2: e = go(k_lu_solve_flags<false, true, 2>, xsb); break;
            case 3: e = go(k_lu_solve_flags<false, true, 3>, xsb); break;
            case 4: e = go(k_lu_solve_flags<false, true, 4>, xsb); break;
            default: e = shared_x ? go(k_lu_solve_flags<false, true, 0>, xsb) : go(k_lu_solve_flags<false, false, 0>, 0);
            }
        }
        if (e != cudaSuccess) return e;
    } else {
        const int64_t ds = lu_dinv_stride(n);
        const size_t sm = persist_smem_bytes<32>();
        if (conj_trans)
            k_lu_solve_persist<32, true><<<g, kSolveThreads, sm, strm>>>(A, n, stride, Dinv, ds, X,
                                                                                 xstride, nrhs, done, bad);
        else
            k_lu_solve_persist<32, false><<<g, kSolveThreads, sm, strm>>>(A, n, stride, Dinv, ds, X,
                                                                                  xstride, nrhs, done, bad);
    }
    ctx->launches += 1;
    return cudaGetLastError();
}

cudaError_t launch_lu_solve_ct(mh_ctx* ctx, int backend, const float2* A, int64_t n, int64_t stride,
                               int nbatch, const float2* Dinv, float2* X, float2* T, int64_t xstride,
                               int nrhs)
{
    if (backend == MH_LU_TCGEN05_F16)
        return solve_blocks_ct<TC_NB>(ctx, A, n, stride, nbatch, Dinv, lu_dinv_stride_tc(n), X, T,
                                      xstride, nrhs);
    return solve_blocks_ct<32>(ctx, A, n, stride, nbatch, Dinv, lu_dinv_stride(n), X, T, xstride, nrhs);
}

cudaError_t launch_lu_solve_tc(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                               const float2* Dinv, float2* X, float2* T, int64_t xstride, int nrhs)
{
    return solve_blocks<TC_NB>(ctx, A, n, stride, nbatch, Dinv, lu_dinv_stride_tc(n), X, T, xstride,
                               nrhs);
}

cudaError_t launch_lu_solve_blocks32(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride,
                                     int nbatch, const float2* Dinv, float2* X, float2* T,
                                     int64_t xstride, int nrhs)
{
    return solve_blocks<32>(ctx, A, n, stride, nbatch, Dinv, lu_dinv_stride(n), X, T, xstride, nrhs);
}

}  // namespace mh
