// mh_solve_mixed_noalloc: the mixed-precision dense solve (FP32 LU of A, FP64
// iterative refinement) with all of its scratch memory in one file-scope
// device array, so a call allocates nothing.
//
// Who needs it: code that drives this library from places where device
// allocation is not allowed or not possible -- a host loop that must not
// block on the allocator (cudaMalloc synchronises the device), an embedding
// application that owns all device memory through its own pool and forbids
// other allocations, or a real-time control loop that must have a fixed
// memory footprint.  Such a caller passes device buffers it already owns for
// the inputs and the output; the scratch (the FP32 LU copy, the inverses of
// its diagonal blocks, residual vectors and a status word) lives in
// g_noalloc_scratch below.
//
// Limits and behaviour:
//  - n <= MH_NOALLOC_MAX_N (1024) and nrhs <= MH_NOALLOC_MAX_RHS (16); the
//    array is sized for that maximum (about 9 MiB) and every GPU that loads
//    this library holds it until the process exits;
//  - the call runs on the calling thread's current device and on `stream`;
//  - every call shares the one array per device and leaves the last call's
//    contents in it; what must start at zero is cleared at the start of each
//    call.  Calls whose work overlaps on the GPU (two host threads, or two
//    streams, at once) race on the array: serialise them;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (this also loads the module on that device); make
//    that first call before any stream capture.  The address is kept for the
//    life of the process: after cudaDeviceReset (or anything else that
//    destroys the device's primary context) the kept address is stale, so do
//    not call this entry point on that device again in the same process;
//  - A, B and X must be device memory of the current device (or managed
//    memory); a pointer into another GPU's memory is rejected with
//    MH_ERR_ARG before anything is launched.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "mh_internal.h"

namespace {

constexpr int64_t kNaMaxN = MH_NOALLOC_MAX_N;
constexpr int64_t kNaMaxRhs = MH_NOALLOC_MAX_RHS;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }
// FP32 LU copy, inverse diagonal blocks (32 x 32, two per block), FP64
// residual, FP32 correction, status.
constexpr size_t kLuBytes = align_up(sizeof(float2) * kNaMaxN * kNaMaxN);
constexpr size_t kDinvBytes = align_up(sizeof(float2) * ((kNaMaxN + 31) / 32) * 2 * 32 * 32);
constexpr size_t kRBytes = align_up(sizeof(double2) * kNaMaxN * kNaMaxRhs);
constexpr size_t kR32Bytes = align_up(sizeof(float2) * kNaMaxN * kNaMaxRhs);
constexpr size_t kStatusBytes = kAlign;
constexpr size_t kScratchBytes = kLuBytes + kDinvBytes + kRBytes + kR32Bytes + kStatusBytes;

}  // namespace

// The scratch of every mh_solve_mixed_noalloc call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct Status {
    int bad;       // set by the LU on a zero / non-finite pivot
    int pad;
    double ratio;  // max over right-hand sides of max|r| / max|b|
};

std::mutex g_mu;
void* g_scratch_ptr[64] = {};

// Device address of the scratch array on the current device (looked up once
// per device).
int scratch_address(int device, void** out)
{
    if (device < 0 || device >= 64) return mh::set_err(nullptr, MH_ERR_NO_DEVICE, "device %d", device);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return mh::set_err(nullptr, MH_ERR_CUDA, "cudaGetSymbolAddress of the scratch array: %s",
                               cudaGetErrorString(e));
        }
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return MH_OK;
}

__global__ void k_na_convert(const double2* __restrict__ A, float2* __restrict__ lo, int64_t count)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) lo[t] = make_float2((float)A[t].x, (float)A[t].y);
}

// X = 0, R = B
__global__ void k_na_start(const double2* __restrict__ B, double2* __restrict__ R,
                           double2* __restrict__ X, int64_t count)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) {
        R[t] = B[t];
        X[t] = make_double2(0.0, 0.0);
    }
}

__global__ void k_na_to_f32(const double2* __restrict__ R, float2* __restrict__ R32, int64_t count)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) R32[t] = make_float2((float)R[t].x, (float)R[t].y);
}

__global__ void k_na_add(double2* __restrict__ X, const float2* __restrict__ D, int64_t count)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) X[t] = make_double2(X[t].x + (double)D[t].x, X[t].y + (double)D[t].y);
}

// R[:, q] = B[:, q] - A X[:, q] in FP64, q = blockIdx.y, one thread per row.
__global__ void k_na_residual(const double2* __restrict__ A, const double2* __restrict__ B,
                              const double2* __restrict__ X, double2* __restrict__ R, int64_t n)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t q = blockIdx.y;
    const double2* x = X + q * n;
    double ar = B[q * n + i].x, ai = B[q * n + i].y;
    for (int64_t j = 0; j < n; ++j) {
        double2 a = A[j * n + i], v = x[j];
        ar -= a.x * v.x - a.y * v.y;
        ai -= a.x * v.y + a.y * v.x;
    }
    R[q * n + i] = make_double2(ar, ai);
}

__global__ void __launch_bounds__(256)
k_na_norm(const double2* __restrict__ R, const double2* __restrict__ B, int64_t n, int nrhs,
          Status* __restrict__ st)
{
    __shared__ double sr[256], sb[256];
    double worst = 0.0;
    for (int q = 0; q < nrhs; ++q) {
        double mr = 0.0, mb = 0.0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            mr = fmax(mr, hypot(R[q * n + i].x, R[q * n + i].y));
            mb = fmax(mb, hypot(B[q * n + i].x, B[q * n + i].y));
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
    if (threadIdx.x == 0) st->ratio = (worst == worst) ? worst : INFINITY;
}

// Memory that kernels launched on `device` may read and write: device memory
// of that device, or managed memory.  Device memory of another GPU is
// rejected: without peer access a kernel touching it faults, which would
// poison the context; the check launches nothing on the pointer.
bool is_local_device_pointer(const void* p, int device)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged) return true;
    return a.type == cudaMemoryTypeDevice && a.device == device;
}

unsigned nblk(int64_t count) { return (unsigned)((count + 255) / 256); }

}  // namespace

extern "C" int mh_solve_mixed_noalloc(int64_t n, const void* A, const void* B, int64_t nrhs, void* X,
                                      double tol, int max_iter, void* stream, int32_t* iterations,
                                      double* rel_residual)
{
    using mh::set_err;
    if (n < 1 || n > kNaMaxN)
        return set_err(nullptr, MH_ERR_ARG, "mh_solve_mixed_noalloc: n = %lld, must be in [1, %lld]",
                       (long long)n, (long long)kNaMaxN);
    if (nrhs < 1 || nrhs > kNaMaxRhs)
        return set_err(nullptr, MH_ERR_ARG, "mh_solve_mixed_noalloc: nrhs = %lld, must be in [1, %lld]",
                       (long long)nrhs, (long long)kNaMaxRhs);
    if (!(tol > 0.0) || max_iter < 1 || max_iter > 100)
        return set_err(nullptr, MH_ERR_ARG, "mh_solve_mixed_noalloc: need tol > 0, 1 <= max_iter <= 100");
    if (!A || !B || !X || X == B || X == A)
        return set_err(nullptr, MH_ERR_ARG, "mh_solve_mixed_noalloc: A, B, X must be distinct non-NULL");
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return set_err(nullptr, MH_ERR_NO_DEVICE, "no current CUDA device");
    }
    if (!is_local_device_pointer(A, device) || !is_local_device_pointer(B, device) ||
        !is_local_device_pointer(X, device))
        return set_err(nullptr, MH_ERR_ARG,
                       "mh_solve_mixed_noalloc: A, B and X must be device memory of the current device "
                       "(%d) or managed memory", device);
    void* base = nullptr;
    int rc = scratch_address(device, &base);
    if (rc) return rc;
    auto* bytes = (unsigned char*)base;
    auto* lu = (float2*)bytes;
    auto* dinv = (float2*)(bytes + kLuBytes);
    auto* R = (double2*)(bytes + kLuBytes + kDinvBytes);
    auto* R32 = (float2*)(bytes + kLuBytes + kDinvBytes + kRBytes);
    auto* st = (Status*)(bytes + kLuBytes + kDinvBytes + kRBytes + kR32Bytes);

    // A stack context carries the stream for the shared LU launchers; it owns
    // no resources.
    mh_ctx local;
    local.stream = (cudaStream_t)stream;
    const auto* dA = (const double2*)A;
    const auto* dB = (const double2*)B;
    auto* dX = (double2*)X;
    const int64_t cnt = n * nrhs;
    cudaError_t e;
#define NA_TRY(expr)                                                                              \
    do {                                                                                          \
        if ((e = (expr)) != cudaSuccess)                                                          \
            return set_err(nullptr, MH_ERR_CUDA, "mh_solve_mixed_noalloc: %s", cudaGetErrorString(e)); \
    } while (0)
    NA_TRY(cudaMemsetAsync(st, 0, sizeof(Status), local.stream));
    k_na_convert<<<nblk(n * n), 256, 0, local.stream>>>(dA, lu, n * n);
    k_na_start<<<nblk(cnt), 256, 0, local.stream>>>(dB, R, dX, cnt);
    NA_TRY(cudaGetLastError());
    NA_TRY(mh::launch_lu_f32(&local, lu, n, n * n, 1, dinv, &st->bad));
    Status h{};
    int it = 0;
    bool converged = false;
    for (it = 1; it <= max_iter; ++it) {
        k_na_to_f32<<<nblk(cnt), 256, 0, local.stream>>>(R, R32, cnt);
        NA_TRY(mh::launch_lu_solve_f32(&local, lu, n, n * n, 1, dinv, R32, cnt, (int)nrhs));
        k_na_add<<<nblk(cnt), 256, 0, local.stream>>>(dX, R32, cnt);
        k_na_residual<<<dim3(nblk(n), (unsigned)nrhs), 256, 0, local.stream>>>(dA, dB, dX, R, n);
        k_na_norm<<<1, 256, 0, local.stream>>>(R, dB, n, (int)nrhs, st);
        NA_TRY(cudaGetLastError());
        NA_TRY(cudaMemcpyAsync(&h, st, sizeof(Status), cudaMemcpyDeviceToHost, local.stream));
        NA_TRY(cudaStreamSynchronize(local.stream));
        if (h.bad) break;
        if (h.ratio <= tol) {
            converged = true;
            break;
        }
    }
#undef NA_TRY
    if (iterations) *iterations = converged ? it : std::min(it, max_iter);
    if (rel_residual) *rel_residual = h.ratio;
    if (h.bad)
        return set_err(nullptr, MH_ERR_NOT_CONVERGED,
                       "mh_solve_mixed_noalloc: zero or non-finite pivot in the FP32 LU");
    if (!converged)
        return set_err(nullptr, MH_ERR_NOT_CONVERGED,
                       "mh_solve_mixed_noalloc: residual %.3e above tol after %d sweeps", h.ratio, max_iter);
    return MH_OK;
}
