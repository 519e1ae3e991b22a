// C ABI of libmarinehydro_b200: contexts, meshes, matrix-level and
// output-level entry points.  Every entry point validates its arguments,
// returns an MH_* status and records a message on the context.
#include <cuComplex.h>
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include <cmath>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <utility>

#include "mh_internal.h"

namespace {
thread_local std::string g_create_err;

bool finite_array(const double* a, int64_t count)
{
    for (int64_t i = 0; i < count; ++i)
        if (!std::isfinite(a[i])) return false;
    return true;
}
}  // namespace

namespace mh {

int set_err(mh_ctx* ctx, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    else g_create_err = buf;
    return code;
}

cudaError_t raise_smem_cap(const void* kernel, size_t bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> caps;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& cur = caps[{kernel, dev}];
    if (bytes <= cur) return cudaSuccess;
    if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes)) != cudaSuccess)
        return e;
    cur = bytes;
    return cudaSuccess;
}

void* ws_get(mh_ctx* ctx, int slot, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    if (ctx->ws_bytes[slot] >= bytes) return ctx->ws[slot];
    // stream-ordered: the old buffer is released after the work already
    // issued on the ctx stream (which the ctx's other streams join), and
    // neither call synchronises the device, so contexts on other host threads
    // keep running
    if (ctx->ws[slot]) {
        cudaFreeAsync(ctx->ws[slot], ctx->stream);
        ctx->ws[slot] = nullptr;
        ctx->ws_bytes[slot] = 0;
    }
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, ctx->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_err(ctx, MH_ERR_OOM, "device allocation of %zu bytes failed: %s", bytes,
                cudaGetErrorString(e));
        return nullptr;
    }
    ctx->ws[slot] = p;
    ctx->ws_bytes[slot] = bytes;
    return p;
}

namespace {
cudaEvent_t pooled_event(mh_ctx* ctx)
{
    if (!ctx->ev_pool.empty()) {
        cudaEvent_t e = ctx->ev_pool.back();
        ctx->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}
}  // namespace

void phase_begin(mh_ctx* ctx, int ph)
{
    if (!ctx->profile) return;
    if (ctx->ev_open[ph]) ctx->ev_pool.push_back(ctx->ev_open[ph]);
    ctx->ev_open[ph] = pooled_event(ctx);
    if (ctx->ev_open[ph]) cudaEventRecord(ctx->ev_open[ph], ctx->stream);
}

void phase_end(mh_ctx* ctx, int ph)
{
    if (!ctx->profile || !ctx->ev_open[ph]) return;
    cudaEvent_t e = pooled_event(ctx);
    if (!e) return;
    cudaEventRecord(e, ctx->stream);
    ctx->ev_recs.push_back({ph, ctx->ev_open[ph], e});
    ctx->ev_open[ph] = nullptr;
    if (ctx->ev_recs.size() >= 512) phase_collect(ctx);
}

void phase_collect(mh_ctx* ctx)
{
    for (auto& r : ctx->ev_recs) {
        float ms = 0.f;
        if (cudaEventSynchronize(r.e) == cudaSuccess && cudaEventElapsedTime(&ms, r.b, r.e) == cudaSuccess) {
            ctx->phase_ms[r.ph] += ms;
            ctx->phase_calls[r.ph] += 1;
        }
        ctx->ev_pool.push_back(r.b);
        ctx->ev_pool.push_back(r.e);
    }
    ctx->ev_recs.clear();
    cudaGetLastError();
}

}  // namespace mh

using mh::set_err;
using mh::ws_get;

namespace {

int check_ctx(mh_ctx* ctx)
{
    if (!ctx) return MH_ERR_ARG;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess)
        return set_err(ctx, MH_ERR_CUDA, "cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
    ctx->err.clear();
    return MH_OK;
}

int check_mesh(mh_ctx* ctx, const mh_mesh* m)
{
    if (!m || !m->geom || m->n <= 0) return set_err(ctx, MH_ERR_ARG, "mesh is NULL or empty");
    if (m->device != ctx->device)
        return set_err(ctx, MH_ERR_ARG, "mesh lives on device %d, context on device %d", m->device,
                       ctx->device);
    return MH_OK;
}

int valid_mask(mh_ctx* ctx, uint32_t mask)
{
    const uint32_t all = MH_GF_RANKINE | MH_GF_RANKINE_REFLECTED | MH_GF_RANKINE_REFLECTED_NEGATIVE |
                         MH_GF_WU | MH_GF_DELHOMMEAU;
    if (mask == 0 || (mask & ~all))
        return set_err(ctx, MH_ERR_ARG, "invalid Green-function mask 0x%x", mask);
    return MH_OK;
}

int sync_status(mh_ctx* ctx, const char* what)
{
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return set_err(ctx, MH_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return MH_OK;
}

// LU-factorise A (n x n, device, overwritten) and solve A X = B in place
// (B: n x nrhs, device) with cuSOLVER zgetrf/zgetrs.
int lu_solve_fp64(mh_ctx* ctx, int64_t n, double2* A, double2* B, int64_t nrhs)
{
    int lwork = 0;
    cusolverStatus_t st = cusolverDnZgetrf_bufferSize(ctx->cusolver, (int)n, (int)n,
                                                      (cuDoubleComplex*)A, (int)n, &lwork);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrf_bufferSize failed (%d)", (int)st);
    auto* work = (cuDoubleComplex*)ws_get(ctx, WS_LWORK, sizeof(cuDoubleComplex) * (size_t)lwork);
    auto* piv = (int*)ws_get(ctx, WS_PIV, sizeof(int) * (size_t)n);
    auto* info = (int*)ws_get(ctx, WS_INFO, sizeof(int) * 2);
    if (!work || !piv || !info) return MH_ERR_OOM;
    st = cusolverDnZgetrf(ctx->cusolver, (int)n, (int)n, (cuDoubleComplex*)A, (int)n, work, piv, info);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrf failed (%d)", (int)st);
    st = cusolverDnZgetrs(ctx->cusolver, CUBLAS_OP_N, (int)n, (int)nrhs, (const cuDoubleComplex*)A,
                          (int)n, piv, (cuDoubleComplex*)B, (int)n, info + 1);
    if (st != CUSOLVER_STATUS_SUCCESS)
        return set_err(ctx, MH_ERR_CUDA, "cusolverDnZgetrs failed (%d)", (int)st);
    int h_info[2] = {0, 0};
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h_info, info, sizeof(h_info), cudaMemcpyDeviceToHost, ctx->stream));
    int rc = sync_status(ctx, "LU solve");
    if (rc) return rc;
    if (h_info[0] > 0) return set_err(ctx, MH_ERR_SINGULAR, "zero pivot at column %d", h_info[0]);
    if (h_info[0] < 0 || h_info[1] < 0)
        return set_err(ctx, MH_ERR_ARG, "LAPACK argument %d invalid", -(h_info[0] ? h_info[0] : h_info[1]));
    return MH_OK;
}

// C = A B for n x n A and n x nrhs B (device, complex128).
int zgemm_nn(mh_ctx* ctx, int64_t n, int64_t nrhs, const double2* A, const double2* B, double2* C)
{
    const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
    cublasStatus_t st = cublasZgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)nrhs, (int)n,
                                    &one, (const cuDoubleComplex*)A, (int)n,
                                    (const cuDoubleComplex*)B, (int)n, &zero, (cuDoubleComplex*)C,
                                    (int)n);
    if (st != CUBLAS_STATUS_SUCCESS) return set_err(ctx, MH_ERR_CUDA, "cublasZgemm failed (%d)", (int)st);
    return MH_OK;
}

// phi = D \ (S bc)  or  phi = S (K \ bc), all device; D is overwritten by its
// LU factors, bc by intermediate results.  (src/matrix_assembly.jl:105-133)
int solve_fp64_device(mh_ctx* ctx, int64_t n, double2* D, const double2* S, double2* bc,
                      int64_t nrhs, int direct, double2* phi)
{
    int rc;
    if (direct) {
        if ((rc = zgemm_nn(ctx, n, nrhs, S, bc, phi))) return rc;
        return lu_solve_fp64(ctx, n, D, phi, nrhs);
    }
    if ((rc = lu_solve_fp64(ctx, n, D, bc, nrhs))) return rc;
    return zgemm_nn(ctx, n, nrhs, S, bc, phi);
}

int dof_upload(mh_ctx* ctx, const mh_mesh* m, const double* dof, int64_t dof_rows, double** d_dof)
{
    if (!dof) return set_err(ctx, MH_ERR_ARG, "dof is NULL");
    if (dof_rows != 1 && dof_rows != m->n)
        return set_err(ctx, MH_ERR_ARG, "dof must be a 3-vector or an nfaces x 3 matrix (got %lld rows)",
                       (long long)dof_rows);
    size_t bytes = sizeof(double) * 3 * (size_t)dof_rows;
    double* p = (double*)ws_get(ctx, WS_DOF, bytes);
    if (!p) return MH_ERR_OOM;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(p, dof, bytes, cudaMemcpyHostToDevice, ctx->stream));
    *d_dof = p;
    return MH_OK;
}

// Shared pipeline of the two front doors: assembly, bc, solve, force.
int front_door(mh_ctx* ctx, const mh_mesh* m, const double* dof, int64_t dof_rows, double omega,
               double rho, double g, uint32_t gf_mask, int direct, int precision, bool diffraction,
               double beta, double2* F_host)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if ((rc = check_mesh(ctx, m))) return rc;
    if ((rc = valid_mask(ctx, gf_mask))) return rc;
    if (!(omega > 0.0) || !std::isfinite(omega) || !(g > 0.0) || !std::isfinite(rho))
        return set_err(ctx, MH_ERR_ARG, "omega and g must be positive and finite");
    if (precision != MH_PRECISION_FP64)
        return set_err(ctx, MH_ERR_ARG, "precision %d is not available on this entry point", precision);
    const int64_t n = m->n;
    const size_t mat = sizeof(double2) * (size_t)n * (size_t)n;
    auto* S = (double2*)ws_get(ctx, WS_S, mat);
    auto* D = (double2*)ws_get(ctx, WS_D, mat);
    auto* bc = (double2*)ws_get(ctx, WS_RHS, sizeof(double2) * (size_t)n);
    auto* phi = (double2*)ws_get(ctx, WS_PHI, sizeof(double2) * (size_t)n);
    auto* F = (double2*)ws_get(ctx, WS_OUT, sizeof(double2));
    if (!S || !D || !bc || !phi || !F) return MH_ERR_OOM;
    double* d_dof = nullptr;
    if ((rc = dof_upload(ctx, m, dof, dof_rows, &d_dof))) return rc;
    const double k = omega * omega / g;
    const double* tab = mh::delh_table_for(ctx, gf_mask, &rc);
    if (rc) return rc;
    MH_CUDA_TRY(ctx, mh::launch_assemble_f64(ctx, m, k, gf_mask, direct, tab, S, D));
    if (diffraction) MH_CUDA_TRY(ctx, mh::launch_airy_bc(ctx, m, omega, beta, g, bc));
    else MH_CUDA_TRY(ctx, mh::launch_radiation_bc(ctx, m, d_dof, dof_rows, omega, bc));
    if ((rc = solve_fp64_device(ctx, n, D, S, bc, 1, direct, phi))) return rc;
    MH_CUDA_TRY(ctx, mh::launch_force(ctx, m, phi, d_dof, dof_rows, rho, omega, F));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(F_host, F, sizeof(double2), cudaMemcpyDeviceToHost, ctx->stream));
    return sync_status(ctx, "front door");
}

}  // namespace

extern "C" {

int mh_version(void) { return 100; }

int mh_device_count(int* count)
{
    if (!count) return MH_ERR_ARG;
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c = 0;
    }
    *count = c;
    return MH_OK;
}

int mh_ctx_create(int device, mh_ctx** out)
{
    if (!out) return set_err(nullptr, MH_ERR_ARG, "out is NULL");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return set_err(nullptr, MH_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    if (device < 0 || device >= count)
        return set_err(nullptr, MH_ERR_NO_DEVICE, "device %d out of range (%d visible)", device, count);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
        return set_err(nullptr, MH_ERR_CUDA, "cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
    auto* ctx = new (std::nothrow) mh_ctx();
    if (!ctx) return set_err(nullptr, MH_ERR_OOM, "host allocation failed");
    ctx->device = device;
    {  // keep freed stream-ordered memory in the device's pool instead of
       // returning it to the driver at every synchronisation (a setting of
       // this process's pool, not of the GPU)
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    }
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if ((e = cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, greatest)) != cudaSuccess ||
        (e = cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, least)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_panel, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_side, cudaEventDisableTiming)) != cudaSuccess) {
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->ev_panel) cudaEventDestroy(ctx->ev_panel);
        delete ctx;
        return set_err(nullptr, MH_ERR_CUDA, "stream/event creation: %s", cudaGetErrorString(e));
    }
    for (int g = 0; g < kLuGroups - 1 && e == cudaSuccess; ++g) {
        if ((e = cudaStreamCreateWithPriority(&ctx->grp_main[g], cudaStreamNonBlocking, greatest)) != cudaSuccess ||
            (e = cudaStreamCreateWithPriority(&ctx->grp_side[g], cudaStreamNonBlocking, least)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ctx->grp_ev_panel[g], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ctx->grp_ev_side[g], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ctx->grp_ev_join[g], cudaEventDisableTiming)) != cudaSuccess)
            break;
    }
    for (int g = 0; g < kLuGroups && e == cudaSuccess; ++g) {
        if ((e = cudaStreamCreateWithPriority(&ctx->lu_strip[g], cudaStreamNonBlocking, greatest)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ctx->lu_ev_strip_go[g], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&ctx->lu_ev_strip_done[g], cudaEventDisableTiming)) != cudaSuccess)
            break;
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        mh_ctx_destroy(ctx);
        return set_err(nullptr, MH_ERR_CUDA, "stream/event creation: %s", cudaGetErrorString(e));
    }
    if (cublasCreate(&ctx->cublas) != CUBLAS_STATUS_SUCCESS ||
        cusolverDnCreate(&ctx->cusolver) != CUSOLVER_STATUS_SUCCESS) {
        mh_ctx_destroy(ctx);
        return set_err(nullptr, MH_ERR_CUDA, "cuBLAS / cuSOLVER handle creation failed");
    }
    cublasSetStream(ctx->cublas, ctx->stream);
    cusolverDnSetStream(ctx->cusolver, ctx->stream);
    // LU schedules the autotuner chose on a B200 (mh_lu_autotune, median of
    // three sweeps over groups 1-4 x 2-8 panels per outer step x both update
    // kernels; ms against the default 2 x 4): 512 panels x 16 matrices, 1
    // group x 4 panels with C staged in tensor memory (0.555 vs 0.651);
    // 1024 x 64, 1 x 4 (1.730 vs 1.736; 1.232 vs 1.413 at 1024 x 16); 1536
    // x 16, 1 x 4 (2.00 vs 2.20); 2048 x 64, 2 x 8 (5.67 vs 6.27).  Other
    // sizes take the nearest entry; mh_ctx_set_lu_schedule or the autotuner
    // replace them.
    ctx->lu_table = {{512, LuSchedule{1, 4, 1}}, {1024, LuSchedule{1, 4, 0}}, {1536, LuSchedule{1, 4, 0}},
                     {2048, LuSchedule{2, 8, 0}}};
    *out = ctx;
    return MH_OK;
}

int mh_ctx_destroy(mh_ctx* ctx)
{
    if (!ctx) return MH_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    for (int g = 0; g < kLuGroups - 1; ++g) {
        if (ctx->grp_main[g]) cudaStreamSynchronize(ctx->grp_main[g]);
        if (ctx->grp_side[g]) cudaStreamSynchronize(ctx->grp_side[g]);
    }
    for (int g = 0; g < kLuGroups; ++g)
        if (ctx->lu_strip[g]) cudaStreamSynchronize(ctx->lu_strip[g]);
    for (int s = 0; s < WS_NSLOTS; ++s)
        if (ctx->ws[s]) cudaFree(ctx->ws[s]);
    if (ctx->delh_table) cudaFree(ctx->delh_table);
    mh::phase_collect(ctx);
    for (int q = 0; q < PH_N; ++q)
        if (ctx->ev_open[q]) cudaEventDestroy(ctx->ev_open[q]);
    for (cudaEvent_t e : ctx->ev_pool) cudaEventDestroy(e);
    if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
    for (int g = 0; g < kLuGroups - 1; ++g)
        if (ctx->cusolver_grp[g]) cusolverDnDestroy(ctx->cusolver_grp[g]);
    if (ctx->cublas) cublasDestroy(ctx->cublas);
    if (ctx->ev_panel) cudaEventDestroy(ctx->ev_panel);
    if (ctx->ev_side) cudaEventDestroy(ctx->ev_side);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    for (int g = 0; g < kLuGroups - 1; ++g) {
        if (ctx->grp_ev_panel[g]) cudaEventDestroy(ctx->grp_ev_panel[g]);
        if (ctx->grp_ev_side[g]) cudaEventDestroy(ctx->grp_ev_side[g]);
        if (ctx->grp_ev_join[g]) cudaEventDestroy(ctx->grp_ev_join[g]);
        if (ctx->grp_side[g]) cudaStreamDestroy(ctx->grp_side[g]);
        if (ctx->grp_main[g]) cudaStreamDestroy(ctx->grp_main[g]);
    }
    for (int g = 0; g < kLuGroups; ++g) {
        if (ctx->lu_ev_strip_go[g]) cudaEventDestroy(ctx->lu_ev_strip_go[g]);
        if (ctx->lu_ev_strip_done[g]) cudaEventDestroy(ctx->lu_ev_strip_done[g]);
        if (ctx->lu_strip[g]) cudaStreamDestroy(ctx->lu_strip[g]);
    }
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MH_OK;
}

const char* mh_last_error(const mh_ctx* ctx)
{
    return ctx ? ctx->err.c_str() : g_create_err.c_str();
}

int mh_ctx_kernel_launches(const mh_ctx* ctx, int64_t* count)
{
    if (!ctx || !count) return MH_ERR_ARG;
    *count = ctx->launches;
    return MH_OK;
}

int mh_ctx_stream(const mh_ctx* ctx, void** stream)
{
    if (!ctx || !stream) return MH_ERR_ARG;
    *stream = (void*)ctx->stream;
    return MH_OK;
}

int mh_ctx_set_profiling(mh_ctx* ctx, int enable)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    mh::phase_collect(ctx);
    ctx->profile = enable != 0;
    for (int q = 0; q < PH_N; ++q) {
        ctx->phase_ms[q] = 0.0;
        ctx->phase_calls[q] = 0;
        if (ctx->ev_open[q]) ctx->ev_pool.push_back(ctx->ev_open[q]);
        ctx->ev_open[q] = nullptr;
    }
    return MH_OK;
}

int mh_ctx_phase_times(mh_ctx* ctx, int nphases, double* ms, int64_t* calls)
{
    if (!ctx || nphases < 0 || (nphases && (!ms || !calls))) return MH_ERR_ARG;
    mh::phase_collect(ctx);
    for (int q = 0; q < nphases; ++q) {
        ms[q] = q < PH_N ? ctx->phase_ms[q] : 0.0;
        calls[q] = q < PH_N ? ctx->phase_calls[q] : 0;
    }
    return MH_OK;
}

int mh_ctx_set_delhommeau_method(mh_ctx* ctx, int method)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (method != MH_DELHOMMEAU_TABLE && method != MH_DELHOMMEAU_EXACT)
        return set_err(ctx, MH_ERR_ARG, "unknown Delhommeau method %d", method);
    ctx->delh_method = method;
    return MH_OK;
}

int mh_ctx_set_lu_backend(mh_ctx* ctx, int backend)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (backend != MH_LU_SIMT_F32 && backend != MH_LU_TCGEN05_F16)
        return set_err(ctx, MH_ERR_ARG, "unknown LU backend %d", backend);
    ctx->lu_backend = backend;
    return MH_OK;
}

int mh_lu_factor_lowp(mh_ctx* ctx, int backend, int64_t n, int64_t nbatch, const double* A_host,
                      float* LU_host, int* bad_host)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (backend != MH_LU_SIMT_F32 && backend != MH_LU_TCGEN05_F16)
        return set_err(ctx, MH_ERR_ARG, "unknown LU backend %d", backend);
    if (n < 1 || nbatch < 1 || !A_host || !LU_host || !bad_host)
        return set_err(ctx, MH_ERR_ARG, "bad arguments to mh_lu_factor_lowp");
    const size_t nn = (size_t)n * (size_t)n, cnt = nn * (size_t)nbatch;
    auto* d64 = (double2*)ws_get(ctx, WS_D, sizeof(double2) * cnt);
    auto* lo = (float2*)ws_get(ctx, WS_LO, sizeof(float2) * cnt);
    const int64_t dst = backend == MH_LU_TCGEN05_F16 ? mh::lu_dinv_stride_tc(n) : mh::lu_dinv_stride(n);
    auto* dinv = (float2*)ws_get(ctx, WS_DINV, sizeof(float2) * (size_t)dst * (size_t)nbatch);
    auto* bad = (int*)ws_get(ctx, WS_MISC, sizeof(int) * (size_t)nbatch);
    if (!d64 || !lo || !dinv || !bad) return MH_ERR_OOM;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d64, A_host, sizeof(double2) * cnt, cudaMemcpyHostToDevice,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, mh::launch_to_f32(ctx, d64, lo, (int64_t)cnt));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(int) * (size_t)nbatch, ctx->stream));
    if (backend == MH_LU_TCGEN05_F16) {
        auto* panels = (unsigned char*)ws_get(ctx, WS_PANEL,
                                              (size_t)mh::lu_panel_bytes_tc(n) * (size_t)nbatch);
        if (!panels) return MH_ERR_OOM;
        MH_CUDA_TRY(ctx, mh::launch_lu_tc(ctx, lo, n, (int64_t)nn, (int)nbatch, dinv, panels, bad));
    }
    else
        MH_CUDA_TRY(ctx, mh::launch_lu_f32(ctx, lo, n, (int64_t)nn, (int)nbatch, dinv, bad));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(LU_host, lo, sizeof(float2) * cnt, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(bad_host, bad, sizeof(int) * (size_t)nbatch,
                                     cudaMemcpyDeviceToHost, ctx->stream));
    return sync_status(ctx, "low-precision LU");
}

int mh_lu_solve_lowp(mh_ctx* ctx, int backend, int64_t n, int64_t nbatch, const double* A_host, int64_t nrhs,
                     int conj_trans, const double* B_host, double* X_host)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (backend != MH_LU_SIMT_F32 && backend != MH_LU_TCGEN05_F16)
        return set_err(ctx, MH_ERR_ARG, "unknown LU backend %d", backend);
    if (n < 1 || nbatch < 1 || nrhs < 1 || nrhs > kMaxRhs || !A_host || !B_host || !X_host)
        return set_err(ctx, MH_ERR_ARG, "bad arguments to mh_lu_solve_lowp");
    const size_t nn = (size_t)n * (size_t)n, cnt = nn * (size_t)nbatch;
    const size_t nv = (size_t)n * (size_t)nrhs, vcnt = nv * (size_t)nbatch;
    auto* d64 = (double2*)ws_get(ctx, WS_D, sizeof(double2) * cnt);
    auto* lo = (float2*)ws_get(ctx, WS_LO, sizeof(float2) * cnt);
    const int64_t dst = backend == MH_LU_TCGEN05_F16 ? mh::lu_dinv_stride_tc(n) : mh::lu_dinv_stride(n);
    auto* dinv = (float2*)ws_get(ctx, WS_DINV, sizeof(float2) * (size_t)dst * (size_t)nbatch);
    auto* bad = (int*)ws_get(ctx, WS_MISC, sizeof(int) * (size_t)nbatch);
    auto* v64 = (double2*)ws_get(ctx, WS_RHS, sizeof(double2) * vcnt);
    auto* v32 = (float2*)ws_get(ctx, WS_TMP32, sizeof(float2) * vcnt);
    if (!d64 || !lo || !dinv || !bad || !v64 || !v32) return MH_ERR_OOM;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d64, A_host, sizeof(double2) * cnt, cudaMemcpyHostToDevice,
                                     ctx->stream));
    MH_CUDA_TRY(ctx, mh::launch_to_f32(ctx, d64, lo, (int64_t)cnt));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(bad, 0, sizeof(int) * (size_t)nbatch, ctx->stream));
    if (backend == MH_LU_TCGEN05_F16) {
        auto* panels = (unsigned char*)ws_get(ctx, WS_PANEL,
                                              (size_t)mh::lu_panel_bytes_tc(n) * (size_t)nbatch);
        if (!panels) return MH_ERR_OOM;
        MH_CUDA_TRY(ctx, mh::launch_lu_tc(ctx, lo, n, (int64_t)nn, (int)nbatch, dinv, panels, bad));
    }
    else
        MH_CUDA_TRY(ctx, mh::launch_lu_f32(ctx, lo, n, (int64_t)nn, (int)nbatch, dinv, bad));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(v64, B_host, sizeof(double2) * vcnt, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, mh::launch_to_f32(ctx, v64, v32, (int64_t)vcnt));
    MH_CUDA_TRY(ctx, mh::launch_lu_solve_persist(ctx, backend, conj_trans != 0, lo, n, (int64_t)nn, (int)nbatch,
                                                 dinv, v32, (int64_t)nv, (int)nrhs, bad));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(v64, 0, sizeof(double2) * vcnt, ctx->stream));
    MH_CUDA_TRY(ctx, mh::launch_add_f32(ctx, v64, v32, (int64_t)vcnt));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(X_host, v64, sizeof(double2) * vcnt, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<int> h_bad((size_t)nbatch);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(h_bad.data(), bad, sizeof(int) * (size_t)nbatch, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    if ((rc = sync_status(ctx, "low-precision solve"))) return rc;
    // marks of the factorisation (1: zero or non-finite pivot; 2: a tensor-core
    // wait ran out) and of the solve (3: a flag wait ran out)
    for (int64_t b = 0; b < nbatch; ++b) {
        if (h_bad[(size_t)b] == 1)
            return set_err(ctx, MH_ERR_SINGULAR, "matrix %lld: zero or non-finite pivot in the low-precision LU",
                           (long long)b);
        if (h_bad[(size_t)b] == 2 || h_bad[(size_t)b] == 3)
            return set_err(ctx, MH_ERR_TIMEOUT, "matrix %lld: a bounded device wait of the %s ran out",
                           (long long)b, h_bad[(size_t)b] == 2 ? "factorisation" : "triangular solve");
    }
    return MH_OK;
}

int mh_ctx_set_lu_schedule(mh_ctx* ctx, int64_t n, int groups, int outer_panels, int update_kernel)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (n < 0 || groups < 1 || groups > kLuGroups || outer_panels < 2 || outer_panels > 8 || (outer_panels & 1) ||
        update_kernel < 0 || update_kernel > 1)
        return set_err(ctx, MH_ERR_ARG,
                       "LU schedule: need n >= 0, 1 <= groups <= %d, outer_panels in {2, 4, 6, 8}, update_kernel 0 or 1",
                       kLuGroups);
    LuSchedule s;
    s.groups = groups;
    s.outer = outer_panels;
    s.update = update_kernel;
    if (n == 0) {
        ctx->lu_default = s;
        return MH_OK;
    }
    for (auto& e : ctx->lu_table)
        if (e.first == n) {
            e.second = s;
            return MH_OK;
        }
    ctx->lu_table.emplace_back(n, s);
    return MH_OK;
}

int mh_ctx_get_lu_schedule(mh_ctx* ctx, int64_t n, int* groups, int* outer_panels, int* update_kernel)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (n < 0 || !groups || !outer_panels || !update_kernel)
        return set_err(ctx, MH_ERR_ARG, "bad arguments to mh_ctx_get_lu_schedule");
    const LuSchedule s = n == 0 ? ctx->lu_default : ctx->lu_schedule(n);
    *groups = s.groups;
    *outer_panels = s.outer;
    *update_kernel = s.update;
    return MH_OK;
}

int mh_lu_autotune(mh_ctx* ctx, int64_t n, int64_t nbatch, int ncand, const int* groups, const int* outer_panels,
                   const int* update_kernel, double* ms, int* best)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (n < 1 || nbatch < 1 || ncand < 1 || !groups || !outer_panels || !update_kernel || !ms)
        return set_err(ctx, MH_ERR_ARG, "bad arguments to mh_lu_autotune");
    for (int c = 0; c < ncand; ++c)
        if (groups[c] < 1 || groups[c] > kLuGroups || outer_panels[c] < 2 || outer_panels[c] > 8 ||
            (outer_panels[c] & 1) || update_kernel[c] < 0 || update_kernel[c] > 1)
            return set_err(ctx, MH_ERR_ARG,
                           "candidate %d: need 1 <= groups <= %d, outer_panels in {2, 4, 6, 8}, update_kernel 0 or 1",
                           c, kLuGroups);
    const size_t nn = (size_t)n * (size_t)n;
    auto* lo = (float2*)ws_get(ctx, WS_LO, sizeof(float2) * nn * (size_t)nbatch);
    auto* dinv = (float2*)ws_get(ctx, WS_DINV, sizeof(float2) * (size_t)mh::lu_dinv_stride_tc(n) * (size_t)nbatch);
    auto* panels = (unsigned char*)ws_get(ctx, WS_PANEL, (size_t)mh::lu_panel_bytes_tc(n) * (size_t)nbatch);
    auto* bad = (int*)ws_get(ctx, WS_MISC, sizeof(int) * (size_t)nbatch);
    if (!lo || !dinv || !panels || !bad) return MH_ERR_OOM;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MH_CUDA_TRY(ctx, cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return set_err(ctx, MH_ERR_CUDA, "event creation failed");
    }
    const auto table = ctx->lu_table;
    const LuSchedule dflt = ctx->lu_default;
    ctx->lu_table.clear();
    cudaError_t e = cudaSuccess;
    int fastest = 0;
    for (int c = 0; c < ncand && e == cudaSuccess; ++c) {
        ctx->lu_default.groups = groups[c];
        ctx->lu_default.outer = outer_panels[c];
        ctx->lu_default.update = update_kernel[c];
        ms[c] = INFINITY;
        // one warm-up factorisation, then one timed; fresh matrices each time
        for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
            if ((e = mh::launch_fill_lu_test(ctx, lo, n, (int)nbatch)) != cudaSuccess) break;
            if ((e = cudaMemsetAsync(bad, 0, sizeof(int) * (size_t)nbatch, ctx->stream)) != cudaSuccess) break;
            if ((e = cudaEventRecord(e0, ctx->stream)) != cudaSuccess) break;
            if ((e = mh::launch_lu_tc(ctx, lo, n, (int64_t)nn, (int)nbatch, dinv, panels, bad)) != cudaSuccess) break;
            if ((e = cudaEventRecord(e1, ctx->stream)) != cudaSuccess) break;
            if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
            float t = 0.f;
            if ((e = cudaEventElapsedTime(&t, e0, e1)) != cudaSuccess) break;
            ms[c] = t;
        }
        if (e == cudaSuccess && ms[c] < ms[fastest]) fastest = c;
    }
    ctx->lu_table = table;
    ctx->lu_default = dflt;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return set_err(ctx, MH_ERR_CUDA, "LU autotune: %s", cudaGetErrorString(e));
    if ((rc = mh_ctx_set_lu_schedule(ctx, n, groups[fastest], outer_panels[fastest], update_kernel[fastest])))
        return rc;
    if (best) *best = fastest;
    return MH_OK;
}

int mh_ctx_set_wave_series_fp32(mh_ctx* ctx, int level)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (level < 0 || level > 2) return set_err(ctx, MH_ERR_ARG, "wave series precision level must be 0, 1 or 2");
    ctx->wave_series_fp32 = level;
    return MH_OK;
}

int mh_ctx_set_wait_injection(mh_ctx* ctx, int enable)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    ctx->inject_wait_timeout = enable != 0;
    return MH_OK;
}

int mh_wave_term(mh_ctx* ctx, uint32_t which, int64_t n, const double* r, const double* z,
                 double* out)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (which != MH_GF_WU && which != MH_GF_DELHOMMEAU)
        return set_err(ctx, MH_ERR_ARG, "mh_wave_term evaluates MH_GF_WU or MH_GF_DELHOMMEAU");
    if (n <= 0 || !r || !z || !out) return set_err(ctx, MH_ERR_ARG, "bad point arrays");
    const double* tab = mh::delh_table_for(ctx, which, &rc);
    if (rc) return rc;
    size_t b = sizeof(double) * (size_t)n;
    auto* d = (double*)ws_get(ctx, WS_TMP, b * 8);
    if (!d) return MH_ERR_OOM;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d, r, b, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(d + n, z, b, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, mh::launch_wave_term(ctx, tab, which, n, d, d + n, d + 2 * n));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(out, d + 2 * n, 6 * b, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_status(ctx, "wave term");
}

int mh_mesh_create(mh_ctx* ctx, int64_t nfaces, int64_t nvertices, const double* vertices,
                   const int64_t* faces, const double* centers, const double* normals,
                   const double* areas, const double* radii, mh_mesh** out)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (!out) return set_err(ctx, MH_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (nfaces <= 0 || nvertices <= 0)
        return set_err(ctx, MH_ERR_ARG, "nfaces and nvertices must be positive");
    if (!vertices || !faces || !centers || !normals || !areas || !radii)
        return set_err(ctx, MH_ERR_ARG, "a mesh array is NULL");
    for (int64_t q = 0; q < 4 * nfaces; ++q)
        if (faces[q] < 0 || faces[q] >= nvertices)
            return set_err(ctx, MH_ERR_ARG, "face vertex index %lld out of range [0, %lld)",
                           (long long)faces[q], (long long)nvertices);
    if (!finite_array(vertices, 3 * nvertices) || !finite_array(centers, 3 * nfaces) ||
        !finite_array(normals, 3 * nfaces) || !finite_array(areas, nfaces) ||
        !finite_array(radii, nfaces))
        return set_err(ctx, MH_ERR_ARG, "mesh arrays must be finite");
    // Host-side staging of the structure-of-arrays geometry.
    const int64_t n = nfaces;
    double* h = new (std::nothrow) double[(size_t)G_NFIELDS * (size_t)n];
    if (!h) return set_err(ctx, MH_ERR_OOM, "host allocation failed");
    for (int64_t i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) {
            h[(G_CX + c) * n + i] = centers[c * n + i];
            h[(G_NX + c) * n + i] = normals[c * n + i];
        }
        h[G_AREA * n + i] = areas[i];
        h[G_RADIUS * n + i] = radii[i];
        for (int a = 0; a < 4; ++a) {
            int64_t v = faces[a * n + i];
            for (int c = 0; c < 3; ++c) h[(G_V + 3 * a + c) * n + i] = vertices[c * nvertices + v];
        }
    }
    auto* m = new (std::nothrow) mh_mesh();
    if (!m) {
        delete[] h;
        return set_err(ctx, MH_ERR_OOM, "host allocation failed");
    }
    m->n = n;
    m->nv = nvertices;
    m->device = ctx->device;
    try {
        m->faces.assign(faces, faces + 4 * n);
        MeshPart part;
        part.nf = n;
        part.nv = nvertices;
        m->parts.push_back(part);
    } catch (...) {
        delete[] h;
        delete m;
        return set_err(ctx, MH_ERR_OOM, "host allocation failed");
    }
    size_t bytes = sizeof(double) * (size_t)G_NFIELDS * (size_t)n;
    // stream-ordered allocation: no device-wide synchronisation, so meshes
    // come and go without stalling other contexts
    cudaError_t e = cudaMallocAsync((void**)&m->geom, bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->geom, h, bytes, cudaMemcpyHostToDevice, ctx->stream);
    // the vertices too, so that the mesh can be combined with generated ones
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&m->verts, sizeof(double) * 3 * (size_t)nvertices, ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m->verts, vertices, sizeof(double) * 3 * (size_t)nvertices, cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    delete[] h;
    if (e != cudaSuccess) {
        if (m->geom) cudaFree(m->geom);
        if (m->verts) cudaFree(m->verts);
        delete m;
        return set_err(ctx, e == cudaErrorMemoryAllocation ? MH_ERR_OOM : MH_ERR_CUDA,
                       "mesh upload failed: %s", cudaGetErrorString(e));
    }
    *out = m;
    return MH_OK;
}

int mh_mesh_destroy(mh_ctx* ctx, mh_mesh* mesh)
{
    if (!mesh) return MH_OK;
    if (ctx) {
        // released after the ctx's work issued so far, without waiting for it
        // or synchronising the device
        cudaSetDevice(ctx->device);
        if (mesh->geom) cudaFreeAsync(mesh->geom, ctx->stream);
        if (mesh->verts) cudaFreeAsync(mesh->verts, ctx->stream);
    } else {
        if (mesh->geom) cudaFree(mesh->geom);
        if (mesh->verts) cudaFree(mesh->verts);
    }
    delete mesh;
    return MH_OK;
}

int mh_mesh_nfaces(const mh_mesh* mesh, int64_t* nfaces)
{
    if (!mesh || !nfaces) return MH_ERR_ARG;
    *nfaces = mesh->n;
    return MH_OK;
}

int mh_assemble_matrices_device(mh_ctx* ctx, const mh_mesh* mesh, double wavenumber,
                                uint32_t gf_mask, int direct, void* S_dev, void* D_dev)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if ((rc = check_mesh(ctx, mesh))) return rc;
    if ((rc = valid_mask(ctx, gf_mask))) return rc;
    if (!std::isfinite(wavenumber) || wavenumber < 0.0)
        return set_err(ctx, MH_ERR_ARG, "wavenumber must be finite and non-negative");
    if ((gf_mask & (MH_GF_WU | MH_GF_DELHOMMEAU)) && !(wavenumber > 0.0))
        return set_err(ctx, MH_ERR_ARG, "wave terms need a positive wavenumber");
    if (!S_dev && !D_dev) return MH_OK;
    const double* tab = mh::delh_table_for(ctx, gf_mask, &rc);
    if (rc) return rc;
    MH_CUDA_TRY(ctx, mh::launch_assemble_f64(ctx, mesh, wavenumber, gf_mask, direct, tab,
                                             (double2*)S_dev, (double2*)D_dev));
    return sync_status(ctx, "assembly");
}

int mh_assemble_matrices(mh_ctx* ctx, const mh_mesh* mesh, double wavenumber, uint32_t gf_mask,
                         int direct, double* S_out, double* D_out)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if ((rc = check_mesh(ctx, mesh))) return rc;
    const int64_t n = mesh->n;
    const size_t mat = sizeof(double2) * (size_t)n * (size_t)n;
    void* S = S_out ? ws_get(ctx, WS_S, mat) : nullptr;
    void* D = D_out ? ws_get(ctx, WS_D, mat) : nullptr;
    if ((S_out && !S) || (D_out && !D)) return MH_ERR_OOM;
    if ((rc = mh_assemble_matrices_device(ctx, mesh, wavenumber, gf_mask, direct, S, D))) return rc;
    if (S_out) MH_CUDA_TRY(ctx, cudaMemcpyAsync(S_out, S, mat, cudaMemcpyDeviceToHost, ctx->stream));
    if (D_out) MH_CUDA_TRY(ctx, cudaMemcpyAsync(D_out, D, mat, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_status(ctx, "copy of S/D to host");
}

int mh_solve(mh_ctx* ctx, int64_t n, const double* D, const double* S, const double* bc,
             int64_t nrhs, int direct, double* phi_out)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if (n <= 0 || nrhs <= 0) return set_err(ctx, MH_ERR_ARG, "n and nrhs must be positive");
    if (!D || !S || !bc || !phi_out) return set_err(ctx, MH_ERR_ARG, "a solve argument is NULL");
    const size_t mat = sizeof(double2) * (size_t)n * (size_t)n;
    const size_t vec = sizeof(double2) * (size_t)n * (size_t)nrhs;
    auto* dD = (double2*)ws_get(ctx, WS_D, mat);
    auto* dS = (double2*)ws_get(ctx, WS_S, mat);
    auto* dB = (double2*)ws_get(ctx, WS_RHS, vec);
    auto* dP = (double2*)ws_get(ctx, WS_PHI, vec);
    if (!dD || !dS || !dB || !dP) return MH_ERR_OOM;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(dD, D, mat, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(dS, S, mat, cudaMemcpyHostToDevice, ctx->stream));
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(dB, bc, vec, cudaMemcpyHostToDevice, ctx->stream));
    if ((rc = solve_fp64_device(ctx, n, dD, dS, dB, nrhs, direct, dP))) return rc;
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(phi_out, dP, vec, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_status(ctx, "solve");
}

int mh_calculate_radiation_forces(mh_ctx* ctx, const mh_mesh* mesh, const double* dof,
                                  int64_t dof_rows, double omega, double rho, double g,
                                  uint32_t gf_mask, int direct, int precision, double out[2])
{
    if (!out) return ctx ? set_err(ctx, MH_ERR_ARG, "out is NULL") : MH_ERR_ARG;
    double2 F;
    int rc = front_door(ctx, mesh, dof, dof_rows, omega, rho, g, gf_mask, direct, precision, false,
                        0.0, &F);
    if (rc) return rc;
    out[0] = F.x / (omega * omega);  // src/waves.jl:36
    out[1] = F.y / omega;
    return MH_OK;
}

int mh_diffraction_force(mh_ctx* ctx, const mh_mesh* mesh, double omega, const double* dof,
                         int64_t dof_rows, double beta, double rho, double g, uint32_t gf_mask,
                         int direct, int precision, double out[2])
{
    if (!out) return ctx ? set_err(ctx, MH_ERR_ARG, "out is NULL") : MH_ERR_ARG;
    double2 F;
    int rc = front_door(ctx, mesh, dof, dof_rows, omega, rho, g, gf_mask, direct, precision, true,
                        beta, &F);
    if (rc) return rc;
    out[0] = F.x;
    out[1] = F.y;
    return MH_OK;
}

}  // extern "C"

namespace {

int check_batch(mh_ctx* ctx, const mh_mesh* mesh, int64_t n_omega, const double* omegas, int64_t n_dof,
                const double* dofs, int64_t n_beta, const double* betas, double rho, double g,
                uint32_t gf_mask, int precision, double tol, int max_iter)
{
    int rc;
    if ((rc = check_ctx(ctx))) return rc;
    if ((rc = check_mesh(ctx, mesh))) return rc;
    if ((rc = valid_mask(ctx, gf_mask))) return rc;
    if (n_omega <= 0 || !omegas) return set_err(ctx, MH_ERR_ARG, "need at least one frequency");
    for (int64_t z = 0; z < n_omega; ++z)
        if (!(omegas[z] > 0.0) || !std::isfinite(omegas[z]))
            return set_err(ctx, MH_ERR_ARG, "frequencies must be positive and finite");
    if (n_dof < 1 || n_beta < 0 || n_dof + n_beta > kMaxRhs)
        return set_err(ctx, MH_ERR_ARG, "need 1 <= n_dof and n_dof + n_beta <= %d", kMaxRhs);
    if (!dofs || (n_beta > 0 && !betas)) return set_err(ctx, MH_ERR_ARG, "dofs / betas is NULL");
    if (!finite_array(dofs, 3 * mesh->n * n_dof) || (n_beta && !finite_array(betas, n_beta)))
        return set_err(ctx, MH_ERR_ARG, "dofs and betas must be finite");
    if (!(g > 0.0) || !std::isfinite(g) || !std::isfinite(rho))
        return set_err(ctx, MH_ERR_ARG, "g must be positive and rho finite");
    if (precision != MH_PRECISION_FP64 && precision != MH_PRECISION_MIXED)
        return set_err(ctx, MH_ERR_ARG, "unknown precision %d", precision);
    if (precision == MH_PRECISION_MIXED) {
        if (!(tol > 0.0) || max_iter < 1 || max_iter > 100)
            return set_err(ctx, MH_ERR_ARG, "mixed precision needs tol > 0 and 1 <= max_iter <= 100");
        if ((gf_mask & MH_GF_WU) && (gf_mask & MH_GF_DELHOMMEAU))
            return set_err(ctx, MH_ERR_ARG, "the mixed path takes one wave term (GFWu or Delhommeau)");
    }
    return MH_OK;
}

}  // namespace

extern "C" {

int mh_hydro_batch(mh_ctx* ctx, const mh_mesh* mesh, int64_t n_omega, const double* omegas,
                   int64_t n_dof, const double* dofs, int64_t n_beta, const double* betas,
                   double rho, double g, uint32_t gf_mask, int direct, int precision, double tol,
                   int max_iter, double* added_mass, double* damping, double* diffraction,
                   double* froude_krylov, mh_batch_info* info)
{
    int rc;
    const bool batched64 = precision == MH_PRECISION_FP64_BATCHED;
    if ((rc = check_batch(ctx, mesh, n_omega, omegas, n_dof, dofs, n_beta, betas, rho, g, gf_mask,
                          batched64 ? MH_PRECISION_FP64 : precision, tol, max_iter)))
        return rc;
    if (batched64 && (gf_mask & MH_GF_WU) && (gf_mask & MH_GF_DELHOMMEAU))
        return set_err(ctx, MH_ERR_ARG, "the batched FP64 path takes one wave term (GFWu or Delhommeau)");
    return mh::hydro_batch(ctx, mesh, n_omega, omegas, n_dof, dofs, n_beta, betas, rho, g, gf_mask,
                           direct, precision, tol, max_iter, added_mass, damping, diffraction,
                           froude_krylov, info);
}

int mh_hydro_batch_vjp(mh_ctx* ctx, const mh_mesh* mesh, int64_t n_omega, const double* omegas,
                       int64_t n_dof, const double* dofs, int64_t n_beta, const double* betas,
                       double rho, double g, uint32_t gf_mask, int direct, int precision, double tol,
                       int max_iter, const double* bar_added_mass, const double* bar_damping,
                       const double* bar_diffraction, const double* bar_froude_krylov,
                       double* added_mass, double* damping, double* diffraction,
                       double* froude_krylov, double* d_vertices, double* d_centers,
                       double* d_normals, double* d_areas, double* d_radii, double* d_omegas,
                       double* d_dofs, mh_batch_info* info)
{
    int rc;
    const bool batched64 = precision == MH_PRECISION_FP64_BATCHED;
    if ((rc = check_batch(ctx, mesh, n_omega, omegas, n_dof, dofs, n_beta, betas, rho, g, gf_mask,
                          batched64 ? MH_PRECISION_FP64 : precision, tol, max_iter)))
        return rc;
    if (batched64 && (gf_mask & MH_GF_WU) && (gf_mask & MH_GF_DELHOMMEAU))
        return set_err(ctx, MH_ERR_ARG, "the batched FP64 path takes one wave term (GFWu or Delhommeau)");
    const int64_t nrad = n_dof * n_dof * n_omega, ndif = 2 * n_dof * n_omega * n_beta;
    if ((bar_added_mass && !finite_array(bar_added_mass, nrad)) ||
        (bar_damping && !finite_array(bar_damping, nrad)) ||
        (bar_diffraction && !finite_array(bar_diffraction, ndif)) ||
        (bar_froude_krylov && !finite_array(bar_froude_krylov, ndif)))
        return set_err(ctx, MH_ERR_ARG, "output cotangents must be finite");
    return mh::hydro_batch_vjp(ctx, mesh, n_omega, omegas, n_dof, dofs, n_beta, betas, rho, g, gf_mask,
                               direct, precision, tol, max_iter, bar_added_mass, bar_damping,
                               bar_diffraction, bar_froude_krylov, added_mass, damping, diffraction,
                               froude_krylov, d_vertices, d_centers, d_normals, d_areas, d_radii,
                               d_omegas, d_dofs, info);
}

int mh_hydro_batch_jvp(mh_ctx* ctx, const mh_mesh* mesh, int64_t n_omega, const double* omegas,
                       int64_t n_dof, const double* dofs, int64_t n_beta, const double* betas,
                       double rho, double g, uint32_t gf_mask, int direct, int precision, double tol,
                       int max_iter, const double* t_vertices, const double* t_centers,
                       const double* t_normals, const double* t_areas, const double* t_omegas,
                       const double* t_dofs, double* added_mass, double* damping, double* diffraction,
                       double* froude_krylov, double* d_added_mass, double* d_damping,
                       double* d_diffraction, double* d_froude_krylov, mh_batch_info* info)
{
    int rc;
    if ((rc = check_batch(ctx, mesh, n_omega, omegas, n_dof, dofs, n_beta, betas, rho, g, gf_mask,
                          precision, tol, max_iter)))
        return rc;
    if ((gf_mask & MH_GF_WU) && (gf_mask & MH_GF_DELHOMMEAU))
        return set_err(ctx, MH_ERR_ARG, "the tangent path takes one wave term (GFWu or Delhommeau)");
    const int64_t n = mesh->n;
    if ((t_vertices && !finite_array(t_vertices, 3 * mesh->nv)) ||
        (t_centers && !finite_array(t_centers, 3 * n)) || (t_normals && !finite_array(t_normals, 3 * n)) ||
        (t_areas && !finite_array(t_areas, n)) || (t_omegas && !finite_array(t_omegas, n_omega)) ||
        (t_dofs && !finite_array(t_dofs, 3 * n * n_dof)))
        return set_err(ctx, MH_ERR_ARG, "tangents must be finite");
    return mh::hydro_batch_jvp(ctx, mesh, n_omega, omegas, n_dof, dofs, n_beta, betas, rho, g, gf_mask,
                               direct, precision, tol, max_iter, t_vertices, t_centers, t_normals, t_areas,
                               t_omegas, t_dofs, added_mass, damping, diffraction, froude_krylov,
                               d_added_mass, d_damping, d_diffraction, d_froude_krylov, info);
}

}  // extern "C"
