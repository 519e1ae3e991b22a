// Internal declarations shared by the library's translation units.
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <stdint.h>

#include <string>

#include "marinehydro_b200.h"

// Device geometry of one mesh: 20 arrays of n doubles (structure of arrays,
// so a warp reading one field of consecutive panels is one coalesced load).
enum GeomField : int {
    G_CX = 0, G_CY, G_CZ,      // panel centres
    G_NX, G_NY, G_NZ,          // unit normals
    G_AREA, G_RADIUS,          // areas, radii
    G_V = 8,                   // vertex a, coord c at field G_V + 3*a + c (a<4, c<3)
    G_NFIELDS = 20
};

struct mh_mesh {
    int64_t n = 0;
    int64_t nv = 0;
    int device = 0;
    double* geom = nullptr;  // device, G_NFIELDS * n doubles
};

// Workspace slots of a context; each is a grow-only device buffer.
enum WsSlot : int {
    WS_S = 0, WS_D, WS_RHS, WS_PHI, WS_TMP, WS_PIV, WS_INFO, WS_LWORK,
    WS_DOF, WS_OUT, WS_LO, WS_DINV, WS_TMP32, WS_MISC, WS_SR, WS_TMP32B, WS_PANEL, WS_NSLOTS
};

// Largest number of right-hand sides (radiating dofs + headings) per frequency.
constexpr int kMaxRhs = 16;

// Phases timed with CUDA events when profiling is on (mh_ctx_set_profiling).
enum Phase : int {
    PH_RANKINE = 0, PH_WAVE, PH_RHS, PH_LU, PH_REFINE, PH_FORCES, PH_FP64_ASSEMBLY, PH_FP64_LU,
    PH_N
};

struct mh_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cublasHandle_t cublas = nullptr;
    cusolverDnHandle_t cusolver = nullptr;
    std::string err;
    int64_t launches = 0;
    int delh_method = MH_DELHOMMEAU_TABLE;
    int lu_backend = MH_LU_TCGEN05_F16;
    double* delh_table = nullptr;  // device, kTabWords doubles (built on first use)
    bool profile = false;
    cudaEvent_t ev[2 * PH_N] = {};
    bool ev_pending[PH_N] = {};
    double phase_ms[PH_N] = {};
    int64_t phase_calls[PH_N] = {};
    void* ws[WS_NSLOTS] = {};
    size_t ws_bytes[WS_NSLOTS] = {};
};

namespace mh {

int set_err(mh_ctx* ctx, int code, const char* fmt, ...);
// Phase timing (no-ops unless ctx->profile): begin/end record events on the
// ctx stream; collect() adds the elapsed times of completed phases.
void phase_begin(mh_ctx* ctx, int ph);
void phase_end(mh_ctx* ctx, int ph);
void phase_collect(mh_ctx* ctx);
// Returns a device buffer of at least `bytes` for `slot` (nullptr + error set on failure).
void* ws_get(mh_ctx* ctx, int slot, size_t bytes);

// ---- kernels (mh_kernels.cu) ----
// S, D: n x n complex128 column-major device buffers (either may be null);
// tab: Delhommeau table or null (adaptive quadrature).
cudaError_t launch_assemble_f64(mh_ctx* ctx, const mh_mesh* m, double k, uint32_t mask,
                                int direct, const double* tab, double2* S, double2* D);
// bc[i] = -i omega (n_i . dof_i); dof is a device 3-vector (dof_rows==1) or n x 3 col-major.
cudaError_t launch_radiation_bc(mh_ctx* ctx, const mh_mesh* m, const double* dof, int64_t dof_rows,
                                double omega, double2* bc);
// bc[i] = -(v_inc(x_i) . n_i) for Airy waves (src/waves.jl:121-142).
cudaError_t launch_airy_bc(mh_ctx* ctx, const mh_mesh* m, double omega, double beta, double g,
                           double2* bc);
// F = sum_j (i rho omega phi_j) * (-(n_j . dof_j)) * area_j, written to F_out (device, 1 complex).
cudaError_t launch_force(mh_ctx* ctx, const mh_mesh* m, const double2* phi, const double* dof,
                         int64_t dof_rows, double rho, double omega, double2* F_out);

// ---- batched FP32 LU (mh_lu.cu) ----
// Elements of the inverse-diagonal-block buffer per matrix.
int64_t lu_dinv_stride(int64_t n);
// Pivot-free LU of nbatch n x n float2 matrices (stride elements apart), in
// place; bad[b] is set when matrix b meets a zero/non-finite pivot.
cudaError_t launch_lu_f32(mh_ctx* ctx, float2* A, int64_t n, int64_t stride, int nbatch,
                          float2* Dinv, int* bad);
// X <- (LU)^-1 X for nrhs <= kMaxRhs right-hand sides per matrix.
cudaError_t launch_lu_solve_f32(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                                const float2* Dinv, float2* X, int64_t xstride, int nrhs);

// ---- tensor-core LU (mh_lu_tc.cu), block size 64 ----
int64_t lu_dinv_stride_tc(int64_t n);
// Bytes of packed FP16 operand panels per matrix (scratch of launch_lu_tc).
int64_t lu_panel_bytes_tc(int64_t n);
cudaError_t launch_lu_tc(mh_ctx* ctx, float2* A, int64_t n, int64_t stride, int nbatch, float2* Dinv,
                         unsigned char* panels, int* bad);
// Block-parallel (LU)^-1 X in place; T: scratch of the same size as X.
cudaError_t launch_lu_solve_tc(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                               const float2* Dinv, float2* X, float2* T, int64_t xstride, int nrhs);
// The same block-parallel solve for the block-size-32 factors of launch_lu_f32.
cudaError_t launch_lu_solve_blocks32(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride,
                                     int nbatch, const float2* Dinv, float2* X, float2* T,
                                     int64_t xstride, int nrhs);

// ---- batched driver (mh_batch.cu) ----
cudaError_t launch_to_f32(mh_ctx* ctx, const double2* a, float2* b, int64_t count);
int hydro_batch(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                const double* dofs, int64_t nbeta, const double* betas, double rho, double g,
                uint32_t mask, int direct, int precision, double tol, int max_iter,
                double* added_mass, double* damping, double* diffraction, double* froude_krylov,
                mh_batch_info* info);

// ---- Delhommeau table (mh_table.cu) ----
int ensure_delh_table(mh_ctx* ctx);
// Table to use for `mask` on this ctx (null: no Delhommeau term or exact quadrature).
const double* delh_table_for(mh_ctx* ctx, uint32_t mask, int* status);
cudaError_t launch_wave_term(mh_ctx* ctx, const double* tab, uint32_t which, int64_t n,
                             const double* r, const double* z, double* out);

}  // namespace mh

#define MH_CUDA_TRY(ctx, expr)                                                             \
    do {                                                                                   \
        cudaError_t _e = (expr);                                                           \
        if (_e != cudaSuccess)                                                             \
            return mh::set_err((ctx), MH_ERR_CUDA, "%s failed: %s", #expr,                 \
                               cudaGetErrorString(_e));                                    \
    } while (0)
