// Internal declarations shared by the library's translation units.
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <utility>
#include <vector>

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

// One generated part of a mesh (mh_mesh_hemisphere, mh_mesh_wavebot), kept so
// that the mesh's fields can be differentiated with respect to the part's
// parameters on the device; a part of kind MESH_UPLOADED has none.
enum MeshKind : int { MESH_UPLOADED = 0, MESH_HEMISPHERE = 1, MESH_WAVEBOT = 2 };
constexpr int kMeshPartParams = 4;
struct MeshPart {
    int kind = MESH_UPLOADED;
    double p[kMeshPartParams] = {};  // hemisphere: radius, cx, cy, cz; wavebot: r1, r2, d1, d2
    int ip[4] = {};                  // hemisphere: bands, sectors; wavebot: n_bottom, n_frustum, n_cylinder, n_theta
    int64_t f0 = 0, nf = 0;          // its faces ...
    int64_t v0 = 0, nv = 0;          // ... and vertices in the mesh
    int radius_max = 0;              // panel radius: 1 largest vertex distance, 0 distance to the first vertex
};

struct mh_mesh {
    int64_t n = 0;
    int64_t nv = 0;
    int device = 0;
    double* geom = nullptr;      // device, G_NFIELDS * n doubles
    std::vector<int64_t> faces;  // host copy, 4 x n column-major (vertex cotangent scatter)
    double* verts = nullptr;     // device, nv x 3 column-major (generated and combined meshes)
    std::vector<MeshPart> parts; // generated and combined meshes: their parts in order
};

// Workspace slots of a context; each is a grow-only device buffer.
enum WsSlot : int {
    WS_S = 0, WS_D, WS_RHS, WS_PHI, WS_TMP, WS_PIV, WS_INFO, WS_LWORK,
    WS_DOF, WS_OUT, WS_LO, WS_DINV, WS_TMP32, WS_MISC, WS_SR, WS_TMP32B, WS_PANEL, WS_FB, WS_COEF32,
    WS_ADJ, WS_WSD, WS_PART, WS_GBAR, WS_TAPE, WS_FLAGS, WS_FLAGS2, WS_NEAR, WS_NEARRES, WS_FALL, WS_REPACK, WS_NSLOTS
};

// Largest number of right-hand sides (radiating dofs + headings) per frequency.
constexpr int kMaxRhs = 16;

// Phases timed with CUDA events when profiling is on (mh_ctx_set_profiling).
enum Phase : int {
    PH_RANKINE = 0, PH_WAVE, PH_RHS, PH_LU, PH_REFINE, PH_FORCES, PH_FP64_ASSEMBLY, PH_FP64_LU,
    PH_ADJ_SOLVE, PH_ADJ_WAVE, PH_ADJ_RANKINE, PH_ADJ_LINEAR, PH_N
};

// Groups of matrices whose blocked LUs run concurrently on their own
// streams, so one group's latency-bound panel work (diagonal blocks, panel
// solves) overlaps another's trailing updates: at most this many.
constexpr int kLuGroups = 4;

// Schedule of the tensor-core LU: groups of matrices on their own stream
// pairs (1 .. kLuGroups), 64-column panels per outer step (even, 2 .. 8) and
// the trailing-update kernel (0: C through shared memory after the MMAs,
// 1: C staged in tensor memory before them).
// The streams and events one group of the tensor-core LU runs on.
struct LuStreams {
    cudaStream_t main, side, strip;
    cudaEvent_t ev_side, ev_panel, ev_strip_go, ev_strip_done;
};

struct LuSchedule {
    int groups = 2;
    int outer = 4;
    int update = 0;
};

struct mh_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;  // every call's work (highest priority)
    cudaStream_t side = nullptr;    // concurrent work inside a call (lowest priority)
    cudaEvent_t ev_panel = nullptr, ev_side = nullptr;
    // further (main, side) stream pairs: the batched LU runs its matrices in
    // kLuGroups groups, group 0 on (stream, side), group g on these; forked
    // from and joined back to stream inside each call
    cudaStream_t grp_main[kLuGroups - 1] = {}, grp_side[kLuGroups - 1] = {};
    cudaEvent_t grp_ev_panel[kLuGroups - 1] = {}, grp_ev_side[kLuGroups - 1] = {}, grp_ev_join[kLuGroups - 1] = {};
    cudaEvent_t ev_fork = nullptr;
    // per LU group: the stream of the in-block strip updates (high priority,
    // concurrent with the next diagonal-block factorisation) and its events
    cudaStream_t lu_strip[kLuGroups] = {};
    cudaEvent_t lu_ev_strip_go[kLuGroups] = {}, lu_ev_strip_done[kLuGroups] = {};
    cublasHandle_t cublas = nullptr;
    cusolverDnHandle_t cusolver = nullptr;
    // cuSOLVER handles on grp_main[g] (created on first use by the batched
    // FP64 path, which factors one frequency per stream concurrently)
    cusolverDnHandle_t cusolver_grp[kLuGroups - 1] = {};
    std::string err;
    int64_t launches = 0;
    int delh_method = MH_DELHOMMEAU_TABLE;
    int lu_backend = MH_LU_TCGEN05_F16;
    // failure injection (tests): the triangular solves' flag waits wait on a
    // flag that nothing publishes, so they expire
    bool inject_wait_timeout = false;
    // reduced-precision levels of the frequency-batched Delhommeau pass
    // (mixed path only): 0 all FP64, 1 the per-frequency Horner series in
    // FP32 (the default: A, B, F within 2e-9 of the FP64 oracle at 2048
    // panels and 64 frequencies), 2 also the alpha contraction in FP32
    int wave_series_fp32 = 1;
    // LU schedules by matrix size (set by hand or by the autotuner); sizes
    // with no entry use the nearest entry in log n, else lu_default
    std::vector<std::pair<int64_t, LuSchedule>> lu_table;
    LuSchedule lu_default;
    LuSchedule lu_schedule(int64_t n) const
    {
        const LuSchedule* best = &lu_default;
        double gap = 1e300;
        for (const auto& e : lu_table) {
            const double d = std::fabs(std::log((double)e.first / (double)n));
            if (d < gap) {
                gap = d;
                best = &e.second;
            }
        }
        return *best;
    }
    // refinement sweeps launched before the first host check, per direction
    // (0: D x = b, 1: D^H x = b): the most any matrix needed in the last call
    int refine_ahead[2] = {2, 2};
    double* delh_table = nullptr;  // device, kTabWords doubles (built on first use)
    bool profile = false;
    // phase timing: events recorded on whichever stream issues the phase
    struct PhaseRec {
        int ph;
        cudaEvent_t b, e;
    };
    std::vector<cudaEvent_t> ev_pool;
    std::vector<PhaseRec> ev_recs;
    cudaEvent_t ev_open[PH_N] = {};
    double phase_ms[PH_N] = {};
    int64_t phase_calls[PH_N] = {};
    void* ws[WS_NSLOTS] = {};
    size_t ws_bytes[WS_NSLOTS] = {};
};

namespace mh {

int set_err(mh_ctx* ctx, int code, const char* fmt, ...);
// Phase timing (no-ops unless ctx->profile): begin/end record events on the
// ctx stream current at the call; collect() waits for the recorded phases and
// adds their elapsed times (a phase issued several times adds every span).
void phase_begin(mh_ctx* ctx, int ph);
void phase_end(mh_ctx* ctx, int ph);
void phase_collect(mh_ctx* ctx);
// Returns a device buffer of at least `bytes` for `slot` (nullptr + error set on failure).
void* ws_get(mh_ctx* ctx, int slot, size_t bytes);

// Opt a kernel in to `bytes` of dynamic shared memory on the current device.
// The limit is per kernel and process-wide, so concurrent contexts that set
// different sizes would race (one lowering it under another's launch): the
// limit is only ever raised, under a process-wide lock.
cudaError_t raise_smem_cap(const void* kernel, size_t bytes);

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
// Diagonally dominant FP32 complex test matrices (the LU autotuner's input).
cudaError_t launch_fill_lu_test(mh_ctx* ctx, float2* A, int64_t n, int nbatch);
cudaError_t launch_lu_tc(mh_ctx* ctx, float2* A, int64_t n, int64_t stride, int nbatch, float2* Dinv,
                         unsigned char* panels, int* bad);
// Block-parallel (LU)^-1 X in place; T: scratch of the same size as X.
cudaError_t launch_lu_solve_tc(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride, int nbatch,
                               const float2* Dinv, float2* X, float2* T, int64_t xstride, int nrhs);
// The same block-parallel solve for the block-size-32 factors of launch_lu_f32.
cudaError_t launch_lu_solve_blocks32(mh_ctx* ctx, const float2* A, int64_t n, int64_t stride,
                                     int nbatch, const float2* Dinv, float2* X, float2* T,
                                     int64_t xstride, int nrhs);

// Persistent (one CTA per matrix, one launch) solve with the factors of
// launch_lu_tc / launch_lu_f32: X <- (LU)^-1 X, or (LU)^-H X when conj_trans.
// bad (device, per matrix, may be null): a flag wait of the tensor-core
// backend that runs out writes 3 there.  done (device, per matrix, may be
// null; needs bad): matrices with done[b] or bad[b] nonzero are skipped.
// stream: where to launch (null: the ctx stream); flags_slot: the workspace
// slot of the hand-off flags (solves running concurrently need their own).
cudaError_t launch_lu_solve_persist(mh_ctx* ctx, int backend, bool conj_trans, const float2* A, int64_t n,
                                    int64_t stride, int nbatch, const float2* Dinv, float2* X, int64_t xstride,
                                    int nrhs, int* bad = nullptr, const int* done = nullptr,
                                    cudaStream_t stream = nullptr, int flags_slot = WS_FLAGS);
// Conjugate-transposed solve D^H X = X with the factors of launch_lu_tc
// (backend MH_LU_TCGEN05_F16) or launch_lu_f32 (MH_LU_SIMT_F32).
cudaError_t launch_lu_solve_ct(mh_ctx* ctx, int backend, const float2* A, int64_t n, int64_t stride,
                               int nbatch, const float2* Dinv, float2* X, float2* T, int64_t xstride,
                               int nrhs);

// ---- batched driver (mh_batch.cu) ----
struct Batch {
    mh_ctx* ctx;
    const mh_mesh* m;
    int64_t n;
    int ndof, nbeta, nrhs;
    const double* d_dofs;
    const double* d_betas;
    double rho, g;
    uint32_t mask;
    int direct;
    // optional (Delhommeau term, mixed path): per pair and frequency the
    // dimensionless (G, G_r), 2 double2 in the layout of S, for the adjoint
    double2* tape = nullptr;
};
// FP64 factors of the problems of a chunk that left the mixed path, kept for
// the adjoint solve (lu: nb matrices, piv: nb x n, used[z] != 0 when set).
struct FallbackStore {
    double2* lu = nullptr;
    int* piv = nullptr;
    std::vector<int> used;
};
cudaError_t launch_to_f32(mh_ctx* ctx, const double2* a, float2* b, int64_t count);
cudaError_t launch_add_f32(mh_ctx* ctx, double2* x, const float2* d, int64_t count);
// R = beta B + alpha op(A) X for nb n x n complex matrices (op = identity or
// ^H), X and B n x nrhs per matrix; B may be R, or null when beta = 0.
// done, bad (device, per matrix, both or neither): skip matrices with either set.
cudaError_t launch_gemv(mh_ctx* ctx, bool conj_trans, const double2* A, int64_t n, int nb, const double2* X,
                        const double2* B, double2* R, int nrhs, double alpha, double beta,
                        const int* done = nullptr, const int* bad = nullptr, cudaStream_t stream = nullptr);
// R = B - op(A) X for nb n x n complex matrices (op = identity or ^H).
cudaError_t launch_residual(mh_ctx* ctx, bool conj_trans, const double2* A, int64_t n, int nb, const double2* X,
                            const double2* B, double2* R, int nrhs);
// out[z] = max over right-hand sides of max|r| / max|b| for nb problems of n x nrhs.
cudaError_t launch_rel_residual(mh_ctx* ctx, const double2* r, const double2* b, int64_t n, int nrhs,
                                int nb, double* out);
// Device force layout (F then FK, see hydro_batch) to the reference's output arrays.
void unpack_outputs(const double2* h, int64_t nomega, const double* omegas, int64_t ndof, int64_t nbeta,
                    double* added_mass, double* damping, double* diffraction, double* froude_krylov);
// C = alpha A B + beta C for nb strided n x n by n x nrhs complex products.
int zgemm_strided(mh_ctx* ctx, int64_t n, int nrhs, const double2* A, const double2* B, double2* C,
                  int nb, double alpha_re, double beta_re);
int fp64_lu_factor(mh_ctx* ctx, int64_t n, double2* A, int* piv);
int fp64_getrs(mh_ctx* ctx, bool conj_trans, int64_t n, const double2* LU, const int* piv, double2* B,
               int nrhs);
int fp64_lu_solve(mh_ctx* ctx, int64_t n, double2* A, double2* B, int nrhs);
int fallback_factor(mh_ctx* ctx, FallbackStore* fb, int64_t n, int nb, int z, const double2* D);
// Per-matrix control of a refinement run, in device memory (one block of
// refine_ctl_bytes(nb)): residual ratios, then marks of bad matrices (low-
// precision LU pivot or wait timeout), of converged ones, and sweep counts.
struct RefineCtl {
    double* res;
    int* bad;
    int* done;
    int* sweeps;
};
size_t refine_ctl_bytes(int nb);
RefineCtl refine_ctl(void* block, int nb);
// Host copy of a RefineCtl after a run.
struct RefineState {
    std::vector<double> res;
    std::vector<int> bad, done, sweeps;
    bool ok(int z) const { return !bad[z] && done[z]; }
    int most_sweeps() const;
};
// Mixed-precision refinement of op(D) X = RHS (op = identity or ^H) for nb
// matrices with the low-precision factors (Dlo, Dinv) and FP64 residuals
// against D64, controlled on the device: each sweep skips the matrices that
// converged (residual ratio <= tol) or are marked bad, and the host checks
// only after the number of sweeps the last call needed (then one sweep at a
// time), at most max_iter sweeps.  c.bad must hold the marks on entry;
// timeouts of the solve add to them.  R (FP64), R32 (FP32): scratch of the
// size of RHS.  Leaves the control block's host copy in h.
int refine_sweeps(mh_ctx* ctx, bool conj_trans, int64_t n, int nb, int nrhs, const double2* D64,
                  const float2* Dlo, const float2* Dinv, const double2* RHS, double2* X, double2* R, float2* R32,
                  const RefineCtl& c, double tol, int max_iter, RefineState& h);
// X = op(D)^-1 RHS for nb problems by refine_sweeps; problems whose forward
// solve fell back (fb.used), are marked bad or do not converge use FP64
// factors.  ctl: a device block of refine_ctl_bytes(nb).
int mixed_refine_solve(mh_ctx* ctx, int64_t n, int nb, int nrhs, const double2* D64, const float2* Dlo,
                       const float2* Dinv, const double2* RHS, double2* X, double2* R, float2* R32, void* ctl,
                       bool conj_trans, double tol, int max_iter, FallbackStore& fb, mh_batch_info* info);
// Frequency-independent Rankine parts SR, DR (n x n real) of the mixed path.
int rankine_real(const Batch& bt, double* SR, double* DR);
// One chunk of the mixed path; leaves S (WS_S), D (WS_D), the low-precision
// factors (WS_LO, WS_DINV), the boundary conditions (WS_RHS), the solution
// (WS_PHI: phi, or sigma when indirect; phi = S sigma in WS_TMP) in place.
int run_mixed_chunk(const Batch& bt, const double* d_omegas, const double* d_k, int nb,
                    const double* SR, const double* DR, double tol, int max_iter, double2* d_F,
                    double2* d_FK, mh_batch_info* info, FallbackStore* fb);
// One chunk of the batched FP64 path (MH_PRECISION_FP64_BATCHED): leaves S
// (WS_S), the pivoted FP64 factors of D (WS_D, pivots in WS_PIV), the
// boundary conditions (WS_RHS), the solution (WS_PHI; phi = S sigma in WS_TMP
// when indirect) in place; writes the wave tape when bt.tape is set.
int run_fp64_chunk(const Batch& bt, const double* d_omegas, const double* d_k, int nb, const double* SR,
                   const double* DR, double2* d_F, double2* d_FK);
// X_z = op(D_z)^-1 X_z with the factors run_fp64_chunk left (op = identity or ^H).
int fp64_batched_getrs(mh_ctx* ctx, bool conj_trans, int64_t n, int nb, int nrhs, double2* X);
cudaError_t launch_bc_batch(const Batch& bt, const double* d_omegas, int nb, double2* BC);
cudaError_t launch_forces_batch(const Batch& bt, const double* d_omegas, int nb, const double2* PHI,
                                double2* d_F, double2* d_FK);
int hydro_batch(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                const double* dofs, int64_t nbeta, const double* betas, double rho, double g,
                uint32_t mask, int direct, int precision, double tol, int max_iter,
                double* added_mass, double* damping, double* diffraction, double* froude_krylov,
                mh_batch_info* info);

// ---- adjoint (mh_adjoint.cu) ----
int hydro_batch_vjp(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                    const double* dofs, int64_t nbeta, const double* betas, double rho, double g,
                    uint32_t mask, int direct, int precision, double tol, int max_iter,
                    const double* bar_added_mass, const double* bar_damping, const double* bar_diffraction,
                    const double* bar_froude_krylov, double* added_mass, double* damping,
                    double* diffraction, double* froude_krylov, double* d_vertices, double* d_centers,
                    double* d_normals, double* d_areas, double* d_radii, double* d_omegas_out,
                    double* d_dofs_out, mh_batch_info* info);

// ---- forward mode (mh_jvp.cu) ----
int hydro_batch_jvp(mh_ctx* ctx, const mh_mesh* m, int64_t nomega, const double* omegas, int64_t ndof,
                    const double* dofs, int64_t nbeta, const double* betas, double rho, double g, uint32_t mask,
                    int direct, int precision, double tol, int max_iter, const double* t_vertices,
                    const double* t_centers, const double* t_normals, const double* t_areas, const double* t_omegas,
                    const double* t_dofs, double* added_mass, double* damping, double* diffraction,
                    double* froude_krylov, double* d_added_mass, double* d_damping, double* d_diffraction,
                    double* d_froude_krylov, mh_batch_info* info);

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
