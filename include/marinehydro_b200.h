/*
 * marinehydro_b200 -- C ABI of the B200 (sm_100a) boundary-element library.
 *
 * Drop-in for the hot path of MarineHydro.jl: influence-matrix assembly of the
 * Rankine / reflected-Rankine / Wu / exact Guevel-Delhommeau Green functions,
 * the dense complex solve (direct or indirect formulation), the pressure
 * integration that gives added mass, radiation damping and diffraction force,
 * and their adjoints.  The reference is pure Julia; its per-pair multiple
 * dispatch (`integral` / `integral_gradient` on `GreensFunction` subtypes,
 * src/green_functions/abstract_greens_function.jl:47-83) is too fine-grained
 * for a foreign call, so this boundary sits at matrix level
 * (`assemble_matrices`, `solve`) and at output level
 * (`calculate_radiation_forces`, `DiffractionForce`, the batched
 * hydrodynamic-coefficient driver and its gradients).
 *
 * Conventions (all follow the reference's Julia storage):
 *  - matrices and N x 3 arrays are column-major; complex numbers are
 *    interleaved (re, im) float64 pairs, i.e. Julia's ComplexF64;
 *  - faces are 0-based vertex indices, N x 4 int64 (src/meshes.jl:179 adds 1);
 *  - every function returns MH_OK (0) or an MH_ERR_* code and never aborts;
 *    mh_last_error() gives the message;
 *  - host pointers are caller-owned and only read/written during the call;
 *  - one mh_ctx owns one CUDA stream; calls on one ctx must not overlap.
 */
#ifndef MARINEHYDRO_B200_H
#define MARINEHYDRO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MH_OK                 0
#define MH_ERR_ARG            1 /* bad shape / NULL / out-of-range, mirrors the reference's @assert checks (src/meshes.jl:28-34) */
#define MH_ERR_CUDA           2 /* a CUDA runtime / library call failed */
#define MH_ERR_NOT_CONVERGED  3 /* iterative refinement hit its iteration cap */
#define MH_ERR_TIMEOUT        4 /* a bounded device-side wait gave up */
#define MH_ERR_OOM            5 /* device allocation failed */
#define MH_ERR_NO_DEVICE      6 /* no CUDA device / requested device absent */
#define MH_ERR_SINGULAR       7 /* zero pivot in the LU factorisation */

/* Green-function terms, summed like the reference's tuples
 * (abstract_greens_function.jl:18,34,49,65,83).  RANKINE_REFLECTED and
 * RANKINE_REFLECTED_NEGATIVE together cancel, as +G - G does in Julia. */
#define MH_GF_RANKINE                     1u  /* Rankine()                  src/green_functions/rankine.jl */
#define MH_GF_RANKINE_REFLECTED           2u  /* RankineReflected()         src/green_functions/rankine_reflected.jl */
#define MH_GF_RANKINE_REFLECTED_NEGATIVE  4u  /* RankineReflectedNegative() src/green_functions/rankine_reflected_negative.jl */
#define MH_GF_WU                          8u  /* GFWu()                     src/green_functions/wu.jl */
#define MH_GF_DELHOMMEAU                 16u  /* ExactGuevelDelhommeau()    src/green_functions/exact_Guevel_Delhommeau.jl */

/* precision of a solve */
#define MH_PRECISION_FP64   0  /* FP64 assembly + FP64 LU (cuSOLVER zgetrf/zgetrs) */
#define MH_PRECISION_MIXED  1  /* FP64-accurate matrices, low-precision LU, FP64 iterative refinement */
/* FP64 everywhere with the batch structure of the mixed path (mh_hydro_batch
 * and mh_hydro_batch_vjp): the frequency-independent Rankine part once, the
 * frequency-batched wave pass, then cuSOLVER zgetrf/zgetrs per frequency on
 * the FP64 matrices, frequencies spread over four streams (the adjoint solves
 * with the same pivoted factors, conjugate transposed).  The plain-FP64
 * denominator of the mixed path's speed-up. */
#define MH_PRECISION_FP64_BATCHED 2

/* evaluation of the ExactGuevelDelhommeau wave term */
#define MH_DELHOMMEAU_TABLE  0  /* 2-D Chebyshev table built on the device from the FP64 quadrature (default) */
#define MH_DELHOMMEAU_EXACT  1  /* adaptive Gauss-Kronrod quadrature per panel pair, as the reference */

/* low-precision LU of the mixed path */
#define MH_LU_SIMT_F32     0  /* FP32 complex blocked LU on the CUDA cores (block 32) */
#define MH_LU_TCGEN05_F16  1  /* block-64 LU, trailing update as FP16 tcgen05 MMA with FP32 accumulation in tensor memory */

typedef struct mh_ctx mh_ctx;
typedef struct mh_mesh mh_mesh;

/* Diagnostics of a batched solve. */
typedef struct mh_batch_info {
    int32_t refine_iterations; /* mixed: largest number of refinement sweeps used */
    int32_t n_fallback;        /* mixed: problems re-solved with the pivoted FP64 LU */
    double max_rel_residual;   /* mixed: largest final max|b - A x| / max|b| per right-hand side */
} mh_batch_info;

/* ---- library / context ------------------------------------------------ */

/* ABI version (major*10000 + minor*100 + patch). */
int mh_version(void);

/* Number of visible CUDA devices (0 on a machine without a GPU). */
int mh_device_count(int* count);

/* Create a context bound to `device`: one CUDA stream, library handles and a
 * grow-only workspace.  No reference counterpart (the reference is
 * single-process Julia); it replaces Julia's implicit global state. */
int mh_ctx_create(int device, mh_ctx** out);
int mh_ctx_destroy(mh_ctx* ctx);

/* Message of the last error on this context (ctx == NULL: last error of
 * mh_ctx_create or of mh_solve_mixed_noalloc on this thread).  Valid until
 * the next call on the ctx (or on this thread, for NULL). */
const char* mh_last_error(const mh_ctx* ctx);

/* Number of this library's own kernels launched on the ctx so far. */
int mh_ctx_kernel_launches(const mh_ctx* ctx, int64_t* count);

/* The ctx's CUDA stream (a cudaStream_t), e.g. to record timing events. */
int mh_ctx_stream(const mh_ctx* ctx, void** stream);

/* Phase timing with CUDA events on the ctx stream (off by default; turning it
 * on or off resets the totals).  Phases, in order: 0 Rankine part, 1 wave
 * part + FP32 copy, 2 right-hand sides S*BC, 3 FP32 LU, 4 refinement,
 * 5 forces, 6 FP64 assembly, 7 FP64 LU (cuSOLVER), and of the adjoint
 * (mh_hydro_batch_vjp): 8 adjoint solve, 9 wave-term contraction,
 * 10 Rankine contraction, 11 force / boundary-condition reverse and
 * frequency sums.  No reference counterpart (instrumentation). */
int mh_ctx_set_profiling(mh_ctx* ctx, int enable);
int mh_ctx_phase_times(mh_ctx* ctx, int nphases, double* ms, int64_t* calls);

/* How ExactGuevelDelhommeau() is evaluated on this ctx: MH_DELHOMMEAU_TABLE
 * (default) or MH_DELHOMMEAU_EXACT (per-pair adaptive quadrature, the
 * reference's method, src/green_functions/exact_Guevel_Delhommeau.jl:8-26). */
int mh_ctx_set_delhommeau_method(mh_ctx* ctx, int method);

/* Low-precision LU backend of the mixed path on this ctx (MH_LU_*).  No
 * reference counterpart (the reference factors in FP64 with LAPACK). */
int mh_ctx_set_lu_backend(mh_ctx* ctx, int backend);

/* Schedule of the tensor-core LU (MH_LU_TCGEN05_F16) for matrices of n
 * panels: `groups` (1 to 4) groups of matrices factored concurrently, each on
 * its own pair of streams, so that one group's latency-bound diagonal blocks
 * and panel solves overlap another's trailing updates; `outer_panels` (2, 4,
 * 6 or 8) 64-column panels per outer step, the trailing matrix being updated
 * once per outer step with all of them accumulated in tensor memory;
 * `update_kernel` 0 (the trailing tile C read and written through shared
 * memory by bulk copies after the MMAs) or 1 (C staged in tensor memory
 * before the MMAs, which accumulate onto it).  n = 0 sets the default for
 * sizes with no entry of their own (2 groups, 4 panels, kernel 0); otherwise
 * a size uses the entry nearest to it (in log n).  A new ctx holds the
 * entries the autotuner chose on a B200: 512 -> (1, 4, 1), 1024 -> (2, 2, 0),
 * 2048 -> (2, 4, 0).  No reference counterpart
 * (the reference factors with LAPACK). */
int mh_ctx_set_lu_schedule(mh_ctx* ctx, int64_t n, int groups, int outer_panels, int update_kernel);
int mh_ctx_get_lu_schedule(mh_ctx* ctx, int64_t n, int* groups, int* outer_panels, int* update_kernel);

/* Autotuner of that schedule: factors nbatch synthetic n x n diagonally
 * dominant matrices (generated on the device) with each of the ncand
 * candidate schedules (groups[c], outer_panels[c], update_kernel[c]), one warm-up and one
 * timed factorisation each (CUDA events on the ctx stream), writes the times
 * to ms[c] (host, milliseconds), sets the fastest as the ctx's schedule for
 * n and returns its index in *best (may be NULL).  Uses the ctx's workspace
 * (n^2 nbatch complex64 plus the LU scratch).  No reference counterpart. */
int mh_lu_autotune(mh_ctx* ctx, int64_t n, int64_t nbatch, int ncand, const int* groups,
                   const int* outer_panels, const int* update_kernel, double* ms, int* best);

/* Reduced-precision levels of the mixed path's frequency-batched
 * tabulated-Delhommeau pass: 0 all FP64; 1 (the default) the per-frequency
 * Horner series in R in FP32; 2 also the per-pair alpha contraction of the
 * polar table in FP32.  Measured at 2048 panels and 64 frequencies against
 * the FP64 oracle's exact quadrature: A, B, F within 6e-10 (level 0), 2e-9
 * (1), 7.5e-8 (2).  The pair geometry, the log terms, the assembly of S and D and their
 * Rankine parts stay FP64, and the FP64 paths never use these levels.  No
 * reference counterpart (the reference integrates in FP64). */
int mh_ctx_set_wave_series_fp32(mh_ctx* ctx, int level);

/* Failure injection for tests (no reference counterpart): while enabled, the
 * flag waits of the tensor-core backend's triangular solves on this ctx wait
 * on a flag that nothing publishes, with a limit of 64 polls, so each wait
 * expires the way a lost hand-off would.  The solve marks its matrices:
 * mh_lu_solve_lowp returns MH_ERR_TIMEOUT, the batched mixed paths solve the
 * marked matrices with the FP64 LU instead (mh_batch_info.n_fallback).  The
 * kernels still end normally and the ctx stays usable. */
int mh_ctx_set_wait_injection(mh_ctx* ctx, int enable);

/* Pivot-free low-precision LU of nbatch n x n complex matrices as the mixed
 * path computes it: A_host is nbatch x n x n complex128 column-major, LU_host
 * receives the factors (unit-lower L below the diagonal, U on and above) as
 * complex64 (interleaved float32), bad_host[b] flags a matrix: 1 a zero or
 * non-finite pivot, 2 a timed-out tensor-core wait.  Test and diagnostic hook
 * of the factorisation that replaces LAPACK's getrf in `solve`
 * (src/matrix_assembly.jl:105-133).
 * Limits: no pivoting, so it is meant for the diagonally dominant
 * second-kind matrices D and K of this path (partial pivoting moves no row on
 * them); the MH_LU_TCGEN05_F16 backend rounds the trailing-update operands to
 * FP16 without scaling, so entries of the Schur complements must stay within
 * FP16's range (|x| < 65504, and well above 6e-5 to keep precision).  Inside
 * the batched mixed path, a matrix outside these limits is caught by the bad
 * marks or by the FP64 residual and solved by the pivoted FP64 LU instead. */
int mh_lu_factor_lowp(mh_ctx* ctx, int backend, int64_t n, int64_t nbatch, const double* A_host,
                      float* LU_host, int* bad_host);

/* Factors like mh_lu_factor_lowp, then solves op(L U) X = B with those
 * low-precision factors as one step of the mixed refinement does (op = the
 * identity, or the conjugate transpose when conj_trans != 0).  B_host and
 * X_host are nbatch x nrhs x n complex128 (right-hand sides contiguous, 1 <=
 * nrhs <= 16); the solve runs in FP32, X is returned widened to FP64.
 * Returns MH_ERR_SINGULAR when a factorisation met a zero or non-finite
 * pivot and MH_ERR_TIMEOUT when a bounded device wait of the factorisation or
 * of the solve ran out (X_host is then written but not meaningful).  Test
 * and diagnostic hook of the substitution that replaces LAPACK's getrs
 * (src/matrix_assembly.jl:105-133). */
int mh_lu_solve_lowp(mh_ctx* ctx, int backend, int64_t n, int64_t nbatch, const double* A_host, int64_t nrhs,
                     int conj_trans, const double* B_host, double* X_host);

/* Dimensionless wave term at n points (r[i], z[i]), z < 0, on the device:
 * out[6*i .. 6*i+5] = (G, dG/dr, dG/dz) as (re, im) pairs.  `which` is
 * MH_GF_WU (wu.jl:19-30) or MH_GF_DELHOMMEAU (exact_Guevel_Delhommeau.jl:15-59
 * through the ctx's method).  Replaces the reference's test hooks
 * `_dimless_wave_term` / `_d_dimless_wave_term_dr`. */
int mh_wave_term(mh_ctx* ctx, uint32_t which, int64_t n, const double* r, const double* z,
                 double* out);

/* ---- meshes ------------------------------------------------------------ */

/* Upload a panel mesh; replaces `Mesh(vertices, faces, centers, normals,
 * areas, radii, nvertices, nfaces)` (src/meshes.jl:21-36) on the device.
 *   vertices  nvertices x 3, column-major float64
 *   faces     nfaces x 4, column-major int64, 0-based
 *   centers, normals  nfaces x 3 column-major; areas, radii  nfaces   */
int mh_mesh_create(mh_ctx* ctx, int64_t nfaces, int64_t nvertices,
                   const double* vertices, const int64_t* faces,
                   const double* centers, const double* normals,
                   const double* areas, const double* radii,
                   mh_mesh** out);
/* Releases a mesh; pass the ctx that created it: its device memory is then
 * released in stream order on that ctx, after the ctx's work issued so far,
 * without synchronising the device (with ctx = NULL it is freed at once). */
int mh_mesh_destroy(mh_ctx* ctx, mh_mesh* mesh);
int mh_mesh_nfaces(const mh_mesh* mesh, int64_t* nfaces);
int mh_mesh_nvertices(const mh_mesh* mesh, int64_t* nvertices);

/* ---- meshes generated on the device, and their derivatives --------------
 * Vertices, faces and panel fields computed by kernels straight into the
 * mesh's device geometry (no host arrays in, one copy of the faces back to
 * the host), with the exact derivative of every field with respect to the
 * generator's parameters.  Replaces the reference's mesh generators
 * (src/meshes.jl:247-479; the hemispheres its tests and paper scripts load
 * from Capytaine's mesh_sphere, src/meshes.jl:122-127) and the
 * finite-difference rrules that differentiate them
 * (paper/MeshGradients_singlebody.jl:85-167, paper/meshGradients_pair.jl:100-210).
 *
 * Immersed half (z <= cz) of a latitude-longitude sphere of the given radius
 * and centre: ceil(ntheta / 2) polar bands of nphi sectors, the bottom band
 * triangles stored as quads with a repeated vertex; panel radius = largest
 * vertex distance.  Parameters, in order: radius, cx, cy, cz. */
int mh_mesh_hemisphere(mh_ctx* ctx, double radius, double cx, double cy, double cz, int ntheta, int nphi,
                       mh_mesh** out);
/* The WaveBot buoy (src/meshes.jl:458-479): top radius r1, bottom radius r2
 * (both > 0), cylinder height d1, frustum height d2, profile points
 * (n_bottom, n_frustum, n_cylinder) revolved with n_theta sectors; panel
 * radius = distance to the first vertex (src/meshes.jl:353-423).
 * Parameters, in order: r1, r2, d1, d2. */
int mh_mesh_wavebot(mh_ctx* ctx, double r1, double r2, double d1, double d2, int n_bottom, int n_frustum,
                    int n_cylinder, int n_theta, mh_mesh** out);
/* Concatenation of meshes of this ctx's device (combine_meshes,
 * src/meshes.jl:53-99, with cumulative vertex offsets); the inputs stay
 * valid.  The parameters of the result are those of its generated parts in
 * order (an uploaded mesh has none). */
int mh_mesh_combine(mh_ctx* ctx, int count, const mh_mesh* const* meshes, mh_mesh** out);
int mh_mesh_nparams(const mh_mesh* mesh, int* nparams);
/* The mesh's fields, in the layouts of mh_mesh_create, into host or device
 * buffers (each may be NULL). */
int mh_mesh_fields(mh_ctx* ctx, const mh_mesh* mesh, double* vertices, int64_t* faces, double* centers,
                   double* normals, double* areas, double* radii);
/* Forward mode: the derivative of every field with respect to parameter
 * `param` (0 <= param < mh_mesh_nparams), computed on the device, into host
 * or device buffers in the layouts of mh_mesh_fields (each may be NULL);
 * these are the t_* arguments of mh_hydro_batch_jvp. */
int mh_mesh_tangent(mh_ctx* ctx, const mh_mesh* mesh, int param, double* t_vertices, double* t_centers,
                    double* t_normals, double* t_areas, double* t_radii);
/* Reverse mode: the cotangents of the parameters (bar_params, host,
 * mh_mesh_nparams of them) from the cotangents of the fields (host or
 * device, each may be NULL = zero), e.g. the d_* outputs of
 * mh_hydro_batch_vjp: bar_params[p] = sum over fields of bar . tangent_p. */
int mh_mesh_param_vjp(mh_ctx* ctx, const mh_mesh* mesh, const double* bar_vertices, const double* bar_centers,
                      const double* bar_normals, const double* bar_areas, const double* bar_radii,
                      double* bar_params);

/* ---- matrix level ------------------------------------------------------ */

/* S and D (direct) or S and K (indirect), FP64, written to HOST buffers of
 * nfaces*nfaces complex128 (column-major); either may be NULL.
 * Replaces `assemble_matrices(green_functions, mesh, wavenumber; direct)`
 * (src/matrix_assembly.jl:4-42, :97). */
int mh_assemble_matrices(mh_ctx* ctx, const mh_mesh* mesh, double wavenumber,
                         uint32_t gf_mask, int direct,
                         double* S_out, double* D_out);

/* Same, into DEVICE buffers (nfaces*nfaces complex128 each, may be NULL). */
int mh_assemble_matrices_device(mh_ctx* ctx, const mh_mesh* mesh, double wavenumber,
                                uint32_t gf_mask, int direct,
                                void* S_dev, void* D_dev);

/* phi = D \ (S bc) (direct) or phi = S (K \ bc) (indirect), FP64, host
 * buffers; D, S: n x n complex128, bc and phi_out: n x nrhs complex128.
 * Replaces `solve(D, S, bc; direct)` (src/matrix_assembly.jl:105-133). */
int mh_solve(mh_ctx* ctx, int64_t n, const double* D, const double* S,
             const double* bc, int64_t nrhs, int direct, double* phi_out);

/* ---- output level ------------------------------------------------------ */

/* [added mass, radiation damping] for one rigid-body motion `dof` at
 * frequency omega: k = omega^2/g, assembly, bc = -i omega (n . dof), solve,
 * p = i rho omega phi, F = sum p (-(n . dof)) area, out = [Re F/omega^2,
 * Im F/omega].  `dof` is a 3-vector (dof_rows = 1) or an nfaces x 3
 * column-major matrix (dof_rows = nfaces).
 * Replaces `calculate_radiation_forces(mesh, dof, omega)` (src/waves.jl:29-37);
 * the reference hard-codes gf = Rankine+RankineReflected+GFWu and direct=true,
 * which are the values a drop-in caller passes. */
int mh_calculate_radiation_forces(mh_ctx* ctx, const mh_mesh* mesh,
                                  const double* dof, int64_t dof_rows,
                                  double omega, double rho, double g,
                                  uint32_t gf_mask, int direct, int precision,
                                  double out[2]);

/* Complex diffraction force (re, im) for incident Airy waves of heading beta:
 * bc = -(v_inc . n) (src/waves.jl:121-142), solve, p = i rho phi omega,
 * F = sum p (-(n . dof)) area.
 * Replaces `DiffractionForce(mesh, omega, dof)` (src/waves.jl:40-59). */
int mh_diffraction_force(mh_ctx* ctx, const mh_mesh* mesh, double omega,
                         const double* dof, int64_t dof_rows, double beta,
                         double rho, double g, uint32_t gf_mask, int direct,
                         int precision, double out[2]);

/* ---- batched driver ---------------------------------------------------- */

/* Hydrodynamic coefficients of one mesh over n_omega frequencies, every
 * degree of freedom radiating and influenced, and n_beta incident-wave
 * headings.  Replaces `compute_hydrodynamic_coefficients(parameters, body)`
 * (src/problems_and_results.jl:231-236) with parameters = (wave_frequencies,
 * radiating_dofs = influenced_dofs = all dofs, wave_directions): the
 * reference solves one problem per (omega, dof) and (omega, beta)
 * re-assembling each time (src/solve.jl:4-13); here each frequency is
 * assembled once and all its right-hand sides share one factorisation.
 *   dofs          n_dof motion fields, each nfaces x 3 column-major
 *                 (FloatingBody dofs, src/bodies.jl:63-89), concatenated
 *   n_dof + n_beta <= 16
 *   added_mass, damping      n_dof x n_dof x n_omega  ([influenced, radiating, omega])
 *   diffraction, froude_krylov  complex n_dof x n_omega x n_beta ([dof, omega, beta])
 *   (any output may be NULL)
 *   precision     MH_PRECISION_FP64, MH_PRECISION_MIXED or (mh_hydro_batch,
 *                 mh_hydro_batch_vjp) MH_PRECISION_FP64_BATCHED
 *   tol, max_iter mixed only: refinement stops when max|b - A x|/max|b| <= tol
 *                 for every right-hand side; problems that do not get there in
 *                 max_iter sweeps are re-solved in FP64 (info->n_fallback).
 * The mixed path accepts at most one wave term (GFWu or Delhommeau). */
int mh_hydro_batch(mh_ctx* ctx, const mh_mesh* mesh,
                   int64_t n_omega, const double* omegas,
                   int64_t n_dof, const double* dofs,
                   int64_t n_beta, const double* betas,
                   double rho, double g, uint32_t gf_mask, int direct, int precision,
                   double tol, int max_iter,
                   double* added_mass, double* damping,
                   double* diffraction, double* froude_krylov,
                   mh_batch_info* info);

/* ---- adjoint gradients -------------------------------------------------- */

/* Reverse-mode derivative of mh_hydro_batch: runs the same forward batch
 * (outputs as mh_hydro_batch, each may be NULL) and, for the cotangents of
 * its outputs (bar_*, same layouts; NULL = zero), returns the cotangents of
 * every input: the mesh fields as given to mh_mesh_create
 *   d_vertices  n_vertices x 3,  d_centers, d_normals  nfaces x 3,
 *   d_areas, d_radii  nfaces  (radii only select branches: zero),
 * d_omegas (n_omega) and d_dofs (same layout as dofs); any may be NULL.
 * For J(A, B, F, FK) the result is dJ/dx = sum bar_A dA/dx + bar_B dB/dx
 * + Re(conj(bar_F) dF/dx) + Re(conj(bar_FK) dFK/dx) for the real and
 * imaginary parts of complex outputs given as (re, im) pairs.
 * Replaces Zygote's pullback through compute_hydrodynamic_coefficients /
 * calculate_radiation_forces / DiffractionForce: the ImplicitAD adjoint of
 * `solve` (src/matrix_assembly.jl:105-133, implicit_linear at :120) and the
 * pullbacks of the pair integrals (src/green_functions/*.jl) that the
 * reference's tests check (test/outputs_differentiation.jl:59-68, :21-35).
 * The adjoint solve reuses the forward factors (FP64: conjugate-transposed
 * zgetrs; mixed: the low-precision factors with FP64 refinement of
 * D^H x = r to tol, FP64 fallback as in the forward).  Arguments and errors
 * as mh_hydro_batch; non-finite cotangents are MH_ERR_ARG. */
int mh_hydro_batch_vjp(mh_ctx* ctx, const mh_mesh* mesh,
                       int64_t n_omega, const double* omegas,
                       int64_t n_dof, const double* dofs,
                       int64_t n_beta, const double* betas,
                       double rho, double g, uint32_t gf_mask, int direct, int precision,
                       double tol, int max_iter,
                       const double* bar_added_mass, const double* bar_damping,
                       const double* bar_diffraction, const double* bar_froude_krylov,
                       double* added_mass, double* damping,
                       double* diffraction, double* froude_krylov,
                       double* d_vertices, double* d_centers, double* d_normals,
                       double* d_areas, double* d_radii, double* d_omegas, double* d_dofs,
                       mh_batch_info* info);

/* Forward-mode derivative of mh_hydro_batch along one direction of the
 * inputs: the tangents of the mesh fields (t_vertices n_vertices x 3,
 * t_centers and t_normals nfaces x 3, t_areas nfaces; radii only select
 * branches and have none), of the frequencies (t_omegas) and of the dof
 * fields (t_dofs, layout of dofs); any may be NULL (zero).  Returns the
 * outputs (as mh_hydro_batch, each may be NULL) and their tangents
 * d_added_mass, d_damping, d_diffraction, d_froude_krylov (same layouts).
 * Replaces the reference's ForwardDiff path: Dual element types through
 * assemble_matrices (src/matrix_assembly.jl:7-11) and `solve`
 * (:108-114), as test/outputs_differentiation.jl:133-151 uses it.  The
 * tangent solve reuses the forward factors.  One wave term at most
 * (GFWu or Delhommeau); otherwise as mh_hydro_batch. */
int mh_hydro_batch_jvp(mh_ctx* ctx, const mh_mesh* mesh,
                       int64_t n_omega, const double* omegas,
                       int64_t n_dof, const double* dofs,
                       int64_t n_beta, const double* betas,
                       double rho, double g, uint32_t gf_mask, int direct, int precision,
                       double tol, int max_iter,
                       const double* t_vertices, const double* t_centers, const double* t_normals,
                       const double* t_areas, const double* t_omegas, const double* t_dofs,
                       double* added_mass, double* damping,
                       double* diffraction, double* froude_krylov,
                       double* d_added_mass, double* d_damping,
                       double* d_diffraction, double* d_froude_krylov,
                       mh_batch_info* info);

/* ---- allocation-free mixed-precision solve ------------------------------ */

#define MH_NOALLOC_MAX_N    1024
#define MH_NOALLOC_MAX_RHS  16

/* X = A^-1 B for a dense complex128 A (n x n) and B (n x nrhs), all three
 * column-major DEVICE buffers owned by the caller, by the same method as the
 * batched mixed path (pivot-free FP32 LU of A, FP64 refinement until
 * max|B - A X| / max|B| <= tol per column, at most max_iter sweeps), WITHOUT
 * allocating any device memory: its scratch is one static device array of
 * fixed size, so it serves callers that cannot call cudaMalloc (a memory
 * pool that owns the whole device, a fixed-footprint real-time loop, a host
 * thread that must not block on the allocator).  No counterpart in the
 * reference.
 * Limits: n <= MH_NOALLOC_MAX_N, nrhs <= MH_NOALLOC_MAX_RHS (beyond them:
 * MH_ERR_ARG); the static array (~9 MiB) is held by every GPU that loads the
 * library until the process exits.  Runs on the calling thread's current
 * device, on `stream` (a cudaStream_t; NULL = default stream), and returns
 * after the work is done.  All calls on a device share the array: calls that
 * overlap on the GPU race, so serialise them.  The first call on a device
 * looks up the array's address (cudaGetSymbolAddress) and should come before
 * any stream capture; the address is kept for the life of the process, so
 * after cudaDeviceReset of a device this entry point must not be called on
 * it again.  A, B and X must be memory of the current device (or managed
 * memory); a pointer to another GPU's memory or to host memory gives
 * MH_ERR_ARG and nothing is launched.  A bad FP32 pivot or no convergence within max_iter
 * gives MH_ERR_NOT_CONVERGED (X then holds the last iterate).
 * iterations / rel_residual (host, may be NULL) report the sweeps used and
 * the final residual ratio; errors go to mh_last_error(NULL). */
int mh_solve_mixed_noalloc(int64_t n, const void* A, const void* B, int64_t nrhs, void* X,
                           double tol, int max_iter, void* stream,
                           int32_t* iterations, double* rel_residual);

#ifdef __cplusplus
}
#endif
#endif
