/*
 * FP64 CPU oracle for the MarineHydro.jl boundary-element hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (Green functions, panel integrals, influence-matrix assembly),
 * used as the checker of the CUDA library and as the timed CPU baseline.
 * Nothing in the product path links, loads or calls it; only tests/,
 * __graft_entry__.smoke() and bench.py's CPU legs do.
 *
 * Layout conventions follow the reference (Julia, column-major):
 *   centers/normals  N x 3 column-major  (x[0..N), y[N..2N), z[2N..3N))
 *   vertices         V x 3 column-major
 *   faces            N x 4 column-major, int64, 0-based vertex indices
 *   S, D             N x N column-major complex128 (re, im interleaved)
 */
#ifndef MH_ORACLE_H
#define MH_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Green-function term bits; the same values as the CUDA library's gf_mask. */
#define ORC_GF_RANKINE            1u
#define ORC_GF_RANKINE_REFLECTED  2u
#define ORC_GF_RANKINE_REFL_NEG   4u
#define ORC_GF_WU                 8u
#define ORC_GF_DELHOMMEAU        16u

/* complex exponential integral E1(z), principal branch; out = (re, im) */
void orc_expint_e1(double zr, double zi, double out[2]);

/* Rankine panel integral (rankine.jl:24-63) */
double orc_rankine_integral(const double x[3], const double center[3],
                            const double normal[3], const double verts[12],
                            double area, double radius);
/* Rankine integral + integral of the gradient (rankine.jl:65-123) */
void orc_rankine_both(const double x[3], const double center[3],
                      const double normal[3], const double verts[12],
                      double area, double radius, int wrt_first,
                      double* integral, double grad[3]);

/* Dimensionless wave terms.  out = (G.re, G.im, Gr.re, Gr.im, Gz.re, Gz.im) */
void orc_wu_dimless(double r, double z, double out[6]);          /* wu.jl:19-30 */
void orc_delhommeau_dimless(double r, double z, double out[6]);  /* exact_Guevel_Delhommeau.jl:15-59 */

/* Pair-level integrals summed over the terms in gf_mask:
 *   integral(gfs, e1, e2, k)           -> s[2] complex
 *   integral_gradient(gfs, e1, e2, k)  -> g[6] complex 3-vector            */
void orc_pair_integrals(const double x[3],
                        const double center[3], const double normal[3],
                        const double verts[12], double area, double radius,
                        double k, uint32_t gf_mask, int wrt_first,
                        double s[2], double g[6]);

/* Influence matrices (matrix_assembly.jl:4-42).  S_out/D_out may be NULL.
 * Returns 0 on success, nonzero on bad arguments.  nthreads<=0: OpenMP default. */
int orc_assemble(int64_t n, int64_t nv,
                 const double* centers, const double* normals,
                 const double* areas, const double* radii,
                 const double* vertices, const int64_t* faces,
                 double k, uint32_t gf_mask, int direct,
                 double* S_out, double* D_out, int nthreads);

/* Same, restricted to columns [j0, j1) (used to time a bounded sample). */
int orc_assemble_columns(int64_t n, int64_t nv,
                         const double* centers, const double* normals,
                         const double* areas, const double* radii,
                         const double* vertices, const int64_t* faces,
                         double k, uint32_t gf_mask, int direct,
                         int64_t j0, int64_t j1,
                         double* S_out, double* D_out, int nthreads);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
