// Meshes generated on the device and their exact derivatives with respect to
// the generators' parameters: the immersed hemisphere (the meshes the
// reference's tests and paper scripts load from Capytaine's mesh_sphere,
// src/meshes.jl:122-127), the WaveBot buoy (src/meshes.jl:247-479), their
// concatenation (combine_meshes, src/meshes.jl:53-99), the derivative of
// every mesh field along one parameter (forward mode) and the contraction of
// mesh-field cotangents into parameter cotangents (reverse mode), which
// replaces the finite-difference rrules of the mesh generators
// (paper/MeshGradients_singlebody.jl:85-167, paper/meshGradients_pair.jl:100-210).
//
// Vertices, faces and the panel fields are computed by kernels straight into
// the mesh's device geometry; the faces also come back to the host once (the
// vertex cotangent scatter of the adjoint reads them there).
#include <cstring>
#include <vector>

#include "mh_internal.h"

using mh::set_err;

namespace {

constexpr double kPiD = 3.14159265358979323846;
constexpr int kGenThreads = 256;
constexpr int64_t kGenMaxPanels = (int64_t)1 << 26;

unsigned gen_blocks(int64_t count) { return (unsigned)((count + kGenThreads - 1) / kGenThreads); }

int gen_ctx(mh_ctx* ctx)
{
    if (!ctx) return MH_ERR_ARG;
    const cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess)
        return set_err(ctx, MH_ERR_CUDA, "cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
    ctx->err.clear();
    return MH_OK;
}

// ---- hemisphere -------------------------------------------------------------
// nb bands of the lower half of a latitude-longitude sphere (polar angle
// theta_b = pi/2 + (pi/2) b / nb) and nphi sectors (phi_s = 2 pi s / nphi):
// vertex b nphi + s for b < nb, the pole last.  which < 0: the vertices;
// which = 0: their derivative with respect to the radius; 1..3: with
// respect to the centre's x, y, z.  V is column-major with leading
// dimension ldv, this part's vertices from row v0.
__global__ void k_hemi_verts(double* __restrict__ V, int64_t ldv, int64_t v0, double R, double cx, double cy,
                             double cz, int nb, int nphi, int which)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nring = (int64_t)nb * nphi;
    if (q > nring) return;
    double x, y, z;
    if (q == nring) {  // the pole
        x = which == 1 ? 1.0 : (which < 0 ? cx : 0.0);
        y = which == 2 ? 1.0 : (which < 0 ? cy : 0.0);
        z = which == 3 ? 1.0 : (which < 0 ? cz - R : (which == 0 ? -1.0 : 0.0));
    } else {
        const int b = (int)(q / nphi), s = (int)(q % nphi);
        const double th = 0.5 * kPiD + 0.5 * kPiD * b / nb;
        const double ph = 2.0 * kPiD * s / nphi;
        const double st = sin(th), ct = cos(th), cp = cos(ph), sp = sin(ph);
        if (which < 0) {
            const double rs = R * st;
            x = cx + rs * cp;
            y = cy + rs * sp;
            z = cz + R * ct;
        } else if (which == 0) {
            x = st * cp;
            y = st * sp;
            z = ct;
        } else {
            x = which == 1 ? 1.0 : 0.0;
            y = which == 2 ? 1.0 : 0.0;
            z = which == 3 ? 1.0 : 0.0;
        }
    }
    V[v0 + q] = x;
    V[ldv + v0 + q] = y;
    V[2 * ldv + v0 + q] = z;
}

// Face (b, s) = (a, b+1 ring, b+1 ring next sector, d); the bottom band's
// faces are triangles through the pole, stored with their last vertex
// repeated.  F: 4 x nf column-major (leading dimension nf), vertex indices
// offset by v0.
__global__ void k_hemi_faces(int64_t* __restrict__ F, int64_t v0, int nb, int nphi)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nf = (int64_t)nb * nphi;
    if (q >= nf) return;
    const int64_t b = q / nphi, s = q % nphi, s2 = (s + 1) % nphi;
    const int64_t a = b * nphi + s, d = b * nphi + s2, pole = nf;
    const bool last = b + 1 == nb;
    F[q] = v0 + a;
    F[nf + q] = v0 + (last ? pole : (b + 1) * nphi + s);
    F[2 * nf + q] = v0 + (last ? d : (b + 1) * nphi + s2);
    F[3 * nf + q] = v0 + d;
}

// ---- WaveBot ----------------------------------------------------------------
// Profile point p (r, z) from the waterline down: a cylinder of radius r1 to
// depth d1 (ncy points), a frustum to radius r2 over d2 (nfr - 1 more), the
// flat bottom to the axis (nbot - 1 more, the last at r = 0).  Linear and
// homogeneous in (d1, d2, r1, r2), so its derivative along one parameter is
// the profile of the unit vector of that parameter.
__device__ __forceinline__ void wb_point(int p, double d1, double d2, double r1, double r2, int nbot, int nfr,
                                         int ncy, double& r, double& z)
{
    if (p < ncy) {
        const double t = (double)p / (ncy - 1);
        r = r1;
        z = -d1 * t;
    } else if (p < ncy + nfr - 1) {
        const double t = (double)(p - ncy + 1) / (nfr - 1);
        r = r1 + (r2 - r1) * t;
        z = -d1 - d2 * t;
    } else {
        const double t = (double)(p - (ncy + nfr - 1) + 1) / (nbot - 1);
        r = r2 * (1.0 - t);
        z = -d1 - d2;
    }
}

// The profile revolved about z: points 0 .. P-2 become rings of nth
// vertices (theta_i = 2 pi i / nth), the last point (r = 0) one vertex on
// the axis.  which < 0: the vertices; 0..3: their derivative with respect
// to r1, r2, d1, d2.
__global__ void k_wb_verts(double* __restrict__ V, int64_t ldv, int64_t v0, double r1, double r2, double d1,
                           double d2, int nbot, int nfr, int ncy, int nth, int which)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int P = ncy + nfr - 1 + nbot - 1;
    const int64_t nring = (int64_t)(P - 1) * nth;
    if (q > nring) return;
    double e1 = d1, e2 = d2, er1 = r1, er2 = r2;
    if (which >= 0) {
        er1 = which == 0 ? 1.0 : 0.0;
        er2 = which == 1 ? 1.0 : 0.0;
        e1 = which == 2 ? 1.0 : 0.0;
        e2 = which == 3 ? 1.0 : 0.0;
    }
    double r, z, x, y;
    if (q == nring) {
        wb_point(P - 1, e1, e2, er1, er2, nbot, nfr, ncy, r, z);
        x = 0.0;
        y = 0.0;
    } else {
        const int p = (int)(q / nth), i = (int)(q % nth);
        wb_point(p, e1, e2, er1, er2, nbot, nfr, ncy, r, z);
        const double th = 2.0 * kPiD * i / nth;
        x = r * cos(th);
        y = r * sin(th);
    }
    V[v0 + q] = x;
    V[ldv + v0 + q] = y;
    V[2 * ldv + v0 + q] = z;
}

// Layer L joins ring L to ring L + 1 by quads (upper i, lower i, lower i+1,
// upper i+1); the last layer joins the last ring to the axis vertex by
// triangles stored with their last vertex repeated.
__global__ void k_wb_faces(int64_t* __restrict__ F, int64_t v0, int P, int nth)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nf = (int64_t)(P - 1) * nth;
    if (q >= nf) return;
    const int64_t L = q / nth, i = q % nth, i2 = (i + 1) % nth;
    const int64_t s1 = L * nth, s2 = (L + 1) * nth;
    int64_t f[4];
    if (L < P - 2) {
        f[0] = s1 + i; f[1] = s2 + i; f[2] = s2 + i2; f[3] = s1 + i2;
    } else {
        f[0] = s1 + i; f[1] = s2; f[2] = s1 + i2; f[3] = s1 + i2;
    }
    for (int k = 0; k < 4; ++k) F[k * nf + q] = v0 + f[k];
}

// ---- panel fields and their derivatives --------------------------------------
struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 v3(const double* V, int64_t ldv, int64_t k) { return {V[k], V[ldv + k], V[2 * ldv + k]}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ V3 operator/(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ V3 cross(V3 u, V3 v)
{
    return {u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
__device__ __forceinline__ double dot(V3 u, V3 v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
__device__ __forceinline__ double norm(V3 u) { return sqrt(u.x * u.x + u.y * u.y + u.z * u.z); }

// Centre (area-weighted centroid of the triangles (a, b, c) and (a, c, d),
// src/meshes.jl:399-408), unit normal of (b - a) x (c - a)
// (src/meshes.jl:413-414), area (both triangles) and radius (radius_max:
// the largest vertex distance, Capytaine's convention for the hemisphere
// meshes; else the distance to the first vertex, src/meshes.jl:353-423) of
// faces f0 .. f0 + nf - 1 (F: leading dimension nf, this part's faces from
// row 0) into the geometry (n panels), with their four vertices.
__global__ void k_face_fields(const double* __restrict__ V, int64_t ldv, const int64_t* __restrict__ F,
                              int64_t f0, int64_t nf, int radius_max, double* __restrict__ geom, int64_t n)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nf) return;
    V3 v[4];
    for (int k = 0; k < 4; ++k) v[k] = v3(V, ldv, F[k * nf + q]);
    const V3 a = v[0], b = v[1], c = v[2], d = v[3];
    const V3 cr1 = cross(b - a, c - a), cr2 = cross(c - a, d - a);
    const double n1 = norm(cr1), area1 = 0.5 * n1, area2 = 0.5 * norm(cr2);
    const double area = area1 + area2;
    const V3 cen = ((a + b + c) / 3.0 * area1 + (a + c + d) / 3.0 * area2) / area;
    const V3 nrm = cr1 / n1;
    double rad = norm(a - cen);
    if (radius_max)
        for (int k = 1; k < 4; ++k) rad = fmax(rad, norm(v[k] - cen));
    const int64_t i = f0 + q;
    geom[G_CX * n + i] = cen.x;
    geom[G_CY * n + i] = cen.y;
    geom[G_CZ * n + i] = cen.z;
    geom[G_NX * n + i] = nrm.x;
    geom[G_NY * n + i] = nrm.y;
    geom[G_NZ * n + i] = nrm.z;
    geom[G_AREA * n + i] = area;
    geom[G_RADIUS * n + i] = rad;
    for (int k = 0; k < 4; ++k) {
        geom[(G_V + 3 * k + 0) * n + i] = v[k].x;
        geom[(G_V + 3 * k + 1) * n + i] = v[k].y;
        geom[(G_V + 3 * k + 2) * n + i] = v[k].z;
    }
}

// Derivative of the fields of k_face_fields along the vertex tangent dV:
// the exact derivatives of the area-weighted centroid, the unit normal, the
// area (a triangle's degenerate second half has none) and the radius (for
// radius_max, that of the farthest vertex).  Outputs column-major with
// leading dimension n: centres and normals n x 3, areas and radii n.
__global__ void k_face_fields_jvp(const double* __restrict__ V, const double* __restrict__ dV, int64_t ldv,
                                  const int64_t* __restrict__ F, int64_t f0, int64_t nf, int radius_max,
                                  double* __restrict__ tc, double* __restrict__ tn, double* __restrict__ ta,
                                  double* __restrict__ tr, int64_t n)
{
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nf) return;
    V3 v[4], w[4];
    for (int k = 0; k < 4; ++k) {
        const int64_t j = F[k * nf + q];
        v[k] = v3(V, ldv, j);
        w[k] = v3(dV, ldv, j);
    }
    const V3 a = v[0], b = v[1], c = v[2], d = v[3];
    const V3 da = w[0], db = w[1], dc = w[2], dd = w[3];
    const V3 cr1 = cross(b - a, c - a), cr2 = cross(c - a, d - a);
    const V3 dcr1 = cross(db - da, c - a) + cross(b - a, dc - da);
    const V3 dcr2 = cross(dc - da, d - a) + cross(c - a, dd - da);
    const double n1 = norm(cr1), n2 = norm(cr2);
    const double area1 = 0.5 * n1, area2 = 0.5 * n2;
    const double dn1 = dot(cr1, dcr1) / n1, dn2 = n2 > 0.0 ? dot(cr2, dcr2) / n2 : 0.0;
    const double darea1 = 0.5 * dn1, darea2 = 0.5 * dn2;
    const double area = area1 + area2, darea = darea1 + darea2;
    const V3 c1 = (a + b + c) / 3.0, c2 = (a + c + d) / 3.0;
    const V3 dc1 = (da + db + dc) / 3.0, dc2 = (da + dc + dd) / 3.0;
    const V3 cen = (c1 * area1 + c2 * area2) / area;
    const V3 dcen = (dc1 * area1 + c1 * darea1 + dc2 * area2 + c2 * darea2 - cen * darea) / area;
    const V3 nrm = cr1 / n1;
    const V3 dnrm = dcr1 / n1 - nrm * (dn1 / n1);
    int kr = 0;
    double rad = norm(a - cen);
    if (radius_max)
        for (int k = 1; k < 4; ++k) {
            const double rk = norm(v[k] - cen);
            if (rk > rad) {
                rad = rk;
                kr = k;
            }
        }
    const double drad = dot(v[kr] - cen, w[kr] - dcen) / rad;
    const int64_t i = f0 + q;
    tc[i] = dcen.x;
    tc[n + i] = dcen.y;
    tc[2 * n + i] = dcen.z;
    tn[i] = dnrm.x;
    tn[n + i] = dnrm.y;
    tn[2 * n + i] = dnrm.z;
    ta[i] = darea;
    tr[i] = drad;
}

// out[0] = sum_k a[k] b[k] over count entries (one CTA, a fixed order).
__global__ void k_dot(const double* __restrict__ a, const double* __restrict__ b, int64_t count, double* out)
{
    __shared__ double red[kGenThreads];
    double acc = 0.0;
    for (int64_t k = threadIdx.x; k < count; k += blockDim.x) acc += a[k] * b[k];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0];
}

// Vertices of one part (which < 0) or their derivative along the part's
// parameter `which`, into V (leading dimension ldv).
void launch_part_verts(const MeshPart& pt, double* V, int64_t ldv, int which, cudaStream_t st)
{
    if (pt.kind == MESH_HEMISPHERE)
        k_hemi_verts<<<gen_blocks(pt.nv), kGenThreads, 0, st>>>(V, ldv, pt.v0, pt.p[0], pt.p[1], pt.p[2], pt.p[3],
                                                               pt.ip[0], pt.ip[1], which);
    else if (pt.kind == MESH_WAVEBOT)
        k_wb_verts<<<gen_blocks(pt.nv), kGenThreads, 0, st>>>(V, ldv, pt.v0, pt.p[0], pt.p[1], pt.p[2], pt.p[3],
                                                             pt.ip[0], pt.ip[1], pt.ip[2], pt.ip[3], which);
}

// A new mesh of one generated part: vertices and faces by the part's
// kernels, panel fields by k_face_fields, faces copied to the host.
int make_generated(mh_ctx* ctx, const MeshPart& part, mh_mesh** out)
{
    const int64_t n = part.nf, nv = part.nv;
    auto* m = new (std::nothrow) mh_mesh();
    if (!m) return set_err(ctx, MH_ERR_OOM, "host allocation failed");
    m->n = n;
    m->nv = nv;
    m->device = ctx->device;
    int64_t* dF = nullptr;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaSuccess;
    try {
        m->faces.resize((size_t)(4 * n));
        m->parts.push_back(part);
    } catch (...) {
        delete m;
        return set_err(ctx, MH_ERR_OOM, "host allocation failed");
    }
    e = cudaMallocAsync((void**)&m->geom, sizeof(double) * G_NFIELDS * (size_t)n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&m->verts, sizeof(double) * 3 * (size_t)nv, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&dF, sizeof(int64_t) * 4 * (size_t)n, st);
    if (e == cudaSuccess) {
        launch_part_verts(part, m->verts, nv, -1, st);
        if (part.kind == MESH_HEMISPHERE)
            k_hemi_faces<<<gen_blocks(n), kGenThreads, 0, st>>>(dF, 0, part.ip[0], part.ip[1]);
        else
            k_wb_faces<<<gen_blocks(n), kGenThreads, 0, st>>>(
                dF, 0, part.ip[2] + part.ip[1] - 1 + part.ip[0] - 1, part.ip[3]);
        k_face_fields<<<gen_blocks(n), kGenThreads, 0, st>>>(m->verts, nv, dF, 0, n, part.radius_max, m->geom, n);
        e = cudaGetLastError();
        ctx->launches += 3;
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->faces.data(), dF, sizeof(int64_t) * 4 * (size_t)n,
                                              cudaMemcpyDeviceToHost, st);
    if (dF) cudaFreeAsync(dF, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        if (m->geom) cudaFreeAsync(m->geom, st);
        if (m->verts) cudaFreeAsync(m->verts, st);
        delete m;
        return set_err(ctx, e == cudaErrorMemoryAllocation ? MH_ERR_OOM : MH_ERR_CUDA, "mesh generation failed: %s",
                       cudaGetErrorString(e));
    }
    *out = m;
    return MH_OK;
}

int nparams_of(const mh_mesh* m)
{
    int np = 0;
    for (const MeshPart& pt : m->parts) np += pt.kind == MESH_UPLOADED ? 0 : kMeshPartParams;
    return np;
}

// Tangents of every field of mesh m along parameter p, into device buffers
// (each zeroed outside the parameter's part): dV nv x 3, tc and tn n x 3,
// ta and tr n.  dF: scratch of 4 x (faces of the part) int64.
int mesh_tangent_device(mh_ctx* ctx, const mh_mesh* m, int p, double* dV, double* tc, double* tn, double* ta,
                        double* tr, int64_t* dF)
{
    const MeshPart* part = nullptr;
    int local = p;
    for (const MeshPart& pt : m->parts) {
        if (pt.kind == MESH_UPLOADED) continue;
        if (local < kMeshPartParams) {
            part = &pt;
            break;
        }
        local -= kMeshPartParams;
    }
    if (!part) return set_err(ctx, MH_ERR_ARG, "parameter %d out of range [0, %d)", p, nparams_of(m));
    const int64_t n = m->n, nv = m->nv;
    cudaStream_t st = ctx->stream;
    MH_CUDA_TRY(ctx, cudaMemsetAsync(dV, 0, sizeof(double) * 3 * nv, st));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(tc, 0, sizeof(double) * 3 * n, st));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(tn, 0, sizeof(double) * 3 * n, st));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(ta, 0, sizeof(double) * n, st));
    MH_CUDA_TRY(ctx, cudaMemsetAsync(tr, 0, sizeof(double) * n, st));
    // the part's faces, from the host copy (global vertex indices)
    std::vector<int64_t> hf((size_t)(4 * part->nf));
    for (int k = 0; k < 4; ++k)
        std::memcpy(hf.data() + k * part->nf, m->faces.data() + k * n + part->f0, sizeof(int64_t) * part->nf);
    MH_CUDA_TRY(ctx, cudaMemcpyAsync(dF, hf.data(), sizeof(int64_t) * hf.size(), cudaMemcpyHostToDevice, st));
    launch_part_verts(*part, dV, nv, local, st);
    k_face_fields_jvp<<<gen_blocks(part->nf), kGenThreads, 0, st>>>(m->verts, dV, nv, dF, part->f0, part->nf,
                                                                   part->radius_max, tc, tn, ta, tr, n);
    ctx->launches += 2;
    MH_CUDA_TRY(ctx, cudaGetLastError());
    // hf must outlive the copy
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MH_OK;
}

bool finite_d(double v) { return std::isfinite(v); }

}  // namespace

extern "C" {

int mh_mesh_hemisphere(mh_ctx* ctx, double radius, double cx, double cy, double cz, int ntheta, int nphi,
                       mh_mesh** out)
{
    int rc;
    if ((rc = gen_ctx(ctx))) return rc;
    if (!out) return set_err(ctx, MH_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!(finite_d(radius) && radius > 0.0) || !finite_d(cx) || !finite_d(cy) || !finite_d(cz))
        return set_err(ctx, MH_ERR_ARG, "the radius must be positive and the centre finite");
    if (ntheta < 2 || nphi < 3) return set_err(ctx, MH_ERR_ARG, "resolution must be at least (2, 3)");
    const int nb = (ntheta + 1) / 2;
    if ((int64_t)nb * nphi > kGenMaxPanels) return set_err(ctx, MH_ERR_ARG, "too many panels");
    MeshPart pt;
    pt.kind = MESH_HEMISPHERE;
    pt.p[0] = radius;
    pt.p[1] = cx;
    pt.p[2] = cy;
    pt.p[3] = cz;
    pt.ip[0] = nb;
    pt.ip[1] = nphi;
    pt.nf = (int64_t)nb * nphi;
    pt.nv = pt.nf + 1;
    pt.radius_max = 1;
    return make_generated(ctx, pt, out);
}

int mh_mesh_wavebot(mh_ctx* ctx, double r1, double r2, double d1, double d2, int n_bottom, int n_frustum,
                    int n_cylinder, int n_theta, mh_mesh** out)
{
    int rc;
    if ((rc = gen_ctx(ctx))) return rc;
    if (!out) return set_err(ctx, MH_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!(finite_d(r1) && r1 > 0.0 && finite_d(r2) && r2 > 0.0) || !finite_d(d1) || !finite_d(d2))
        return set_err(ctx, MH_ERR_ARG, "r1 and r2 must be positive, d1 and d2 finite");
    if (n_bottom < 2 || n_frustum < 2 || n_cylinder < 2)
        return set_err(ctx, MH_ERR_ARG, "each part of the profile needs at least 2 points");
    if (n_theta < 3) return set_err(ctx, MH_ERR_ARG, "n_theta must be at least 3");
    const int64_t P = (int64_t)n_cylinder + n_frustum - 1 + n_bottom - 1;
    if ((P - 1) * n_theta > kGenMaxPanels) return set_err(ctx, MH_ERR_ARG, "too many panels");
    MeshPart pt;
    pt.kind = MESH_WAVEBOT;
    pt.p[0] = r1;
    pt.p[1] = r2;
    pt.p[2] = d1;
    pt.p[3] = d2;
    pt.ip[0] = n_bottom;
    pt.ip[1] = n_frustum;
    pt.ip[2] = n_cylinder;
    pt.ip[3] = n_theta;
    pt.nf = (P - 1) * n_theta;
    pt.nv = pt.nf + 1;
    pt.radius_max = 0;
    return make_generated(ctx, pt, out);
}

int mh_mesh_combine(mh_ctx* ctx, int count, const mh_mesh* const* meshes, mh_mesh** out)
{
    int rc;
    if ((rc = gen_ctx(ctx))) return rc;
    if (!out) return set_err(ctx, MH_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (count < 1 || !meshes) return set_err(ctx, MH_ERR_ARG, "need at least one mesh");
    int64_t n = 0, nv = 0;
    for (int k = 0; k < count; ++k) {
        const mh_mesh* m = meshes[k];
        if (!m || !m->geom || !m->verts) return set_err(ctx, MH_ERR_ARG, "mesh %d is NULL or empty", k);
        if (m->device != ctx->device) return set_err(ctx, MH_ERR_ARG, "mesh %d lives on another device", k);
        n += m->n;
        nv += m->nv;
    }
    auto* c = new (std::nothrow) mh_mesh();
    if (!c) return set_err(ctx, MH_ERR_OOM, "host allocation failed");
    c->n = n;
    c->nv = nv;
    c->device = ctx->device;
    cudaStream_t st = ctx->stream;
    cudaError_t e = cudaMallocAsync((void**)&c->geom, sizeof(double) * G_NFIELDS * (size_t)n, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&c->verts, sizeof(double) * 3 * (size_t)nv, st);
    try {
        c->faces.resize((size_t)(4 * n));
    } catch (...) {
        e = cudaErrorMemoryAllocation;
    }
    int64_t off = 0, voff = 0;
    for (int k = 0; k < count && e == cudaSuccess; ++k) {
        const mh_mesh* m = meshes[k];
        for (int f = 0; f < G_NFIELDS && e == cudaSuccess; ++f)
            e = cudaMemcpyAsync(c->geom + f * n + off, m->geom + f * m->n, sizeof(double) * m->n,
                                cudaMemcpyDeviceToDevice, st);
        for (int q = 0; q < 3 && e == cudaSuccess; ++q)
            e = cudaMemcpyAsync(c->verts + q * nv + voff, m->verts + q * m->nv, sizeof(double) * m->nv,
                                cudaMemcpyDeviceToDevice, st);
        for (int a = 0; a < 4; ++a)
            for (int64_t i = 0; i < m->n; ++i) c->faces[a * n + off + i] = m->faces[a * m->n + i] + voff;
        for (MeshPart pt : m->parts) {
            pt.f0 += off;
            pt.v0 += voff;
            c->parts.push_back(pt);
        }
        off += m->n;
        voff += m->nv;
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        if (c->geom) cudaFreeAsync(c->geom, st);
        if (c->verts) cudaFreeAsync(c->verts, st);
        delete c;
        return set_err(ctx, e == cudaErrorMemoryAllocation ? MH_ERR_OOM : MH_ERR_CUDA, "mesh combination failed: %s",
                       cudaGetErrorString(e));
    }
    *out = c;
    return MH_OK;
}

int mh_mesh_nvertices(const mh_mesh* mesh, int64_t* nvertices)
{
    if (!mesh || !nvertices) return MH_ERR_ARG;
    *nvertices = mesh->nv;
    return MH_OK;
}

int mh_mesh_nparams(const mh_mesh* mesh, int* nparams)
{
    if (!mesh || !nparams) return MH_ERR_ARG;
    *nparams = nparams_of(mesh);
    return MH_OK;
}

int mh_mesh_fields(mh_ctx* ctx, const mh_mesh* mesh, double* vertices, int64_t* faces, double* centers,
                   double* normals, double* areas, double* radii)
{
    int rc;
    if ((rc = gen_ctx(ctx))) return rc;
    if (!mesh || !mesh->geom) return set_err(ctx, MH_ERR_ARG, "mesh is NULL");
    if (mesh->device != ctx->device) return set_err(ctx, MH_ERR_ARG, "the mesh lives on another device");
    if (vertices && !mesh->verts) return set_err(ctx, MH_ERR_ARG, "the mesh keeps no device vertices");
    const int64_t n = mesh->n, nv = mesh->nv;
    cudaStream_t st = ctx->stream;
    if (vertices) MH_CUDA_TRY(ctx, cudaMemcpyAsync(vertices, mesh->verts, sizeof(double) * 3 * nv, cudaMemcpyDefault, st));
    if (faces) MH_CUDA_TRY(ctx, cudaMemcpyAsync(faces, mesh->faces.data(), sizeof(int64_t) * 4 * n, cudaMemcpyDefault, st));
    if (centers)
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(centers, mesh->geom + G_CX * n, sizeof(double) * 3 * n, cudaMemcpyDefault, st));
    if (normals)
        MH_CUDA_TRY(ctx, cudaMemcpyAsync(normals, mesh->geom + G_NX * n, sizeof(double) * 3 * n, cudaMemcpyDefault, st));
    if (areas) MH_CUDA_TRY(ctx, cudaMemcpyAsync(areas, mesh->geom + G_AREA * n, sizeof(double) * n, cudaMemcpyDefault, st));
    if (radii) MH_CUDA_TRY(ctx, cudaMemcpyAsync(radii, mesh->geom + G_RADIUS * n, sizeof(double) * n, cudaMemcpyDefault, st));
    MH_CUDA_TRY(ctx, cudaStreamSynchronize(st));
    return MH_OK;
}

int mh_mesh_tangent(mh_ctx* ctx, const mh_mesh* mesh, int param, double* t_vertices, double* t_centers,
                    double* t_normals, double* t_areas, double* t_radii)
{
    int rc;
    if ((rc = gen_ctx(ctx))) return rc;
    if (!mesh || !mesh->geom) return set_err(ctx, MH_ERR_ARG, "mesh is NULL");
    if (mesh->device != ctx->device) return set_err(ctx, MH_ERR_ARG, "the mesh lives on another device");
    if (param < 0 || param >= nparams_of(mesh))
        return set_err(ctx, MH_ERR_ARG, "parameter %d out of range [0, %d)", param, nparams_of(mesh));
    const int64_t n = mesh->n, nv = mesh->nv;
    const size_t words = (size_t)(3 * nv + 8 * n);
    double* buf = nullptr;
    int64_t* dF = nullptr;
    cudaStream_t st = ctx->stream;
    MH_CUDA_TRY(ctx, cudaMallocAsync((void**)&buf, sizeof(double) * words, st));
    cudaError_t e = cudaMallocAsync((void**)&dF, sizeof(int64_t) * 4 * (size_t)n, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(buf, st);
        return set_err(ctx, MH_ERR_OOM, "device allocation failed");
    }
    double *dV = buf, *tc = dV + 3 * nv, *tn = tc + 3 * n, *ta = tn + 3 * n, *tr = ta + n;
    rc = mesh_tangent_device(ctx, mesh, param, dV, tc, tn, ta, tr, dF);
    if (!rc) {
        struct {
            double* dst;
            const double* src;
            size_t count;
        } cp[5] = {{t_vertices, dV, (size_t)(3 * nv)}, {t_centers, tc, (size_t)(3 * n)},
                   {t_normals, tn, (size_t)(3 * n)}, {t_areas, ta, (size_t)n}, {t_radii, tr, (size_t)n}};
        for (auto& c : cp)
            if (c.dst && !rc && cudaMemcpyAsync(c.dst, c.src, sizeof(double) * c.count, cudaMemcpyDefault, st))
                rc = set_err(ctx, MH_ERR_CUDA, "copying a tangent out failed");
        if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = set_err(ctx, MH_ERR_CUDA, "tangent copy failed");
    }
    cudaFreeAsync(buf, st);
    cudaFreeAsync(dF, st);
    return rc;
}

int mh_mesh_param_vjp(mh_ctx* ctx, const mh_mesh* mesh, const double* bar_vertices, const double* bar_centers,
                      const double* bar_normals, const double* bar_areas, const double* bar_radii,
                      double* bar_params)
{
    int rc;
    if ((rc = gen_ctx(ctx))) return rc;
    if (!mesh || !mesh->geom) return set_err(ctx, MH_ERR_ARG, "mesh is NULL");
    if (mesh->device != ctx->device) return set_err(ctx, MH_ERR_ARG, "the mesh lives on another device");
    if (!bar_params) return set_err(ctx, MH_ERR_ARG, "bar_params is NULL");
    const int np = nparams_of(mesh);
    const int64_t n = mesh->n, nv = mesh->nv;
    const size_t words = (size_t)(2 * (3 * nv + 8 * n) + np);
    double* buf = nullptr;
    int64_t* dF = nullptr;
    cudaStream_t st = ctx->stream;
    MH_CUDA_TRY(ctx, cudaMallocAsync((void**)&buf, sizeof(double) * words, st));
    cudaError_t e = cudaMallocAsync((void**)&dF, sizeof(int64_t) * 4 * (size_t)n, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(buf, st);
        return set_err(ctx, MH_ERR_OOM, "device allocation failed");
    }
    // cotangents (zero where not given) in the layout of the tangents
    double* bars = buf;
    double* tang = bars + 3 * nv + 8 * n;
    double* dots = tang + 3 * nv + 8 * n;
    const double* src[5] = {bar_vertices, bar_centers, bar_normals, bar_areas, bar_radii};
    const size_t cnt[5] = {(size_t)(3 * nv), (size_t)(3 * n), (size_t)(3 * n), (size_t)n, (size_t)n};
    size_t at = 0;
    for (int k = 0; k < 5 && !rc; ++k) {
        e = src[k] ? cudaMemcpyAsync(bars + at, src[k], sizeof(double) * cnt[k], cudaMemcpyDefault, st)
                   : cudaMemsetAsync(bars + at, 0, sizeof(double) * cnt[k], st);
        if (e != cudaSuccess) rc = set_err(ctx, MH_ERR_CUDA, "cotangent upload failed: %s", cudaGetErrorString(e));
        at += cnt[k];
    }
    for (int p = 0; p < np && !rc; ++p) {
        double *dV = tang, *tc = dV + 3 * nv, *tn = tc + 3 * n, *ta = tn + 3 * n, *tr = ta + n;
        rc = mesh_tangent_device(ctx, mesh, p, dV, tc, tn, ta, tr, dF);
        if (!rc) {
            k_dot<<<1, kGenThreads, 0, st>>>(bars, tang, (int64_t)(3 * nv + 8 * n), dots + p);
            ctx->launches += 1;
        }
    }
    if (!rc && np > 0 &&
        (cudaMemcpyAsync(bar_params, dots, sizeof(double) * np, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
         cudaStreamSynchronize(st) != cudaSuccess))
        rc = set_err(ctx, MH_ERR_CUDA, "parameter cotangent copy failed");
    cudaFreeAsync(buf, st);
    cudaFreeAsync(dF, st);
    return rc;
}

}  // extern "C"
