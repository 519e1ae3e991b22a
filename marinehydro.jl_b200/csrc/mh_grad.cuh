// Device helpers shared by the gradient kernels (reverse mode in
// mh_adjoint.cu, forward mode in mh_jvp.cu): panel staging, warp sums, the
// r, z derivatives of the dimensionless wave terms and the pair geometry of
// the wave term.  Included inside an anonymous namespace of each unit.
#pragma once

constexpr int kGradCols = 16;  // columns (panels in shared memory) per CTA of the pair kernels

using d2 = dualn<2>;
using d6 = dualn<6>;

__device__ __forceinline__ double re_mul(const cplx& a, const cplx& b) { return a.re * b.re - a.im * b.im; }

__device__ __forceinline__ double warp_sum(double v)
{
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ void stage(Panel* sp, const double* __restrict__ geom, int64_t n, int64_t j0)
{
    for (int t = threadIdx.x; t < kGradCols * G_NFIELDS; t += blockDim.x) {
        const int f = t / kGradCols, jj = t % kGradCols;
        const int64_t j = j0 + jj;
        const double v = (j < n) ? geom[(int64_t)f * n + j] : 0.0;
        Panel& p = sp[jj];
        if (f < 3) p.c[f] = v;
        else if (f < 6) p.n[f - 3] = v;
        else if (f == G_AREA) p.area = v;
        else if (f == G_RADIUS) p.radius = v;
        else p.v[f - G_V] = v;
    }
}

// Sum over the block of one value per thread; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    return s;
}

// ---------------------------------------------------------------------------
// wave term
// ---------------------------------------------------------------------------

// Dimensionless wave term (G, G_r, G_z) with its r and z derivatives.
struct GDer {
    cplx G[3];
    cplx Gr[3];
    cplx Gz[3];
};

__device__ __forceinline__ void from_duals(const cx<d2>* o, GDer& g)
{
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        g.G[m] = mk(o[m].re.v, o[m].im.v);
        g.Gr[m] = mk(o[m].re.d[0], o[m].im.d[0]);
        g.Gz[m] = mk(o[m].re.d[1], o[m].im.d[1]);
    }
}

// (r, z) derivatives of Wu's formulas by 2-way dual numbers.
__device__ __noinline__ void wave_dimless_dual(int kind, double r, double z, GDer* g)
{
    d2 rd, zd;
    rd.v = r;
    rd.d[0] = 1.0;
    rd.d[1] = 0.0;
    zd.v = z;
    zd.d[0] = 0.0;
    zd.d[1] = 1.0;
    cx<d2> o[3];
    (void)kind;
    wu_dimless(rd, zd, o);
    from_duals(o, *g);
}

// r, z derivatives of the Delhommeau wave term from its values: with
// G_r = G1 and G_z = G2 = G + 2/R (exact_Guevel_Delhommeau.jl:56), the wave
// part is harmonic in the fluid, so G_zz = G_z - 2z/R^3, G_rz = G_r - 2r/R^3
// and G_rr = -G_r/r - G_zz (-G_zz/2 as r -> 0).  These are the derivatives
// of the function itself (what the reference's AD of its quadrature
// gives), whichever way its values were obtained.
__device__ __forceinline__ void gder_identities(const cplx G[3], double r, double z, double R, GDer& o)
{
    const double iR = 1.0 / R, iR3 = iR * iR * iR;
    const cplx Gzz = G[2] - mk(2.0 * z * iR3, 0.0);
    const cplx Grz = G[1] - mk(2.0 * r * iR3, 0.0);
    const cplx Grr = (r > 1e-3) ? -(G[1] / r) - Gzz : mk(-0.5 * Gzz.re, -0.5 * Gzz.im);
#pragma unroll
    for (int m = 0; m < 3; ++m) o.G[m] = G[m];
    o.Gr[0] = G[1];
    o.Gz[0] = G[2];
    o.Gr[1] = Grr;
    o.Gz[1] = Grz;
    o.Gr[2] = Grz;
    o.Gz[2] = Gzz;
}

// The same with the reciprocals 1/R and 1/r given (hoisted out of a
// frequency loop: R = k rho, r = k dis).
__device__ __forceinline__ void gder_identities_inv(const cplx G[3], double r, double z, double iR, double ir,
                                                    GDer& o)
{
    const double iR3 = iR * iR * iR;
    const cplx Gzz = G[2] - mk(2.0 * z * iR3, 0.0);
    const cplx Grz = G[1] - mk(2.0 * r * iR3, 0.0);
    const cplx Grr = (r > 1e-3) ? -(G[1] * ir) - Gzz : mk(-0.5 * Gzz.re, -0.5 * Gzz.im);
#pragma unroll
    for (int m = 0; m < 3; ++m) o.G[m] = G[m];
    o.Gr[0] = G[1];
    o.Gz[0] = G[2];
    o.Gr[1] = Grr;
    o.Gz[1] = Grz;
    o.Gr[2] = Grz;
    o.Gz[2] = Gzz;
}

// Delhommeau term and its r, z derivatives at one point: the forward's
// value (table, or the quadrature outside it / without a table), then the
// identities.
__device__ __noinline__ void delh_point_grad(const double* __restrict__ tab, double r, double z, GDer* out)
{
    cplx G[3];
    if (tab) delh_dimless_table(tab, r, z, G);
    else delh_dimless(r, z, G);
    gder_identities(G, r, z, hypot(r, z), *out);
}

// kind 1: Wu (exact derivatives of its formulas); kind 2: Delhommeau.
__device__ __forceinline__ void wave_dimless_grad(int kind, const double* __restrict__ tab, double r, double z,
                                                  GDer& g)
{
    if (kind == 2) delh_point_grad(tab, r, z, &g);
    else wave_dimless_dual(kind, r, z, &g);
}

// Pair geometry of the wave term (abstract_greens_function.jl:88-155 at k = 1).
struct WaveGeom {
    double dx, dy, zs, dis, u0, u1, invd;
};

__device__ __forceinline__ WaveGeom wave_geom(const double x[3], const Panel& p)
{
    WaveGeom w;
    w.dx = x[0] - p.c[0];
    w.dy = x[1] - p.c[1];
    w.zs = x[2] + p.c[2];
    const double dis2 = w.dx * w.dx + w.dy * w.dy;
    const double purt = 1e-18;
    w.dis = (dis2 == 0.0) ? sqrt(dis2 + purt * purt) - purt : sqrt(dis2);
    w.invd = w.dis > 0.0 ? 1.0 / w.dis : 0.0;
    w.u0 = w.dx * w.invd;
    w.u1 = w.dy * w.invd;
    return w;
}

