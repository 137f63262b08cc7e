// vof.cu -- volume fraction of the cells (VOF): front tracking and THINC/WLIC.
//
// Replaces front_tracking (fronttrack.cu:628-944 of the reference, with its
// matrix and source kernels 27-625 and the red-black SOR of
// matrix_solver.cu:112-216) and thinc_wlic (thincwlic.cu:12-420).
//
// The field vf lives on the internal lattice [z][y][x] in FP64: BUFF planes
// (and the shear mode's BUFF columns) are periodic images, so they are not
// stored; wall nodes hold 0, as wlic1d4md_st3 leaves them.
//
// Front tracking.  The gradient of the cells' indicator is spread from every
// triangle (inward normal times area, 4-point cosine delta about the
// centroid) with FP64 atomics; raw stencil nodes outside the reference lattice
// are dropped, nodes of fluid columns wrap (that is the fold of
// front_tracking_source3 into COMP nodes), nodes of wall columns keep only what
// lands in the reference's COMP planes (the reference folds COMP nodes only,
// and the divergence reads wall nodes only beside COMP nodes in the same
// plane).  The divergence on fluid nodes gives the right-hand side of the
// Jacobi-scaled Poisson system of front_tracking_matrix: x_i - (1/6) sum of the
// fluid neighbours' x = b_i = dg_i / (-6 / dx^2), with x = 0 on walls and the
// BUFF rows eliminated by the periodic index.  The reference solves it from
// x = 0 by red-black SOR with a host-synchronised residual every sweep; here
// one cooperative kernel runs conjugate gradients on it (the matrix is
// symmetric positive definite) from the current vf, with deterministic
// block-partial reductions and the reference's stopping rule
// |r| / |b| < RESIDUAL.  Both converge to the same solution.
//
// THINC/WLIC.  One kernel per sweep direction (x, y, z, in that order, each
// on the result of the one before): every fluid node computes the fluxes
// through its low and high faces (wlic1d4md_st1) and updates its value
// (wlic1d4md_st2) into a second buffer.  The flux through the face between
// a = b - e and b follows wlic1d4md_st1 for node b: 0 when b sits on the
// reference's outermost two layers at a low end or its last layer at a high
// end of a non-periodic axis, 0 at a wall; else upwind, and where the upwind
// node is an interface node with a normal (the average of the vf gradients at
// its eight cell corners, normal3d_st1/st2), the THINC flux weighted by the
// normal's share along the sweep.  Its transcendental steps use the float
// expf / coshf of the reference, on the same double arguments.
#include "rbc_internal.cuh"

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace rbc {

namespace {

constexpr int VOF_THREADS = 256;

__device__ __forceinline__ bool fluid_col(const uint32_t *mask2d, int nx, int x, int y)
{
    return (__ldg(&mask2d[y * nx + x]) & MASK_FLUID) != 0;
}

// ---- THINC/WLIC ---------------------------------------------------------

struct Node { int x, y, z; };

// n + s e_D with the periodic axes wrapped (z always, x in the shear mode)
template <int D>
__device__ __forceinline__ Node step(const Geom &g, Node n, int s)
{
    if (D == 0) n.x = g.xper ? wrap_x(n.x + s, g.nx) : n.x + s;
    if (D == 1) n.y += s;
    if (D == 2) n.z = wrap_z(n.z + s, g.nzc);
    return n;
}

__device__ __forceinline__ long long lin(const Geom &g, Node n) { return (long long)n.z * g.plane + (long long)n.y * g.nx + n.x; }

// vf at n + (ox, oy, oz), o in {-1, 0, 1}; the offsets never leave the lattice
// along a non-periodic axis for the interior nodes this is called for
__device__ __forceinline__ double vf_at(const Geom &g, const double *vf, Node n, int ox, int oy, int oz)
{
    int x = n.x + ox;
    if (g.xper) x = wrap_x(x, g.nx);
    const int z = wrap_z(n.z + oz, g.nzc);
    return __ldg(&vf[(long long)z * g.plane + (long long)(n.y + oy) * g.nx + x]);
}

// normal3d_st1 + normal3d_st2 (thincwlic.cu:12-106) at node n
__device__ void interface_normal(const Geom &g, const double *vf, Node n, double nrm[3])
{
    double V[3][3][3];   // V[oz + 1][oy + 1][ox + 1]
#pragma unroll
    for (int oz = -1; oz <= 1; oz++)
#pragma unroll
        for (int oy = -1; oy <= 1; oy++)
#pragma unroll
            for (int ox = -1; ox <= 1; ox++) V[oz + 1][oy + 1][ox + 1] = vf_at(g, vf, n, ox, oy, oz);
    const double c = 0.25 / g.dx;
    double s[3] = {0.0, 0.0, 0.0};
    // corners in the reference's summation order: i, i+z, i+x, i+x+z, i+y, i+y+z, i+x+y, i+x+y+z
    const int cx[8] = {0, 0, 1, 1, 0, 0, 1, 1}, cy[8] = {0, 0, 0, 0, 1, 1, 1, 1}, cz[8] = {0, 1, 0, 1, 0, 1, 0, 1};
#pragma unroll
    for (int k = 0; k < 8; k++) {
        // W(dx, dy, dz) = vf at corner - (dx, dy, dz); corner (cx, cy, cz) relative to n
#define W(a, b, d) V[cz[k] - (d) + 1][cy[k] - (b) + 1][cx[k] - (a) + 1]
        s[0] += c * (W(0, 0, 0) - W(1, 0, 0) + W(0, 1, 0) - W(1, 1, 0) + W(0, 0, 1) - W(1, 0, 1) + W(0, 1, 1) - W(1, 1, 1));
        s[1] += c * (W(0, 0, 0) - W(0, 1, 0) + W(1, 0, 0) - W(1, 1, 0) + W(0, 0, 1) - W(0, 1, 1) + W(1, 0, 1) - W(1, 1, 1));
        s[2] += c * (W(0, 0, 0) - W(0, 0, 1) + W(1, 0, 0) - W(1, 0, 1) + W(0, 1, 0) - W(0, 1, 1) + W(1, 1, 0) - W(1, 1, 1));
#undef W
    }
    nrm[0] = 0.125 * s[0];
    nrm[1] = 0.125 * s[1];
    nrm[2] = 0.125 * s[2];
}

// flux through the low face of node b along D (wlic1d4md_st1, thincwlic.cu:108-238)
template <int D>
__device__ double face_flux(const Geom &g, const double *vf, const float4 *uvr, const uint32_t *mask2d, Node b,
                            double dt)
{
    // wlic1d4md_st1 returns for raw index 0 or 1 along any axis and for the last
    // raw index; on the periodic axes those nodes are BUFF images whose faces no
    // fluid node uses
    if (b.y <= 1 || b.y >= g.ny - 1) return 0.0;
    if (!g.xper && (b.x <= 1 || b.x >= g.nx - 1)) return 0.0;
    const Node a = step<D>(g, b, -1);
    if (!fluid_col(mask2d, g.nx, b.x, b.y) || !fluid_col(mask2d, g.nx, a.x, a.y)) return 0.0;
    const long long ib = lin(g, b), ia = lin(g, a);
    const float4 qb = __ldg(&uvr[ib]), qa = __ldg(&uvr[ia]);
    const double up = D == 0 ? qb.x : D == 1 ? qb.y : qb.z;
    const double um = D == 0 ? qa.x : D == 1 ? qa.y : qa.z;
    const double uc = (up + um) / 2.0;
    const int isgn = uc <= 0.0 ? 0 : 1;
    const Node ii = isgn ? a : b;
    const double v = __ldg(&vf[isgn ? ia : ib]);
    if (v >= 1.0 - 1.0e-6 || v <= 1.0e-6) return v * uc * dt;
    double nrm[3];
    interface_normal(g, vf, ii, nrm);
    const double nn = fabs(nrm[0]) + fabs(nrm[1]) + fabs(nrm[2]);
    if (nn <= 1.0e-6) return v * uc * dt;
    const double beta = 2.0;
    const double vlo = __ldg(&vf[lin(g, step<D>(g, ii, -1))]), vhi = __ldg(&vf[lin(g, step<D>(g, ii, 1))]);
    const double alpha = vlo <= vhi ? 1.0 : -1.0;
    const double a1 = expf(beta * (2.0 * v - 1.0) / alpha);
    const double a3 = expf(beta);
    const double xc = 0.5 / beta * log((a3 * a3 - a1 * a3) / (a1 * a3 - 1.0));
    const double a4 = coshf(beta * ((double)isgn - uc * dt / g.dx - xc));
    const double a5 = coshf(beta * ((double)isgn - xc));
    const double f = 0.5 * (uc * dt - alpha * g.dx / beta * log(a4 / a5));
    const double w = fabs(nrm[D]) / nn;
    return f * w + v * uc * dt * (1.0 - w);
}

template <int D>
__global__ void __launch_bounds__(VOF_THREADS)
thinc_sweep_kernel(const Geom g, const double *__restrict__ vin, double *__restrict__ vout,
                   const float4 *__restrict__ uvr, const uint32_t *__restrict__ mask2d, double dt)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nint) return;
    Node n;
    n.z = (int)(i / g.plane);
    const int r = (int)(i - (long long)n.z * g.plane);
    n.y = r / g.nx;
    n.x = r - n.y * g.nx;
    if (!fluid_col(mask2d, g.nx, n.x, n.y)) { vout[i] = 0.0; return; }   // wlic1d4md_st3
    const double flo = face_flux<D>(g, vin, uvr, mask2d, n, dt);
    const double fhi = face_flux<D>(g, vin, uvr, mask2d, step<D>(g, n, 1), dt);
    vout[i] = vin[i] - (fhi - flo) / g.dx;   // wlic1d4md_st2
}

// ---- front tracking -------------------------------------------------------

// front_tracking_source2 (fronttrack.cu:351-455) for one triangle per thread
__global__ void __launch_bounds__(VOF_THREADS)
indicator_gradient_kernel(const Geom g, const double *__restrict__ X, long long nv, const int *__restrict__ tri,
                          int V, int E, int ncell, const uint32_t *__restrict__ mask2d, double *__restrict__ G)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)ncell * E) return;
    const int c = (int)(e / E), k = (int)(e - (long long)c * E);
    const long long base = (long long)c * V;
    const long long j1 = base + __ldg(&tri[3 * k]), j2 = base + __ldg(&tri[3 * k + 1]), j3 = base + __ldg(&tri[3 * k + 2]);
    const double *xs = X, *ys = X + nv, *zs = X + 2 * nv;
    double tx1 = xs[j1], tx2 = xs[j2], tx3 = xs[j3];
    const double ty1 = ys[j1], ty2 = ys[j2], ty3 = ys[j3];
    double tz1 = zs[j1], tz2 = zs[j2], tz3 = zs[j3];
    const double LX = g.LX, LZ = g.LZ, dx = g.dx;
    double xx1 = tx2 - tx1, zz1 = tz2 - tz1;
    const double yy1 = ty2 - ty1;
    if (xx1 > LX * 0.5) { xx1 -= LX; tx1 += LX; } else if (xx1 < -LX * 0.5) { xx1 += LX; tx2 += LX; }
    if (zz1 > LZ * 0.5) { zz1 -= LZ; tz1 += LZ; } else if (zz1 < -LZ * 0.5) { zz1 += LZ; tz2 += LZ; }
    double xx2 = tx3 - tx1, zz2 = tz3 - tz1;
    const double yy2 = ty3 - ty1;
    if (xx2 > LX * 0.5) { xx2 -= LX; tx1 += LX; } else if (xx2 < -LX * 0.5) { xx2 += LX; tx3 += LX; }
    if (zz2 > LZ * 0.5) { zz2 -= LZ; tz1 += LZ; } else if (zz2 < -LZ * 0.5) { zz2 += LZ; tz3 += LZ; }
    const double xg = (tx1 + tx2 + tx3) / 3.0, yg = (ty1 + ty2 + ty3) / 3.0, zg = (tz1 + tz2 + tz3) / 3.0;
    const double xtr = xg + (double)(g.nxr - 1) * dx / 2.0, ytr = yg + (double)(g.ny - 1) * dx / 2.0,
                 ztr = zg + (double)(g.nzr - 1) * dx / 2.0;
    double nvx = -(yy1 * zz2 - zz1 * yy2), nvy = -(zz1 * xx2 - xx1 * zz2), nvz = -(xx1 * yy2 - yy1 * xx2);
    const double nn = sqrt(nvx * nvx + nvy * nvy + nvz * nvz), ds = nn / 2.0;
    nvx /= nn; nvy /= nn; nvz /= nn;
    const int x1 = (int)floor(xtr / dx) - 1, x2 = (int)ceil(xtr / dx) + 1;
    const int y1 = (int)floor(ytr / dx) - 1, y2 = (int)ceil(ytr / dx) + 1;
    const int z1 = (int)floor(ztr / dx) - 1, z2 = (int)ceil(ztr / dx) + 1;
    const double inv64 = 1.0 / (64.0 * dx * dx * dx);
    double *Gx = G, *Gy = G + g.nint, *Gz = G + 2 * g.nint;
    for (int iz = z1; iz <= z2; iz++) {
        if (iz < 0 || iz >= g.nzr) continue;
        const double zcos = 1.0 + cospi(((double)iz * dx - ztr) / (2.0 * dx));
        for (int iy = y1; iy <= y2; iy++) {
            if (iy < 0 || iy >= g.ny) continue;
            const double ycos = 1.0 + cospi(((double)iy * dx - ytr) / (2.0 * dx));
            for (int ix = x1; ix <= x2; ix++) {
                if (ix < 0 || ix >= g.nxr) continue;
                int xi = ix - g.xb;
                const bool in_x = xi >= 0 && xi < g.nx;
                if (g.xper) xi = wrap_x(xi, g.nx);
                else if (!in_x) continue;
                int zc = iz - 2;
                if (fluid_col(mask2d, g.nx, xi, iy)) {
                    zc = wrap_z(zc, g.nzc);
                } else if (zc < 0 || zc >= g.nzc || !in_x) {
                    continue;   // a wall node outside the COMP range: never read
                }
                const double xcos = 1.0 + cospi(((double)ix * dx - xtr) / (2.0 * dx));
                const double dlt = xcos * ycos * zcos * inv64;
                const long long idx = (long long)zc * g.plane + (long long)iy * g.nx + xi;
                atomicAdd(&Gx[idx], dlt * nvx * ds);
                atomicAdd(&Gy[idx], dlt * nvy * ds);
                atomicAdd(&Gz[idx], dlt * nvz * ds);
            }
        }
    }
}

// front_tracking_source4 + jacobi_source (fronttrack.cu:540-583, 300-319):
// b = div G / (-6 / dx^2) on fluid nodes, 0 on walls
__global__ void __launch_bounds__(VOF_THREADS)
indicator_rhs_kernel(const Geom g, const double *__restrict__ G, const uint32_t *__restrict__ mask2d,
                     double *__restrict__ b)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nint) return;
    const int z = (int)(i / g.plane), r = (int)(i - (long long)z * g.plane), y = r / g.nx, x = r - y * g.nx;
    if (!fluid_col(mask2d, g.nx, x, y)) { b[i] = 0.0; return; }
    const double *Gx = G, *Gy = G + g.nint, *Gz = G + 2 * g.nint;
    const int xm = g.xper ? wrap_x(x - 1, g.nx) : x - 1, xp = g.xper ? wrap_x(x + 1, g.nx) : x + 1;
    const long long zo = (long long)z * g.plane;
    const long long izm = (long long)wrap_z(z - 1, g.nzc) * g.plane + r, izp = (long long)wrap_z(z + 1, g.nzc) * g.plane + r;
    const double gxp = xp < g.nx ? Gx[zo + (long long)y * g.nx + xp] : 0.0, gxm = xm >= 0 ? Gx[zo + (long long)y * g.nx + xm] : 0.0;
    const double d = (gxp - gxm + Gy[i + g.nx] - Gy[i - g.nx] + Gz[izp] - Gz[izm]) / (2.0 * g.dx);
    b[i] = d / (-6.0 / (g.dx * g.dx));
}

// ---- conjugate gradients on the scaled system -----------------------------

struct CgArgs {
    Geom g;
    const uint32_t *mask2d;
    const double *b;
    double *x, *r, *p, *q;
    double *partial;          // [2][2 * nblocks]
    double tol;
    int itrmax;
    int *iters_out;           // device: sweeps taken, -1 = not converged
    int *flags;
};

constexpr int CG_THREADS = 256;

// A v at node i: v_i - (1/6) sum of the fluid neighbours' v (walls hold 0)
__device__ __forceinline__ double apply_a(const Geom &g, const uint32_t *mask2d, const double *v, long long i, int x, int y,
                                          int z)
{
    const double off = (1.0 / (g.dx * g.dx)) / (-6.0 / (g.dx * g.dx));
    double s = v[i];
    auto nb = [&](int xx, int yy, int zz) -> double {
        if (g.xper) xx = wrap_x(xx, g.nx);
        else if (xx < 0 || xx >= g.nx) return 0.0;
        if (yy < 0 || yy >= g.ny) return 0.0;
        zz = wrap_z(zz, g.nzc);
        if (!fluid_col(mask2d, g.nx, xx, yy)) return 0.0;
        return v[(long long)zz * g.plane + (long long)yy * g.nx + xx];
    };
    s += off * nb(x, y, z - 1);
    s += off * nb(x, y - 1, z);
    s += off * nb(x - 1, y, z);
    s += off * nb(x + 1, y, z);
    s += off * nb(x, y + 1, z);
    s += off * nb(x, y, z + 1);
    return s;
}

// deterministic grid sum of two values: block tree -> partial[bank] -> every
// block adds the partials in block order after the grid barrier
__device__ void grid_sum2(cg::grid_group &grid, double *partial, int bank, double a, double b, double &sa, double &sb)
{
    __shared__ double sh[2][CG_THREADS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wid] = a; sh[1][wid] = b; }
    __syncthreads();
    double *pb = partial + (size_t)bank * 2 * gridDim.x;
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int w = 0; w < CG_THREADS / 32; w++) { ta += sh[0][w]; tb += sh[1][w]; }
        pb[blockIdx.x] = ta;
        pb[gridDim.x + blockIdx.x] = tb;
    }
    grid.sync();
    __shared__ double res[2];
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (unsigned k = 0; k < gridDim.x; k++) { ta += pb[k]; tb += pb[gridDim.x + k]; }
        res[0] = ta;
        res[1] = tb;
    }
    __syncthreads();
    sa = res[0];
    sb = res[1];
    __syncthreads();
}

__global__ void __launch_bounds__(CG_THREADS)
indicator_cg_kernel(const CgArgs a)
{
    cg::grid_group grid = cg::this_grid();
    const Geom &g = a.g;
    const long long stride = (long long)gridDim.x * blockDim.x, first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    auto coords = [&](long long i, int &x, int &y, int &z) {
        z = (int)(i / g.plane);
        const int r = (int)(i - (long long)z * g.plane);
        y = r / g.nx;
        x = r - y * g.nx;
    };
    double lr = 0.0, lb = 0.0;
    for (long long i = first; i < g.nint; i += stride) {
        int x, y, z;
        coords(i, x, y, z);
        if (!fluid_col(a.mask2d, g.nx, x, y)) { a.x[i] = 0.0; a.r[i] = 0.0; a.p[i] = 0.0; a.q[i] = 0.0; continue; }
        const double ri = a.b[i] - apply_a(g, a.mask2d, a.x, i, x, y, z);
        a.r[i] = ri;
        a.p[i] = ri;
        lr += ri * ri;
        lb += a.b[i] * a.b[i];
    }
    double rr, bb;
    int bank = 0;
    grid_sum2(grid, a.partial, bank, lr, lb, rr, bb);
    bank ^= 1;
    int it = 0;
    if (bb > 0.0) {
        while (it < a.itrmax && !(sqrt(rr / bb) < a.tol)) {
            double lpq = 0.0;
            for (long long i = first; i < g.nint; i += stride) {
                int x, y, z;
                coords(i, x, y, z);
                if (!fluid_col(a.mask2d, g.nx, x, y)) continue;
                const double qi = apply_a(g, a.mask2d, a.p, i, x, y, z);
                a.q[i] = qi;
                lpq += a.p[i] * qi;
            }
            double pq, unused;
            grid_sum2(grid, a.partial, bank, lpq, 0.0, pq, unused);
            bank ^= 1;
            const double alpha = rr / pq;
            double lrr = 0.0;
            for (long long i = first; i < g.nint; i += stride) {
                const double ri = a.r[i] - alpha * a.q[i];
                a.x[i] += alpha * a.p[i];
                a.r[i] = ri;
                lrr += ri * ri;
            }
            double rr_new;
            grid_sum2(grid, a.partial, bank, lrr, 0.0, rr_new, unused);
            bank ^= 1;
            const double beta = rr_new / rr;
            rr = rr_new;
            for (long long i = first; i < g.nint; i += stride) a.p[i] = a.r[i] + beta * a.p[i];
            grid.sync();
            it++;
        }
    } else {
        for (long long i = first; i < g.nint; i += stride) a.x[i] = 0.0;
    }
    if (first == 0) {
        const bool ok = bb == 0.0 || sqrt(rr / bb) < a.tol;
        *a.iters_out = ok ? it : -1;
        if (!ok) atomicOr(a.flags, RBC_FLAG_VOF_NOT_CONVERGED);
    }
}

int g_cg_blocks = 0;   // co-resident blocks of the CG kernel on this device

}  // namespace

int vof_cg_blocks()
{
    return g_cg_blocks;
}

cudaError_t vof_setup()
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, indicator_cg_kernel, CG_THREADS, 0);
    if (e == cudaSuccess) g_cg_blocks = sms * (per_sm < 2 ? per_sm : 2);
    return e;
}

void launch_thinc_wlic(const Geom &g, double *vf, double *s1, double *s2, const float4 *uvr, const uint32_t *mask2d,
                       double dt, cudaStream_t s)
{
    const unsigned blocks = (unsigned)((g.nint + VOF_THREADS - 1) / VOF_THREADS);
    thinc_sweep_kernel<0><<<blocks, VOF_THREADS, 0, s>>>(g, vf, s1, uvr, mask2d, dt);
    thinc_sweep_kernel<1><<<blocks, VOF_THREADS, 0, s>>>(g, s1, s2, uvr, mask2d, dt);
    thinc_sweep_kernel<2><<<blocks, VOF_THREADS, 0, s>>>(g, s2, vf, uvr, mask2d, dt);
}

cudaError_t launch_front_tracking(const Geom &g, const FrontArgs &a, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(a.G, 0, sizeof(double) * 3 * (size_t)g.nint, s);
    if (e != cudaSuccess) return e;
    const long long ntri = (long long)a.ncell * a.E;
    if (ntri > 0)
        indicator_gradient_kernel<<<(unsigned)((ntri + VOF_THREADS - 1) / VOF_THREADS), VOF_THREADS, 0, s>>>(
            g, a.X, a.nv, a.tri, a.V, a.E, a.ncell, a.mask2d, a.G);
    const unsigned blocks = (unsigned)((g.nint + VOF_THREADS - 1) / VOF_THREADS);
    indicator_rhs_kernel<<<blocks, VOF_THREADS, 0, s>>>(g, a.G, a.mask2d, a.b);
    // the gradient is consumed: its storage holds the CG vectors r, p, q
    CgArgs c{};
    c.g = g; c.mask2d = a.mask2d; c.b = a.b; c.x = a.vf;
    c.r = a.G; c.p = a.G + g.nint; c.q = a.G + 2 * g.nint;
    c.partial = a.partial; c.tol = a.tol; c.itrmax = a.itrmax; c.iters_out = a.iters; c.flags = a.flags;
    void *args[] = {&c};
    return cudaLaunchCooperativeKernel((const void *)indicator_cg_kernel, dim3((unsigned)g_cg_blocks), dim3(CG_THREADS),
                                       args, 0, s);
}

}  // namespace rbc
