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

#include <vector>

namespace cg = cooperative_groups;

namespace rbc {

namespace {

constexpr int VOF_THREADS = 256;

__device__ __forceinline__ bool fluid_col(const uint32_t *mask2d, int nx, int x, int y)
{
    return (__ldg(&mask2d[y * nx + x]) & MASK_FLUID) != 0;
}

// ---- THINC/WLIC ---------------------------------------------------------

// A CTA sweeps a tile of TX x TY x TZ nodes.  It stages vf of the tile and a
// halo of two nodes in shared memory, computes the interface normal
// (normal3d_st1/st2) once for every node of the tile and its two neighbour
// layers along the sweep, then each node computes the fluxes through its two
// faces along the sweep from the staged values.
// The staged box: two halo layers along the sweep (a face's upwind node is one
// beyond the tile and its normal and THINC neighbours one more), one across.
constexpr int TX = 32, TY = 4, TZ = 4, HALO = 2;
constexpr int SX = TX + 2 * HALO, SY = TY + 2 * HALO, SZ = TZ + 2 * HALO;
template <int D> struct Staged {   // the part of the SZ x SY x SX box a sweep along D loads
    static constexpr int hx = D == 0 ? 2 : 1, hy = D == 1 ? 2 : 1, hz = D == 2 ? 2 : 1;
    static constexpr int nx = TX + 2 * hx, ny = TY + 2 * hy, nz = TZ + 2 * hz;
};
constexpr int NMAX = (TX + 2) * TY * TZ > TX * (TY + 2) * TZ ? (TX + 2) * TY * TZ : TX * (TY + 2) * TZ;

template <int D> struct NormalRegion {   // the tile extended by one node each way along D
    static constexpr int nx = TX + (D == 0 ? 2 : 0), ny = TY + (D == 1 ? 2 : 0), nz = TZ + (D == 2 ? 2 : 0);
    static constexpr int ox = D == 0 ? 1 : 0, oy = D == 1 ? 1 : 0, oz = D == 2 ? 1 : 0;   // region origin = tile - o
};

// normal at staged node (sx, sy, sz) (shared coordinates, >= 1 and < S - 1).
// The average over the eight cell corners of normal3d_st1's corner gradients
// is, per component, the central difference across the node weighted (1, 2,
// 1) x (1, 2, 1) over the two other axes, divided by 32 dx: the 27 staged
// values are read once.
__device__ __forceinline__ void staged_normal(const double (&sv)[SZ][SY][SX], int sx, int sy, int sz, double inv32dx,
                                              double n[3])
{
    double V[3][3][3];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
#pragma unroll
            for (int c = 0; c < 3; c++) V[a][b][c] = sv[sz + a - 1][sy + b - 1][sx + c - 1];
    const double w[3] = {1.0, 2.0, 1.0};
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            s0 += w[a] * w[b] * (V[a][b][2] - V[a][b][0]);   // x: weights over (z, y)
            s1 += w[a] * w[b] * (V[a][2][b] - V[a][0][b]);   // y: weights over (z, x)
            s2 += w[a] * w[b] * (V[2][a][b] - V[0][a][b]);   // z: weights over (y, x)
        }
    n[0] = s0 * inv32dx;
    n[1] = s1 * inv32dx;
    n[2] = s2 * inv32dx;
}

// p wrapped into [0, n) for |p| within a few periods (tile and halo offsets)
__device__ __forceinline__ int wrap_near(int p, int n)
{
    while (p < 0) p += n;
    while (p >= n) p -= n;
    return p;
}

template <int D> struct FaceRegion {   // faces along D: the tile's nodes and one beyond it along D
    static constexpr int nx = TX + (D == 0), ny = TY + (D == 1), nz = TZ + (D == 2);
};
constexpr int FMAX = TX * TY * (TZ + 1) > TX * (TY + 1) * TZ ? TX * TY * (TZ + 1) : TX * (TY + 1) * TZ;

// flux through the face between a = b - e_D and b (wlic1d4md_st1,
// thincwlic.cu:108-238).  (bx, by, bz): b in lattice coordinates; (tx, ty, tz):
// b in tile coordinates (the upwind node is b or a, inside the normal region).
template <int D>
__device__ double face_flux(const Geom &g, const double (&sv)[SZ][SY][SX], const double (&sn)[3][NMAX],
                            const float4 *__restrict__ uvr, const uint32_t *__restrict__ mask2d,
                            int bx, int by, int bz, int tx, int ty, int tz, double dt)
{
    using R = NormalRegion<D>;
    // wlic1d4md_st1 returns for raw index 0 or 1 along any axis and for the last
    // raw index; on the periodic axes those nodes are BUFF images whose faces no
    // fluid node uses
    if (by <= 1 || by >= g.ny - 1) return 0.0;
    if (!g.xper && (bx <= 1 || bx >= g.nx - 1)) return 0.0;
    int ax = bx, ay = by, az = bz;
    if (D == 0) ax = g.xper ? wrap_near(bx - 1, g.nx) : bx - 1;
    if (D == 1) ay = by - 1;
    if (D == 2) az = wrap_near(bz - 1, g.nzc);
    if (!fluid_col(mask2d, g.nx, bx, by) || !fluid_col(mask2d, g.nx, ax, ay)) return 0.0;
    const float4 qb = __ldg(&uvr[(long long)bz * g.plane + (long long)by * g.nx + bx]);
    const float4 qa = __ldg(&uvr[(long long)az * g.plane + (long long)ay * g.nx + ax]);
    const double up = D == 0 ? qb.x : D == 1 ? qb.y : qb.z;
    const double um = D == 0 ? qa.x : D == 1 ? qa.y : qa.z;
    const double uc = (up + um) / 2.0;
    const int isgn = uc <= 0.0 ? 0 : 1;
    // upwind node ii in tile coordinates
    const int ix = tx - (D == 0 ? isgn : 0), iy = ty - (D == 1 ? isgn : 0), iz = tz - (D == 2 ? isgn : 0);
    const double v = sv[iz + HALO][iy + HALO][ix + HALO];
    if (v >= 1.0 - 1.0e-6 || v <= 1.0e-6) return v * uc * dt;
    const int ni = ((iz + R::oz) * R::ny + (iy + R::oy)) * R::nx + (ix + R::ox);
    const double n0 = sn[0][ni], n1 = sn[1][ni], n2 = sn[2][ni];
    const double nn = fabs(n0) + fabs(n1) + fabs(n2);
    if (nn <= 1.0e-6) return v * uc * dt;
    const double beta = 2.0;
    const double vlo = sv[iz + HALO - (D == 2)][iy + HALO - (D == 1)][ix + HALO - (D == 0)];
    const double vhi = sv[iz + HALO + (D == 2)][iy + HALO + (D == 1)][ix + HALO + (D == 0)];
    const double alpha = vlo <= vhi ? 1.0 : -1.0;
    const double a1 = expf(beta * (2.0 * v - 1.0) * alpha);   // / alpha: alpha = +-1, the same value
    const double a3 = expf(beta);
    const double xc = 0.5 / beta * log((a3 * a3 - a1 * a3) / (a1 * a3 - 1.0));
    const double a4 = coshf(beta * ((double)isgn - uc * dt * g.inv_dx - xc));
    const double a5 = coshf(beta * ((double)isgn - xc));
    const double f = 0.5 * (uc * dt - alpha * g.dx / beta * log(a4 / a5));
    const double w = fabs(D == 0 ? n0 : D == 1 ? n1 : n2) / nn;
    return f * w + v * uc * dt * (1.0 - w);
}

template <int D>
__global__ void __launch_bounds__(VOF_THREADS)
thinc_sweep_kernel(const Geom g, const double *__restrict__ vin, double *__restrict__ vout,
                   const float4 *__restrict__ uvr, const uint32_t *__restrict__ mask2d, double dt)
{
    using R = NormalRegion<D>;
    using F = FaceRegion<D>;
    __shared__ double sv[SZ][SY][SX];
    __shared__ double sn[3][NMAX];
    __shared__ double sf[FMAX];
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    // stage vf of the tile and its halo; nodes beyond a non-periodic end read 0
    // (they only enter normals of wall nodes, which no face uses)
    using St = Staged<D>;
    for (int k = threadIdx.x; k < St::nx * St::ny * St::nz; k += blockDim.x) {
        const int lx = k % St::nx + (HALO - St::hx), ly = (k / St::nx) % St::ny + (HALO - St::hy),
                  lz = k / (St::nx * St::ny) + (HALO - St::hz);
        int x = x0 + lx - HALO;
        const int y = y0 + ly - HALO, z = wrap_near(z0 + lz - HALO, g.nzc);
        double v = 0.0;
        if (g.xper) x = wrap_near(x, g.nx);
        if (x >= 0 && x < g.nx && y >= 0 && y < g.ny) v = __ldg(&vin[(long long)z * g.plane + (long long)y * g.nx + x]);
        sv[lz][ly][lx] = v;
    }
    __syncthreads();
    const double inv32dx = 1.0 / (32.0 * g.dx);
    for (int k = threadIdx.x; k < R::nx * R::ny * R::nz; k += blockDim.x) {
        const int rx = k % R::nx, ry = (k / R::nx) % R::ny, rz = k / (R::nx * R::ny);
        const int sx = rx - R::ox + HALO, sy = ry - R::oy + HALO, sz = rz - R::oz + HALO;
        const double v = sv[sz][sy][sx];
        double n[3] = {0.0, 0.0, 0.0};
        // a full or empty node's flux is plain upwind: its normal is never read
        if (v > 1.0e-6 && v < 1.0 - 1.0e-6) staged_normal(sv, sx, sy, sz, inv32dx, n);
        sn[0][k] = n[0];
        sn[1][k] = n[1];
        sn[2][k] = n[2];
    }
    __syncthreads();
    // every face along D of the tile once: the low faces of the tile's nodes and
    // the high face of its last layer
    for (int k = threadIdx.x; k < F::nx * F::ny * F::nz; k += blockDim.x) {
        const int fx = k % F::nx, fy = (k / F::nx) % F::ny, fz = k / (F::nx * F::ny);
        int x = x0 + fx, y = y0 + fy, z = z0 + fz;
        double f = 0.0;
        if (g.xper) x = wrap_near(x, g.nx);
        z = wrap_near(z, g.nzc);
        if (x < g.nx && y < g.ny) f = face_flux<D>(g, sv, sn, uvr, mask2d, x, y, z, fx, fy, fz, dt);
        sf[k] = f;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < TX * TY * TZ; k += blockDim.x) {
        const int tx = k % TX, ty = (k / TX) % TY, tz = k / (TX * TY);
        const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
        if (x >= g.nx || y >= g.ny || z >= g.nzc) continue;
        const long long i = (long long)z * g.plane + (long long)y * g.nx + x;
        if (!fluid_col(mask2d, g.nx, x, y)) { vout[i] = 0.0; continue; }   // wlic1d4md_st3
        const int lo = (tz * F::ny + ty) * F::nx + tx;
        const int hi = ((tz + (D == 2)) * F::ny + ty + (D == 1)) * F::nx + tx + (D == 0);
        vout[i] = sv[tz + HALO][ty + HALO][tx + HALO] - (sf[hi] - sf[lo]) * g.inv_dx;   // wlic1d4md_st2
    }
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
    double *partial;          // [2][2 * nblocks]; lattice indices fit 32 bits (checked at setup)
    double tol;
    int itrmax;
    int *iters_out;           // device: sweeps taken, -1 = not converged
    int *flags;
};

constexpr int CG_THREADS = 256;
constexpr int CG_BLOCKS_PER_SM = 4;

// A v at node i = (x, y, z) of a fluid column: v_i - (1/6) sum of the fluid
// neighbours' v (walls hold 0)
__device__ __forceinline__ double apply_a(const Geom &g, const uint32_t *mask2d, const double *v, unsigned i, int x, int y,
                                          int z)
{
    const double off = (1.0 / (g.dx * g.dx)) / (-6.0 / (g.dx * g.dx));
    const unsigned pl = (unsigned)g.plane, row = (unsigned)(y * g.nx);
    const unsigned zo = (unsigned)z * pl;
    const unsigned zm = (z == 0 ? (unsigned)(g.nzc - 1) * pl : zo - pl), zp = (z == g.nzc - 1 ? 0u : zo + pl);
    int xm = x - 1, xp = x + 1;
    if (g.xper) { if (xm < 0) xm += g.nx; if (xp >= g.nx) xp -= g.nx; }
    double s = v[i];
    s += off * v[zm + row + x];   // the node's own column is fluid, so are its z neighbours
    if (y > 0 && fluid_col(mask2d, g.nx, x, y - 1)) s += off * v[zo + row - g.nx + x];
    if (xm >= 0 && fluid_col(mask2d, g.nx, xm, y)) s += off * v[zo + row + xm];
    if (xp < g.nx && fluid_col(mask2d, g.nx, xp, y)) s += off * v[zo + row + xp];
    if (y + 1 < g.ny && fluid_col(mask2d, g.nx, x, y + 1)) s += off * v[zo + row + g.nx + x];
    s += off * v[zp + row + x];
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
    if (threadIdx.x < 32) {   // one warp adds the partials: strided lanes, then a fixed tree
        double ta = 0.0, tb = 0.0;
        for (unsigned k = threadIdx.x; k < gridDim.x; k += 32) { ta += pb[k]; tb += pb[gridDim.x + k]; }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ta += __shfl_down_sync(0xffffffffu, ta, o);
            tb += __shfl_down_sync(0xffffffffu, tb, o);
        }
        if (threadIdx.x == 0) { res[0] = ta; res[1] = tb; }
    }
    __syncthreads();
    sa = res[0];
    sb = res[1];
    __syncthreads();
}

// Conjugate gradients with the search direction and A p updated in one pass:
// p = r + beta p and q = A p = A r + beta q, so an iteration is two passes
// over the lattice and two grid barriers.
__global__ void __launch_bounds__(CG_THREADS, CG_BLOCKS_PER_SM)
indicator_cg_kernel(const CgArgs a)
{
    cg::grid_group grid = cg::this_grid();
    const Geom &g = a.g;
    const unsigned n = (unsigned)g.nint, pl = (unsigned)g.plane;
    const unsigned stride = gridDim.x * blockDim.x, first = blockIdx.x * blockDim.x + threadIdx.x;
    double lr = 0.0, lb = 0.0;
    for (unsigned i = first; i < n; i += stride) {
        const unsigned z = i / pl, rr = i - z * pl, y = rr / (unsigned)g.nx, x = rr - y * (unsigned)g.nx;
        a.p[i] = 0.0;
        a.q[i] = 0.0;
        if (!fluid_col(a.mask2d, g.nx, (int)x, (int)y)) { a.x[i] = 0.0; a.r[i] = 0.0; continue; }
        const double ri = a.b[i] - apply_a(g, a.mask2d, a.x, i, (int)x, (int)y, (int)z);
        a.r[i] = ri;
        lr += ri * ri;
        lb += a.b[i] * a.b[i];
    }
    double rr, bb;
    int bank = 0;
    grid_sum2(grid, a.partial, bank, lr, lb, rr, bb);
    bank ^= 1;
    int it = 0;
    double beta = 0.0;
    if (bb > 0.0) {
        while (it < a.itrmax && !(sqrt(rr / bb) < a.tol)) {
            double lpq = 0.0;
            for (unsigned i = first; i < n; i += stride) {
                const unsigned z = i / pl, rw = i - z * pl, y = rw / (unsigned)g.nx, x = rw - y * (unsigned)g.nx;
                if (!fluid_col(a.mask2d, g.nx, (int)x, (int)y)) continue;
                const double pi = a.r[i] + beta * a.p[i];
                const double qi = apply_a(g, a.mask2d, a.r, i, (int)x, (int)y, (int)z) + beta * a.q[i];
                a.p[i] = pi;
                a.q[i] = qi;
                lpq += pi * qi;
            }
            double pq, unused;
            grid_sum2(grid, a.partial, bank, lpq, 0.0, pq, unused);
            bank ^= 1;
            const double alpha = rr / pq;
            double lrr = 0.0;
            for (unsigned i = first; i < n; i += stride) {
                const double ri = a.r[i] - alpha * a.q[i];
                a.x[i] += alpha * a.p[i];
                a.r[i] = ri;
                lrr += ri * ri;
            }
            double rr_new;
            grid_sum2(grid, a.partial, bank, lrr, 0.0, rr_new, unused);
            bank ^= 1;
            beta = rr_new / rr;
            rr = rr_new;
            it++;
        }
    } else {
        for (unsigned i = first; i < n; i += stride) a.x[i] = 0.0;
    }
    if (first == 0) {
        const bool ok = bb == 0.0 || sqrt(rr / bb) < a.tol;
        *a.iters_out = ok ? it : -1;
        if (!ok) atomicOr(a.flags, RBC_FLAG_VOF_NOT_CONVERGED);
    }
}

// ---- multigrid-preconditioned CG ------------------------------------------

// (A_l v)_i at node i = (x, y, z) of level L (0 on wall columns); v(j, c, x, y, z)
// gives the vector's value at node j = (x, y, z) of column c
template <typename Val>
__device__ __forceinline__ double apply_level_fn(const MgLevel &L, int x, int y, int z, Val v)
{
    const unsigned ncol = (unsigned)(L.nx * L.ny), col = (unsigned)(y * L.nx + x);
    const double *c = L.coef;
    const double d = c[col];
    if (d == 0.0) return 0.0;
    const unsigned zo = (unsigned)z * ncol;
    double s = d * v(zo + col, col, x, y, z);
    const double cxm = c[ncol + col], cxp = c[2 * ncol + col], cym = c[3 * ncol + col], cyp = c[4 * ncol + col];
    const double cz = c[5 * ncol + col];
    if (cxm != 0.0) {
        const int xl = x > 0 ? x - 1 : L.nx - 1;
        const unsigned cl = (unsigned)(y * L.nx + xl);
        s += cxm * v(zo + cl, cl, xl, y, z);
    }
    if (cxp != 0.0) {
        const int xr = x < L.nx - 1 ? x + 1 : 0;
        const unsigned cr = (unsigned)(y * L.nx + xr);
        s += cxp * v(zo + cr, cr, xr, y, z);
    }
    if (cym != 0.0) s += cym * v(zo + col - (unsigned)L.nx, col - (unsigned)L.nx, x, y - 1, z);
    if (cyp != 0.0) s += cyp * v(zo + col + (unsigned)L.nx, col + (unsigned)L.nx, x, y + 1, z);
    if (cz != 0.0) {
        const int zm = z == 0 ? L.nz - 1 : z - 1, zp = z == L.nz - 1 ? 0 : z + 1;
        s += cz * (v((unsigned)zm * ncol + col, col, x, y, zm) + v((unsigned)zp * ncol + col, col, x, y, zp));
    }
    return s;
}

__device__ __forceinline__ double apply_level(const MgLevel &L, const double *v, unsigned, int x, int y, int z)
{
    return apply_level_fn(L, x, y, z, [v](unsigned j, unsigned, int, int, int) { return v[j]; });
}

struct PcgArgs {
    MgHierarchy mg;           // level 0: b = r, y = z
    const double *b;          // right-hand side of the scaled system
    double *x, *r, *p, *q;
    double *partial;
    double tol;
    int itrmax;
    int *iters_out;
    int *flags;
};

constexpr double MG_OMEGA = 0.8;   // damped-Jacobi smoothing weight
constexpr int MG_COARSE_SWEEPS = 40;

// z = M r: one symmetric V-cycle (one damped-Jacobi sweep from 0 before and
// one after the coarse correction, the coarsest level by Jacobi sweeps in
// block 0), so M is symmetric positive definite and CG stays CG.  The
// pre-smoothed iterate x = w D^-1 b is never stored: the restriction of its
// residual and the post-smoothing (with x = w D^-1 b + P y_coarse) evaluate
// it at the stencil's nodes, so each level costs one pass and one barrier on
// the way down and one on the way up.
__device__ void vcycle(cg::grid_group &grid, const PcgArgs &a, unsigned first, unsigned stride)
{
    const int L = a.mg.nlev;
    for (int l = 0; l < L - 1; l++) {
        const MgLevel &F = a.mg.lev[l], &C = a.mg.lev[l + 1];
        const unsigned ncf = (unsigned)(F.nx * F.ny);
        const double *fb = F.b, *fc = F.coef;
        auto xpre = [fb, fc, ncf](unsigned j, unsigned c, int, int, int) { return MG_OMEGA * fb[j] * fc[6 * ncf + c]; };
        const unsigned nc = (unsigned)C.n, ncc = (unsigned)(C.nx * C.ny);
        for (unsigned I = first; I < nc; I += stride) {
            const unsigned Z = I / ncc, rc = I - Z * ncc, Y = rc / (unsigned)C.nx, X = rc - Y * (unsigned)C.nx;
            double s = 0.0;
            for (int dz = 0; dz < F.bz; dz++)
                for (int dy = 0; dy < F.by; dy++)
                    for (int dx = 0; dx < F.bx; dx++) {
                        const int x = (int)X * F.bx + dx, y = (int)Y * F.by + dy, z = (int)Z * F.bz + dz;
                        if (x >= F.nx || y >= F.ny) continue;
                        const unsigned col = (unsigned)(y * F.nx + x), i = (unsigned)z * ncf + col;
                        if (fc[col] == 0.0) continue;
                        s += fb[i] - apply_level_fn(F, x, y, z, xpre);
                    }
            C.b[I] = s;
        }
        grid.sync();
    }
    {   // coarsest level: Jacobi sweeps from 0 in block 0 (x and y alternate)
        const MgLevel &C = a.mg.lev[L - 1];
        if (blockIdx.x == 0) {
            const unsigned nc = (unsigned)C.n, ncc = (unsigned)(C.nx * C.ny);
            for (unsigned i = threadIdx.x; i < nc; i += blockDim.x) C.y[i] = 0.0;
            __syncthreads();
            double *src = C.y, *dst = C.x;
            for (int sw = 0; sw < MG_COARSE_SWEEPS; sw++) {
                for (unsigned i = threadIdx.x; i < nc; i += blockDim.x) {
                    const unsigned Z = i / ncc, rc = i - Z * ncc, Y = rc / (unsigned)C.nx, X = rc - Y * (unsigned)C.nx;
                    const double id = C.coef[6 * ncc + rc];
                    dst[i] = id != 0.0 ? src[i] + MG_OMEGA * (C.b[i] - apply_level(C, src, i, (int)X, (int)Y, (int)Z)) * id : 0.0;
                }
                __syncthreads();
                double *t = src; src = dst; dst = t;
            }
            if (src != C.y)
                for (unsigned i = threadIdx.x; i < nc; i += blockDim.x) C.y[i] = src[i];
        }
        grid.sync();
    }
    for (int l = L - 2; l >= 0; l--) {
        const MgLevel &F = a.mg.lev[l], &C = a.mg.lev[l + 1];
        const unsigned nf = (unsigned)F.n, ncf = (unsigned)(F.nx * F.ny), ncc = (unsigned)(C.nx * C.ny);
        const double *fb = F.b, *fc = F.coef, *cy = C.y;
        const int sx = F.bx >> 1, sy = F.by >> 1, sz = F.bz >> 1, cnx = C.nx;   // aggregation factors are 1 or 2
        // x = w D^-1 b + P y_coarse at any node of the level
        auto xcor = [fb, fc, cy, ncf, ncc, sx, sy, sz, cnx](unsigned j, unsigned c, int x, int y, int z) {
            const double id = fc[6 * ncf + c];
            if (id == 0.0) return 0.0;
            return MG_OMEGA * fb[j] * id + cy[(unsigned)(z >> sz) * ncc + (unsigned)((y >> sy) * cnx + (x >> sx))];
        };
        for (unsigned i = first; i < nf; i += stride) {
            const unsigned z = i / ncf, rc = i - z * ncf, y = rc / (unsigned)F.nx, x = rc - y * (unsigned)F.nx;
            const double id = fc[6 * ncf + rc];
            F.y[i] = id != 0.0 ? xcor(i, rc, (int)x, (int)y, (int)z)
                                     + MG_OMEGA * (fb[i] - apply_level_fn(F, (int)x, (int)y, (int)z, xcor)) * id
                               : 0.0;
        }
        grid.sync();
    }
}

constexpr int PCG_BLOCKS_PER_SM = 3;

__global__ void __launch_bounds__(CG_THREADS, PCG_BLOCKS_PER_SM)
indicator_pcg_kernel(const PcgArgs a)
{
    cg::grid_group grid = cg::this_grid();
    const MgLevel &L0 = a.mg.lev[0];
    const unsigned n = (unsigned)L0.n, ncol = (unsigned)(L0.nx * L0.ny);
    const unsigned stride = gridDim.x * blockDim.x, first = blockIdx.x * blockDim.x + threadIdx.x;
    double lr = 0.0, lb = 0.0;
    for (unsigned i = first; i < n; i += stride) {
        const unsigned z = i / ncol, rc = i - z * ncol, y = rc / (unsigned)L0.nx, x = rc - y * (unsigned)L0.nx;
        if (L0.coef[rc] == 0.0) { a.x[i] = 0.0; a.r[i] = 0.0; a.p[i] = 0.0; continue; }
        const double ri = a.b[i] - apply_level(L0, a.x, i, (int)x, (int)y, (int)z);
        a.r[i] = ri;
        lr += ri * ri;
        lb += a.b[i] * a.b[i];
    }
    double rr, bb;
    int bank = 0;
    grid_sum2(grid, a.partial, bank, lr, lb, rr, bb);
    bank ^= 1;
    int it = 0;
    if (bb > 0.0 && !(sqrt(rr / bb) < a.tol)) {
        vcycle(grid, a, first, stride);   // z = M r (level 0's y)
        double lrz = 0.0;
        for (unsigned i = first; i < n; i += stride) { a.p[i] = L0.y[i]; lrz += a.r[i] * L0.y[i]; }
        double rz, unused;
        grid_sum2(grid, a.partial, bank, lrz, 0.0, rz, unused);
        bank ^= 1;
        while (it < a.itrmax) {
            double lpq = 0.0;
            for (unsigned i = first; i < n; i += stride) {
                const unsigned z = i / ncol, rc = i - z * ncol, y = rc / (unsigned)L0.nx, x = rc - y * (unsigned)L0.nx;
                const double qi = apply_level(L0, a.p, i, (int)x, (int)y, (int)z);
                a.q[i] = qi;
                lpq += a.p[i] * qi;
            }
            double pq;
            grid_sum2(grid, a.partial, bank, lpq, 0.0, pq, unused);
            bank ^= 1;
            const double alpha = rz / pq;
            double lrr = 0.0;
            for (unsigned i = first; i < n; i += stride) {
                const double ri = a.r[i] - alpha * a.q[i];
                a.x[i] += alpha * a.p[i];
                a.r[i] = ri;
                lrr += ri * ri;
            }
            grid_sum2(grid, a.partial, bank, lrr, 0.0, rr, unused);
            bank ^= 1;
            it++;
            if (sqrt(rr / bb) < a.tol) break;
            vcycle(grid, a, first, stride);
            double lrz2 = 0.0;
            for (unsigned i = first; i < n; i += stride) lrz2 += a.r[i] * L0.y[i];
            double rz_new;
            grid_sum2(grid, a.partial, bank, lrz2, 0.0, rz_new, unused);
            bank ^= 1;
            const double beta = rz_new / rz;
            rz = rz_new;
            for (unsigned i = first; i < n; i += stride) a.p[i] = L0.y[i] + beta * a.p[i];
            grid.sync();
        }
    }
    if (bb == 0.0)
        for (unsigned i = first; i < n; i += stride) a.x[i] = 0.0;
    if (first == 0) {
        const bool ok = bb == 0.0 || sqrt(rr / bb) < a.tol;
        *a.iters_out = ok ? it : -1;
        if (!ok) atomicOr(a.flags, RBC_FLAG_VOF_NOT_CONVERGED);
    }
}

int g_cg_blocks = 0;    // co-resident blocks of the CG kernel on this device
int g_pcg_blocks = 0;   // and of the preconditioned one

}  // namespace

int vof_cg_blocks()
{
    return g_cg_blocks > g_pcg_blocks ? g_cg_blocks : g_pcg_blocks;
}

cudaError_t vof_setup()
{
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, indicator_cg_kernel, CG_THREADS, 0);
    int per_sm2 = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, indicator_pcg_kernel, CG_THREADS, 0);
    if (e == cudaSuccess) g_cg_blocks = sms * (per_sm < CG_BLOCKS_PER_SM ? per_sm : CG_BLOCKS_PER_SM);
    if (e == cudaSuccess) g_pcg_blocks = sms * (per_sm2 < PCG_BLOCKS_PER_SM ? per_sm2 : PCG_BLOCKS_PER_SM);
    return e;
}

void launch_thinc_wlic(const Geom &g, double *vf, double *s1, double *s2, const float4 *uvr, const uint32_t *mask2d,
                       double dt, cudaStream_t s)
{
    const dim3 tiles((unsigned)((g.nx + TX - 1) / TX), (unsigned)((g.ny + TY - 1) / TY), (unsigned)((g.nzc + TZ - 1) / TZ));
    thinc_sweep_kernel<0><<<tiles, VOF_THREADS, 0, s>>>(g, vf, s1, uvr, mask2d, dt);
    thinc_sweep_kernel<1><<<tiles, VOF_THREADS, 0, s>>>(g, s1, s2, uvr, mask2d, dt);
    thinc_sweep_kernel<2><<<tiles, VOF_THREADS, 0, s>>>(g, s2, vf, uvr, mask2d, dt);
}

cudaError_t vof_mg_build(const Geom &g, const uint32_t *mask, MgHierarchy &mg)
{
    mg = MgHierarchy{};
    struct HostLevel { int nx, ny, nz, bx = 1, by = 1, bz = 1; std::vector<double> coef; };
    std::vector<HostLevel> lv(1);
    HostLevel &l0 = lv[0];
    l0.nx = g.nx; l0.ny = g.ny; l0.nz = g.nzc;
    const int nc0 = g.nx * g.ny;
    l0.coef.assign(7 * (size_t)nc0, 0.0);
    const double off = (1.0 / (g.dx * g.dx)) / (-6.0 / (g.dx * g.dx));
    auto fl = [&](int x, int y) { return (mask[(size_t)y * g.nx + x] & MASK_FLUID) != 0; };
    for (int y = 0; y < g.ny; y++)
        for (int x = 0; x < g.nx; x++) {
            if (!fl(x, y)) continue;
            const int c = y * g.nx + x;
            l0.coef[c] = 1.0;
            const int xl = x > 0 ? x - 1 : (g.xper ? g.nx - 1 : -1), xr = x < g.nx - 1 ? x + 1 : (g.xper ? 0 : -1);
            if (xl >= 0 && fl(xl, y)) l0.coef[nc0 + c] = off;
            if (xr >= 0 && fl(xr, y)) l0.coef[2 * nc0 + c] = off;
            if (y > 0 && fl(x, y - 1)) l0.coef[3 * nc0 + c] = off;
            if (y < g.ny - 1 && fl(x, y + 1)) l0.coef[4 * nc0 + c] = off;
            l0.coef[5 * nc0 + c] = off;
        }
    // Galerkin coarsening with piecewise-constant aggregation
    while ((int)lv.size() < MG_MAX_LEVELS) {
        HostLevel &f = lv.back();
        if ((long long)f.nx * f.ny * f.nz <= 512) break;
        const int bx = (f.nx >= 4 && !(g.xper && f.nx % 2)) ? 2 : 1, by = f.ny >= 4 ? 2 : 1;
        const int bz = (f.nz >= 4 && f.nz % 2 == 0) ? 2 : 1;
        if (bx * by * bz == 1) break;
        f.bx = bx; f.by = by; f.bz = bz;
        HostLevel c;
        c.nx = (f.nx + bx - 1) / bx; c.ny = (f.ny + by - 1) / by; c.nz = f.nz / bz;
        const int ncf = f.nx * f.ny, ncc = c.nx * c.ny;
        c.coef.assign(7 * (size_t)ncc, 0.0);
        for (int y = 0; y < f.ny; y++)
            for (int x = 0; x < f.nx; x++) {
                const int col = y * f.nx + x;
                const double d = f.coef[col];
                if (d == 0.0) continue;
                const int X = x / bx, Y = y / by, C = Y * c.nx + X;
                const double cxm = f.coef[ncf + col], cxp = f.coef[2 * ncf + col];
                const double cym = f.coef[3 * ncf + col], cyp = f.coef[4 * ncf + col], cz = f.coef[5 * ncf + col];
                c.coef[C] += bz * d + (bz == 2 ? 2.0 * cz : 0.0);   // the z link inside the block, both ways
                const int xl = x > 0 ? x - 1 : f.nx - 1, xr = x < f.nx - 1 ? x + 1 : 0;
                if (cxm != 0.0) { if (xl / bx == X) c.coef[C] += bz * cxm; else c.coef[ncc + C] += bz * cxm; }
                if (cxp != 0.0) { if (xr / bx == X) c.coef[C] += bz * cxp; else c.coef[2 * ncc + C] += bz * cxp; }
                if (cym != 0.0) { if ((y - 1) / by == Y) c.coef[C] += bz * cym; else c.coef[3 * ncc + C] += bz * cym; }
                if (cyp != 0.0) { if ((y + 1) / by == Y) c.coef[C] += bz * cyp; else c.coef[4 * ncc + C] += bz * cyp; }
                c.coef[5 * ncc + C] += cz;   // one link per fine column crosses each block boundary in z
            }
        lv.push_back(std::move(c));
    }
    const int L = (int)lv.size();
    if (L < 2) return cudaSuccess;
    for (HostLevel &h : lv) {   // row 6: the inverse diagonal (0 on wall columns)
        const size_t nc = (size_t)h.nx * h.ny;
        for (size_t c = 0; c < nc; c++) h.coef[6 * nc + c] = h.coef[c] != 0.0 ? 1.0 / h.coef[c] : 0.0;
    }
    // one allocation: every level's coefficients, level 0's x and y, the coarse levels' b, x, y
    size_t words = 0;
    for (int l = 0; l < L; l++) {
        const long long n = (long long)lv[l].nx * lv[l].ny * lv[l].nz;
        words += lv[l].coef.size() + (size_t)n * (l == 0 ? 2 : 3);
    }
    double *mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, 8 * words);
    if (e != cudaSuccess) return e;
    mg.mem = mem;
    double *cur = mem;
    for (int l = 0; l < L; l++) {
        MgLevel &d = mg.lev[l];
        const HostLevel &h = lv[l];
        d.nx = h.nx; d.ny = h.ny; d.nz = h.nz; d.bx = h.bx; d.by = h.by; d.bz = h.bz; d.xper = g.xper;
        d.n = (long long)h.nx * h.ny * h.nz;
        if ((e = cudaMemcpy(cur, h.coef.data(), 8 * h.coef.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        d.coef = cur; cur += h.coef.size();
        d.b = nullptr;
        if (l > 0) { d.b = cur; cur += d.n; }
        d.x = cur; cur += d.n;
        d.y = cur; cur += d.n;
    }
    mg.nlev = L;
    return cudaSuccess;
}

void vof_mg_free(MgHierarchy &mg)
{
    if (mg.mem) cudaFree(mg.mem);
    mg = MgHierarchy{};
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
    if (a.mg && a.mg->nlev >= 2) {
        PcgArgs c{};
        c.mg = *a.mg;
        c.mg.lev[0].b = a.G;   // the residual r is level 0's right-hand side
        c.b = a.b; c.x = a.vf; c.r = a.G; c.p = a.G + g.nint; c.q = a.G + 2 * g.nint;
        c.partial = a.partial; c.tol = a.tol; c.itrmax = a.itrmax; c.iters_out = a.iters; c.flags = a.flags;
        void *args[] = {&c};
        return cudaLaunchCooperativeKernel((const void *)indicator_pcg_kernel, dim3((unsigned)g_pcg_blocks),
                                           dim3(CG_THREADS), args, 0, s);
    }
    CgArgs c{};
    c.g = g; c.mask2d = a.mask2d; c.b = a.b; c.x = a.vf;
    c.r = a.G; c.p = a.G + g.nint; c.q = a.G + 2 * g.nint;
    c.partial = a.partial; c.tol = a.tol; c.itrmax = a.itrmax; c.iters_out = a.iters; c.flags = a.flags;
    void *args[] = {&c};
    return cudaLaunchCooperativeKernel((const void *)indicator_cg_kernel, dim3((unsigned)g_cg_blocks), dim3(CG_THREADS),
                                       args, 0, s);
}

}  // namespace rbc
