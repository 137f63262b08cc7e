// ibm.cu -- immersed-boundary force spreading and velocity interpolation.
//
// Spreading replaces ibm_st1a/ibm_st1b/ibm_st1c (ibm.cu:27-131, 214-296 of the
// reference).  The reference adds every vertex's 4x4x4 stencil straight into
// the FP64 lattice with CAS-loop atomics (about 192 contended atomics per
// vertex) and folds the BUFF planes afterwards.  Here one CTA owns one cell:
// it finds the cell's lattice bounding box, accumulates the cell's stencils in
// a shared-memory box with shared atomics, then adds each non-zero box node to
// the lattice once with a global FP32 atomic (cells may overlap).  z indices
// wrap periodically, which is what the BUFF planes plus the fold compute.
// A cell whose box does not fit in shared memory takes a direct-atomic path.
//
// Interpolation + advection replaces ibm_st2a (ibm.cu:372-639): four
// interpolations of the averaged velocity in a frozen field, classical RK4 in
// FP64 positions, periodic wrap in x and z as the reference does.
#include "rbc_internal.cuh"

#include <climits>

namespace rbc {

constexpr int SPREAD_THREADS = 512;
constexpr int SPREAD_SMEM = 100 * 1024;          // two CTAs per SM
constexpr int SPREAD_BOX_CAP = SPREAD_SMEM / (3 * (int)sizeof(float));

int spread_smem_bytes() { return SPREAD_SMEM; }

__device__ __forceinline__ double unwrap_near(double l, double ref, int n) {
    const double h = 0.5 * n;
    if (l - ref > h) l -= n; else if (l - ref < -h) l += n;
    return l;
}

__global__ void __launch_bounds__(SPREAD_THREADS)
spread_kernel(const Geom g, const double *__restrict__ X, long long nv, int V,
              const float *__restrict__ Fv, float *__restrict__ Fx, float *__restrict__ Fy,
              float *__restrict__ Fz, const uint32_t *__restrict__ mask2d, int *__restrict__ flags)
{
    extern __shared__ float sbox[];
    __shared__ int s_lo[3], s_hi[3];
    const int cell = blockIdx.x, tid = threadIdx.x;
    const double *xs = X + (long long)cell * V, *ys = X + nv + (long long)cell * V, *zs = X + 2 * nv + (long long)cell * V;
    const float *fxs = Fv + (long long)cell * V, *fys = Fv + nv + (long long)cell * V, *fzs = Fv + 2 * nv + (long long)cell * V;
    const float wscale = (float)(1.0 / (g.dx * g.dx * g.dx));   // 1/(64 dx^3) of ibm.cu:108 with the 1/4s in delta4
    const double az = lat_z(g, zs[0]);

    if (tid < 3) { s_lo[tid] = INT_MAX; s_hi[tid] = INT_MIN; }
    __syncthreads();
    int lo0 = INT_MAX, lo1 = INT_MAX, lo2 = INT_MAX, hi0 = INT_MIN, hi1 = INT_MIN, hi2 = INT_MIN;
    for (int v = tid; v < V; v += blockDim.x) {
        const int ix = (int)floor(lat_x(g, xs[v])), iy = (int)floor(lat_y(g, ys[v]));
        const int iz = (int)floor(unwrap_near(lat_z(g, zs[v]), az, g.nzc));
        lo0 = min(lo0, ix - 1); hi0 = max(hi0, ix + 2);
        lo1 = min(lo1, iy - 1); hi1 = max(hi1, iy + 2);
        lo2 = min(lo2, iz - 1); hi2 = max(hi2, iz + 2);
    }
    atomicMin(&s_lo[0], lo0); atomicMin(&s_lo[1], lo1); atomicMin(&s_lo[2], lo2);
    atomicMax(&s_hi[0], hi0); atomicMax(&s_hi[1], hi1); atomicMax(&s_hi[2], hi2);
    __syncthreads();
    const int bx0 = s_lo[0], by0 = s_lo[1], bz0 = s_lo[2];
    const int bx = s_hi[0] - bx0 + 1, by = s_hi[1] - by0 + 1, bz = s_hi[2] - bz0 + 1;
    const long long nb = (long long)bx * by * bz;
    const bool use_box = nb <= SPREAD_BOX_CAP;
    if (!use_box && tid == 0) atomicOr(flags, RBC_FLAG_SPREAD_OVERFLOW);

    if (use_box) {
        for (int i = tid; i < 3 * nb; i += blockDim.x) sbox[i] = 0.f;
        __syncthreads();
    }
    // One warp per vertex: lane l owns stencil nodes k = l and l + 32 with
    // (a, b, c) = (k & 3, (k >> 2) & 3, k >> 4), so the 32 atomics of one warp
    // instruction go to 32 different box nodes (lanes working on neighbouring
    // vertices would collide on the same nodes).
    const int lane = tid & 31, nwarp = blockDim.x >> 5;
    for (int v = tid >> 5; v < V; v += nwarp) {
        const double lx = lat_x(g, xs[v]), ly = lat_y(g, ys[v]);
        const double lzr = lat_z(g, zs[v]);
        const double lz = unwrap_near(lzr, az, g.nzc);
        const double flx = floor(lx), fly = floor(ly), flz = floor(lz);
        // lanes 0..2 evaluate sin/cos of the three fractions, the warp shares them
        float sv = 0.f, cv = 0.f;
        if (lane < 3) sincospif(0.5f * (float)(lane == 0 ? lx - flx : (lane == 1 ? ly - fly : lz - flz)), &sv, &cv);
        const int ix0 = (int)flx - 1, iy0 = (int)fly - 1, iz0 = (int)flz - 1;
        const int izr0 = iz0 - (int)lrint(lz - lzr);   // stencil start in the vertex's own (unshifted) frame
        const float f0 = fxs[v] * wscale, f1 = fys[v] * wscale, f2 = fzs[v] * wscale;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int k = lane + 32 * half;
            const int ka = k & 3, kb = (k >> 2) & 3, kc = k >> 4;
            // phi at offset 0..3 = (1 - s, 1 + c, 1 + s, 1 - c) / 4 (delta4)
            const float sx = __shfl_sync(0xffffffffu, sv, 0), cx = __shfl_sync(0xffffffffu, cv, 0);
            const float sy = __shfl_sync(0xffffffffu, sv, 1), cy = __shfl_sync(0xffffffffu, cv, 1);
            const float sz = __shfl_sync(0xffffffffu, sv, 2), cz = __shfl_sync(0xffffffffu, cv, 2);
            const float wa = 0.25f * (ka == 0 ? 1.f - sx : ka == 1 ? 1.f + cx : ka == 2 ? 1.f + sx : 1.f - cx);
            const float wb = 0.25f * (kb == 0 ? 1.f - sy : kb == 1 ? 1.f + cy : kb == 2 ? 1.f + sy : 1.f - cy);
            const float wc = 0.25f * (kc == 0 ? 1.f - sz : kc == 1 ? 1.f + cz : kc == 2 ? 1.f + sz : 1.f - cz);
            const int gx = ix0 + ka, gy = iy0 + kb;
            // the reference's lattice ends two BUFF planes beyond the periodic
            // range; stencil nodes past them are skipped (ibm.cu:107-110)
            if (izr0 + kc < -2 || izr0 + kc >= g.nzc + 2) continue;
            if (gx < 0 || gx >= g.nx || gy < 0 || gy >= g.ny) continue;
            if (!(__ldg(&mask2d[gx + g.nx * gy]) & MASK_FLUID)) continue;
            const float w = wa * wb * wc;
            if (use_box) {
                const long long li = (gx - bx0) + (long long)bx * ((gy - by0) + (long long)by * (iz0 + kc - bz0));
                atomicAdd(&sbox[li], w * f0);
                atomicAdd(&sbox[nb + li], w * f1);
                atomicAdd(&sbox[2 * nb + li], w * f2);
            } else {
                const long long gi = (long long)wrap_z(iz0 + kc, g.nzc) * g.plane + gx + (long long)g.nx * gy;
                atomicAdd(&Fx[gi], w * f0);
                atomicAdd(&Fy[gi], w * f1);
                atomicAdd(&Fz[gi], w * f2);
            }
        }
    }
    if (!use_box) return;
    __syncthreads();
    for (long long li = tid; li < nb; li += blockDim.x) {
        const float a = sbox[li], b = sbox[nb + li], c = sbox[2 * nb + li];
        if (a == 0.f && b == 0.f && c == 0.f) continue;
        const int lx = (int)(li % bx), rest = (int)(li / bx);
        const int ly = rest % by, lz = rest / by;
        const int gx = bx0 + lx, gy = by0 + ly;
        if (gx < 0 || gx >= g.nx || gy < 0 || gy >= g.ny) continue;   // never written; kept as a guard
        const long long gi = (long long)wrap_z(bz0 + lz, g.nzc) * g.plane + gx + (long long)g.nx * gy;
        if (a != 0.f) atomicAdd(&Fx[gi], a);
        if (b != 0.f) atomicAdd(&Fy[gi], b);
        if (c != 0.f) atomicAdd(&Fz[gi], c);
    }
}

cudaError_t spread_setup()
{
    return cudaFuncSetAttribute(spread_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SPREAD_SMEM);
}

void launch_spread(const Geom &g, const SpreadArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    spread_kernel<<<a.ncell, SPREAD_THREADS, SPREAD_SMEM, s>>>(g, a.X, a.nv, a.V, a.Fv, a.Fx, a.Fy, a.Fz,
                                                              a.mask2d, a.flags);
}

// ---- interpolation + RK4 advection ---------------------------------------

// Four lanes per vertex: lane c of the group gathers stencil plane c (16 nodes,
// one float4 (u, v, w, rho) each); the group sums its partial velocities with
// two butterfly shuffles, so every lane holds the interpolated velocity.
__device__ __forceinline__ void interp4(const Geom &g, const float4 *__restrict__ uvr, double px, double py,
                                        double pz, int c, float &ur, float &vr, float &wr)
{
    const double lx = lat_x(g, px), ly = lat_y(g, py), lz = lat_z(g, pz);
    const double flx = floor(lx), fly = floor(ly), flz = floor(lz);
    float wx[4], wy[4], wz[4];
    delta4((float)(lx - flx), wx); delta4((float)(ly - fly), wy); delta4((float)(lz - flz), wz);
    const int ix0 = (int)flx - 1, iy0 = (int)fly - 1, iz = (int)flz - 1 + c;
    float su = 0.f, sv = 0.f, sw = 0.f;
    if (iz >= -2 && iz < g.nzc + 2) {   // beyond the BUFF planes (ibm.cu:453-455)
        const long long zb = (long long)wrap_z(iz, g.nzc) * g.plane;
        const float wzc = c == 0 ? wz[0] : c == 1 ? wz[1] : c == 2 ? wz[2] : wz[3];
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int gy = iy0 + b;
            if (gy < 0 || gy >= g.ny) continue;
            const float wyz = wy[b] * wzc;
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const int gx = ix0 + a;
                if (gx < 0 || gx >= g.nx) continue;
                const float4 q = __ldg(&uvr[zb + gx + (long long)g.nx * gy]);
                const float w = wx[a] * wyz;
                su += w * q.x; sv += w * q.y; sw += w * q.z;
            }
        }
    }
#pragma unroll
    for (int o = 1; o <= 2; o <<= 1) {
        su += __shfl_xor_sync(0xffffffffu, su, o);
        sv += __shfl_xor_sync(0xffffffffu, sv, o);
        sw += __shfl_xor_sync(0xffffffffu, sw, o);
    }
    ur = su; vr = sv; wr = sw;
}

constexpr int ADVECT_THREADS = 256;

__global__ void __launch_bounds__(ADVECT_THREADS, 4)
advect_kernel(const Geom g, double *__restrict__ X, double *__restrict__ Xd, float *__restrict__ U,
              const float4 *__restrict__ uvr, long long nv, double dtM, int *__restrict__ flags)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = (int)(t & 3);
    const bool live = (t >> 2) < nv;
    const long long j = live ? (t >> 2) : nv - 1;   // idle lanes shadow the last vertex for the shuffles
    const double xn = X[j], yn = X[nv + j], zn = X[2 * nv + j];
    float u1, v1, w1, u2, v2, w2, u3, v3, w3, u4, v4, w4;
    interp4(g, uvr, xn, yn, zn, c, u1, v1, w1);
    interp4(g, uvr, xn + u1 * dtM * 0.5, yn + v1 * dtM * 0.5, zn + w1 * dtM * 0.5, c, u2, v2, w2);
    interp4(g, uvr, xn + u2 * dtM * 0.5, yn + v2 * dtM * 0.5, zn + w2 * dtM * 0.5, c, u3, v3, w3);
    interp4(g, uvr, xn + u3 * dtM, yn + v3 * dtM, zn + w3 * dtM, c, u4, v4, w4);
    if (!live || c != 0) return;
    const double um = ((double)u1 + 2.0 * u2 + 2.0 * u3 + u4) / 6.0;
    const double vm = ((double)v1 + 2.0 * v2 + 2.0 * v3 + v4) / 6.0;
    const double wm = ((double)w1 + 2.0 * w2 + 2.0 * w3 + w4) / 6.0;
    double xr = xn + um * dtM, yr = yn + vm * dtM, zr = zn + wm * dtM;
    if (xr < g.xmin) xr += g.LX;   // ibm.cu:629-632
    if (xr > g.xmax) xr -= g.LX;
    if (zr < g.zmin) zr += g.LZ;
    if (zr > g.zmax) zr -= g.LZ;
    if (!isfinite(xr) || !isfinite(yr) || !isfinite(zr)) atomicOr(flags, RBC_FLAG_NONFINITE);
    X[j] = xr; X[nv + j] = yr; X[2 * nv + j] = zr;
    Xd[j] = xr; Xd[nv + j] = yr; Xd[2 * nv + j] = zr;
    U[j] = (float)um; U[nv + j] = (float)vm; U[2 * nv + j] = (float)wm;
}

void launch_advect(const Geom &g, const AdvectArgs &a, cudaStream_t s)
{
    if (a.nv <= 0) return;
    const long long threads = 4 * a.nv;
    advect_kernel<<<(unsigned)((threads + ADVECT_THREADS - 1) / ADVECT_THREADS), ADVECT_THREADS, 0, s>>>(
        g, a.X, a.Xd, a.U, a.uvr, a.nv, a.dtM, a.flags);
}

}  // namespace rbc
