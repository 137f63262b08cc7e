// ibm.cu -- immersed-boundary force spreading and velocity interpolation.
//
// Spreading replaces ibm_st1a/ibm_st1b/ibm_st1c (ibm.cu:27-131, 214-296 of the
// reference).  The reference adds every vertex's 4x4x4 stencil straight into
// the FP64 lattice with CAS-loop atomics (about 192 contended atomics per
// vertex) and folds the BUFF planes afterwards.  Here one CTA owns one surface
// patch of one cell: it finds the patch's lattice bounding box, accumulates
// the patch's stencils in a shared-memory box with shared atomics, then adds
// each non-zero box node to the lattice once with a global 64-bit integer
// atomic (patches and cells overlap) into the fixed-point force field
// (ForceField), whose sums do not depend on the order of the atomics.  z
// indices wrap periodically, which is what the BUFF planes plus the fold
// compute.  A patch whose box does not fit in shared memory takes a
// direct-atomic path (into the same fixed point, so it is deterministic too).
//
// Interpolation + advection replaces ibm_st2a (ibm.cu:372-639): four
// interpolations of the averaged velocity in a frozen field, classical RK4 in
// FP64 positions, periodic wrap in x and z as the reference does.
#include <cfloat>
#include "rbc_internal.cuh"

#include <climits>

namespace rbc {

constexpr int SPREAD_THREADS = 256;
constexpr int SPREAD_SMEM = 48 * 1024;           // up to four CTAs per SM
constexpr int SPREAD_BOX_CAP = SPREAD_SMEM / (3 * (int)sizeof(unsigned));

int spread_smem_bytes() { return SPREAD_SMEM; }

// A lattice coordinate that the box arithmetic can take: finite and within
// 2^24 nodes (positions outside are a blown-up state; they raise
// RBC_FLAG_NONFINITE instead of indexing anything).
__device__ __forceinline__ bool sane_lattice(double l) { return fabs(l) < 16777216.0; }

// v * 2^shift rounded to the nearest integer (ties to even) into out; false
// when its magnitude reaches 2^62 (no add is then made).
__device__ __forceinline__ bool to_fixed(double v, int shift, long long &out) {
    const double d = ldexp(v, shift);   // exact: a power-of-two scaling
    if (!(fabs(d) < 4.611686018427387904e18)) return false;
    out = __double2ll_rn(d);
    return true;
}

// v * 2^shift rounded to the nearest integer, ties to even (as __double2ll_rn
// of the exact FP64 product, in integer arithmetic); false beyond 2^62 in
// magnitude.  v: a box sum (|v| < 2^31).
__device__ __forceinline__ bool box_to_fixed(int v, int shift, long long &out) {
    if (shift >= 0) {
        if (shift > 62) { out = 0; return v == 0; }
        const long long lim = 1LL << (62 - shift);
        if (v >= lim || -(long long)v >= lim) return false;
        out = (long long)v << shift;
        return true;
    }
    const int k = -shift;
    if (k > 32) { out = 0; return true; }
    const long long x = v, q = x >> k, r = x - (q << k), half = 1LL << (k - 1);
    out = (r > half || (r == half && (q & 1))) ? q + 1 : q;
    return true;
}

// Adds one node's fixed-point force (three components; zeros skipped).
// *added: whether anything was added (the node's occupancy bit must be set).
// Returns false if a component was out of range.
__device__ __forceinline__ bool add_force(const ForceField &F, long long nint, long long gi, double a, double b,
                                          double c, int sa, int sb, int sc, bool *added) {
    long long ia = 0, ib = 0, ic = 0;
    const bool ok = to_fixed(a, sa, ia) & to_fixed(b, sb, ib) & to_fixed(c, sc, ic);
    if (ia) atomicAdd(reinterpret_cast<unsigned long long *>(&F.F[gi]), (unsigned long long)ia);
    if (ib) atomicAdd(reinterpret_cast<unsigned long long *>(&F.F[nint + gi]), (unsigned long long)ib);
    if (ic) atomicAdd(reinterpret_cast<unsigned long long *>(&F.F[2 * nint + gi]), (unsigned long long)ic);
    *added = (ia | ib | ic) != 0;
    return ok;
}

__device__ __forceinline__ double unwrap_near(double l, double ref, int n) {
    const double h = 0.5 * n;
    if (l - ref > h) l -= n; else if (l - ref < -h) l += n;
    return l;
}

// One CTA per (cell, surface patch).  Patches are compact groups of mesh
// vertices (recursive coordinate bisection of the reference shape, the same
// for every cell), so a patch's stencils fit a small box and a step has many
// more CTAs than cells.  Box layout: x fastest, rows of bx, planes of ps >= bx*by
// with ps = 8 (mod 32) so the four stencil planes of one vertex sit in
// different shared-memory banks.
// bid: the block's (cell, patch) index, blockIdx.x of a one-lattice launch
template <bool XPER>
__device__ __forceinline__ void
spread_body(const Geom &g, const double *__restrict__ X, long long nv, int V,
            const int *__restrict__ patch_off, const int *__restrict__ patch_vtx,
            const int *__restrict__ patch_stride, int npatch,
            const float *__restrict__ Fv, const ForceField &F, const uint32_t *__restrict__ mask2d,
            int *__restrict__ flags, int bid)
{
    extern __shared__ __align__(16) unsigned sbox[];
    // each patch vertex's lattice cell, unwrap shifts and fractions, from the bounds pass
    __shared__ int4 s_cell[MAX_PATCH_VERTICES];      // floor(lx), floor(ly), floor(lz), z unwrap shift
    __shared__ float4 s_frac[MAX_PATCH_VERTICES];    // lx - floor(lx), ly - floor(ly), lz - floor(lz), x shift
    __shared__ int s_lo[3], s_hi[3];
    __shared__ unsigned s_fmax[3], s_wmax;
    const int cell = bid / npatch, patch = bid - cell * npatch, tid = threadIdx.x;
    const int p0 = patch_off[patch], np = patch_off[patch + 1] - p0, vstride = patch_stride[patch];
    const double *xs = X + (long long)cell * V, *ys = X + nv + (long long)cell * V, *zs = X + 2 * nv + (long long)cell * V;
    const float *fxs = Fv + (long long)cell * V, *fys = Fv + nv + (long long)cell * V, *fzs = Fv + 2 * nv + (long long)cell * V;
    const float wscale = (float)(1.0 / (g.dx * g.dx * g.dx));   // 1/(64 dx^3) of ibm.cu:108 with the 1/4s in delta4
    const double az = lat_z(g, zs[0]);   // one anchor per cell: every patch unwraps z the same way
    const double ax = lat_x(g, xs[0]);   // and x, when x is periodic (shear mode)

    if (tid < 3) { s_lo[tid] = INT_MAX; s_hi[tid] = INT_MIN; }
    if (tid < 3) s_fmax[tid] = 0u;
    if (tid == 0) s_wmax = 0u;
    __syncthreads();
    int lo0 = INT_MAX, lo1 = INT_MAX, lo2 = INT_MAX, hi0 = INT_MIN, hi1 = INT_MIN, hi2 = INT_MIN;
    float fmax0 = 0.f, fmax1 = 0.f, fmax2 = 0.f;
    bool nonfinite = false;
#pragma unroll 2
    for (int k = tid; k < np; k += blockDim.x) {
        const int v = patch_vtx[p0 + k];
        const float afx = fabsf(fxs[v]), afy = fabsf(fys[v]), afz = fabsf(fzs[v]);
        nonfinite |= !(afx <= FLT_MAX && afy <= FLT_MAX && afz <= FLT_MAX);
        fmax0 = fmaxf(fmax0, afx); fmax1 = fmaxf(fmax1, afy); fmax2 = fmaxf(fmax2, afz);
        const double lxr = lat_x(g, xs[v]), lxv = XPER ? unwrap_near(lxr, ax, g.nx) : lxr;
        const double lzr = lat_z(g, zs[v]);
        const double lyv = lat_y(g, ys[v]), lzv = unwrap_near(lzr, az, g.nzc);
        if (!(sane_lattice(lxv) && sane_lattice(lyv) && sane_lattice(lzv) && sane_lattice(az) && sane_lattice(ax))) { nonfinite = true; continue; }
        const double flx = floor(lxv), fly = floor(lyv), flz = floor(lzv);
        const int ix = (int)flx, iy = (int)fly;
        const int iz = (int)flz;
        const int xsh = XPER ? (int)lrint(lxv - lxr) : 0, zsh = (int)lrint(lzv - lzr);   // unwrapped minus raw frame
        s_cell[k] = make_int4(ix, iy, iz, zsh);
        s_frac[k] = make_float4((float)(lxv - flx), (float)(lyv - fly), (float)(lzv - flz), (float)xsh);
        lo0 = min(lo0, ix - 1); hi0 = max(hi0, ix + 2);
        lo1 = min(lo1, iy - 1); hi1 = max(hi1, iy + 2);
        lo2 = min(lo2, iz - 1); hi2 = max(hi2, iz + 2);
    }
    atomicMin(&s_lo[0], lo0); atomicMin(&s_lo[1], lo1); atomicMin(&s_lo[2], lo2);
    atomicMax(&s_hi[0], hi0); atomicMax(&s_hi[1], hi1); atomicMax(&s_hi[2], hi2);
    // non-negative floats order like their bit patterns
    atomicMax(&s_fmax[0], __float_as_uint(fmax0));
    atomicMax(&s_fmax[1], __float_as_uint(fmax1));
    atomicMax(&s_fmax[2], __float_as_uint(fmax2));
    if (__syncthreads_or(nonfinite)) {
        if (tid == 0) atomicOr(flags, RBC_FLAG_NONFINITE);
        return;
    }
    if ((s_fmax[0] | s_fmax[1] | s_fmax[2]) == 0u) return;   // no force on this patch
    const int bx0 = s_lo[0], by0 = s_lo[1], bz0 = s_lo[2];
    const int bx = s_hi[0] - bx0 + 1, by = s_hi[1] - by0 + 1, bz = s_hi[2] - bz0 + 1;
    const long long ps = (((long long)bx * by + 31) & ~31LL) + 8;   // plane stride = 8 (mod 32)
    const long long nb = ps * bz;
    const bool use_box = bx >= 4 && by >= 4 && bz >= 4 && nb <= SPREAD_BOX_CAP;
    if (!use_box && tid == 0) atomicOr(flags, RBC_FLAG_SPREAD_OVERFLOW);
    const int psi = use_box ? (int)ps : 0, nbi = use_box ? (int)nb : 0;   // box indices fit in int

    // Box sums in 32-bit fixed point, one power-of-two scale per force
    // component.  A vertex whose stencil starts at node b - 1 (b = floor of
    // its lattice position) gives node b - 1 + a a 1-D weight of at most
    // k[a] = (1, 2, 2, 1) / 4 (the largest values of delta4's weights), so
    // Wn = sum over base cells b of count(b) * k[ax] * k[ay] * k[az] bounds
    // the sum of the weights at node n, and no node's force sum exceeds
    // max(Wn) * fmax.  A scale of at most 2^31 / that keeps every FINAL sum in
    // range; partial sums may wrap, but the adds are modular (unsigned), so
    // the final sums are still exact.  Each term is an FP32 product rounded
    // once to an integer, the integer sums do not depend on the order of the
    // atomics, and converting back costs one rounding to FP32 (the scale is
    // capped at 2^126 so that it and its inverse stay normal floats).  The
    // flush converts each box sum exactly (a power-of-two scaling, rounded
    // only where the box resolves finer than 2^-FORCE_FRAC) to the lattice's
    // fixed point, whose integer sums are again order independent.
    float qs[3] = {0.f, 0.f, 0.f};
    int qe[3] = {0, 0, 0};
    if (use_box) {
        // Wn in units of 1/64: each vertex adds 4 k[a] * 4 k[b] to the 16
        // nodes (x, y) of its stencil in its base plane; a walk down each
        // column then applies 4 k along z with a sliding window.
        unsigned *cnt = sbox + 2 * nbi;
        for (int i = tid; i < nbi / 4; i += SPREAD_THREADS) reinterpret_cast<uint4 *>(cnt)[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        for (int k = tid; k < np; k += SPREAD_THREADS) {
            const int4 cl = s_cell[k];
            const int li0 = (cl.x - 1 - bx0) + bx * (cl.y - 1 - by0) + psi * (cl.z - bz0);
#pragma unroll
            for (int b = 0; b < 4; b++)
#pragma unroll
                for (int a = 0; a < 4; a++)
                    atomicAdd(&cnt[li0 + a + bx * b], (unsigned)((a == 0 || a == 3 ? 1 : 2) * (b == 0 || b == 3 ? 1 : 2)));
        }
        __syncthreads();
        unsigned wmax = 0u;
        for (int r = tid; r < bx * by; r += SPREAD_THREADS) {
            unsigned c2 = 0u, c1 = 0u, c0 = 0u, nx1 = cnt[r];   // base planes z-2, z-1, z, z+1
            for (int z = 0; z < bz; z++) {
                c2 = c1; c1 = c0; c0 = nx1;
                nx1 = z + 1 < bz ? cnt[(z + 1) * psi + r] : 0u;
                wmax = max(wmax, nx1 + 2u * (c0 + c1) + c2);
            }
        }
        atomicMax(&s_wmax, wmax);
        __syncthreads();
        const float wb = (float)s_wmax * (1.0f / 64.0f);
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float fm = __uint_as_float(s_fmax[k]) * wscale;
            // 2.147e9 < 2^31 leaves room for the rounding of the terms
            const float e = fminf(floorf(log2f(2.147e9f / (wb * fm))), 126.f);
            qs[k] = exp2f(e);
            qe[k] = (int)e;
        }
        for (int i = tid; i < 3 * nbi / 4; i += blockDim.x) reinterpret_cast<uint4 *>(sbox)[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
    }
    // Four tasks per vertex: task i handles stencil plane c = i & 3 of the
    // patch's vertex (i >> 2) * vstride mod np.  vstride is coprime with np, so
    // the lanes of a warp hold vertices spread over the patch and rarely add
    // to the same box node in one instruction.  The fluid test is applied once
    // per node at the flush (wall columns accumulate in shared memory and are
    // dropped there).
    // SPREAD_THREADS is a multiple of 4, so a thread keeps one plane c and
    // steps through j = tid / 4 + k * SPREAD_THREADS / 4, whose patch slot
    // j * vstride mod np advances by a constant.
    const int c = tid & 3, jstep = SPREAD_THREADS / 4;
    const int vstep = (int)(((long long)jstep * vstride) % np);
    int jv = (int)(((long long)(tid >> 2) * vstride) % np);
    for (int j = tid >> 2; j < np; j += jstep) {
        const int v = patch_vtx[p0 + jv];
        const int4 cl = s_cell[jv];
        const float4 fr = s_frac[jv];
        jv += vstep;
        if (jv >= np) jv -= np;
        const int xsh = (int)fr.w, zsh = cl.w;   // unwrapped minus raw frame (x shift exact in FP32: |x| < 2^24)
        const int iz = cl.z - 1 + c;
        // the reference's lattice ends two BUFF planes beyond the periodic
        // range; stencil nodes past them are skipped (ibm.cu:107-110)
        const int izr = iz - zsh;
        if (izr < -2 || izr >= g.nzc + 2) continue;
        float wx[4], wy[4], wz[4];
        delta4(fr.x, wx); delta4(fr.y, wy); delta4(fr.z, wz);
        const float wzc = c == 0 ? wz[0] : c == 1 ? wz[1] : c == 2 ? wz[2] : wz[3];
        const int ix0 = cl.x - 1, iy0 = cl.y - 1;
        const float sc = wscale * wzc;
        const float f0 = fxs[v] * sc, f1 = fys[v] * sc, f2 = fzs[v] * sc;
        const float q0 = f0 * qs[0], q1 = f1 * qs[1], q2 = f2 * qs[2];
        const int zoff = psi * (iz - bz0);
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int gy = iy0 + b;
            if (gy < 0 || gy >= g.ny) continue;
            const float wyb = wy[b];
#pragma unroll
            for (int a = 0; a < 4; a++) {
                const int gx = ix0 + a;
                // x: outside the lattice; periodic (shear mode): nodes beyond the two BUFF
                // columns of the vertex's raw frame are dropped as ibm.cu:107-110 drops them,
                // the rest fold periodically (ibm.cu:239-294)
                if (!XPER && (gx < 0 || gx >= g.nx)) continue;
                if (XPER && (gx - xsh < -g.xb || gx - xsh >= g.nx + g.xb)) continue;
                const float w = wx[a] * wyb;
                const int gxw = XPER ? wrap_x(gx, g.nx) : gx;
                if (use_box) {
                    const int li = (gx - bx0) + bx * (gy - by0) + zoff;
                    atomicAdd(&sbox[li], (unsigned)__float2int_rn(w * q0));
                    atomicAdd(&sbox[nbi + li], (unsigned)__float2int_rn(w * q1));
                    atomicAdd(&sbox[2 * nbi + li], (unsigned)__float2int_rn(w * q2));
                } else if (__ldg(&mask2d[gxw + g.nx * gy]) & MASK_FLUID) {
                    const int zw = wrap_z(iz, g.nzc);
                    const long long xy = gxw + (long long)g.nx * gy, gi = (long long)zw * g.plane + xy;
                    bool added = false;
                    if (!add_force(F, g.nint, gi, (double)(w * f0), (double)(w * f1), (double)(w * f2),
                                   FORCE_FRAC, FORCE_FRAC, FORCE_FRAC, &added))
                        atomicOr(flags, RBC_FLAG_NONFINITE);
                    if (added) atomicOr(&F.bits[(long long)zw * F.wpp + (xy >> 5)], 1u << (xy & 31));
                }
            }
        }
    }
    if (!use_box) return;
    __syncthreads();
    const int rowplane = bx * by;
    // one item = one box column (x, y) and ZC consecutive planes: the column's lattice
    // position and wall test once per item, the planes' box reads independent of each other
    constexpr int ZC = 2;
    const int items = rowplane * ((bz + ZC - 1) / ZC);
    for (int it = tid; it < items; it += SPREAD_THREADS) {
        const int zc = it / rowplane, r = it - zc * rowplane;
        const int ly = r / bx, lx = r - ly * bx;
        const int gx = XPER ? wrap_x(bx0 + lx, g.nx) : bx0 + lx, gy = by0 + ly;
        if (gx < 0 || gx >= g.nx || gy < 0 || gy >= g.ny) continue;   // never written; kept as a guard
        if (!(__ldg(&mask2d[gx + g.nx * gy]) & MASK_FLUID)) continue;   // wall column: the LBM never reads it
        const long long xy = gx + (long long)g.nx * gy;
#pragma unroll
        for (int u = 0; u < ZC; u++) {
            const int lz = zc * ZC + u;
            if (lz >= bz) break;
            const int li = lz * psi + r;
            const int ia = (int)sbox[li], ib = (int)sbox[nbi + li], ic = (int)sbox[2 * nbi + li];
            if ((ia | ib | ic) == 0) continue;
            int zw = bz0 + lz;   // the box spans less than a period: one correction, the modulo as a fallback
            if (zw < 0) zw += g.nzc;
            if (zw >= g.nzc) zw -= g.nzc;
            if ((unsigned)zw >= (unsigned)g.nzc) zw = wrap_z(zw, g.nzc);
            const long long gi = (long long)zw * g.plane + xy;
            long long fa = 0, fb = 0, fc = 0;
            const bool ok = box_to_fixed(ia, FORCE_FRAC - qe[0], fa) & box_to_fixed(ib, FORCE_FRAC - qe[1], fb) &
                            box_to_fixed(ic, FORCE_FRAC - qe[2], fc);
            if (!ok) atomicOr(flags, RBC_FLAG_NONFINITE);
            if (fa) atomicAdd(reinterpret_cast<unsigned long long *>(&F.F[gi]), (unsigned long long)fa);
            if (fb) atomicAdd(reinterpret_cast<unsigned long long *>(&F.F[g.nint + gi]), (unsigned long long)fb);
            if (fc) atomicAdd(reinterpret_cast<unsigned long long *>(&F.F[2 * g.nint + gi]), (unsigned long long)fc);
            if (fa | fb | fc) atomicOr(&F.bits[(long long)zw * F.wpp + (xy >> 5)], 1u << (xy & 31));
        }
    }
}

template <bool XPER>
__global__ void __launch_bounds__(SPREAD_THREADS)
spread_kernel(const Geom g, const double *__restrict__ X, long long nv, int V,
              const int *__restrict__ patch_off, const int *__restrict__ patch_vtx,
              const int *__restrict__ patch_stride, int npatch,
              const float *__restrict__ Fv, const ForceField F, const uint32_t *__restrict__ mask2d,
              int *__restrict__ flags)
{
    pdl_start();
    spread_body<XPER>(g, X, nv, V, patch_off, patch_vtx, patch_stride, npatch, Fv, F, mask2d, flags, blockIdx.x);
}

cudaError_t spread_setup()
{
    cudaError_t e = cudaFuncSetAttribute(spread_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, SPREAD_SMEM);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(spread_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, SPREAD_SMEM);
}

void launch_spread(const Geom &g, const SpreadArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    auto k = g.xper ? spread_kernel<true> : spread_kernel<false>;
    launch_pdl(k, dim3(a.ncell * a.npatch), dim3(SPREAD_THREADS), SPREAD_SMEM, s,
               g, a.X, a.nv, a.V, a.patch_off, a.patch_vtx, a.patch_stride, a.npatch, a.Fv, a.F, a.mask2d, a.flags);
}

// ---- interpolation + RK4 advection ---------------------------------------

// Four lanes per vertex: lane c of the group owns stencil plane c (16 nodes).
// The stage-1 stencil is loaded once into registers (u, v, w of 16 nodes) and
// reused by the later RK stages, whose positions move by u dt / 2 ~ 1e-3 and
// almost never leave the stage-1 lattice cell; a stage that does re-gathers.
// The group sums its partial velocities with two butterfly shuffles.  Stage 1
// locates the vertex in FP64 (positions ~100 lattice units); the later stages'
// fractions are the stage-1 fraction plus the move u h / dx in FP32 (one more
// FP32 rounding of a number below 1, where the FP64 position would round the
// same move to about 1e-14).
struct Plane16 {
    float u[16], v[16], w[16];
};

// xm: bit a = stencil column a is inside the reference lattice (x periodic:
// within the two BUFF columns of the vertex's raw frame, ibm.cu:453-455)
__device__ __forceinline__ void gather_plane(const Geom &g, const float4 *__restrict__ uvr, int ix0, int iy0, int iz,
                                             unsigned xm, Plane16 &P)
{
    const bool zin = iz >= -2 && iz < g.nzc + 2;   // beyond the BUFF planes (ibm.cu:453-455)
    const long long zb = (long long)wrap_z(iz, g.nzc) * g.plane;
#pragma unroll
    for (int b = 0; b < 4; b++) {
        const int gy = iy0 + b;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int gx = ix0 + a;
            float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
            const int gxw = g.xper ? wrap_x(gx, g.nx) : gx;
            if (zin && ((xm >> a) & 1u) && gy >= 0 && gy < g.ny && gxw >= 0 && gxw < g.nx)
                q = __ldg(&uvr[zb + gxw + (long long)g.nx * gy]);
            P.u[4 * b + a] = q.x; P.v[4 * b + a] = q.y; P.w[4 * b + a] = q.z;
        }
    }
}

__device__ __forceinline__ void lattice_cell(const Geom &g, double px, double py, double pz, int &ix0, int &iy0,
                                             int &iz0, float &fx, float &fy, float &fz)
{
    const double lx = lat_x(g, px), ly = lat_y(g, py), lz = lat_z(g, pz);
    const double flx = floor(lx), fly = floor(ly), flz = floor(lz);
    ix0 = (int)flx - 1; iy0 = (int)fly - 1; iz0 = (int)flz - 1;
    fx = (float)(lx - flx); fy = (float)(ly - fly); fz = (float)(lz - flz);
}

__device__ __forceinline__ void contract(const Plane16 &P, const float wx[4], const float wy[4], float wzc,
                                         float &ur, float &vr, float &wr)
{
    float su = 0.f, sv = 0.f, sw = 0.f;
#pragma unroll
    for (int b = 0; b < 4; b++) {
        const float wyz = wy[b] * wzc;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const float w = wx[a] * wyz;
            su += w * P.u[4 * b + a]; sv += w * P.v[4 * b + a]; sw += w * P.w[4 * b + a];
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
constexpr int ADVECT_MAX_PATCH = MAX_PATCH_VERTICES;
constexpr int ADVECT_BOX_BYTES = 48 * 1024;
constexpr int ADVECT_BOX_CAP = ADVECT_BOX_BYTES / (int)sizeof(float4);
constexpr int ADVECT_SMEM = ADVECT_BOX_BYTES + ADVECT_MAX_PATCH * (3 * (int)sizeof(double) + (int)sizeof(int));

// Stage-1 stencil plane of one lane from the patch's shared-memory box; false
// when the plane is not inside the box (the caller then gathers from global
// memory).  (xi, yi, zi) = stencil corner relative to the box origin.
__device__ __forceinline__ bool box_plane(const float4 *box, int bxs, int bys, int bzs, int bps, int xi, int yi,
                                          int zi, bool zin, unsigned xm, Plane16 &P)
{
    if (xi < 0 || xi + 3 >= bxs || yi < 0 || yi + 3 >= bys || zi < 0 || zi >= bzs) return false;
    const float4 *row = box + zi * bps + yi * bxs + xi;
#pragma unroll
    for (int b = 0; b < 4; b++)
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const float4 q = (zin && ((xm >> a) & 1u)) ? row[b * bxs + a] : make_float4(0.f, 0.f, 0.f, 0.f);
            P.u[4 * b + a] = q.x; P.v[4 * b + a] = q.y; P.w[4 * b + a] = q.z;
        }
    return true;
}

// One CTA per (cell, surface patch), as for the spread.  The CTA loads the
// lattice box of its patch's stage-1 stencils, widened by one node on every
// side for the later RK stages, into shared memory with coalesced row reads,
// so a stencil gather is 16 shared-memory reads instead of 16 scattered L1/L2
// reads.  Box nodes outside the lattice in x or y hold 0 (the reference reads
// nothing there); z wraps periodically, and nodes beyond the two BUFF planes
// of the vertex's own (unwrapped) frame are dropped per vertex as
// ibm.cu:453-455 does.  A box larger than ADVECT_SMEM, or a later-stage
// stencil outside the box, gathers from global memory instead.
// bid: the block's (cell, patch) index, blockIdx.x of a one-lattice launch.
// RK: RUNGE_KUTTA, the stages of ibm.cu:430-517 (4), 518-574 (2) or 575-617 (1).
template <bool XPER, int RK>
__device__ __forceinline__ void
advect_body(const Geom &g, double *__restrict__ X, double *__restrict__ Xd, float *__restrict__ U,
            const float4 *__restrict__ uvr, long long nv, int V, const int *__restrict__ patch_off,
            const int *__restrict__ patch_vtx, int npatch, double dtM, int *__restrict__ flags, int bid)
{
    extern __shared__ float4 abox[];   // [ADVECT_BOX_CAP] box, then the patch's positions and vertex ids
    double *spos = reinterpret_cast<double *>(abox + ADVECT_BOX_CAP);   // [3][ADVECT_MAX_PATCH]
    int *svid = reinterpret_cast<int *>(spos + 3 * ADVECT_MAX_PATCH);    // [ADVECT_MAX_PATCH]
    __shared__ int s_lo[3], s_hi[3];
    const int cell = bid / npatch, patch = bid - cell * npatch, tid = threadIdx.x;
    const int p0 = patch_off[patch], np = patch_off[patch + 1] - p0;
    const long long vb = (long long)cell * V;
    const double *xs = X + vb, *ys = X + nv + vb, *zs = X + 2 * nv + vb;
    const double az = lat_z(g, zs[0]);   // one anchor per cell: every patch unwraps z the same way
    const double ax = lat_x(g, xs[0]);   // and x, when x is periodic (shear mode)

    if (tid < 3) { s_lo[tid] = INT_MAX; s_hi[tid] = INT_MIN; }
    __syncthreads();
    int lo0 = INT_MAX, lo1 = INT_MAX, lo2 = INT_MAX, hi0 = INT_MIN, hi1 = INT_MIN, hi2 = INT_MIN;
    bool bad = false;
    for (int k = tid; k < np; k += ADVECT_THREADS) {
        const int v = patch_vtx[p0 + k];
        const double px = xs[v], py = ys[v], pz = zs[v];
        svid[k] = v; spos[k] = px; spos[ADVECT_MAX_PATCH + k] = py; spos[2 * ADVECT_MAX_PATCH + k] = pz;
        const double lxr = lat_x(g, px), lxv = XPER ? unwrap_near(lxr, ax, g.nx) : lxr;
        const double lyv = lat_y(g, py), lzv = unwrap_near(lat_z(g, pz), az, g.nzc);
        if (!(sane_lattice(lxv) && sane_lattice(lyv) && sane_lattice(lzv) && sane_lattice(az) && sane_lattice(ax))) { bad = true; continue; }
        const int ix = (int)floor(lxv), iy = (int)floor(lyv);
        const int iz = (int)floor(lzv);
        lo0 = min(lo0, ix - 2); hi0 = max(hi0, ix + 3);
        lo1 = min(lo1, iy - 2); hi1 = max(hi1, iy + 3);
        lo2 = min(lo2, iz - 2); hi2 = max(hi2, iz + 3);
    }
    atomicMin(&s_lo[0], lo0); atomicMin(&s_lo[1], lo1); atomicMin(&s_lo[2], lo2);
    atomicMax(&s_hi[0], hi0); atomicMax(&s_hi[1], hi1); atomicMax(&s_hi[2], hi2);
    if (__syncthreads_or(bad)) {   // a blown-up patch: flag it, leave its vertices as they are
        if (tid == 0) atomicOr(flags, RBC_FLAG_NONFINITE);
        return;
    }
    const int bx0 = s_lo[0], by0 = s_lo[1], bz0 = s_lo[2];
    const long long bxl = (long long)s_hi[0] - bx0 + 1, byl = (long long)s_hi[1] - by0 + 1, bzl = (long long)s_hi[2] - bz0 + 1;
    // plane stride bps = bxs * bys rounded up to odd: the four planes of a vertex's stencil, read
    // by four lanes of one quarter-warp, then fall in four different 16-byte bank groups
    const long long bpl = (bxl * byl) | 1;
    const bool use_box = np > 0 && bxl >= 6 && byl >= 6 && bzl >= 6 && bpl * bzl <= ADVECT_BOX_CAP;
    const int bxs = use_box ? (int)bxl : 0, bys = use_box ? (int)byl : 0, bzs = use_box ? (int)bzl : 0;
    const int bps = use_box ? (int)bpl : 0;
    if (use_box) {
        // node li = (z * bys + y) * bxs + x, stored at z * bps + y * bxs + x; each thread steps li
        // by ADVECT_THREADS
        const int nb = bxs * bys * bzs;
        int x = tid % bxs, y = (tid / bxs) % bys, z = tid / (bxs * bys);
        const int sx = ADVECT_THREADS % bxs, sy = (ADVECT_THREADS / bxs) % bys, sz = ADVECT_THREADS / (bxs * bys);
        // eight nodes per thread and round, their loads issued before any store: a mean box of
        // ~2000 nodes is one round, one wait on the L2 instead of two
        constexpr int UF = 8;
        for (int li = tid; li < nb; li += UF * ADVECT_THREADS) {
            float4 q[UF];
            int si[UF];
#pragma unroll
            for (int u = 0; u < UF; u++) {
                si[u] = z * bps + y * bxs + x;
                const int gx = XPER ? wrap_x(bx0 + x, g.nx) : bx0 + x, gy = by0 + y;
                // the box spans less than a period: one correction, the modulo only as a fallback
                int gz = bz0 + z;
                if (gz < 0) gz += g.nzc;
                if (gz >= g.nzc) gz -= g.nzc;
                if ((unsigned)gz >= (unsigned)g.nzc) gz = wrap_z(gz, g.nzc);
                q[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (li + u * ADVECT_THREADS < nb && gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny)
                    q[u] = __ldg(&uvr[(long long)gz * g.plane + gx + (long long)g.nx * gy]);
                x += sx; y += sy; z += sz;
                if (x >= bxs) { x -= bxs; y++; }
                if (y >= bys) { y -= bys; z++; }
            }
#pragma unroll
            for (int u = 0; u < UF; u++)
                if (li + u * ADVECT_THREADS < nb) abox[si[u]] = q[u];
        }
    }
    __syncthreads();

    // four lanes per vertex (lane c owns stencil plane c), 64 vertices per pass;
    // every lane of a warp runs the same passes (shuffles), idle lanes shadow vertex 0
    const int c = tid & 3;
    const int npass = (np + ADVECT_THREADS / 4 - 1) / (ADVECT_THREADS / 4);
    for (int pass = 0; pass < npass; pass++) {
        const int j = pass * (ADVECT_THREADS / 4) + (tid >> 2);
        const bool live = j < np;
        const int jj = live ? j : 0;
        const long long vj = vb + svid[jj];
        const double xn = spos[jj], yn = spos[ADVECT_MAX_PATCH + jj], zn = spos[2 * ADVECT_MAX_PATCH + jj];
        Plane16 P;
        int bx, by, bz;
        float fx, fy, fz, wx[4], wy[4], wz[4];
        lattice_cell(g, xn, yn, zn, bx, by, bz, fx, fy, fz);
        // shift from the raw z (and, periodic, x) frame to the cell's unwrapped frame
        const double lzr = lat_z(g, zn);
        const int zsh = (int)lrint(unwrap_near(lzr, az, g.nzc) - lzr);
        const double lxr = lat_x(g, xn);
        const int xsh = XPER ? (int)lrint(unwrap_near(lxr, ax, g.nx) - lxr) : 0;
        auto fetch = [&](int cx, int cy, int cz) {
            const int izr = cz + c;
            const bool zin = izr >= -2 && izr < g.nzc + 2;   // beyond the BUFF planes (ibm.cu:453-455)
            unsigned xm = 0xFu;
            if (XPER) {   // the same rule for the x BUFF columns (cx: raw frame)
                xm = 0u;
#pragma unroll
                for (int a = 0; a < 4; a++) xm |= (cx + a >= -g.xb && cx + a < g.nx + g.xb) ? (1u << a) : 0u;
            }
            if (!use_box || !box_plane(abox, bxs, bys, bzs, bps, cx + xsh - bx0, cy - by0, izr + zsh - bz0, zin, xm, P))
                gather_plane(g, uvr, cx, cy, izr, xm, P);
        };
        fetch(bx, by, bz);
        // the later stages' lattice positions relative to the stage-1 cell, in FP32:
        // x_k = x_n + u_{k-1} h moves the vertex by u h / dx lattice units (~1e-2)
        const int bx1 = bx, by1 = by, bz1 = bz;
        const float f1x = fx, f1y = fy, f1z = fz;
        float us[RK], vs[RK], ws[RK];
#pragma unroll
        for (int k = 0; k < RK; k++) {
            if (k > 0) {
                // RK4: x + u1 M dt / 2, x + u2 M dt / 2, x + u3 M dt (ibm.cu:487-505);
                // RK2: x + u1 M (ibm.cu:560-562; dt = 1 there)
                const float hs = (float)((RK == 4 && k < 3 ? 0.5 : 1.0) * dtM * g.inv_dx);
                const float gxs = fmaf(us[k - 1], hs, f1x), gys = fmaf(vs[k - 1], hs, f1y), gzs = fmaf(ws[k - 1], hs, f1z);
                const float sx = floorf(gxs), sy = floorf(gys), sz = floorf(gzs);
                fx = gxs - sx; fy = gys - sy; fz = gzs - sz;
                const int cx = bx1 + (int)sx, cy = by1 + (int)sy, cz = bz1 + (int)sz;
                if (cx != bx || cy != by || cz != bz) {   // uniform across the 4 lanes of the vertex
                    bx = cx; by = cy; bz = cz;
                    fetch(bx, by, bz);
                }
            }
            delta4(fx, wx); delta4(fy, wy); delta4(fz, wz);
            const float wzc = c == 0 ? wz[0] : c == 1 ? wz[1] : c == 2 ? wz[2] : wz[3];
            contract(P, wx, wy, wzc, us[k], vs[k], ws[k]);
        }
        if (!live || c != 0) continue;
        double um, vm, wm;
        if constexpr (RK == 4) {
            um = ((double)us[0] + 2.0 * us[1] + 2.0 * us[2] + us[3]) / 6.0;
            vm = ((double)vs[0] + 2.0 * vs[1] + 2.0 * vs[2] + vs[3]) / 6.0;
            wm = ((double)ws[0] + 2.0 * ws[1] + 2.0 * ws[2] + ws[3]) / 6.0;
        } else if constexpr (RK == 2) {   // ibm.cu:570-572
            um = ((double)us[0] + (double)us[1]) / 2.0;
            vm = ((double)vs[0] + (double)vs[1]) / 2.0;
            wm = ((double)ws[0] + (double)ws[1]) / 2.0;
        } else {                          // ibm.cu:614-616
            um = us[0]; vm = vs[0]; wm = ws[0];
        }
        double xr = xn + um * dtM, yr = yn + vm * dtM, zr = zn + wm * dtM;
        if (xr < g.xmin) xr += g.LX;   // ibm.cu:629-632
        if (xr > g.xmax) xr -= g.LX;
        if (zr < g.zmin) zr += g.LZ;
        if (zr > g.zmax) zr -= g.LZ;
        if (!isfinite(xr) || !isfinite(yr) || !isfinite(zr)) atomicOr(flags, RBC_FLAG_NONFINITE);
        X[vj] = xr; X[nv + vj] = yr; X[2 * nv + vj] = zr;
        Xd[vj] = xr; Xd[nv + vj] = yr; Xd[2 * nv + vj] = zr;
        U[vj] = (float)um; U[nv + vj] = (float)vm; U[2 * nv + vj] = (float)wm;
    }
}

template <bool XPER, int RK>
__global__ void __launch_bounds__(ADVECT_THREADS)
advect_kernel(const Geom g, double *__restrict__ X, double *__restrict__ Xd, float *__restrict__ U,
              const float4 *__restrict__ uvr, long long nv, int V, const int *__restrict__ patch_off,
              const int *__restrict__ patch_vtx, int npatch, double dtM, int *__restrict__ flags)
{
    pdl_start();
    advect_body<XPER, RK>(g, X, Xd, U, uvr, nv, V, patch_off, patch_vtx, npatch, dtM, flags, blockIdx.x);
}

cudaError_t advect_setup()
{
    const void *ks[] = {(const void *)advect_kernel<false, 4>, (const void *)advect_kernel<true, 4>,
                        (const void *)advect_kernel<false, 2>, (const void *)advect_kernel<true, 2>,
                        (const void *)advect_kernel<false, 1>, (const void *)advect_kernel<true, 1>};
    for (const void *k : ks) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, ADVECT_SMEM);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void launch_advect(const Geom &g, const AdvectArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    auto k = a.rk == 1 ? (g.xper ? advect_kernel<true, 1> : advect_kernel<false, 1>)
           : a.rk == 2 ? (g.xper ? advect_kernel<true, 2> : advect_kernel<false, 2>)
                       : (g.xper ? advect_kernel<true, 4> : advect_kernel<false, 4>);
    launch_pdl(k, dim3(a.ncell * a.npatch), dim3(ADVECT_THREADS), ADVECT_SMEM, s,
               g, a.X, a.Xd, a.U, a.uvr, a.nv, a.V, a.patch_off, a.patch_vtx, a.npatch, a.dtM, a.flags);
}

// ---- fused batches ---------------------------------------------------------

template <bool XPER>
__global__ void __launch_bounds__(SPREAD_THREADS)
spread_fused_kernel(const DomainArgs *__restrict__ dom, const int *__restrict__ boff, int ndom)
{
    const int d = fused_domain(boff, ndom, blockIdx.x);
    const DomainArgs &D = dom[d];
    const SpreadArgs &a = D.spread;
    spread_body<XPER>(D.g, a.X, a.nv, a.V, a.patch_off, a.patch_vtx, a.patch_stride, a.npatch, a.Fv, a.F, a.mask2d,
                      a.flags, blockIdx.x - boff[d]);
}

template <bool XPER>
__global__ void __launch_bounds__(ADVECT_THREADS)
advect_fused_kernel(const DomainArgs *__restrict__ dom, const int *__restrict__ boff, int ndom)
{
    const int d = fused_domain(boff, ndom, blockIdx.x);
    const DomainArgs &D = dom[d];
    const AdvectArgs &a = D.adv;
    advect_body<XPER, 4>(D.g, a.X, a.Xd, a.U, a.uvr, a.nv, a.V, a.patch_off, a.patch_vtx, a.npatch, a.dtM, a.flags,
                      blockIdx.x - boff[d]);
}

cudaError_t ibm_fused_setup()
{
    const void *ks[] = {(const void *)spread_fused_kernel<false>, (const void *)spread_fused_kernel<true>};
    for (const void *k : ks) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SPREAD_SMEM);
        if (e != cudaSuccess) return e;
    }
    const void *ka[] = {(const void *)advect_fused_kernel<false>, (const void *)advect_fused_kernel<true>};
    for (const void *k : ka) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, ADVECT_SMEM);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void launch_spread_fused(const FusedLaunch &f, bool xper, cudaStream_t s)
{
    if (f.nblocks <= 0) return;
    auto k = xper ? spread_fused_kernel<true> : spread_fused_kernel<false>;
    k<<<f.nblocks, SPREAD_THREADS, SPREAD_SMEM, s>>>(f.dom, f.boff, f.ndom);
}

void launch_advect_fused(const FusedLaunch &f, bool xper, cudaStream_t s)
{
    if (f.nblocks <= 0) return;
    auto k = xper ? advect_fused_kernel<true> : advect_fused_kernel<false>;
    k<<<f.nblocks, ADVECT_THREADS, ADVECT_SMEM, s>>>(f.dom, f.boff, f.ndom);
}

}  // namespace rbc
