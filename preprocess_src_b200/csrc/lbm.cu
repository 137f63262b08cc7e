// lbm.cu -- fused D3Q19 BGK collide-stream with Guo forcing, pull scheme.
//
// Replaces lbm_CapsuleCHANNELFLOW + lbm_CHANNELFLOW_Boundary + lbm_AVERAGE
// (lbm.cu:983-1313, 1378-1460 of the reference).  The reference pushes
// post-collision populations to the neighbours (scattered stores into AoS
// fn[i*19+q]); here each node pulls the post-collision populations of the
// previous step from its upstream neighbours (coalesced SoA loads), collides and
// stores its own post-collision populations.  Both orders produce the same
// pre-collision field; the half-way bounce-back of the push form
// (fm[i][opp q] = f*_q(i) when i + e_q is a wall) becomes, in pull form,
// f_q(i) = f*_{opp q}(i) when i - e_q is a wall.  The BUFF planes of the
// reference are replaced by a periodic z index.
//
// Populations are stored as g = f - w (FP32) or (f - w) * scale (FP16), which
// keeps their rounding error relative to the deviation from rest rather than to
// w itself.  Arithmetic is FP32.
#include "rbc_internal.cuh"

namespace rbc {

template <int STORE> struct Store;
template <> struct Store<RBC_STORE_F32> {
    using T = float;
    static constexpr float scale = 1.0f;
    static __device__ __forceinline__ float ld(const T *p, float) { return __ldg(p); }
    static __device__ __forceinline__ void st(T *p, float v, float) { __stcs(p, v); }
    // the collision kernel's loads and stores in storage units (= physical here)
    static __device__ __forceinline__ float ld_raw(const T *p) { return __ldg(p); }
    static __device__ __forceinline__ void st_raw(T *p, float v) { __stcs(p, v); }
};
template <> struct Store<RBC_STORE_F16> {
    using T = __half;
    static constexpr float scale = F16_SCALE;
    static __device__ __forceinline__ float ld(const T *p, float inv_scale) { return __half2float(__ldg(p)) * inv_scale; }
    static __device__ __forceinline__ void st(T *p, float v, float scale) { __stcs(reinterpret_cast<unsigned short *>(p), __half_as_ushort(__float2half_rn(v * scale))); }
    // storage units (f - w) * scale: the collision kernel applies the scale to
    // its per-node moments and coefficients instead of to each population
    static __device__ __forceinline__ float ld_raw(const T *p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ void st_raw(T *p, float v) { __stcs(reinterpret_cast<unsigned short *>(p), __half_as_ushort(__float2half_rn(v))); }
};

constexpr int LBM_THREADS = 256;

// BGK + Guo forcing (lbm.cu:1129-1213 of the reference).  With G the half
// force rho (P drive z^ + B F) (lbm.cu:1116-1118), u = (j + G) / (rho Cr) and
//   f_eq,q = w_q [drho + rho (3 Cr e.u + 4.5 Cr^2 (e.u)^2 - 1.5 Cr^2 u.u)]
//   F_q    = (1 - om/2) 2 w_q [3 e.G - 3 Cr u.G + 9 Cr (e.u)(e.G)]
// the post-collision value (1 - om) g_q + om f_eq,q + F_q is evaluated as
//   (1 - om) g_q + w_q (A + e.u (B + C e.u + E e.G) + D e.G)
// with per-node scalars A..E.  With scaled storage (g in units of 1/SCALE, a
// power of two) the moments are divided and A..E multiplied by SCALE once per
// node, so the populations are used as stored: 5 multiplies per node instead
// of 38 (each population scaled on its load and its store).
struct Collision {
    float u, v, w, r;
    float Gx, Gy, Gz;
    float A, B, C, D, E;
};

// Every product-sum below is an explicit __fmaf_rn / __fmul_rn / __fadd_rn, so
// no step is left to the compiler's contraction: the kernels that inline this
// code (one simulation, the fused batch, each with the om = 1 and general
// forms) round every node the same way, bit for bit.
template <int SCALE>
__device__ __forceinline__ Collision collision_terms(const float (&g)[Q], float fx, float fy, float fz, float pd,
                                                     float omega, float Cr, float Bc)
{
    constexpr float scale = (float)SCALE, inv_scale = 1.0f / (float)SCALE;
    float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        drho += g[q];
        if (ex(q) == 1) jx += g[q]; else if (ex(q) == -1) jx -= g[q];
        if (ey(q) == 1) jy += g[q]; else if (ey(q) == -1) jy -= g[q];
        if (ez(q) == 1) jz += g[q]; else if (ez(q) == -1) jz -= g[q];
    }
    if (SCALE != 1) { drho *= inv_scale; jx *= inv_scale; jy *= inv_scale; jz *= inv_scale; }
    Collision c;
    c.r = 1.0f + drho;
    const float rB = __fmul_rn(c.r, Bc);
    c.Gx = __fmul_rn(rB, fx); c.Gy = __fmul_rn(rB, fy); c.Gz = __fmul_rn(c.r, __fmaf_rn(Bc, fz, pd));
    const float inv = 1.0f / __fmul_rn(c.r, Cr);
    c.u = __fmul_rn(__fadd_rn(jx, c.Gx), inv); c.v = __fmul_rn(__fadd_rn(jy, c.Gy), inv);
    c.w = __fmul_rn(__fadd_rn(jz, c.Gz), inv);
    const float fo = __fmul_rn(__fmaf_rn(-0.5f, omega, 1.0f), 2.0f);
    const float uu = __fmaf_rn(c.w, c.w, __fmaf_rn(c.v, c.v, __fmul_rn(c.u, c.u)));
    const float usq = __fmul_rn(-1.5f * Cr * Cr, uu);
    const float uG = __fmul_rn(3.0f * Cr, __fmaf_rn(c.w, c.Gz, __fmaf_rn(c.v, c.Gy, __fmul_rn(c.u, c.Gx))));
    c.A = __fmaf_rn(-fo, uG, __fmul_rn(omega, __fmaf_rn(c.r, usq, drho)));
    c.B = __fmul_rn(3.0f * Cr * omega, c.r);
    c.C = __fmul_rn(4.5f * Cr * Cr * omega, c.r);
    c.D = __fmul_rn(3.0f, fo);
    c.E = __fmul_rn(9.0f * Cr, fo);
    if (SCALE != 1) { c.A *= scale; c.B *= scale; c.C *= scale; c.D *= scale; c.E *= scale; }
    return c;
}

// e_q . (x, y, z) for the lattice directions (components 0 or +-1): additions only
__device__ __forceinline__ float edot(int q, float x, float y, float z)
{
    float d = 0.f;
    if (ex(q) == 1) d = x; else if (ex(q) == -1) d = -x;
    if (ey(q) == 1) d = __fadd_rn(d, y); else if (ey(q) == -1) d = __fsub_rn(d, y);
    if (ez(q) == 1) d = __fadd_rn(d, z); else if (ez(q) == -1) d = __fsub_rn(d, z);
    return d;
}

// The post-collision values of an opposite pair (q, q + 1 = opp(q)): with
// e_{q+1} = -e_q the polynomial splits into its even and odd parts,
//   S = w_q (A + eu (C eu + E eG)),   T = w_q (B eu + D eG),
//   f*_q = (1 - om) g_q + S + T,   f*_{q+1} = (1 - om) g_{q+1} + S - T,
// so it is evaluated once per pair.  TAU1 (om = 1, tau = 1 as in every named
// workload): (1 - om) g = 0 exactly, and the pulled values enter only through
// the moments (the same results as the general form with om1 = 0).
template <bool TAU1>
__device__ __forceinline__ void post_pair(const Collision &c, int q, float gq, float gp, float om1, float &oq,
                                          float &op)
{
    const float eu = edot(q, c.u, c.v, c.w);
    const float eG = edot(q, c.Gx, c.Gy, c.Gz);
    const float w = wq(q);
    const float S = __fmul_rn(w, __fmaf_rn(eu, __fmaf_rn(c.C, eu, __fmul_rn(c.E, eG)), c.A));
    const float T = __fmul_rn(w, __fmaf_rn(c.B, eu, __fmul_rn(c.D, eG)));
    const float sp = __fadd_rn(S, T), sm = __fsub_rn(S, T);
    oq = TAU1 ? sp : __fmaf_rn(om1, gq, sp);
    op = TAU1 ? sm : __fmaf_rn(om1, gp, sm);
}

template <bool TAU1>
__device__ __forceinline__ float post_rest(const Collision &c, float g0, float om1)
{
    const float a = __fmul_rn(wq(0), c.A);
    return TAU1 ? a : __fmaf_rn(om1, g0, a);
}

// FP16 storage rounds stochastically (cvt.rs.f16x2.f32, sm_100a): each stored
// value goes to one of its two FP16 neighbours with probability proportional to
// its closeness, so the storage error has zero mean instead of being a fixed
// function of the value.  A steady flow stores nearly the same values step
// after step; rounded to nearest, their errors repeat and add up in the flow,
// while stochastic errors average out (M. Croci et al., "Stochastic rounding:
// implementation, error analysis and applications", R. Soc. Open Sci. 9, 2022).
// cvt.rs takes 13 random bits per value: rbits[12:0] for the low half (the
// value in the second operand), rbits[28:16] for the high half.  The bits come
// from a hash of the node index and the step counter, so runs are repeatable:
// one 32-bit hash per node (the murmur3 finaliser), then per pair of
// populations a 32 x 32 -> 64-bit product with an odd constant, whose high word
// supplies the low field and whose low word the high field (the well-mixed
// bits of each word).
__device__ __forceinline__ uint32_t node_hash(uint32_t idx, uint32_t step) {
    uint32_t h = idx * 0x9E3779B1u ^ step * 0x85EBCA77u;
    h ^= h >> 16; h *= 0x85EBCA6Bu;
    h ^= h >> 13; h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}
__device__ __forceinline__ uint32_t pair_bits(uint32_t h, uint32_t mult) {
    const unsigned long long p = (unsigned long long)h * mult;
    return ((uint32_t)(p >> 32) & 0x0000FFFFu) | ((uint32_t)p & 0xFFFF0000u);
}
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float hi, float lo, uint32_t rbits) {
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}
__device__ __forceinline__ void st_u16(__half *p, uint32_t v) {
    __stcs(reinterpret_cast<unsigned short *>(p), (unsigned short)v);
}

// Collision of one node from its pulled populations g (storage units) and
// stores of the post-collision values (0 for wall lanes) at element offset idx of every
// population array; I is the offset type (int when Q * nint < 2^31).  has_force:
// the node's occupancy bit (F holds its IB force; read only here).
// SUB: the rho / u store follows acc (LBM_ACC_*, sub-cycling) instead of
// overwriting.
template <int STORE, bool ALL_FLUID, bool TAU1, bool SUB, typename I>
__device__ __forceinline__ void collide_store(float (&g)[Q], bool fluid, bool has_force, I idx, I nint,
                                              typename Store<STORE>::T *__restrict__ gout, float4 *__restrict__ uvr,
                                              const long long *__restrict__ F, uint32_t step,
                                              float pd, float omega, float om1, float Cr, float Bc, int acc, float Mf)
{
    using S = Store<STORE>;
    const bool live = ALL_FLUID || fluid;
    float fx = 0.f, fy = 0.f, fz = 0.f;
    if (live && has_force) {
        constexpr float inv = 1.0f / (float)(1ULL << FORCE_FRAC);
        fx = (float)__ldg(&F[idx]) * inv; fy = (float)__ldg(&F[nint + idx]) * inv;
        fz = (float)__ldg(&F[2 * nint + idx]) * inv;
    }
    const Collision c = collision_terms<(int)S::scale>(g, fx, fy, fz, pd, omega, Cr, Bc);
    float4 m = live ? make_float4(c.u, c.v, c.w, c.r) : make_float4(0.f, 0.f, 0.f, 1.f);
    if (SUB && live && acc != LBM_ACC_WRITE) {
        // um += tu (lbm.cu:1122-1126), then um /= M at the last step (lbm.cu:1455-1457);
        // the density sum dm is not averaged
        const float4 o = uvr[idx];
        m.x += o.x; m.y += o.y; m.z += o.z; m.w += o.w;
        if (acc == LBM_ACC_AVERAGE) { m.x = __fdiv_rn(m.x, Mf); m.y = __fdiv_rn(m.y, Mf); m.z = __fdiv_rn(m.z, Mf); }
    }
    uvr[idx] = m;
    typename S::T *ob = gout + idx;
    if constexpr (STORE == RBC_STORE_F16) {
        const uint32_t h = node_hash((uint32_t)idx, step);
        // slot 0 alone, then the opposite pairs (1, 2), (3, 4), ..., (17, 18)
        const uint32_t d0 = cvt_rs_f16x2(0.f, live ? post_rest<TAU1>(c, g[0], om1) : 0.f, pair_bits(h, 0x2545F491u));
        st_u16(ob, d0);
#pragma unroll
        for (int q = 1; q < Q; q += 2) {
            float lo, hi;
            post_pair<TAU1>(c, q, g[q], g[q + 1], om1, lo, hi);
            if (!live) { lo = 0.f; hi = 0.f; }
            const uint32_t d = cvt_rs_f16x2(hi, lo, pair_bits(h, 0x9E3779B1u + 0x3C6EF372u * (uint32_t)q));
            st_u16(ob + (I)q * nint, d);
            st_u16(ob + (I)(q + 1) * nint, d >> 16);
        }
    } else {
        S::st_raw(ob, live ? post_rest<TAU1>(c, g[0], om1) : 0.f);
#pragma unroll
        for (int q = 1; q < Q; q += 2) {
            float a, b;
            post_pair<TAU1>(c, q, g[q], g[q + 1], om1, a, b);
            S::st_raw(ob + (I)q * nint, live ? a : 0.f);
            S::st_raw(ob + (I)(q + 1) * nint, live ? b : 0.f);
        }
    }
}

// One thread per (x, y) column and a few planes: blockIdx.x * blockDim.x +
// threadIdx.x indexes the node in its (x, y) plane, blockIdx.y + k gridDim.y
// the planes z.  Per
// fluid node: 19 pulled loads, 12 B of IB force, 19 stores, 16 B of rho/u.
//
// Full-sector stores: a warp that holds any fluid node stores all 32 of its
// nodes in the same store instructions, its wall nodes writing 0 (their
// populations are never read) and rho 1, u 0 (what the interpolation reads at
// walls).  Leaving the wall columns of a row unwritten would leave the first
// and last 32-byte sectors of the row partly written, which the L2 completes
// with a DRAM read before writing them back.
//
// A warp none of whose nodes has a wall link takes a path without the
// bounce-back selects: such a warp holds only fluid nodes, because a wall node
// next (in x) to a fluid node gives that node a wall link, and the first and
// last node of every row are walls.
#ifndef LBM_MIN_BLOCKS
#define LBM_MIN_BLOCKS 4   // resident CTAs per SM the register allocation must allow
#endif
// VISC: omega of each node from the volume fraction, 1 / (df3 (1 + lm1 vf) + 1/2)
// (lbm.cu:1131 with LAMBDA1 != 1); the omega argument otherwise.
// (bx, by, gy): the block's column tile, its first plane and the plane stride
// (blockIdx.x, blockIdx.y, gridDim.y of a one-lattice launch).
template <int STORE, typename I, bool VISC, bool TAU1, bool SUB = false>
__device__ __forceinline__ void
lbm_collide_stream_body(const typename Store<STORE>::T *__restrict__ gin, typename Store<STORE>::T *__restrict__ gout,
                        float4 *__restrict__ uvr,
                        const long long *__restrict__ F, const uint32_t *__restrict__ Fbits, int wpp,
                        const uint32_t *__restrict__ mask2d, const float *__restrict__ drive,
                        const int *__restrict__ iter,
                        const float *__restrict__ wall, const double *__restrict__ vf, float lm1, float df3,
                        int nx, int ny, int nzc, I nint,
                        float omega, float Cr, float Bc, int bx, int by, int gy, int acc = 0, float Mf = 1.f)
{
    using S = Store<STORE>;
    const int plane = nx * ny;
    const int xy = bx * blockDim.x + threadIdx.x;
    if (xy >= plane) return;
    const uint32_t m = __ldg(&mask2d[xy]);
    const bool fluid = (m & MASK_FLUID) != 0;
    const unsigned act = __activemask();
    if (!__any_sync(act, fluid)) return;   // a warp of wall nodes stores nothing
    const bool warp_links = __any_sync(act, (m & ~MASK_FLUID) != 0u);
    const float pd = __ldg(drive);
    const uint32_t step = (STORE == RBC_STORE_F16) ? (uint32_t)__ldg(iter) : 0u;
    float om1 = 1.0f - omega;
    // a warp's 32 nodes of a plane are the 32 bits of one occupancy word
    // (blockDim.x is a multiple of 32), read by every lane (one address); the
    // reset before the next step's spread clears them
    const int lane = threadIdx.x & 31;
    const int fword = xy >> 5;
    for (int z = by; z < nzc; z += gy) {
        const uint32_t fw = __ldg(Fbits + ((long long)z * wpp + fword));
        const bool has_force = (fw >> lane) & 1u;
        // offsets of the source planes z - 1 and z + 1 from plane z (periodic);
        // with them every pull offset from the node is uniform over the block
        const I dzm = (z == 0) ? (I)(nzc - 1) * plane : -(I)plane;
        const I dzp = (z == nzc - 1) ? -(I)(nzc - 1) * plane : (I)plane;
        const I idx = (I)z * plane + xy;
        if (VISC) {
            omega = 1.0f / __fmaf_rn(df3, __fmaf_rn(lm1, (float)__ldg(&vf[idx]), 1.0f), 0.5f);
            om1 = 1.0f - omega;
        }
        const typename S::T *gb = gin + idx;
        float g[Q];
        if (!warp_links) {
#pragma unroll
            for (int q = 0; q < Q; q++)
                g[q] = S::ld_raw(gb + ((I)q * nint + ((ez(q) == 1) ? dzm : (ez(q) == -1) ? dzp : (I)0) - ex(q) - nx * ey(q)));
            collide_store<STORE, true, TAU1, SUB, I>(g, true, has_force, idx, nint, gout, uvr, F, step, pd, omega, om1,
                                                     Cr, Bc, acc, Mf);
        } else {
#pragma unroll
            for (int q = 0; q < Q; q++) {
                // a periodic x (shear mode) wraps the pull of the first and last column
                const I xw = (ex(q) == 1 && (m & MASK_XLO)) ? (I)nx : (ex(q) == -1 && (m & MASK_XHI)) ? -(I)nx : (I)0;
                const I pull = (I)q * nint + ((ez(q) == 1) ? dzm : (ez(q) == -1) ? dzp : (I)0) - ex(q) - nx * ey(q) + xw;
                const bool bb = (m >> q) & 1u;   // i - e_q is a wall: half-way bounce-back of f*_{opp q}(i)
                g[q] = fluid ? S::ld_raw(gb + (bb ? (I)opp(q) * nint : pull)) : 0.f;
            }
            if (fluid && (m & (MASK_TOPW | MASK_BOTW))) {
                // moving wall (shear mode, lbm.cu:946-964): the bounced population gains
                // 6 w_q rho Cr (e_q . u_w), rho = the node's density of the previous collision
                // = 1 + the sum of its own post-collision slots (the collision conserves it)
                float rs = S::scale;
#pragma unroll
                for (int q = 0; q < Q; q++) rs += S::ld_raw(gb + (I)q * nint);
                const float rho = rs * (1.0f / S::scale);
                const float uw = __ldg(&wall[(m & MASK_TOPW) ? 0 : 1]);
#pragma unroll
                for (int q = 0; q < Q; q++)
                    if (ez(q) != 0 && ((m >> q) & 1u)) {
                        const float t = __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(6.0f * wq(q), rho), Cr) * (float)ez(q), uw),
                                                  S::scale);
                        g[q] = __fadd_rn(g[q], t);
                    }
            }
            collide_store<STORE, false, TAU1, SUB, I>(g, fluid, has_force, idx, nint, gout, uvr, F, step, pd, omega,
                                                      om1, Cr, Bc, acc, Mf);
        }
    }
}

template <int STORE, typename I, bool VISC, bool TAU1, bool SUB>
__global__ void __launch_bounds__(LBM_THREADS, LBM_MIN_BLOCKS)
lbm_collide_stream(const typename Store<STORE>::T *__restrict__ gin, typename Store<STORE>::T *__restrict__ gout,
                   float4 *__restrict__ uvr,
                   const long long *__restrict__ F, const uint32_t *__restrict__ Fbits, int wpp,
                   const uint32_t *__restrict__ mask2d, const float *__restrict__ drive, const int *__restrict__ iter,
                   const float *__restrict__ wall, const double *__restrict__ vf, float lm1, float df3,
                   int nx, int ny, int nzc, I nint,
                   float omega, float Cr, float Bc, int acc, float Mf)
{
    pdl_start();
    lbm_collide_stream_body<STORE, I, VISC, TAU1, SUB>(gin, gout, uvr, F, Fbits, wpp, mask2d, drive, iter, wall, vf,
                                                       lm1, df3, nx, ny, nzc, nint, omega, Cr, Bc, blockIdx.x,
                                                       blockIdx.y, gridDim.y, acc, Mf);
}

// z planes per thread: the per-thread setup (mask, warp votes, drive) is paid
// once for that many nodes.  Dense suspension (256 planes of 128 x 128):
// FP32 0.1352 / 0.1312 / 0.1337 ms and FP16 0.1292 / 0.1209 / 0.1182 ms at
// 1 / 2 / 4 planes per thread.  A lattice that would leave fewer than
// LBM_MIN_THREADS threads (~3.5 waves of 148 SMs x 1024 resident threads) keeps
// fewer planes per thread: the single-cell duct (57,600 nodes) takes 0.0086 ms
// at one plane per thread and 0.0098 ms at two.
constexpr int LBM_PLANES_F32 = 2, LBM_PLANES_F16 = 4;
constexpr long long LBM_MIN_THREADS = 1LL << 19;

void launch_lbm(const Geom &g, int storage, const LbmArgs &a, cudaStream_t s)
{
    int zpt = (storage == RBC_STORE_F16) ? LBM_PLANES_F16 : LBM_PLANES_F32;
    while (zpt > 1 && (long long)g.plane * g.nzc / zpt < LBM_MIN_THREADS) zpt >>= 1;
    if (a.planes > 0) zpt = a.planes;   // a launch shape set through rbc_set_launch_shape
    const int gz = (g.nzc + zpt - 1) / zpt;
    const dim3 blocks((unsigned)((g.plane + LBM_THREADS - 1) / LBM_THREADS), (unsigned)(gz < 65535 ? gz : 65535));
    const bool off32 = (long long)Q * g.nint < (1LL << 31);   // every element offset fits in an int
#define LBM_LAUNCH(ST, I, V, T1, SB)                                                                          \
    launch_pdl(lbm_collide_stream<ST, I, V, T1, SB>, blocks, dim3(LBM_THREADS), 0, s,                            \
        (const Store<ST>::T *)a.gin, (Store<ST>::T *)a.gout, a.uvr, a.F.F, a.F.bits, a.F.wpp, a.mask2d, a.drive, a.iter, \
        a.wall, a.vf, \
        a.lm1, a.df3, g.nx, g.ny, g.nzc, (I)g.nint, a.omega, a.Cr, a.Bc, a.acc, a.Mf)
    // tau = 1 without a viscosity ratio: the om = 1 form of the collision.  The
    // sums of a sub-cycled step take the general form (with om = 1 it gives the
    // same values: (1 - om) g = 0 exactly); the volume fraction runs with M = 1.
    const bool tau1 = !a.vf && a.omega == 1.0f;
#define LBM_LAUNCH_V(ST, I)                                                                                   \
    do {                                                                                                      \
        if (a.vf) LBM_LAUNCH(ST, I, true, false, false);                                                      \
        else if (a.acc != LBM_ACC_WRITE) LBM_LAUNCH(ST, I, false, false, true);                               \
        else if (tau1) LBM_LAUNCH(ST, I, false, true, false);                                                 \
        else LBM_LAUNCH(ST, I, false, false, false);                                                          \
    } while (0)
    if (storage == RBC_STORE_F16) {
        if (off32) LBM_LAUNCH_V(RBC_STORE_F16, int); else LBM_LAUNCH_V(RBC_STORE_F16, long long);
    } else {
        if (off32) LBM_LAUNCH_V(RBC_STORE_F32, int); else LBM_LAUNCH_V(RBC_STORE_F32, long long);
    }
#undef LBM_LAUNCH_V
#undef LBM_LAUNCH
}

// Fused batches: the collide-stream of every domain in one launch of TPB
// threads per block; domain d's block b is its column tile b % lbm_bx and
// first plane b / lbm_bx, planes stepping by lbm_gy.
template <int STORE, typename I, int TPB>
__global__ void __launch_bounds__(TPB, (LBM_MIN_BLOCKS * LBM_THREADS) / TPB)
lbm_fused_kernel(const DomainArgs *__restrict__ dom, const int *__restrict__ boff, int ndom)
{
    using T = typename Store<STORE>::T;
    const int d = fused_domain(boff, ndom, blockIdx.x);
    const DomainArgs &D = dom[d];
    const LbmArgs &a = D.lbm;
    const int b = blockIdx.x - boff[d];
    if (a.omega == 1.0f)   // uniform over the block: the om = 1 form, as a one-simulation launch takes it
        lbm_collide_stream_body<STORE, I, false, true>((const T *)a.gin, (T *)a.gout, a.uvr, a.F.F, a.F.bits, a.F.wpp,
                                                       a.mask2d, a.drive, a.iter, a.wall, nullptr, 0.f, 0.f, D.g.nx,
                                                       D.g.ny, D.g.nzc, (I)D.g.nint, a.omega, a.Cr, a.Bc,
                                                       b % D.lbm_bx, b / D.lbm_bx, D.lbm_gy);
    else
        lbm_collide_stream_body<STORE, I, false, false>((const T *)a.gin, (T *)a.gout, a.uvr, a.F.F, a.F.bits,
                                                        a.F.wpp, a.mask2d, a.drive, a.iter, a.wall, nullptr, 0.f,
                                                        0.f, D.g.nx, D.g.ny, D.g.nzc, (I)D.g.nint, a.omega, a.Cr,
                                                        a.Bc, b % D.lbm_bx, b / D.lbm_bx, D.lbm_gy);
}

void launch_lbm_fused(const FusedLaunch &f, int storage, bool off32, int threads, cudaStream_t s)
{
    if (f.nblocks <= 0) return;
#define LBM_FUSED(ST, I, TPB) lbm_fused_kernel<ST, I, TPB><<<f.nblocks, TPB, 0, s>>>(f.dom, f.boff, f.ndom)
#define LBM_FUSED_T(ST, I) do { if (threads == 128) LBM_FUSED(ST, I, 128); else LBM_FUSED(ST, I, 256); } while (0)
    if (storage == RBC_STORE_F16) {
        if (off32) LBM_FUSED_T(RBC_STORE_F16, int); else LBM_FUSED_T(RBC_STORE_F16, long long);
    } else {
        if (off32) LBM_FUSED_T(RBC_STORE_F32, int); else LBM_FUSED_T(RBC_STORE_F32, long long);
    }
#undef LBM_FUSED_T
#undef LBM_FUSED
}

// one warp per 32 words (whole warps: every lane takes part in the ballot)
__global__ void force_reset_kernel(const ForceField F, long long nwords, long long plane, long long nint)
{
    pdl_start();
    const long long w0 = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32;
    if (w0 < nwords) force_reset_words(F.F, F.bits, w0, nwords, F.wpp, plane, nint, threadIdx.x & 31);
}

void launch_force_reset(const Geom &g, const ForceField &F, cudaStream_t s)
{
    const long long nw = (long long)g.nzc * F.wpp;
    launch_pdl(force_reset_kernel, dim3((unsigned)((nw + 255) / 256)), dim3(256), 0, s, F, nw, (long long)g.plane,
               (long long)g.nint);
}

// ---- circular tube: interpolated bounce-back ------------------------------

// lbm_BounceBack_GPU + BounceBackLinearInterpolation_DEV (lbm_cylinder.cu:61-87,
// 190-231) in pull form, after the collide-stream of a step: for a wall link of
// node i in pull direction p crossing the circle at fraction t, the slot the
// next pull bounces back from, f*_{opp p}(i) (read by no other node: its
// regular reader i - e_p is the wall), becomes
//   t < 1/2:  2t f1 + (1 - 2t) f2,    t >= 1/2:  f1 / 2t + (2t - 1) / 2t f3
// with f1 = f*_{opp p}(i) (half-way), f2 = f*_{opp p}(i + e_p) (what i pulls
// along opp p) and f3 = f*_p(i).  The weights sum to 1, so the same holds for
// g = f - w.  No listed link reads a slot another one writes (a slot is
// written only by its own node's link, and links with walls on both sides
// are not listed).  One thread per (link, plane).
template <int STORE>
__global__ void tube_bounce_kernel(const Geom g, typename Store<STORE>::T *__restrict__ gs,
                                   const int *__restrict__ links, const float *__restrict__ frac, int nlinks,
                                   float inv_scale, float scale)
{
    using S = Store<STORE>;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlinks) return;
    const int z = blockIdx.y;
    const int code = __ldg(&links[k]), xy = code >> 5, p = code & 31, o = opp(p);
    const float t = __ldg(&frac[k]);
    const long long zb = (long long)z * g.plane, i = zb + xy;
    const int zn = wrap_z(z + ez(p), g.nzc), dxy = ex(p) + g.nx * ey(p);   // node i + e_p
    typename S::T *slot = gs + (long long)o * g.nint + i;
    const float f1 = S::ld(slot, inv_scale);
    float f;
    if (t < 0.5f) {
        const float f2 = S::ld(gs + (long long)o * g.nint + (long long)zn * g.plane + xy + dxy, inv_scale);
        f = 2.0f * t * f1 + (1.0f - 2.0f * t) * f2;
    } else {
        const float f3 = S::ld(gs + (long long)p * g.nint + i, inv_scale);
        f = f1 / (2.0f * t) + (2.0f * t - 1.0f) / (2.0f * t) * f3;
    }
    S::st(slot, f, scale);
}

void launch_tube_bounce(const Geom &g, int storage, void *gout, const int *links, const float *frac, int nlinks,
                        float inv_scale, float scale, cudaStream_t s)
{
    if (nlinks <= 0) return;
    const dim3 grid((unsigned)((nlinks + 127) / 128), (unsigned)g.nzc);
    if (storage == RBC_STORE_F16)
        tube_bounce_kernel<RBC_STORE_F16><<<grid, 128, 0, s>>>(g, (__half *)gout, links, frac, nlinks, inv_scale, scale);
    else
        tube_bounce_kernel<RBC_STORE_F32><<<grid, 128, 0, s>>>(g, (float *)gout, links, frac, nlinks, inv_scale, scale);
}

// ---- reference layout <-> internal layout ---------------------------------

__device__ __forceinline__ int nb_x(const Geom &g, int x, int d) { return g.xper ? wrap_x(x + d, g.nx) : x + d; }

// The moving-wall term of a bounced population in direction q at a node of
// density rho (shear mode, lbm.cu:946-964): 6 w_q rho Cr (e_q . u_w), u_w along z.
__device__ __forceinline__ double wall_term(int q, uint32_t m, double rho, const WallVel &w) {
    const double uw = (m & MASK_TOPW) ? w.top : (m & MASK_BOTW) ? w.bot : 0.0;
    return 6.0 * wqd(q) * rho * w.Cr * (double)ez(q) * uw;
}

// Reference fn (pre-collision, AoS FP64) -> internal post-collision g*:
// f*_q(i) = fn[i + e_q][q] when i + e_q is fluid, else fn[i][opp q]
// (inverse of the push of lbm.cu:1272-1310).  At a moving wall the bounced
// value excludes the wall term the next step's pull adds (w: the walls'
// velocities in that step; rho = 1 + the sum of the node's slots, which the
// terms leave unchanged since the two linked directions have opposite e_z).
template <int STORE>
__global__ void import_lattice_kernel(const Geom g, const ImportPlanes src, typename Store<STORE>::T *__restrict__ gout,
                                      const uint32_t *__restrict__ mask2d, float scale, const WallVel w, int z0, int z1)
{
    using S = Store<STORE>;
    const long long idx = (long long)z0 * g.plane + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)z1 * g.plane) return;
    const int z = (int)(idx / g.plane);
    const int xy = (int)(idx - (long long)z * g.plane);
    const int y = xy / g.nx, x = xy - y * g.nx;
    const uint32_t m = mask2d[xy];
    // reference plane of internal plane zz in [-1, nzc] (the periodic images -1 -> nzc - 1, nzc -> 0
    // are the two edge planes)
    auto plane = [&](int zz) -> const double * {
        if (zz < 0) return src.edge;
        if (zz >= g.nzc) return src.edge + src.plane_vals;
        return src.ring + (long long)(zz % src.ring_planes) * src.plane_vals;
    };
    auto at = [&](const double *pl, int xx, int yy) -> const double * {
        return pl + ((long long)(xx + g.xb) + (long long)g.nxr * yy) * Q;
    };
    double val[Q];
    double rho = 1.0;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        val[q] = 0.0;
        if (m & MASK_FLUID) {
            double f;
            if ((m >> opp(q)) & 1u) f = at(plane(z), x, y)[opp(q)];
            else f = at(plane(z + ez(q)), nb_x(g, x, ex(q)), y + ey(q))[q];
            val[q] = f - wqd(q);
            rho += val[q];
        }
    }
    if ((m & MASK_FLUID) && (m & (MASK_TOPW | MASK_BOTW)))
#pragma unroll
        for (int q = 0; q < Q; q++)
            if ((m >> opp(q)) & 1u) val[q] -= wall_term(opp(q), m, rho, w);
#pragma unroll
    for (int q = 0; q < Q; q++) S::st(gout + (long long)q * g.nint + idx, (float)val[q], scale);
}

// Internal g* -> reference pre-collision fn (the pull of the LBM kernel without
// the collision), plus rho/u with BUFF planes as periodic images
// (lbm.cu:1378-1432).  Non-COMP fn entries are set to 0, WALL macroscopic
// entries to the reference's untouched initial values (rho 1, u 0).
template <int STORE>
__global__ void export_lattice_kernel(const Geom g, const typename Store<STORE>::T *__restrict__ gin,
                                      const uint32_t *__restrict__ mask2d, const float4 *__restrict__ uvr,
                                      float inv_scale, double *__restrict__ fn, double *__restrict__ dn,
                                      double *__restrict__ un, double *__restrict__ vn, double *__restrict__ wn,
                                      const WallVel w)
{
    using S = Store<STORE>;
    const long long pref = (long long)g.nxr * g.ny, nref = pref * g.nzr;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nref) return;
    const int zr = (int)(i / pref);
    const int xyr = (int)(i - (long long)zr * pref);
    const int y = xyr / g.nxr, xr = xyr - y * g.nxr;
    // internal column; x BUFF columns (shear mode) are periodic images
    const int x = g.xper ? wrap_x(xr - g.xb, g.nx) : xr;
    const int xy = x + g.nx * y;
    const uint32_t m = mask2d[xy];
    const bool comp = (m & MASK_FLUID) && zr >= 2 && zr < g.nzr - 2 && xr >= g.xb && xr < g.nxr - g.xb;
    if (fn) {
        const bool moving = comp && (m & (MASK_TOPW | MASK_BOTW));
        double rho = 1.0;   // the node's density: 1 + the sum of its own slots
        if (moving) {
            const long long idx = (long long)(zr - 2) * g.plane + xy;
            for (int q = 0; q < Q; q++) rho += S::ld(gin + (long long)q * g.nint + idx, inv_scale);
        }
#pragma unroll
        for (int q = 0; q < Q; q++) {
            double f = 0.0;
            if (comp) {
                const int z = zr - 2;
                const long long idx = (long long)z * g.plane + xy;
                float gv;
                if ((m >> q) & 1u) {
                    gv = S::ld(gin + (long long)opp(q) * g.nint + idx, inv_scale);
                    if (moving) f += wall_term(q, m, rho, w);
                } else {
                    const long long src = (long long)wrap_z(z - ez(q), g.nzc) * g.plane + nb_x(g, x, -ex(q)) + (long long)g.nx * (y - ey(q));
                    gv = S::ld(gin + (long long)q * g.nint + src, inv_scale);
                }
                f += (double)gv + wqd(q);
            }
            fn[i * Q + q] = f;
        }
    }
    if (dn) {
        double r = 1.0, a = 0.0, b = 0.0, c = 0.0;
        if (m & MASK_FLUID) {
            const long long idx = (long long)wrap_z(zr - 2, g.nzc) * g.plane + xy;
            const float4 q = uvr[idx];
            r = q.w; a = q.x; b = q.y; c = q.z;
        }
        dn[i] = r; un[i] = a; vn[i] = b; wn[i] = c;
    }
}

// The spread's result in the reference layout (ltc->fx/fy/fz): the fixed-point
// sums as FP64 (exact below 2^53 units of 2^-56); the collide-stream kernel
// rounds them once more, to FP32.
__global__ void export_force_kernel(const Geom g, const long long *__restrict__ F, const uint32_t *__restrict__ mask2d,
                                    double *__restrict__ out)
{
    const long long pref = (long long)g.nxr * g.ny, nref = pref * g.nzr;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nref) return;
    const int zr = (int)(i / pref);
    const int xyr = (int)(i - (long long)zr * pref);
    const int y = xyr / g.nxr, xr = xyr - y * g.nxr;
    const int xy = (xr - g.xb) + g.nx * y;
    double a = 0.0, b = 0.0, c = 0.0;
    if (xr >= g.xb && xr < g.nxr - g.xb && (mask2d[xy] & MASK_FLUID) && zr >= 2 && zr < g.nzr - 2) {
        const long long idx = (long long)(zr - 2) * g.plane + xy;
        constexpr double inv = 1.0 / (double)(1ULL << FORCE_FRAC);
        a = (double)F[idx] * inv; b = (double)F[g.nint + idx] * inv; c = (double)F[2 * g.nint + idx] * inv;
    }
    out[i] = a; out[nref + i] = b; out[2 * nref + i] = c;
}

// The force each node's collision reads, FP32 [3][nint] (what the adjoint keeps).
__global__ void force_to_f32_kernel(const long long *__restrict__ F, long long n3, float *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    constexpr float inv = 1.0f / (float)(1ULL << FORCE_FRAC);
    out[i] = (float)F[i] * inv;
}

void launch_force_to_f32(const Geom &g, const long long *F, float *out3, cudaStream_t s)
{
    const long long n3 = 3 * g.nint;
    force_to_f32_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(F, n3, out3);
}

__global__ void fill_f32_kernel(float *p, long long n, float v)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void fill_f4_kernel(float4 *p, long long n, float4 v)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

void launch_fill_f4(float4 *p, long long n, float4 v, cudaStream_t s)
{
    if (n <= 0) return;
    fill_f4_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, n, v);
}

cudaError_t lattice_io_setup()
{
    // load the import and export kernels now (lazy module loading would load each in its first call)
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)import_lattice_kernel<RBC_STORE_F32>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)import_lattice_kernel<RBC_STORE_F16>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)export_lattice_kernel<RBC_STORE_F32>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)export_lattice_kernel<RBC_STORE_F16>);
    return e;
}

void launch_import_lattice(const Geom &g, int storage, const ImportPlanes &src, void *gout, const uint32_t *mask2d,
                           float scale, const WallVel &w, int z0, int z1, cudaStream_t s)
{
    const unsigned blocks = (unsigned)(((long long)(z1 - z0) * g.plane + 255) / 256);
    if (blocks == 0) return;
    if (storage == RBC_STORE_F16)
        import_lattice_kernel<RBC_STORE_F16><<<blocks, 256, 0, s>>>(g, src, (__half *)gout, mask2d, scale, w, z0, z1);
    else
        import_lattice_kernel<RBC_STORE_F32><<<blocks, 256, 0, s>>>(g, src, (float *)gout, mask2d, scale, w, z0, z1);
}

void launch_export_lattice(const Geom &g, int storage, const void *gin, const uint32_t *mask2d,
                           const float4 *uvr, float inv_scale, double *fn_ref, double *dn, double *un,
                           double *vn, double *wn, const WallVel &w, cudaStream_t s)
{
    const long long nref = (long long)g.nxr * g.ny * g.nzr;
    const unsigned blocks = (unsigned)((nref + 255) / 256);
    if (storage == RBC_STORE_F16)
        export_lattice_kernel<RBC_STORE_F16><<<blocks, 256, 0, s>>>(g, (const __half *)gin, mask2d, uvr,
                                                                     inv_scale, fn_ref, dn, un, vn, wn, w);
    else
        export_lattice_kernel<RBC_STORE_F32><<<blocks, 256, 0, s>>>(g, (const float *)gin, mask2d, uvr,
                                                                     inv_scale, fn_ref, dn, un, vn, wn, w);
}

void launch_export_force(const Geom &g, const long long *F, const uint32_t *mask2d, double *out3, cudaStream_t s)
{
    const long long nref = (long long)g.nxr * g.ny * g.nzr;
    export_force_kernel<<<(unsigned)((nref + 255) / 256), 256, 0, s>>>(g, F, mask2d, out3);
}

void launch_fill_f32(float *p, long long n, float v, cudaStream_t s)
{
    if (n <= 0) return;
    fill_f32_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, n, v);
}

}  // namespace rbc
