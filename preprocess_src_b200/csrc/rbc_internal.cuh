// rbc_internal.cuh -- shared definitions of the sm_100a step kernels.
//
// Internal layout in HBM (one handle):
//   populations  g[q][z][y][x], q = 0..18 in the reference's slot order,
//                x fastest, z = periodic axis without BUFF planes (nzc = nz - 4
//                planes).  Each value is f_q - w_q of the post-collision state
//                of the previous step (pull scheme), FP32 or scaled FP16.
//   macroscopic  uvr[z][y][x] float4 (u, v, w, rho): the reference's um/vm/wm
//                (M = 1, with the half-force shift) and dn, interleaved so one
//                16-byte load serves an interpolation stencil point.
//   IB force     F[3][z][y][x] int64 fixed point (ForceField) with one
//                occupancy bit per node; the LBM kernel converts, reads and
//                zeroes the nodes whose bit is set, and clears the bits.
//   wall mask    mask2d[y][x] uint32: bit 31 = fluid column, bit q = the pull
//                source of direction q is a wall (half-way bounce-back).  The
//                reference channel is z-invariant, so one plane serves all z.
//   cells        X, Xd [3][nv] FP64 (cel->x/y/z and fem->xd), U, Fv [3][nv]
//                FP32; gref [ne] double4 reference covariant metric
//                (G11, G12, G22, -); the contravariant metric n = G^-1.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <string>
#include <utility>

#include "rbc_step.h"

namespace rbc {

// Programmatic dependent launch: the step's kernels on one stream are launched
// with programmatic stream serialization, so a kernel's blocks may be placed on
// the multiprocessors while its predecessor's last blocks still run.  Each such
// kernel first lets its own successor do the same, then waits until the
// predecessor has completed and its writes are visible, before it touches
// memory.  Without the launch attribute both instructions return at once.
__device__ __forceinline__ void pdl_start()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at; cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}


constexpr int Q = 19;
constexpr float F16_SCALE = 32768.0f;   // FP16 storage (f - w) * 2^15 keeps |g| < 2 inside FP16 range
constexpr uint32_t MASK_FLUID = 0x80000000u;
// shear mode (x periodic, moving y walls): column flags beside the link bits 1..18
constexpr uint32_t MASK_XLO = 1u << 20;    // first column: x - 1 is the last column (periodic)
constexpr uint32_t MASK_XHI = 1u << 21;    // last column: x + 1 is the first column
constexpr uint32_t MASK_TOPW = 1u << 22;   // the column's wall links touch the top (+y) wall
constexpr uint32_t MASK_BOTW = 1u << 23;   // ... the bottom (-y) wall

// D3Q19 in the reference's slot order (lbm.cu:1038-1047):
// ___ p__ m__ _p_ _m_ __p __m pp_ mm_ mp_ pm_ _pp _mm _mp _pm p_p m_m p_m m_p
__host__ __device__ constexpr int ex(int q) {
    return (q == 1 || q == 7 || q == 10 || q == 15 || q == 17) ? 1
         : (q == 2 || q == 8 || q == 9 || q == 16 || q == 18) ? -1 : 0;
}
__host__ __device__ constexpr int ey(int q) {
    return (q == 3 || q == 7 || q == 9 || q == 11 || q == 14) ? 1
         : (q == 4 || q == 8 || q == 10 || q == 12 || q == 13) ? -1 : 0;
}
__host__ __device__ constexpr int ez(int q) {
    return (q == 5 || q == 11 || q == 13 || q == 15 || q == 18) ? 1
         : (q == 6 || q == 12 || q == 14 || q == 16 || q == 17) ? -1 : 0;
}
__host__ __device__ constexpr int opp(int q) { return q == 0 ? 0 : ((q & 1) ? q + 1 : q - 1); }
__host__ __device__ constexpr float wq(int q) { return q == 0 ? (1.0f / 3.0f) : (q <= 6 ? (1.0f / 18.0f) : (1.0f / 36.0f)); }
__host__ __device__ constexpr double wqd(int q) { return q == 0 ? (1.0 / 3.0) : (q <= 6 ? (1.0 / 18.0) : (1.0 / 36.0)); }

// Geometry of one handle, passed by value to kernels.
struct Geom {
    int nx, ny, nzc, nzr;      // internal dims; nzr = reference nz (nzc + 4)
    int nxr, xb, xper;         // reference nx; x columns stripped at each end (2 in the shear
                               // mode, whose x is periodic with BUFF columns; else 0); x periodic
    long long plane, nint;     // nx*ny, nx*ny*nzc
    double dx, inv_dx;
    double xoff, yoff, zoff;   // lattice coordinate = (pos + off)/dx (ibm.cu:100-102)
    double LX, LZ, xmin, xmax, zmin, zmax;
};

// Lattice coordinates of a position in the internal frame (z without BUFF).
// (multiplication by 1/dx; exact for the unit lattice spacing the workloads use)
__device__ __forceinline__ double lat_x(const Geom &g, double x) { return (x + g.xoff) * g.inv_dx - g.xb; }
__device__ __forceinline__ double lat_y(const Geom &g, double y) { return (y + g.yoff) * g.inv_dx; }
__device__ __forceinline__ double lat_z(const Geom &g, double z) { return (z + g.zoff) * g.inv_dx - 2.0; }

__device__ __forceinline__ int wrap_z(int iz, int nzc) {
    iz %= nzc;
    return iz < 0 ? iz + nzc : iz;
}
__device__ __forceinline__ int wrap_x(int ix, int nx) { return wrap_z(ix, nx); }

// 4-point cosine delta, phi(r) = (1 + cos(pi r / 2)) / 4 (ibm.cu:103-128), at the
// four nodes floor(l)-1 .. floor(l)+2 for fraction f = l - floor(l):
// r = 1+f, f, 1-f, 2-f  ->  (1 - s, 1 + c, 1 + s, 1 - c) / 4 with s = sin(pi f/2),
// c = cos(pi f/2).  For f = 0 this is the reference's 3-node stencil plus a zero.
// s and c come from polynomials in t = f^2 on [0, 1], s = f P(t) (degree 4) and
// c = Q(t) (degree 5, Q(0) = 1), least-squares fits to sin(pi f / 2) and
// cos(pi f / 2) at the 8000 Chebyshev nodes f_k = (1 + cos(pi (k + 1/2) / 8000)) / 2,
// rounded to FP32: fit errors 3.7e-9 and 2.5e-10, about one FP32
// rounding of 1 when evaluated in FP32 with fused multiply-adds.  They take
// eleven multiply-adds on the FMA pipe where a library sincospi reduces its
// argument first.  s(f) in [0, 1), c(f) in (0, 1] for f in [0, 1), so the weights
// keep the bounds (1, 2, 2, 1) / 4 the spread's fixed-point scale relies on.
__device__ __forceinline__ void delta4(float f, float w[4]) {
    const float t = f * f;
    const float p = fmaf(fmaf(fmaf(fmaf(1.50956082e-4f, t, -4.67254827e-3f), t, 7.96887353e-2f), t,
                              -6.45963430e-1f), t, 1.57079625f);
    const float s = f * p;
    const float c = fmaf(fmaf(fmaf(fmaf(fmaf(-2.38483281e-5f, t, 9.17786616e-4f), t, -2.08627470e-2f), t,
                                   2.53669351e-1f), t, -1.23370051f), t, 1.0f);
    w[0] = fmaf(-0.25f, s, 0.25f);
    w[1] = fmaf(0.25f, c, 0.25f);
    w[2] = fmaf(0.25f, s, 0.25f);
    w[3] = fmaf(-0.25f, c, 0.25f);
}

// IB force on the lattice: the three components as int64 fixed point
// F * 2^FORCE_FRAC in arrays [3][nint], and one occupancy bit per node in words
// [nzc][wpp] (word xy / 32 of plane z, bit xy % 32) that the spread sets for every
// node it adds to.  Integer sums are exact, so the spread's result does not depend
// on the order of its global atomics (several patches and cells add to a node).
// The collide-stream kernel reads, converts (one rounding to FP32) and zeroes the
// nodes whose bit is set, so only nodes near membranes cost force traffic.
// After that read a reset kernel zeroes the forces of the nodes whose bit is
// set and clears the words (force_reset_words).  The collide-stream kernel only
// reads the field: zeroing it there made that kernel 2x slower.  Sums are exact while |F| < 2^(63 - FORCE_FRAC) = 128 at
// every node (partial sums may wrap; the adds are modular); a contribution of
// 64 or more raises RBC_FLAG_NONFINITE (a lattice force density of that size
// has long broken the LBM).
constexpr int FORCE_FRAC = 56;
struct ForceField {
    long long *F;              // [3][nint]
    uint32_t *bits;            // [nzc][wpp]
    int wpp;                   // occupancy words per plane, ceil(plane / 32)
};
__host__ __device__ constexpr int force_words_per_plane(long long plane) { return (int)((plane + 31) / 32); }

// ---- launchers (defined in the .cu files, called by rbc_abi.cu) ----------

struct LbmArgs {
    const void *gin; void *gout;
    float4 *uvr;
    ForceField F;              // read and converted where the occupancy bit is set
    const uint32_t *mask2d;
    const float *drive;        // device scalar: P * drive factor of this step
    const int *iter;           // device: the step counter, which seeds the FP16 stochastic rounding
    const float *wall;         // device [2]: z velocity of the top and bottom walls (shear mode), else NULL
    const double *vf;          // volume fraction: omega = 1 / (df3 (1 + lm1 vf) + 1/2) per node; NULL: omega
    float lm1, df3;            // LAMBDA1 - 1 and 3 Df (lbm.cu:1131)
    float omega, Cr, Bc;
    float scale, inv_scale;    // FP16 storage scale
    int planes;                // z planes per thread; 0 = chosen from the lattice size
    // sub-cycling (M > 1, lbm.cu:1097-1126, 1435-1460): LBM_ACC_WRITE stores the
    // node's u and rho (every step of M = 1, the first of M), LBM_ACC_ADD adds
    // them to the stored sums, LBM_ACC_AVERAGE adds and divides the velocity sum
    // by Mf (the last of M)
    int acc;
    float Mf;
};
enum { LBM_ACC_WRITE = 0, LBM_ACC_ADD = 1, LBM_ACC_AVERAGE = 2 };
void launch_lbm(const Geom &g, int storage, const LbmArgs &a, cudaStream_t s);
// z velocities of the top and bottom walls in the next step (shear mode; 0 otherwise)
struct WallVel { double top, bot, Cr; };
// Reference planes an import reads: internal planes 0 .. nzc-1 in a ring of
// ring_planes planes (plane z at z % ring_planes), and the two periodic images
// (edge: plane nzc - 1, then plane 0), each plane_vals = nxr * ny * 19 doubles
struct ImportPlanes { const double *ring, *edge; int ring_planes; long long plane_vals; };
cudaError_t lattice_io_setup();   // loads the import / export kernels
// Reference fn -> internal g* for internal planes [z0, z1)
void launch_import_lattice(const Geom &g, int storage, const ImportPlanes &src, void *gout, const uint32_t *mask2d,
                           float scale, const WallVel &w, int z0, int z1, cudaStream_t s);
void launch_export_lattice(const Geom &g, int storage, const void *gin, const uint32_t *mask2d,
                           const float4 *uvr, float inv_scale, double *fn_ref, double *dn, double *un,
                           double *vn, double *wn, const WallVel &w, cudaStream_t s);
// Circular tube: after each collide-stream, the slot each listed wall link bounces
// back from becomes the interpolated bounce-back value (lbm_cylinder.cu:190-231).
// links[k] = xy * 32 + p (pull direction p, wall at i - e_p), frac[k] = crossing fraction.
void launch_tube_bounce(const Geom &g, int storage, void *gout, const int *links, const float *frac, int nlinks,
                        float inv_scale, float scale, cudaStream_t s);
void launch_export_force(const Geom &g, const long long *F, const uint32_t *mask2d, double *out3, cudaStream_t s);
// the lattice force as FP32 [3][nint] (the value the collide-stream kernel reads)
void launch_force_to_f32(const Geom &g, const long long *F, float *out3, cudaStream_t s);
void launch_fill_f32(float *p, long long n, float v, cudaStream_t s);
void launch_fill_f4(float4 *p, long long n, float4 v, cudaStream_t s);

// Volume fraction (vof.cu).  THINC/WLIC: three sweeps vf -> s1 -> s2 -> vf.
void launch_thinc_wlic(const Geom &g, double *vf, double *s1, double *s2, const float4 *uvr, const uint32_t *mask2d,
                       double dt, cudaStream_t s);
// Multigrid preconditioner of the front-tracking solve: levels of the
// Jacobi-scaled Poisson operator on the internal lattice, each the Galerkin
// product with piecewise-constant aggregation of 2 x 2 x 2 nodes (fewer along
// an axis that is too short or periodic with odd length).  Coefficients per
// level column [7][nx * ny]: diagonal, x-, x+, y-, y+, z (the z coupling to
// both neighbours), inverse diagonal; a column with diagonal 0 is a wall column.
constexpr int MG_MAX_LEVELS = 12;
struct MgLevel {
    int nx, ny, nz;          // dimensions
    int bx, by, bz;          // aggregation factors to the next level
    int xper;
    long long n;
    const double *coef;
    double *b, *x, *y;       // right-hand side, pre-smoothed iterate, V-cycle result
};
struct MgHierarchy {
    int nlev = 0;
    MgLevel lev[MG_MAX_LEVELS];
    void *mem = nullptr;     // one device allocation holding every level's coefficients and vectors
};
// mask2d_host: the handle's column mask; level 0's b and y are the CG's r and z
cudaError_t vof_mg_build(const Geom &g, const uint32_t *mask2d_host, MgHierarchy &mg);
void vof_mg_free(MgHierarchy &mg);

// Front tracking of one cell population into vf (warm start from vf).
struct FrontArgs {
    const double *X; long long nv;
    const int *tri; int V, E, ncell;
    const uint32_t *mask2d;
    double *G;                 // [3][nint] scratch: the indicator gradient, then the CG vectors
    double *b;                 // [nint] scratch: right-hand side
    double *vf;                // [nint] solution
    double *partial;           // [4 * vof_cg_blocks()] scratch
    const MgHierarchy *mg;     // preconditioner levels (nlev >= 2), or nullptr / nlev < 2 for plain CG
    double tol; int itrmax;
    int *iters;                // device: sweeps of the solve, -1 = not converged
    int *flags;
};
cudaError_t launch_front_tracking(const Geom &g, const FrontArgs &a, cudaStream_t s);
int vof_cg_blocks();



// Surface patches (spread and advection work units) hold at most this many vertices.
constexpr int MAX_PATCH_VERTICES = 512;

struct SpreadArgs {
    const double *X; long long nv; int V, ncell;
    const int *patch_off, *patch_vtx, *patch_stride;   // surface patches of the shared mesh
    int npatch;
    const float *Fv;
    ForceField F;
    const uint32_t *mask2d;
    int *flags;
};
int  spread_smem_bytes();
void launch_spread(const Geom &g, const SpreadArgs &a, cudaStream_t s);

struct AdvectArgs {
    double *X, *Xd; float *U;
    const float4 *uvr;
    long long nv;
    int V, ncell;
    const int *patch_off, *patch_vtx;   // surface patches of the shared mesh
    int npatch;
    double dtM;                // dt * M
    int rk;                    // RUNGE_KUTTA: 1, 2 or 4 stages
    int *flags;
};
void launch_advect(const Geom &g, const AdvectArgs &a, cudaStream_t s);

struct MembraneArgs {
    const double *Xd; long long nv, ne;
    const double4 *gref;      // [ne] reference covariant metric (G11, G12, G22, 1 / det G)
    void *erec;               // [ne][3] element records (Real 4-vectors): scratch written and read by each CTA
    const int *tri, *v2e_off, *v2e;
    const int16_t *nbr;       // [6][V] local neighbour ids, -1 = none
    const int16_t *nbrp;      // [6][V] the same neighbours as positions in the solve order, by position
    const int *vord;          // [V] solve order: the vertex at each position
    float *Fv;
    int V, E, ncell;
    double C, rgs; int law;
    double LX, LZ;
    int niter;
    int *flags;
    int priority;             // launch priority (cudaLaunchAttributePriority)
};
int  membrane_smem_bytes(int V);

// host helpers of the reference-format files (rbc_abi.cu)
int reference_mn(int V);
int output_averages(rbc_handle *h, int group, double *qi, double *tp, bool set);   // group 0 red, 1 white cells
int reference_bc(rbc_handle *h, int *bc);
int import_macro(rbc_handle *h, const double *dm, const double *um, const double *vm, const double *wm);
int clear_force(rbc_handle *h);
int import_vertex_velocity(rbc_handle *h, int group, const double *u, const double *v, const double *w);
int reference_ele(rbc_handle *h, int group, int *ele);   // cel->eleH(_w): [ncell * E * 3] global vertex ids
int group_sizes(const rbc_handle *h, int group, int *ncell, int *vertex, int *element);
void set_handle_error(rbc_handle *h, const std::string &msg);

// Output-interval averages of the load and the principal tensions (fem->qi,
// fem->tp of the reference's output files), after the membrane kernel.
struct AccumArgs {
    const double *Xd; const float *Fv;
    const double4 *gref;
    const int *tri, *v2e_off, *v2e;
    const int *iter;                 // device iteration counter of the step
    double *qi;                      // [ncell][3 V] AoS per vertex (the reference's qd layout)
    double *tp;                      // [ne][2]
    long long nv, ne;
    int V, E, ncell, fileoutput, M;
    double C, LX, LZ;
};
void launch_output_accum(const AccumArgs &a, cudaStream_t s);

// fourpoint_bend (stress.cu:448-578): added to Fv after the membrane forces
struct BendArgs {
    const double *X; long long nv;   // cel->x, [3][nv]
    int V;
    const int *v2e_off, *v2e;        // vertex -> element incidence of the shared mesh
    const int4 *visit;               // [E][3]: (k1, k2, k3, k4) local ids per edge-neighbour visit, k1 < 0: none
    const double2 *cs0;              // [ncell][E][3] spontaneous angle (cos, sin) per visit; nullptr: (1, 0)
    int E, ncell;
    double *rec;                     // [ncell][E][3][3][3] scratch: each visit's forces on k1, k2, k3
    double LX, LZ;
    double coef;                     // (2 / sqrt 3) BR
    float *Fv;
};
void launch_bend(const BendArgs &a, cudaStream_t s);
void launch_membrane(const MembraneArgs &a, bool fp64, cudaStream_t s);

// 18 x the volume contribution and 2 x the area of triangle (a, b, c): with
// c = (b - a) x (c - a), (a + b + c) . c and |c|.  This is the normal form of
// CalcEleNormal_GPU / CalcVolume (volume_correction.cu:138-200, 246-281:
// (r . n) dS / 3 with r the centroid, n = c / |c|, dS = |c| / 2) without its
// divisions; the volume correction and its adjoint's replay both use it.
__device__ __forceinline__ void tri_measure(const double (&A)[3], const double (&B)[3], const double (&C)[3],
                                            double &s18v, double &s2a)
{
    const double v1x = B[0] - A[0], v1y = B[1] - A[1], v1z = B[2] - A[2];
    const double v2x = C[0] - A[0], v2y = C[1] - A[1], v2z = C[2] - A[2];
    const double c0 = v1y * v2z - v1z * v2y, c1 = v1z * v2x - v1x * v2z, c2 = v1x * v2y - v1y * v2x;
    s2a += sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    s18v += (A[0] + B[0] + C[0]) * c0 + (A[1] + B[1] + C[1]) * c1 + (A[2] + B[2] + C[2]) * c2;
}

struct VolumeArgs {
    double *X; long long nv;
    const int *tri, *v2e_off, *v2e;
    const double *vol0;
    double *gx;               // [3][ncell]
    double *vol_out, *area_out;
    double *cen_out;          // [3][ncell] centroid when correct == 0
    int V, E, ncell;
    int *flags, *vc_max, *vc_last;
    int correct;              // 0: metrics only (volume, area, centroid), positions untouched
};
int  volume_smem_bytes(int V);
void launch_volume(const Geom &g, const VolumeArgs &a, cudaStream_t s);

// one-time kernel attribute setup (dynamic shared memory limits); called by
// rbc_create before any launch or graph capture.  Returns a cudaError_t value;
// *membrane_max_smem receives the dynamic shared memory the membrane kernel may use.
int  setup_kernel_attributes(int *membrane_max_smem);

// Step begin: iteration counter, drive P * factor (lbm.cu:1030-1035) and, in the
// shear mode, the walls' z velocities (lbm.cu:752, 946-964).
struct StepBeginArgs {
    int *iter; float *drive;
    double P, freq, dt; int flowstart;
    float *wall;               // [2] top, bottom; NULL outside the shear mode
    double sr, LY; int walls;  // shear rate, wall distance, 0 both walls / 1 top wall
    float *drive_rec; double *factor_rec;   // where the adjoint keeps the step's drive (may be NULL)
    int *vc_last;              // when set, zeroed (the volume correction's count of this step; fused batches)
};
void launch_step_begin(const StepBeginArgs &a, cudaStream_t s);

// The force field's reset after the collide-stream kernel read it: every word
// of occupancy bits that is set zeroes its nodes' forces (only those: the rest
// is zero already), then itself.  One warp per 32 consecutive words: lane l
// loads word w0 + l (one coalesced load), then the warp zeroes the nodes of
// each set word in turn (lane l owns node xy = 32 ((w0 + j) mod wpp) + l of
// word j) and every lane clears its own word.
__device__ __forceinline__ void force_reset_words(long long *__restrict__ F, uint32_t *__restrict__ bits, long long w0,
                                                  long long nwords, int wpp, long long plane, long long nint, int lane)
{
    const long long wl = w0 + lane;
    const uint32_t mine = wl < nwords ? bits[wl] : 0u;
    unsigned pending = __ballot_sync(0xffffffffu, mine != 0u);
    while (pending) {
        const int j = __ffs(pending) - 1;
        pending &= pending - 1;
        const uint32_t word = __shfl_sync(0xffffffffu, mine, j);
        const long long w = w0 + j, z = w / wpp, xy = (w - z * wpp) * 32 + lane;
        if (((word >> lane) & 1u) && xy < plane) {
            const long long idx = z * plane + xy;
            F[idx] = 0; F[nint + idx] = 0; F[2 * nint + idx] = 0;
        }
    }
    if (mine) bits[wl] = 0u;
}
void launch_force_reset(const Geom &g, const ForceField &F, cudaStream_t s);

// ---- adjoint of one step (adjoint.cu); FP32 populations ----------------------

struct LbmAdjArgs {
    const float *gin;          // g_t, [Q][n]
    const float *Fx, *Fy, *Fz; // spread force of the step
    const uint32_t *mask2d;
    const float *gbar_out;     // adjoint of g_t+1, [Q][n]
    const float4 *ubar;        // adjoint of the velocity, [n]
    float *gbar_in;            // out: adjoint of g_t, [Q][n] (fluid slots)
    float *Fbar;               // out: adjoint of the force, [3][n]
    double *pbar;              // += (dfac dL/dpd, dL/dB)
    const float *pd;           // device: drive P * factor of the step
    const double *dfac;        // device: drive factor of the step (dpd / dP)
    float Bc, omega, Cr;       // B, 1 / tau, Cr
};
void launch_lbm_adjoint(const Geom &g, const LbmAdjArgs &a, cudaStream_t s);
void launch_advect_adjoint(const Geom &g, const double *X, const float4 *uvr, const double *xa_bar, double *X_bar,
                           float *ubar, long long nv, double dtM, int *flags, cudaStream_t s);
void launch_spread_adjoint(const Geom &g, const double *X, const float *Fv, const float *Fbar, const uint32_t *mask2d,
                           double *Fv_bar, double *X_bar, long long nv, cudaStream_t s);

struct MembraneAdjArgs {
    const double *Xd; long long nv, ne;
    const double4 *gref;
    const int *tri, *v2e_off, *v2e;
    const int16_t *nbr;
    const float *Fv;           // the step's membrane forces
    const double *Fv_bar;      // their adjoint, [3][nv]
    double *Xd_bar;            // out, [3][nv]
    double *scratch;           // [ne][7]: gab, adjoints of the edge vectors
    float4 *lam, *qv;          // [nv] scratch: lambda = M^-1 q_bar and q per vertex
    float *dsb;                // [nv] scratch: adjoint of the one-ring area / 3
    double *cbar;              // += dL/dC
    int V, E, ncell;
    double C, rgs; int law;
    double LX, LZ;
    int niter;
};
void launch_membrane_adjoint(const MembraneAdjArgs &a, cudaStream_t s);

struct VolumeAdjArgs {
    const double *Xa;          // positions before the correction, [3][nv]
    const double *gx;          // centroids the correction unwraps about, [3][ncell]
    const double *vol0;
    const int *tri, *v2e_off, *v2e;
    const double *X_bar;       // adjoint of the corrected positions
    const double *Xd_bar;      // adjoint of fem->xd after the step (= Xa)
    double *Xa_bar;            // out: adjoint of Xa
    double *hist;              // [ncell][kmax][3][V]
    double *escr;              // [ne][9]
    int *status;               // bit 0: more moves than kmax (only kmax reversed)
    long long nv;
    int V, E, ncell, kmax;
};
int  volume_adjoint_smem_bytes(int V);
void launch_volume_adjoint(const Geom &g, const VolumeAdjArgs &a, cudaStream_t s);

// packed vertex -> element incidence: element id (bits 0..23), local position
// of the vertex in the element (bits 24..25), neighbour slots of the two other
// vertices (bits 26..28 and 29..31)
__host__ __device__ __forceinline__ int v2e_elem(int p) { return p & 0xFFFFFF; }
__host__ __device__ __forceinline__ int v2e_en(int p) { return (p >> 24) & 3; }
__host__ __device__ __forceinline__ int v2e_sa(int p) { return (p >> 26) & 7; }
__host__ __device__ __forceinline__ int v2e_sb(int p) { return (p >> 29) & 7; }

// ---- fused batches: one launch per stage for many simulations -------------
//
// Every simulation of a fused batch is a "domain": its geometry and the
// arguments of each stage kernel, exactly as its own handle would launch them
// (one buffer parity).  A fused launch runs the blocks of all domains of one
// stage: block b belongs to the domain d with boff[d] <= b < boff[d + 1] and is
// that domain's block b - boff[d].  The kernels run the same device code as the
// one-simulation launches, so a fused step equals each simulation's own step
// bit for bit.
struct DomainArgs {
    Geom g;
    StepBeginArgs sb;
    ForceField F;
    MembraneArgs mem;
    SpreadArgs spread;
    LbmArgs lbm;
    int lbm_bx, lbm_gy;        // collide-stream: column tiles per plane, plane stride (tiles along z)
    AdvectArgs adv;
    VolumeArgs vol;
};
struct FusedLaunch {
    const DomainArgs *dom;     // device [ndom]
    const int *boff;           // device [ndom + 1]
    int ndom, nblocks;
};
__device__ __forceinline__ int fused_domain(const int *__restrict__ boff, int ndom, int b)
{
    int lo = 0, hi = ndom;     // the last domain whose first block is at or before b
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(&boff[mid]) <= b) lo = mid; else hi = mid;
    }
    return lo;
}
constexpr int FUSED_CLEAR_THREADS = 256;
void launch_step_begin_fused(const FusedLaunch &f, cudaStream_t s);   // one thread per domain
void launch_clear_bits_fused(const FusedLaunch &f, cudaStream_t s);   // the force reset, FUSED_CLEAR_THREADS words per block
void launch_membrane_fused(const FusedLaunch &f, bool fp64, int V, int vpt, cudaStream_t s);   // a block per cell
void launch_spread_fused(const FusedLaunch &f, bool xper, cudaStream_t s);    // a block per (cell, patch)
void launch_lbm_fused(const FusedLaunch &f, int storage, bool off32, int threads, cudaStream_t s);
void launch_advect_fused(const FusedLaunch &f, bool xper, cudaStream_t s);    // a block per (cell, patch)
void launch_volume_fused(const FusedLaunch &f, int V, cudaStream_t s);        // a block per cell
int  membrane_threads(int V, int vpt);     // threads of a membrane block with vpt vertices per thread
int  membrane_default_vpt(int V);          // the vertices per thread of a one-population launch

}  // namespace rbc
