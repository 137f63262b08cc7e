// membrane.cu -- Skalak membrane FEM nodal forces, one CTA per cell.
//
// Replaces calc_tension, calc_load (with its per-cell BiCGSTAB) and q2f
// (stress.cu:29-445, matrix_solver.cu:279-377 of the reference).  The
// reference computes per-element contravariant tensions t^{ab}, assembles for
// each cell the P1 consistent mass matrix M (gab/12 on the diagonal, gab/24 off
// it, gab = 2 x area) and the load vector
//   b_i = sum_e gab/4 sum_ab t^{ab} (v_a f_b + v_b f_a)      (stress.cu:256-260)
// solves the Jacobi-scaled system D^-1 M q = D^-1 b per cell with BiCGSTAB
// (5 blocking device-to-host reductions per iteration, cells in sequence), and
// converts q to forces f_i = -q_i * (area of the one-ring / 3).
//
// Here one CTA owns one cell and does all of it on chip:
//  1. the cell's FP64 positions go to shared memory, relative to vertex 0;
//     edge vectors take the minimum image in x and z per edge, as the
//     reference does (stress.cu), so cells of any size relative to LX / 2
//     and cells across the periodic boundary are handled alike;
//  2. element pass: each element's tension is evaluated once and its record
//     (twice the area gab and the load contributions of its second and third
//     vertex; the first vertex's is minus their sum) goes to an L2-resident
//     scratch array;
//  3. vertex pass: each thread gathers the rows of its vertices through the
//     vertex -> element incidence list (fixed order, no atomics): matrix row,
//     right-hand side and nodal area;
//     Threads own solve positions, not vertex ids: the host orders the
//     vertices breadth first around the surface and sorts each neighbour list
//     by position, so the lanes of a warp gather neighbours at nearby
//     positions in every slot (fewer shared-memory bank conflicts in step 4:
//     3.7 against 5.6 us per iteration on the dense suspension);
//  4. the scaled system is solved by Chebyshev iteration.  For any P1 triangle
//     mesh the element mass matrix is (A/12)(1 + delta_ij), so every
//     eigenvalue of D^-1 M lies in [1/2, 2] (Rayleigh quotients of an assembled
//     sum of element matrices stay inside the element bounds).  With these
//     bounds Chebyshev needs no inner products: the error falls by at least
//     (sqrt(4)-1)/(sqrt(4)+1) = 1/3 per iteration, one barrier per iteration.
//     (Chebyshev iteration as in Y. Saad, Iterative Methods for Sparse Linear
//     Systems, 2nd ed., Alg. 12.1.)
//  5. f_i = -q_i * ds_i is written out.
//
// Tension without cancellation.  The reference evaluates
//   t = ca n + cb g^-1,  ca = rgs (I1 + 1) / Js,  cb = (C I2 - 1) Js
// where the two O(1) terms cancel to O(strain); in FP32 that turns round-off
// into tension noise of order C * 1e-7.  Here the deformed metric enters only
// through its difference from the reference metric, D = g - G, formed in FP64
// from FP64 edge vectors, and everything after that works on small numbers:
//   I1 = n : D,   I2 = det(n) (G11 D22 + G22 D11 - 2 G12 D12 + det D),
//   Js - 1 = I2 / (Js + 1),
//   t = (ca - 1) n + (cb + 1) g^-1 + n D g^-1        (n - g^-1 = n D g^-1),
//   ca - 1 = (rgs I1 + (rgs - 1) - (Js - 1)) / Js,   cb + 1 = C I2 Js - (Js - 1)
// (neo-Hookean: ca = rgs / Js, cb = -rgs / Js^3), algebraically the same
// tension as stress.cu:94-99.
// Element mechanics after the FP64 metric difference run in FP32 or FP64
// (Real); the solve runs in FP32.
#include "rbc_internal.cuh"

namespace rbc {

constexpr int MEM_MAX_THREADS = 1024;

// pos 24V (then the solve's two d-buffers, 3 x V floats each), coef 24V, and 12V that the adjoint's
// membrane pass uses for its neighbour table (this kernel reads its neighbours
// from global memory once, into registers)
int membrane_smem_bytes(int V) { return 68 * V; }

__device__ __forceinline__ double mimage(double d, double L) {
    if (d > L * 0.5) d -= L; else if (d < -L * 0.5) d += L;
    return d;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    T s = 0;
    for (int k = 0; k < nw; k++) s += red[k];
    return s;
}

// Element records: for each vertex slot en of an element, the load that the
// element puts on that vertex and the element's gab, one 4-vector per slot.
template <typename Real> struct Vec4;
template <> struct Vec4<float> { using T = float4; };
template <> struct Vec4<double> { using T = double4; };

__device__ __forceinline__ float4 make_vec4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
__device__ __forceinline__ double4 make_vec4(double x, double y, double z, double w) { return make_double4(x, y, z, w); }
__device__ __forceinline__ void store_vec4(float4 *p, const float4 &v) { *p = v; }
__device__ __forceinline__ void store_vec4(double4 *p, const double4 &v) {
    double2 *q = reinterpret_cast<double2 *>(p);
    q[0] = make_double2(v.x, v.y); q[1] = make_double2(v.z, v.w);
}
__device__ __forceinline__ float4 load_vec4(const float4 *p) { return *p; }
__device__ __forceinline__ double4 load_vec4(const double4 *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 x = q[0], y = q[1];
    return make_double4(x.x, x.y, y.x, y.y);
}

constexpr int MAX_VALENCE = 6;   // checked when the topology is built

// threads per CTA for VPT vertices per thread: at most 896 for VPT >= 3 (72
// registers a thread), 1024 otherwise
template <int VPT> constexpr int mem_max_threads() { return VPT >= 3 ? 896 : MEM_MAX_THREADS; }

// cell: the block's cell, blockIdx.x of a one-population launch
template <typename Real, int VPT>
__device__ __forceinline__ void membrane_body(const MembraneArgs &a, int cell)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float red[32];
    const int V = a.V, E = a.E, tid = threadIdx.x, T = blockDim.x;
    double *pos = reinterpret_cast<double *>(smem);                    // [3][V]
    float *dbuf = reinterpret_cast<float *>(smem);                     // [2][3][V], after assembly
    float *coef = reinterpret_cast<float *>(smem + 32 * (size_t)V);    // [6][V]

    const long long vb = (long long)cell * V, eb = (long long)cell * E, nv = a.nv;
    const double ax = a.Xd[vb], ay = a.Xd[nv + vb], az = a.Xd[2 * nv + vb];
    for (int v = tid; v < V; v += T) {
        pos[v] = a.Xd[vb + v] - ax;
        pos[V + v] = a.Xd[nv + vb + v] - ay;
        pos[2 * V + v] = a.Xd[2 * nv + vb + v] - az;
    }
    __syncthreads();

    // element pass: tension of each element once (stress.cu:29-110, 195-270)
    const Real C = (Real)a.C, rgs = (Real)a.rgs;
    using R4 = typename Vec4<Real>::T;
    R4 *rec = reinterpret_cast<R4 *>(a.erec) + (size_t)eb * 3;   // [E][3 slots]: load on the slot's vertex, gab
    for (int e = tid; e < E; e += T) {
        const int ia = __ldg(&a.tri[3 * e]), ib = __ldg(&a.tri[3 * e + 1]), ic = __ldg(&a.tri[3 * e + 2]);
        const double e1x = mimage(pos[ib] - pos[ia], a.LX), e1y = pos[V + ib] - pos[V + ia];
        const double e1z = mimage(pos[2 * V + ib] - pos[2 * V + ia], a.LZ);
        const double e2x = mimage(pos[ic] - pos[ia], a.LX), e2y = pos[V + ic] - pos[V + ia];
        const double e2z = mimage(pos[2 * V + ic] - pos[2 * V + ia], a.LZ);
        // deformed covariant metric (stress.cu:75-84) and its difference from the reference, in FP64
        const double g11d = e1x * e1x + e1y * e1y + e1z * e1z;
        const double g12d = e1x * e2x + e1y * e2y + e1z * e2z;
        const double g22d = e2x * e2x + e2y * e2y + e2z * e2z;
        // reference metric: covariant G and 1 / det G (one aligned 32-byte record per element);
        // its inverse n as set_contravariant forms it (init2.cu:241-249)
        const double2 *gp = reinterpret_cast<const double2 *>(a.gref + eb + e);
        const double2 Ga = __ldg(gp), Gb = __ldg(gp + 1);
        const double G11 = Ga.x, G12 = Ga.y, G22 = Gb.x, idG = Gb.y;
        const Real d11 = (Real)(g11d - G11), d12 = (Real)(g12d - G12), d22 = (Real)(g22d - G22);
        const Real g11 = (Real)g11d, g12 = (Real)g12d, g22 = (Real)g22d;
        const Real n00 = (Real)(G22 * idG), n01 = (Real)(-G12 * idG), n11 = (Real)(G11 * idG);
        const Real detn = (Real)idG;
        const Real det = g11 * g22 - g12 * g12;
        const Real idet = (Real)1 / det;
        // invariants (stress.cu:90-93) from the metric difference
        const Real i1 = n00 * d11 + (Real)2 * n01 * d12 + n11 * d22;
        const Real i2 = detn * ((Real)G11 * d22 + (Real)G22 * d11 - (Real)2 * (Real)G12 * d12 + d11 * d22 - d12 * d12);
        const Real js = sqrt(i2 + (Real)1);
        const Real jsm1 = i2 / (js + (Real)1);
        Real al, be;   // ca - 1 and cb + 1 of the law (stress.cu:94-99)
        if (a.law == RBC_LAW_SKALAK) {
            al = (rgs * i1 + (rgs - (Real)1) - jsm1) / js;
            be = C * i2 * js - jsm1;
        } else {
            const Real js3 = js * js * js;
            al = ((rgs - (Real)1) - jsm1) / js;
            be = (jsm1 * (js * js + js + (Real)1) - (rgs - (Real)1)) / js3;
        }
        const Real gi00 = g22 * idet, gi01 = -g12 * idet, gi11 = g11 * idet;
        // n D g^-1 = n - g^-1, symmetrised
        const Real p00 = n00 * d11 + n01 * d12, p01 = n00 * d12 + n01 * d22;
        const Real p10 = n01 * d11 + n11 * d12, p11 = n01 * d12 + n11 * d22;
        const Real t00 = al * n00 + be * gi00 + (p00 * gi00 + p01 * gi01);
        const Real t01 = al * n01 + be * gi01 + (Real)0.5 * ((p00 * gi01 + p01 * gi11) + (p10 * gi00 + p11 * gi01));
        const Real t11 = al * n11 + be * gi11 + (p10 * gi01 + p11 * gi11);
        const Real v1x = (Real)e1x, v1y = (Real)e1y, v1z = (Real)e1z;
        const Real v2x = (Real)e2x, v2y = (Real)e2y, v2z = (Real)e2z;
        const Real gab = sqrt(det), h = gab * (Real)0.5;
        // load of the element's vertex en (stress.cu:204, shape-function gradients
        // en 0 (-1,-1), 1 (1,0), 2 (0,1)): h (t^{a0} v1 + t^{a1} v2) for en = 1 (a = 0), 2 (a = 1)
        const Real bx = h * (t00 * v1x + t01 * v2x), by = h * (t00 * v1y + t01 * v2y), bz = h * (t00 * v1z + t01 * v2z);
        const Real cx = h * (t01 * v1x + t11 * v2x), cy = h * (t01 * v1y + t11 * v2y), cz = h * (t01 * v1z + t11 * v2z);
        store_vec4(rec + (size_t)3 * e, make_vec4(-(bx + cx), -(by + cy), -(bz + cz), gab));
        store_vec4(rec + (size_t)3 * e + 1, make_vec4(bx, by, bz, gab));
        store_vec4(rec + (size_t)3 * e + 2, make_vec4(cx, cy, cz, gab));
    }
    __syncthreads();   // the records are written by this CTA and read below (plain loads, not __ldg)

    // vertex pass: matrix row, right-hand side and nodal area of each vertex.
    // Thread tid owns solve positions p = tid + m T, the vertex vord[p] at each.
    float rhs[VPT][3], ds[VPT];
    int vid[VPT];
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int p = tid + m * T;
        rhs[m][0] = rhs[m][1] = rhs[m][2] = 0.f; ds[m] = 0.f;
        vid[m] = 0;
        if (p >= V) continue;
        const int i = __ldg(&a.vord[p]);
        vid[m] = i;
        Real diag = 0, off[6] = {0, 0, 0, 0, 0, 0}, b0 = 0, b1 = 0, b2 = 0, dsum = 0;
        const int k0 = __ldg(&a.v2e_off[i]), k1 = __ldg(&a.v2e_off[i + 1]);
        // all incidence entries first, then all records, then the sums (in list order)
        int pk[MAX_VALENCE];
#pragma unroll
        for (int j = 0; j < MAX_VALENCE; j++) pk[j] = k0 + j < k1 ? __ldg(&a.v2e[k0 + j]) : 0;
        R4 r[MAX_VALENCE];
#pragma unroll
        for (int j = 0; j < MAX_VALENCE; j++)
            if (k0 + j < k1) r[j] = load_vec4(rec + (size_t)3 * v2e_elem(pk[j]) + v2e_en(pk[j]));
#pragma unroll
        for (int j = 0; j < MAX_VALENCE; j++) {
            if (k0 + j >= k1) break;
            const int sa = v2e_sa(pk[j]), sb = v2e_sb(pk[j]);
            const Real gab = r[j].w;
            diag += gab * (Real)(1.0 / 12.0);
            const Real o = gab * (Real)(1.0 / 24.0);
#pragma unroll
            for (int t = 0; t < 6; t++) off[t] += (t == sa ? o : (Real)0) + (t == sb ? o : (Real)0);
            b0 += r[j].x; b1 += r[j].y; b2 += r[j].z;
            dsum += gab * (Real)(1.0 / 6.0);
        }
        const Real idg = (Real)1 / diag;
#pragma unroll
        for (int s = 0; s < 6; s++) coef[s * V + p] = (float)(off[s] * idg);
        rhs[m][0] = (float)(b0 * idg); rhs[m][1] = (float)(b1 * idg); rhs[m][2] = (float)(b2 * idg);
        ds[m] = (float)dsum;
    }
    __syncthreads();   // positions are dead from here; dbuf reuses their space

    const float theta = 1.25f, delta = 0.75f, sigma = theta / delta;
    float x[VPT][3], r[VPT][3], d[VPT][3];
    float rho = 1.0f / sigma, bb = 0.f;
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int p = tid + m * T;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[m][c] = 0.f; r[m][c] = rhs[m][c]; d[m][c] = rhs[m][c] / theta;
            bb += rhs[m][c] * rhs[m][c];
        }
        if (p < V) { dbuf[p] = d[m][0]; dbuf[V + p] = d[m][1]; dbuf[2 * V + p] = d[m][2]; }
    }
    // each vertex's neighbours and row coefficients stay in registers for the
    // whole solve (a missing sixth neighbour points at the vertex itself with
    // coefficient 0)
    unsigned nb[VPT][3];   // two 16-bit neighbour ids per register
    float cf[VPT][6];
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int p = tid + m * T;
#pragma unroll
        for (int s = 0; s < 6; s++) {
            const int j = p < V ? (int)__ldg(&a.nbrp[s * V + p]) : -1;   // neighbours by solve position
            const unsigned id = (unsigned)(j >= 0 ? j : (p < V ? p : 0));
            if (s & 1) nb[m][s >> 1] |= id << 16; else nb[m][s >> 1] = id;
            cf[m][s] = j >= 0 ? coef[s * V + p] : 0.f;
        }
    }
    __syncthreads();
    for (int it = 0; it < a.niter; it++) {
        // one array per component: three 4-byte gathers per neighbour, whose
        // warp-wide reads of nearby positions take one wavefront each
        const float *cur = dbuf + (it & 1) * 3 * V;
        float *nxt = dbuf + ((it + 1) & 1) * 3 * V;
        const float rho_n = 1.0f / (2.0f * sigma - rho);
        const float c1 = rho_n * rho, c2 = 2.0f * rho_n / delta;
#pragma unroll
        for (int m = 0; m < VPT; m++) {
            const int p = tid + m * T;
            if (p >= V) continue;
            float ad0 = d[m][0], ad1 = d[m][1], ad2 = d[m][2];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                const float w = cf[m][s];
                const unsigned j = (s & 1) ? nb[m][s >> 1] >> 16 : nb[m][s >> 1] & 0xFFFFu;
                ad0 += w * cur[j]; ad1 += w * cur[V + j]; ad2 += w * cur[2 * V + j];
            }
            x[m][0] += d[m][0]; x[m][1] += d[m][1]; x[m][2] += d[m][2];
            r[m][0] -= ad0; r[m][1] -= ad1; r[m][2] -= ad2;
#pragma unroll
            for (int c = 0; c < 3; c++) d[m][c] = c1 * d[m][c] + c2 * r[m][c];
            nxt[p] = d[m][0]; nxt[V + p] = d[m][1]; nxt[2 * V + p] = d[m][2];
        }
        rho = rho_n;
        __syncthreads();
    }
    // residual of the scaled system, relative to its right-hand side: the flag
    // is |r| / |b| > 1e-3, compared as squared norms
    float rr = 0.f;
#pragma unroll
    for (int m = 0; m < VPT; m++)
        if (tid + m * T < V)
#pragma unroll
            for (int c = 0; c < 3; c++) rr += r[m][c] * r[m][c];
    rr = block_sum(rr, red);
    bb = block_sum(bb, red);
    if (tid == 0 && rr > 1e-6f * bb && a.flags) atomicOr(a.flags, RBC_FLAG_SOLVE_RESIDUAL);
    // q2f (stress.cu:440-442)
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        if (tid + m * T >= V) continue;
        const int i = vid[m];
        a.Fv[vb + i] = -x[m][0] * ds[m];
        a.Fv[nv + vb + i] = -x[m][1] * ds[m];
        a.Fv[2 * nv + vb + i] = -x[m][2] * ds[m];
    }
}

template <typename Real, int VPT>
__global__ void __launch_bounds__(mem_max_threads<VPT>(), 1)
membrane_kernel(const MembraneArgs a)
{
    pdl_start();
    membrane_body<Real, VPT>(a, blockIdx.x);
}

template <typename Real, int VPT>
static void launch_vpt(const MembraneArgs &a, cudaStream_t s)
{
    const int smem = membrane_smem_bytes(a.V);
    auto k = membrane_kernel<Real, VPT>;
    int T = (a.V + VPT - 1) / VPT;
    T = ((T + 31) / 32) * 32;
    // launched at the given stream priority: when the previous step's volume
    // correction runs beside it, the membrane CTAs are dispatched first
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)a.ncell);
    cfg.blockDim = dim3((unsigned)T);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = a.priority;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, k, a);
}

template <typename Real>
static void launch_real(const MembraneArgs &a, cudaStream_t s)
{
    // fewest vertices per thread whose CTA (rounded to warps) fits the thread cap
    auto fits = [&](int vpt, int cap) { return ((a.V + vpt - 1) / vpt + 31) / 32 * 32 <= cap; };
    if (fits(1, mem_max_threads<1>())) launch_vpt<Real, 1>(a, s);
    else if (fits(2, mem_max_threads<2>())) launch_vpt<Real, 2>(a, s);
    else if (fits(3, mem_max_threads<3>())) launch_vpt<Real, 3>(a, s);
    else launch_vpt<Real, 4>(a, s);   // V <= 3418 (shared-memory limit) fits 4 x 896
}

cudaError_t set_max_dyn_smem(const void *kernel, int optin, int *granted);

// the smallest limit over all instantiations bounds the vertices per cell
cudaError_t membrane_setup(int optin, int *max_bytes)
{
    const void *ks[] = {(const void *)membrane_kernel<float, 1>, (const void *)membrane_kernel<float, 2>,
                        (const void *)membrane_kernel<float, 3>, (const void *)membrane_kernel<float, 4>,
                        (const void *)membrane_kernel<double, 1>, (const void *)membrane_kernel<double, 2>,
                        (const void *)membrane_kernel<double, 3>, (const void *)membrane_kernel<double, 4>};
    int lo = optin;
    for (const void *k : ks) {
        int g = 0;
        cudaError_t e = set_max_dyn_smem(k, optin, &g);
        if (e != cudaSuccess) return e;
        lo = g < lo ? g : lo;
    }
    if (max_bytes) *max_bytes = lo;
    return cudaSuccess;
}

void launch_membrane(const MembraneArgs &a, bool fp64, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    if (fp64) launch_real<double>(a, s);
    else launch_real<float>(a, s);
}

// ---- fused batches ---------------------------------------------------------

template <typename Real, int VPT>
__global__ void __launch_bounds__(mem_max_threads<VPT>(), 1)
membrane_fused_kernel(const DomainArgs *__restrict__ dom, const int *__restrict__ boff, int ndom)
{
    const int d = fused_domain(boff, ndom, blockIdx.x);
    membrane_body<Real, VPT>(dom[d].mem, blockIdx.x - boff[d]);
}

int membrane_threads(int V, int vpt) { return ((V + vpt - 1) / vpt + 31) / 32 * 32; }

int membrane_default_vpt(int V)
{
    if (membrane_threads(V, 1) <= mem_max_threads<1>()) return 1;
    if (membrane_threads(V, 2) <= mem_max_threads<2>()) return 2;
    if (membrane_threads(V, 3) <= mem_max_threads<3>()) return 3;
    return 4;
}

template <typename Real, int VPT>
static void launch_fused_vpt(const FusedLaunch &f, int V, cudaStream_t s)
{
    membrane_fused_kernel<Real, VPT><<<f.nblocks, membrane_threads(V, VPT), membrane_smem_bytes(V), s>>>(
        f.dom, f.boff, f.ndom);
}

template <typename Real>
static void launch_fused_real(const FusedLaunch &f, int V, int vpt, cudaStream_t s)
{
    switch (vpt) {
    case 1: launch_fused_vpt<Real, 1>(f, V, s); break;
    case 2: launch_fused_vpt<Real, 2>(f, V, s); break;
    case 3: launch_fused_vpt<Real, 3>(f, V, s); break;
    default: launch_fused_vpt<Real, 4>(f, V, s); break;
    }
}

void launch_membrane_fused(const FusedLaunch &f, bool fp64, int V, int vpt, cudaStream_t s)
{
    if (f.nblocks <= 0) return;
    if (fp64) launch_fused_real<double>(f, V, vpt, s);
    else launch_fused_real<float>(f, V, vpt, s);
}

cudaError_t membrane_fused_setup(int optin)
{
    const void *ks[] = {(const void *)membrane_fused_kernel<float, 1>, (const void *)membrane_fused_kernel<float, 2>,
                        (const void *)membrane_fused_kernel<float, 3>, (const void *)membrane_fused_kernel<float, 4>,
                        (const void *)membrane_fused_kernel<double, 1>, (const void *)membrane_fused_kernel<double, 2>,
                        (const void *)membrane_fused_kernel<double, 3>, (const void *)membrane_fused_kernel<double, 4>};
    for (const void *k : ks) {
        int g = 0;
        cudaError_t e = set_max_dyn_smem(k, optin, &g);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace rbc
