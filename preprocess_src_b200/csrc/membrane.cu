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
//  1. the cell's FP64 positions go to shared memory, unwrapped about vertex 0
//     (the reference applies the same minimum-image shift per edge);
//  2. each thread gathers the rows of its vertices through the vertex ->
//     element incidence list (fixed order, no atomics): tension, matrix row,
//     right-hand side and nodal area;
//  3. the scaled system is solved by Chebyshev iteration.  For any P1 triangle
//     mesh the element mass matrix is (A/12)(1 + delta_ij), so every
//     eigenvalue of D^-1 M lies in [1/2, 2] (Rayleigh quotients of an assembled
//     sum of element matrices stay inside the element bounds).  With these
//     bounds Chebyshev needs no inner products: the error falls by at least
//     (sqrt(4)-1)/(sqrt(4)+1) = 1/3 per iteration, one barrier per iteration.
//     (Chebyshev iteration as in Y. Saad, Iterative Methods for Sparse Linear
//     Systems, 2nd ed., Alg. 12.1.)
//  4. f_i = -q_i * ds_i is written out.
// Element mechanics run in FP32 or FP64 (Real); the solve runs in FP32.
#include "rbc_internal.cuh"

namespace rbc {

constexpr int MEM_MAX_THREADS = 1024;

int membrane_smem_bytes(int V) { return 60 * V; }   // pos 24V (later 2x3 FP32 d-buffers), coef 24V, nbr 12V

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

template <typename Real, int VPT>
__global__ void __launch_bounds__(MEM_MAX_THREADS, 1)
membrane_kernel(const MembraneArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ float red[32];
    const int V = a.V, E = a.E, tid = threadIdx.x, T = blockDim.x;
    double *pos = reinterpret_cast<double *>(smem);                    // [3][V]
    float *dbuf = reinterpret_cast<float *>(smem);                     // [2][3][V], after assembly
    float *coef = reinterpret_cast<float *>(smem + 24 * (size_t)V);    // [6][V]
    int16_t *snbr = reinterpret_cast<int16_t *>(smem + 48 * (size_t)V);// [6][V]

    const int cell = blockIdx.x;
    const long long vb = (long long)cell * V, eb = (long long)cell * E, nv = a.nv, ne = a.ne;
    const double ax = a.Xd[vb], ay = a.Xd[nv + vb], az = a.Xd[2 * nv + vb];
    for (int v = tid; v < V; v += T) {
        pos[v] = mimage(a.Xd[vb + v] - ax, a.LX);
        pos[V + v] = a.Xd[nv + vb + v] - ay;
        pos[2 * V + v] = mimage(a.Xd[2 * nv + vb + v] - az, a.LZ);
    }
    for (int k = tid; k < 6 * V; k += T) snbr[k] = a.nbr[k];
    __syncthreads();

    const Real C = (Real)a.C, rgs = (Real)a.rgs;
    float rhs[VPT][3], ds[VPT];
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
        rhs[m][0] = rhs[m][1] = rhs[m][2] = 0.f; ds[m] = 0.f;
        if (i >= V) continue;
        Real diag = 0, off[6] = {0, 0, 0, 0, 0, 0}, b0 = 0, b1 = 0, b2 = 0, dsum = 0;
        const int k0 = __ldg(&a.v2e_off[i]), k1 = __ldg(&a.v2e_off[i + 1]);
        for (int k = k0; k < k1; k++) {
            const int pk = __ldg(&a.v2e[k]);
            const int e = v2e_elem(pk), en = v2e_en(pk);
            const int ia = __ldg(&a.tri[3 * e]), ib = __ldg(&a.tri[3 * e + 1]), ic = __ldg(&a.tri[3 * e + 2]);
            const Real v1x = (Real)(pos[ib] - pos[ia]), v1y = (Real)(pos[V + ib] - pos[V + ia]), v1z = (Real)(pos[2 * V + ib] - pos[2 * V + ia]);
            const Real v2x = (Real)(pos[ic] - pos[ia]), v2y = (Real)(pos[V + ic] - pos[V + ia]), v2z = (Real)(pos[2 * V + ic] - pos[2 * V + ia]);
            // deformed covariant metric and its inverse (stress.cu:75-88)
            const Real g11 = v1x * v1x + v1y * v1y + v1z * v1z;
            const Real g12 = v1x * v2x + v1y * v2y + v1z * v2z;
            const Real g22 = v2x * v2x + v2y * v2y + v2z * v2z;
            const Real det = g11 * g22 - g12 * g12;
            const Real idet = (Real)1 / det;
            const Real n00 = (Real)__ldg(&a.nref[eb + e]), n01 = (Real)__ldg(&a.nref[ne + eb + e]), n11 = (Real)__ldg(&a.nref[2 * ne + eb + e]);
            // invariants (stress.cu:90-93)
            const Real i1 = n00 * g11 + (Real)2 * n01 * g12 + n11 * g22 - (Real)2;
            const Real i2 = det * (n00 * n11 - n01 * n01) - (Real)1;
            const Real js = sqrt(i2 + (Real)1);
            Real ca, cb;   // t = ca * n_ref + cb * g^-1 (stress.cu:94-99)
            if (a.law == RBC_LAW_SKALAK) { ca = rgs * (i1 + (Real)1) / js; cb = (C * i2 - (Real)1) * js; }
            else { ca = rgs / js; cb = -rgs * js / ((i2 + (Real)1) * (i2 + (Real)1)); }
            const Real t00 = ca * n00 + cb * g22 * idet;
            const Real t01 = ca * n01 - cb * g12 * idet;
            const Real t11 = ca * n11 + cb * g11 * idet;
            const Real gab = sqrt(det);
            diag += gab * (Real)(1.0 / 12.0);
            const Real o = gab * (Real)(1.0 / 24.0);
            off[v2e_sa(pk)] += o;
            off[v2e_sb(pk)] += o;
            // shape-function gradients (stress.cu:204): en 0 (-1,-1), 1 (1,0), 2 (0,1)
            const Real f0 = en == 1 ? (Real)1 : (en == 0 ? (Real)-1 : (Real)0);
            const Real f1 = en == 2 ? (Real)1 : (en == 0 ? (Real)-1 : (Real)0);
            const Real h = gab * (Real)0.5;
            const Real c0 = h * (t00 * f0 + t01 * f1), c1 = h * (t01 * f0 + t11 * f1);
            b0 += c0 * v1x + c1 * v2x;
            b1 += c0 * v1y + c1 * v2y;
            b2 += c0 * v1z + c1 * v2z;
            dsum += gab * (Real)(1.0 / 6.0);
        }
        const Real idg = (Real)1 / diag;
#pragma unroll
        for (int s = 0; s < 6; s++) coef[s * V + i] = (float)(off[s] * idg);
        rhs[m][0] = (float)(b0 * idg); rhs[m][1] = (float)(b1 * idg); rhs[m][2] = (float)(b2 * idg);
        ds[m] = (float)dsum;
    }
    __syncthreads();   // positions are dead from here; dbuf reuses their space

    const float theta = 1.25f, delta = 0.75f, sigma = theta / delta;
    float x[VPT][3], r[VPT][3], d[VPT][3];
    float rho = 1.0f / sigma, bb = 0.f;
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
#pragma unroll
        for (int c = 0; c < 3; c++) {
            x[m][c] = 0.f; r[m][c] = rhs[m][c]; d[m][c] = rhs[m][c] / theta;
            bb += rhs[m][c] * rhs[m][c];
            if (i < V) dbuf[c * V + i] = d[m][c];
        }
    }
    __syncthreads();
    for (int it = 0; it < a.niter; it++) {
        const float *cur = dbuf + (it & 1) * 3 * V;
        float *nxt = dbuf + ((it + 1) & 1) * 3 * V;
        const float rho_n = 1.0f / (2.0f * sigma - rho);
        const float c1 = rho_n * rho, c2 = 2.0f * rho_n / delta;
#pragma unroll
        for (int m = 0; m < VPT; m++) {
            const int i = tid + m * T;
            if (i >= V) continue;
            float ad0 = d[m][0], ad1 = d[m][1], ad2 = d[m][2];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                const int j = snbr[s * V + i];
                if (j >= 0) {
                    const float w = coef[s * V + i];
                    ad0 += w * cur[j]; ad1 += w * cur[V + j]; ad2 += w * cur[2 * V + j];
                }
            }
            x[m][0] += d[m][0]; x[m][1] += d[m][1]; x[m][2] += d[m][2];
            r[m][0] -= ad0; r[m][1] -= ad1; r[m][2] -= ad2;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                d[m][c] = c1 * d[m][c] + c2 * r[m][c];
                nxt[c * V + i] = d[m][c];
            }
        }
        rho = rho_n;
        __syncthreads();
    }
    // residual of the scaled system, relative to its right-hand side
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
        const int i = tid + m * T;
        if (i >= V) continue;
        a.Fv[vb + i] = -x[m][0] * ds[m];
        a.Fv[nv + vb + i] = -x[m][1] * ds[m];
        a.Fv[2 * nv + vb + i] = -x[m][2] * ds[m];
    }
}

template <typename Real, int VPT>
static void launch_vpt(const MembraneArgs &a, cudaStream_t s)
{
    const int smem = membrane_smem_bytes(a.V);
    auto k = membrane_kernel<Real, VPT>;
    int T = (a.V + VPT - 1) / VPT;
    T = ((T + 31) / 32) * 32;
    k<<<a.ncell, T, smem, s>>>(a);
}

template <typename Real>
static void launch_real(const MembraneArgs &a, cudaStream_t s)
{
    const int vpt = (a.V + MEM_MAX_THREADS - 1) / MEM_MAX_THREADS;
    switch (vpt) {
    case 1: launch_vpt<Real, 1>(a, s); break;
    case 2: launch_vpt<Real, 2>(a, s); break;
    case 3: launch_vpt<Real, 3>(a, s); break;
    default: launch_vpt<Real, 4>(a, s); break;
    }
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

}  // namespace rbc
