// volume.cu -- FP64 per-cell volume correction, one CTA per cell.
//
// Replaces volume_correction() (volume_correction.cu:453-524 of the reference)
// with CapsulePeriodicBefore/After (28-94), CalcEleNormal (138-200), CalcVolume
// (246-281), CalcLambda1 (378-399), VolumeCorrection_GPU (97-135) and
// CalcCenter (310-352).  The reference iterates on the host: per iteration one
// normal kernel, two thrust::reduce calls per cell and a host->device copy of
// lambda, until every cell has |V - V0| / V0 * 100 < 1e-3 or 1000 iterations.
// A converged cell gets lambda = 0 and never moves again, so each cell's
// sequence of moves does not depend on the other cells: one CTA per cell runs
// that cell's loop on the device with block reductions.  The reference's
// return value (iterations - 1 of the slowest cell) is kept as an atomic max.
// Also the step-begin kernel (iteration counter, drive factor and wall
// velocities, main.cu:75, lbm.cu:752, 1030-1035).
#include "rbc_internal.cuh"

namespace rbc {

constexpr int VOL_THREADS = 1024;
constexpr double COEFF_VOL_CHANGE = 0.1;   // volume_correction.cu:14
constexpr double VC_EPS = 1.0e-3;          // volume_correction.cu:15, percent
constexpr int VC_ITRMAX = 1000;            // volume_correction.cu:487

int volume_smem_bytes(int V) { return 24 * V; }

// block sums of K values at once: per value a warp butterfly, then the warps' sums in warp order
template <int K>
__device__ __forceinline__ void block_sum_k(double (&v)[K], double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < K; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) red[32 * k + wid] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) {
        double s = 0.0;
        for (int w = 0; w < nw; w++) s += red[32 * k + w];
        v[k] = s;
    }
}

// tri_measure of local element e
__device__ __forceinline__ void ele_measure(const double *__restrict__ p, int V, const int *__restrict__ tri, int e,
                                            double &s18v, double &s2a)
{
    const int na = __ldg(&tri[3 * e]), nb = __ldg(&tri[3 * e + 1]), nc = __ldg(&tri[3 * e + 2]);
    const double A[3] = {p[na], p[V + na], p[2 * V + na]};
    const double B[3] = {p[nb], p[V + nb], p[2 * V + nb]};
    const double C[3] = {p[nc], p[V + nc], p[2 * V + nc]};
    tri_measure(A, B, C, s18v, s2a);
}

// unit normal, area and volume contribution of local element e (CalcEleNormal_GPU)
__device__ __forceinline__ void ele_normal(const double *__restrict__ p, int V, const int *__restrict__ tri, int e,
                                           double n[3], double &dS, double &vt)
{
    const int na = __ldg(&tri[3 * e]), nb = __ldg(&tri[3 * e + 1]), nc = __ldg(&tri[3 * e + 2]);
    const double ax = p[na], ay = p[V + na], az = p[2 * V + na];
    const double bx = p[nb], by = p[V + nb], bz = p[2 * V + nb];
    const double cx = p[nc], cy = p[V + nc], cz = p[2 * V + nc];
    const double v1x = bx - ax, v1y = by - ay, v1z = bz - az;
    const double v2x = cx - ax, v2y = cy - ay, v2z = cz - az;
    const double c0 = v1y * v2z - v1z * v2y, c1 = v1z * v2x - v1x * v2z, c2 = v1x * v2y - v1y * v2x;
    const double nc_ = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    n[0] = c0 / nc_; n[1] = c1 / nc_; n[2] = c2 / nc_;
    dS = nc_ / 2.0;
    const double rx = (ax + bx + cx) / 3.0, ry = (ay + by + cy) / 3.0, rz = (az + bz + cz) / 3.0;
    vt = 1.0 / 3.0 * (rx * n[0] + ry * n[1] + rz * n[2]) * dS;
}

// cell: the block's cell, blockIdx.x of a one-population launch
__device__ __forceinline__ void volume_body(const Geom &g, const VolumeArgs &a, int cell)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[3 * 32];
    double *p = reinterpret_cast<double *>(smem);   // [3][V]
    const int V = a.V, E = a.E, tid = threadIdx.x, T = blockDim.x, N = a.ncell;
    const long long vb = (long long)cell * V, nv = a.nv;
    const double gz = a.gx[2 * N + cell], gxx = a.gx[cell];
    // up to four vertices per thread and round, their loads issued before any store
    for (int v0 = tid; v0 < V; v0 += 4 * T) {
        double q[4][3];
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int v = v0 + m * T;
            if (v < V) { q[m][0] = a.X[vb + v]; q[m][1] = a.X[nv + vb + v]; q[m][2] = a.X[2 * nv + vb + v]; }
        }
#pragma unroll
        for (int m = 0; m < 4; m++) {
            const int v = v0 + m * T;
            if (v >= V) break;
            double x = q[m][0], z = q[m][2];
            if (g.xper) {                                   // CapsulePeriodicBefore, x (shear mode)
                const double dxx = x - gxx;
                if (dxx > g.LX * 0.5) x -= g.LX; else if (dxx < -g.LX * 0.5) x += g.LX;
            }
            const double dz = z - gz;                       // CapsulePeriodicBefore, z
            if (dz > g.LZ * 0.5) z -= g.LZ; else if (dz < -g.LZ * 0.5) z += g.LZ;
            p[v] = x; p[V + v] = q[m][1]; p[2 * V + v] = z;
        }
    }
    __syncthreads();

    const double V0 = a.correct ? a.vol0[cell] : 0.0;
    double vol = 0.0, area = 0.0;
    int it = 0;
    for (;;) {
        double s[2] = {0.0, 0.0};
#pragma unroll 2
        for (int e = tid; e < E; e += T) ele_measure(p, V, a.tri, e, s[0], s[1]);
        block_sum_k<2>(s, red);
        vol = s[0] / 18.0;
        area = s[1] / 2.0;
        if (!a.correct) break;
        it++;
        if (fabs(vol - V0) / V0 * 100.0 < VC_EPS) break;
        const double lambda = 18.0 * (vol - V0) / area;
        double disp[4][3];
        for (int m = 0; m < 4; m++) {
            const int v = tid + m * T;
            disp[m][0] = disp[m][1] = disp[m][2] = 0.0;
            if (v >= V) continue;
            const int k0 = __ldg(&a.v2e_off[v]), k1 = __ldg(&a.v2e_off[v + 1]);
            const int nne = k1 - k0;
            double nn0 = 0.0, nn1 = 0.0, nn2 = 0.0;
            for (int k = k0; k < k1; k++) {
                double n[3], dS, vt;
                ele_normal(p, V, a.tri, v2e_elem(__ldg(&a.v2e[k])), n, dS, vt);
                nn0 += n[0] / nne; nn1 += n[1] / nne; nn2 += n[2] / nne;
            }
            disp[m][0] = -lambda / 6.0 * nn0 * COEFF_VOL_CHANGE;
            disp[m][1] = -lambda / 6.0 * nn1 * COEFF_VOL_CHANGE;
            disp[m][2] = -lambda / 6.0 * nn2 * COEFF_VOL_CHANGE;
        }
        __syncthreads();
        for (int m = 0; m < 4; m++) {
            const int v = tid + m * T;
            if (v >= V) continue;
            p[v] += disp[m][0]; p[V + v] += disp[m][1]; p[2 * V + v] += disp[m][2];
        }
        __syncthreads();
        if (it >= VC_ITRMAX) { if (tid == 0) atomicOr(a.flags, RBC_FLAG_VC_NOT_CONVERGED); break; }
    }
    // CalcCenter: vertex mean, wrapped into [zmin, zmax]; with a correction, the same pass
    // stores the positions (CapsulePeriodicAfter)
    double sc[3] = {0.0, 0.0, 0.0};
    for (int v = tid; v < V; v += T) {
        double x = p[v], z = p[2 * V + v];
        sc[0] += x; sc[1] += p[V + v]; sc[2] += z;
        if (a.correct) {
            if (z < g.zmin) z += g.LZ; else if (z > g.zmax) z -= g.LZ;
            if (g.xper) { if (x < g.xmin) x += g.LX; else if (x > g.xmax) x -= g.LX; }   // volume_correction.cu:88-91
            a.X[vb + v] = x;
            a.X[nv + vb + v] = p[V + v];
            a.X[2 * nv + vb + v] = z;
        }
    }
    block_sum_k<3>(sc, red);
    double sx = sc[0] / (double)V, sy = sc[1] / (double)V, sz = sc[2] / (double)V;
    if (sz < g.zmin) sz += g.LZ; else if (sz > g.zmax) sz -= g.LZ;
    if (g.xper) { if (sx < g.xmin) sx += g.LX; else if (sx > g.xmax) sx -= g.LX; }   // volume_correction.cu:319-325
    if (tid == 0) {
        if (a.vol_out) a.vol_out[cell] = vol;
        if (a.area_out) a.area_out[cell] = area;
        double *cen = a.correct ? a.gx : a.cen_out;
        if (cen) { cen[cell] = sx; cen[N + cell] = sy; cen[2 * N + cell] = sz; }
        if (a.correct) { atomicMax(a.vc_max, it - 1); atomicMax(a.vc_last, it - 1); }
    }
}

__global__ void __launch_bounds__(VOL_THREADS)
volume_kernel(const Geom g, const VolumeArgs a)
{
    pdl_start();
    volume_body(g, a, blockIdx.x);
}

void launch_volume(const Geom &g, const VolumeArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    const int smem = volume_smem_bytes(a.V);
    launch_pdl(volume_kernel, dim3(a.ncell), dim3(VOL_THREADS), smem, s, g, a);
}

cudaError_t membrane_setup(int optin, int *max_bytes);
cudaError_t spread_setup();
cudaError_t advect_setup();
cudaError_t adjoint_setup(int optin);
cudaError_t vof_setup();
cudaError_t membrane_fused_setup(int optin);
cudaError_t ibm_fused_setup();
cudaError_t volume_fused_setup(int optin);

// Dynamic shared memory limit of a kernel: the device's per-block opt-in
// maximum minus the kernel's static shared memory.
cudaError_t set_max_dyn_smem(const void *kernel, int optin, int *granted)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    const int bytes = optin - (int)fa.sharedSizeBytes;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (granted) *granted = bytes;
    return e;
}

int setup_kernel_attributes(int *membrane_max_smem)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return (int)e;
    if ((e = set_max_dyn_smem((const void *)volume_kernel, optin, nullptr)) != cudaSuccess) return (int)e;
    if ((e = membrane_setup(optin, membrane_max_smem)) != cudaSuccess) return (int)e;
    if ((e = spread_setup()) != cudaSuccess) return (int)e;
    if ((e = advect_setup()) != cudaSuccess) return (int)e;
    if ((e = adjoint_setup(optin)) != cudaSuccess) return (int)e;
    if ((e = vof_setup()) != cudaSuccess) return (int)e;
    if ((e = membrane_fused_setup(optin)) != cudaSuccess) return (int)e;
    if ((e = ibm_fused_setup()) != cudaSuccess) return (int)e;
    if ((e = volume_fused_setup(optin)) != cudaSuccess) return (int)e;
    return 0;
}

__device__ __forceinline__ void step_begin_body(const StepBeginArgs &a)
{
    const int it = *a.iter + 1;
    *a.iter = it;
    const double wi = (it > a.flowstart) ? 1.0 + 0.5 * sin(M_PI * a.dt * (double)it / a.freq) : 0.0;
    *a.drive = (float)(a.P * wi);
    if (a.drive_rec) *a.drive_rec = (float)(a.P * wi);   // kept for the adjoint of the step
    if (a.factor_rec) *a.factor_rec = wi;
    if (a.vc_last) *a.vc_last = 0;
    if (a.wall) {   // lbm.cu:752 (sra), 946-964: allwall -/+ sra LY/2, topwall sra LY at the top
        const double sra = (it < a.flowstart) ? 0.0 : a.sr;
        a.wall[0] = (float)(a.walls == 0 ? sra * a.LY / 2.0 : sra * a.LY);
        a.wall[1] = (float)(a.walls == 0 ? -sra * a.LY / 2.0 : 0.0);
    }
}

__global__ void step_begin_kernel(const StepBeginArgs a)
{
    pdl_start();
    step_begin_body(a);
}

void launch_step_begin(const StepBeginArgs &a, cudaStream_t s)
{
    launch_pdl(step_begin_kernel, dim3(1), dim3(1), 0, s, a);
}

// ---- fused batches ---------------------------------------------------------

__global__ void step_begin_fused_kernel(const DomainArgs *__restrict__ dom, int ndom)
{
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d < ndom) step_begin_body(dom[d].sb);
}

void launch_step_begin_fused(const FusedLaunch &f, cudaStream_t s)
{
    step_begin_fused_kernel<<<(f.ndom + 127) / 128, 128, 0, s>>>(f.dom, f.ndom);
}

// the force reset of every domain after its collide-stream launch, one warp
// per 32 occupancy words
__global__ void __launch_bounds__(FUSED_CLEAR_THREADS)
clear_bits_fused_kernel(const DomainArgs *__restrict__ dom, const int *__restrict__ boff, int ndom)
{
    const int d = fused_domain(boff, ndom, blockIdx.x);
    const DomainArgs &D = dom[d];
    const long long nw = (long long)D.g.nzc * D.F.wpp;
    const long long w0 = (((long long)(blockIdx.x - boff[d]) * FUSED_CLEAR_THREADS + threadIdx.x) >> 5) * 32;
    if (w0 < nw) force_reset_words(D.F.F, D.F.bits, w0, nw, D.F.wpp, D.g.plane, D.g.nint, threadIdx.x & 31);
}

void launch_clear_bits_fused(const FusedLaunch &f, cudaStream_t s)
{
    if (f.nblocks > 0) clear_bits_fused_kernel<<<f.nblocks, FUSED_CLEAR_THREADS, 0, s>>>(f.dom, f.boff, f.ndom);
}

__global__ void __launch_bounds__(VOL_THREADS)
volume_fused_kernel(const DomainArgs *__restrict__ dom, const int *__restrict__ boff, int ndom)
{
    const int d = fused_domain(boff, ndom, blockIdx.x);
    volume_body(dom[d].g, dom[d].vol, blockIdx.x - boff[d]);
}

cudaError_t volume_fused_setup(int optin)
{
    return set_max_dyn_smem((const void *)volume_fused_kernel, optin, nullptr);
}

void launch_volume_fused(const FusedLaunch &f, int V, cudaStream_t s)
{
    if (f.nblocks > 0)
        volume_fused_kernel<<<f.nblocks, VOL_THREADS, volume_smem_bytes(V), s>>>(f.dom, f.boff, f.ndom);
}

}  // namespace rbc
