// metrics_noalloc.cu -- per-cell volume / area / centroid without allocating.
//
// rbc_cell_metrics computes these through a handle, whose creation allocates
// device memory and whose metrics kernel writes into device buffers the handle
// owns.  Some callers cannot allocate: code inside a framework that owns the
// whole device memory pool, real-time loops that must not call the allocator,
// or host code that only holds device pointers handed to it.  This entry point
// takes the caller's device positions and triangle list and writes the results
// to the caller's host arrays; its only device scratch is the file-scope array
// below, sized for RBC_NOALLOC_MAX_CELLS cells (160 KB, resident on every GPU
// that loads the library until the process exits).
#include <mutex>
#include <string>

#include "rbc_internal.cuh"

namespace rbc {
void set_last_error(const std::string &msg);   // rbc_last_error(NULL) text (rbc_abi.cu)
}

namespace {

constexpr int kMaxDevices = 64;
constexpr int kThreads = 1024;
constexpr int kMaxVertex = RBC_NOALLOC_MAX_VERTEX;

// Scratch of the kernel: volume [N], area [N], then the centroids [N][3]
// (x, y, z of each cell in turn, the layout of rbc_cell_metrics' centroid
// output).  Every call overwrites the first 5 * ncell entries, so nothing
// there needs clearing.  The last slot counts triangle entries outside
// [0, vertex); each call clears it before its kernel.  Calls that overlap on
// the GPU share this array and race.
constexpr int kFlagSlot = 5 * RBC_NOALLOC_MAX_CELLS;
static __device__ __align__(256) double g_metrics_scratch[5 * RBC_NOALLOC_MAX_CELLS + 1];

// In host code g_metrics_scratch names a host-side stand-in, not device
// memory; the device address is looked up once per device with that device
// current (cudaGetSymbolAddress) and cached here.
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

__device__ __forceinline__ double block_sum(double v, double *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    for (int k = 0; k < nw; k++) s += red[k];
    return s;
}

// One CTA per cell: positions unwrapped about the cell's first vertex along z
// and, when x is periodic (LX > 0, the shear mode), along x; then the volume
// sum (r . n) dS / 3, the area and the vertex mean of CalcEleNormal_GPU /
// CalcCenter (volume_correction.cu:138-200, 310-352), the centroid wrapped
// into [zmin, zmax] (and [xmin, xmax]) as volume_correction.cu:319-325 does.
// A triangle entry outside [0, V) is skipped and counted in *bad.
__global__ void __launch_bounds__(kThreads)
metrics_noalloc_kernel(const double *__restrict__ X, long long nv, const int *__restrict__ tri, int V, int E,
                       int ncell, double LX, double xmin, double xmax, double LZ, double zmin, double zmax,
                       double *__restrict__ out, unsigned int *__restrict__ bad)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[32];
    double *p = reinterpret_cast<double *>(smem);   // [3][V]
    const int cell = blockIdx.x, tid = threadIdx.x, T = blockDim.x;
    const long long vb = (long long)cell * V;
    const double x0 = X[vb], z0 = X[2 * nv + vb];
    const bool xper = LX > 0.0;
    for (int v = tid; v < V; v += T) {
        double x = X[vb + v];
        if (xper) {
            const double dx = x - x0;
            if (dx > 0.5 * LX) x -= LX; else if (dx < -0.5 * LX) x += LX;
        }
        p[v] = x;
        p[V + v] = X[nv + vb + v];
        double z = X[2 * nv + vb + v];
        const double dz = z - z0;
        if (dz > 0.5 * LZ) z -= LZ; else if (dz < -0.5 * LZ) z += LZ;
        p[2 * V + v] = z;
    }
    __syncthreads();
    double sv = 0.0, sa = 0.0;
    unsigned int nbad = 0;
    for (int e = tid; e < E; e += T) {
        const int na = tri[3 * e], nb = tri[3 * e + 1], nc = tri[3 * e + 2];
        if ((unsigned)na >= (unsigned)V || (unsigned)nb >= (unsigned)V || (unsigned)nc >= (unsigned)V) {
            nbad++;
            continue;
        }
        const double ax = p[na], ay = p[V + na], az = p[2 * V + na];
        const double bx = p[nb], by = p[V + nb], bz = p[2 * V + nb];
        const double cx = p[nc], cy = p[V + nc], cz = p[2 * V + nc];
        const double v1x = bx - ax, v1y = by - ay, v1z = bz - az, v2x = cx - ax, v2y = cy - ay, v2z = cz - az;
        const double c0 = v1y * v2z - v1z * v2y, c1 = v1z * v2x - v1x * v2z, c2 = v1x * v2y - v1y * v2x;
        const double nn = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
        const double dS = nn / 2.0;
        const double rx = (ax + bx + cx) / 3.0, ry = (ay + by + cy) / 3.0, rz = (az + bz + cz) / 3.0;
        sv += 1.0 / 3.0 * (rx * c0 / nn + ry * c1 / nn + rz * c2 / nn) * dS;
        sa += dS;
    }
    if (nbad) atomicAdd(bad, nbad);
    const double vol = block_sum(sv, red);
    const double area = block_sum(sa, red);
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int v = tid; v < V; v += T) { sx += p[v]; sy += p[V + v]; sz += p[2 * V + v]; }
    sx = block_sum(sx, red) / (double)V;
    sy = block_sum(sy, red) / (double)V;
    sz = block_sum(sz, red) / (double)V;
    if (sz < zmin) sz += LZ; else if (sz > zmax) sz -= LZ;
    if (xper) { if (sx < xmin) sx += LX; else if (sx > xmax) sx -= LX; }
    if (tid == 0) {
        out[cell] = vol;
        out[ncell + cell] = area;
        out[2 * ncell + 3 * cell] = sx;
        out[2 * ncell + 3 * cell + 1] = sy;
        out[2 * ncell + 3 * cell + 2] = sz;
    }
}

// Once per device, with that device current: the scratch array's device
// address and the kernel's shared-memory limit.  Neither allocates.
int setup_device(int dev, double **addr)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_addr[dev]) { *addr = g_scratch_addr[dev]; return RBC_OK; }
    double *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_metrics_scratch);
    if (e != cudaSuccess) {
        rbc::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    e = cudaFuncSetAttribute(metrics_noalloc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 24 * kMaxVertex);
    if (e != cudaSuccess) {
        rbc::set_last_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    g_scratch_addr[dev] = ptr;
    *addr = ptr;
    return RBC_OK;
}

}  // namespace

namespace {

// Runs the call on device dev (current on entry); the caller restores its own
// current device afterwards.
int metrics_on_device(int dev, const double *x, int ncell, int vertex, int element, const int *tri, double LX,
                      double xmin, double xmax, double LZ, double zmin, double zmax, void *stream, double *volume,
                      double *area, double *centroid)
{
    double *scratch = nullptr;
    int rc = setup_device(dev, &scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const long long nv = (long long)ncell * vertex;
    unsigned int *bad = reinterpret_cast<unsigned int *>(scratch + kFlagSlot);
    unsigned int nbad = 0;
    cudaError_t e = cudaMemsetAsync(bad, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        metrics_noalloc_kernel<<<ncell, kThreads, 24 * vertex, s>>>(x, nv, tri, vertex, element, ncell, LX, xmin,
                                                                    xmax, LZ, zmin, zmax, scratch, bad);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(volume, scratch, sizeof(double) * ncell, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(area, scratch + ncell, sizeof(double) * ncell, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(centroid, scratch + 2 * ncell, sizeof(double) * 3 * ncell, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&nbad, bad, sizeof(unsigned int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        rbc::set_last_error(std::string("rbc_cell_metrics_noalloc: ") + cudaGetErrorString(e));
        return RBC_ERR_CUDA;
    }
    if (nbad) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: " + std::to_string(nbad) +
                            " triangle entries outside 0..vertex-1 (those triangles were skipped)");
        return RBC_ERR_ARG;
    }
    return RBC_OK;
}

}  // namespace

extern "C" int rbc_cell_metrics_noalloc(const double *x, int ncell, int vertex, int element, const int *tri,
                                        double LX, double xmin, double xmax, double LZ, double zmin, double zmax,
                                        int device, void *stream, double *volume, double *area, double *centroid)
{
    if (!x || !tri || !volume || !area || !centroid) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: NULL pointer argument");
        return RBC_ERR_ARG;
    }
    if (ncell < 1 || ncell > RBC_NOALLOC_MAX_CELLS) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: ncell = " + std::to_string(ncell) +
                            " is outside 1.." + std::to_string(RBC_NOALLOC_MAX_CELLS) +
                            " (its static scratch holds RBC_NOALLOC_MAX_CELLS cells)");
        return RBC_ERR_ARG;
    }
    if (vertex < 4 || vertex > kMaxVertex || element < 4) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: vertex = " + std::to_string(vertex) + " must be 4.." +
                            std::to_string(kMaxVertex) + " and element >= 4");
        return RBC_ERR_ARG;
    }
    if (!(LZ > 0)) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: LZ must be > 0");
        return RBC_ERR_ARG;
    }
    if (LX > 0 && !(xmax > xmin)) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: a periodic x (LX > 0) needs xmin < xmax");
        return RBC_ERR_ARG;
    }
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) {
        rbc::set_last_error(std::string("rbc_cell_metrics_noalloc: no current CUDA device: ") + cudaGetErrorString(e));
        return RBC_ERR_NO_DEVICE;
    }
    const int dev = device < 0 ? prev : device;
    if (dev >= kMaxDevices) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: device ordinal above 63");
        return RBC_ERR_ARG;
    }
    if (dev != prev && cudaSetDevice(dev) != cudaSuccess) {
        rbc::set_last_error("rbc_cell_metrics_noalloc: cannot select device " + std::to_string(dev));
        return RBC_ERR_CUDA;
    }
    const int rc = metrics_on_device(dev, x, ncell, vertex, element, tri, LX > 0 ? LX : 0.0, xmin, xmax, LZ, zmin,
                                     zmax, stream, volume, area, centroid);
    if (dev != prev) cudaSetDevice(prev);   // the caller's current device is left as it was
    return rc;
}
