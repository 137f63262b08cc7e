// accum.cu -- output-interval averages of the load and the principal tensions.
//
// The reference keeps two diagnostics for its output files: fem->qi, the load
// q of the membrane solve averaged over the FILEOUTPUT steps of an output
// interval (substitute_load, stress.cu:280-300), and fem->tp, the two
// principal tensions of every element averaged the same way (calc_tension,
// stress.cu:101-118).  Both are reset in the first step of an interval
// ((iter - 1) % FILEOUTPUT == 0) and gain M / FILEOUTPUT times the step's
// value in every step.  They run only when an output interval is set, after
// the membrane kernel and before bending (the reference's load excludes it).
//
// The load comes back from the membrane forces: the membrane kernel stores
// Fv = -q ds with ds = one-ring area / 3 (q2f, stress.cu:440-442), so
// q = -Fv / ds with ds recomputed from the same positions.
#include "rbc_internal.cuh"

namespace rbc {

__device__ __forceinline__ double mimage_acc(double d, double L) {
    if (d > L * 0.5) d -= L; else if (d < -L * 0.5) d += L;
    return d;
}

// edge vectors of local element e (minimum image in x and z, stress.cu:61-70)
__device__ __forceinline__ void acc_edges(const AccumArgs &a, long long vb, int e, double (&v1)[3], double (&v2)[3]) {
    const int ia = __ldg(&a.tri[3 * e]), ib = __ldg(&a.tri[3 * e + 1]), ic = __ldg(&a.tri[3 * e + 2]);
    const double *xs = a.Xd + vb, *ys = a.Xd + a.nv + vb, *zs = a.Xd + 2 * a.nv + vb;
    v1[0] = mimage_acc(xs[ib] - xs[ia], a.LX); v1[1] = ys[ib] - ys[ia]; v1[2] = mimage_acc(zs[ib] - zs[ia], a.LZ);
    v2[0] = mimage_acc(xs[ic] - xs[ia], a.LX); v2[1] = ys[ic] - ys[ia]; v2[2] = mimage_acc(zs[ic] - zs[ia], a.LZ);
}

// One thread per element of any cell: principal tensions (stress.cu:76-118).
__global__ void accum_tension_kernel(const AccumArgs a)
{
    const long long eg = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (eg >= a.ne) return;
    const int cell = (int)(eg / a.E), e = (int)(eg - (long long)cell * a.E);
    double v1[3], v2[3];
    acc_edges(a, (long long)cell * a.V, e, v1, v2);
    const double l1 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
    const double l2 = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2];
    const double i12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
    const double dv12 = l1 * l2 - i12 * i12;
    const double4 G = a.gref[eg];   // covariant reference metric, G.w = 1 / det G = det n
    const double n00 = G.z * G.w, n01 = -G.y * G.w, n11 = G.x * G.w;
    const double i1 = n00 * l1 + 2.0 * n01 * i12 + n11 * l2 - 2.0;
    const double i2 = dv12 * G.w - 1.0;
    const double judge = fabs((i1 + 2.0) * (i1 + 2.0) - 4.0 * (i2 + 1.0));
    const double root = sqrt(judge);
    const double lam1_2 = 0.5 * (i1 + 2.0 + root), lam2_2 = 0.5 * (i1 + 2.0 - root);
    const double lam1_1 = sqrt(lam1_2), lam2_1 = sqrt(lam2_2);
    const double w = (double)a.M / (double)a.fileoutput;
    const bool reset = (*a.iter - 1) % a.fileoutput == 0;
    double *tp = a.tp + 2 * eg;
    tp[0] = (reset ? 0.0 : tp[0]) + w * lam1_1 / lam2_1 * (lam1_2 - 1.0 + a.C * lam2_2 * i2);
    tp[1] = (reset ? 0.0 : tp[1]) + w * lam2_1 / lam1_1 * (lam2_2 - 1.0 + a.C * lam1_2 * i2);
}

// One thread per vertex of any cell: q = -Fv / ds, stored per cell as the
// reference's qd (3 V values per cell, AoS per vertex, cell stride 3 V).
__global__ void accum_load_kernel(const AccumArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.nv) return;
    const int cell = (int)(t / a.V), i = (int)(t - (long long)cell * a.V);
    const long long vb = (long long)cell * a.V;
    double ds = 0.0;
    for (int k = __ldg(&a.v2e_off[i]); k < __ldg(&a.v2e_off[i + 1]); k++) {
        double v1[3], v2[3];
        acc_edges(a, vb, v2e_elem(__ldg(&a.v2e[k])), v1, v2);
        const double c0 = v1[1] * v2[2] - v1[2] * v2[1], c1 = v1[2] * v2[0] - v1[0] * v2[2], c2 = v1[0] * v2[1] - v1[1] * v2[0];
        ds += 0.5 * sqrt(c0 * c0 + c1 * c1 + c2 * c2) / 3.0;
    }
    const double w = (double)a.M / (double)a.fileoutput;
    const bool reset = (*a.iter - 1) % a.fileoutput == 0;
    double *qi = a.qi + 3 * t;
    for (int c = 0; c < 3; c++) {
        const double q = -(double)a.Fv[(long long)c * a.nv + t] / ds;
        qi[c] = (reset ? 0.0 : qi[c]) + w * q;
    }
}

void launch_output_accum(const AccumArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0 || a.fileoutput <= 0) return;
    accum_tension_kernel<<<(unsigned)((a.ne + 127) / 128), 128, 0, s>>>(a);
    accum_load_kernel<<<(unsigned)((a.nv + 127) / 128), 128, 0, s>>>(a);
}

}  // namespace rbc
