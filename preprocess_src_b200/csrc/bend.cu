// bend.cu -- four-point dihedral bending forces.
//
// Replaces fourpoint_bend (stress.cu:448-578 of the reference), which runs one
// thread per element, visits the element's three edge neighbours and adds the
// forces of each pair to the pair's vertices with FP64 atomics.  Here one
// thread computes one visit in FP64 and writes the forces on its three vertices
// to a record -- the whole force on the visiting element's vertex off the
// shared edge (k1), half on the shared edge's (k2, k3) -- and a second pass
// gives each vertex the sum of its shares over the visits of its incident
// elements, in incidence order, added to its membrane force once:
// deterministic, no atomics, each visit evaluated once.
//
// Per visit (e1 with neighbour e2 across the edge k2 -> k3 in e1's winding,
// k1 the third vertex of e1, k4 the vertex of e2 off the edge): positions are
// taken as minimum images about k1 (x with LX, z with LZ), xi and ze are the
// two outward normals, pairs with 1 - cos^2 < 1e-6 contribute nothing, and
// the force is beta times the gradient of cos theta with beta = (2 / sqrt 3)
// BR sgn (sin c0 - cos s0) / |sin| (stress.cu:531-535): (2 / sqrt 3) BR with
// the spontaneous angle 0 the reference leaves (c0 = 1, s0 = 0,
// init1.cu:849-850), or with the initial shape's angle of the visit (cs0).
#include "rbc_internal.cuh"

namespace rbc {

__device__ __forceinline__ double min_image(double d, double L) {
    if (d > L * 0.5) d -= L; else if (d < -L * 0.5) d += L;
    return d;
}

constexpr int BEND_THREADS = 128;

// The forces of visit s of element e1 of a cell on its three vertices k1
// (whole), k2 and k3 (half each; e2's visit of the same pair adds the rest):
// f[role][xyz].  false when the visit contributes nothing.
__device__ __forceinline__ bool visit_forces(const BendArgs &a, const double *xs, const double *ys, const double *zs,
                                             int e1, int s, const int4 q, double f[3][3])
{
    const double a1x = xs[q.x], a1y = ys[q.x], a1z = zs[q.x];
    const double a2x = a1x + min_image(xs[q.y] - a1x, a.LX), a2y = ys[q.y], a2z = a1z + min_image(zs[q.y] - a1z, a.LZ);
    const double a3x = a1x + min_image(xs[q.z] - a1x, a.LX), a3y = ys[q.z], a3z = a1z + min_image(zs[q.z] - a1z, a.LZ);
    const double a4x = a1x + min_image(xs[q.w] - a1x, a.LX), a4y = ys[q.w], a4z = a1z + min_image(zs[q.w] - a1z, a.LZ);
    const double a21x = a2x - a1x, a31x = a3x - a1x, a34x = a3x - a4x, a24x = a2x - a4x, a23x = a2x - a3x;
    const double a21y = a2y - a1y, a31y = a3y - a1y, a34y = a3y - a4y, a24y = a2y - a4y, a23y = a2y - a3y;
    const double a21z = a2z - a1z, a31z = a3z - a1z, a34z = a3z - a4z, a24z = a2z - a4z, a23z = a2z - a3z;
    const double xix = a21y * a31z - a21z * a31y, xiy = a21z * a31x - a21x * a31z, xiz = a21x * a31y - a21y * a31x;
    const double zex = a34y * a24z - a34z * a24y, zey = a34z * a24x - a34x * a24z, zez = a34x * a24y - a34y * a24x;
    // the reference's divisions by |xi|, |ze| and sqrt(1 - cos^2) as products with their reciprocals
    const double ixi = 1.0 / sqrt(xix * xix + xiy * xiy + xiz * xiz), ize = 1.0 / sqrt(zex * zex + zey * zey + zez * zez);
    const double cost = (xix * zex + xiy * zey + xiz * zez) * ixi * ize;
    const double cost2 = 1.0 - cost * cost;
    if (cost2 < 1.0e-6) return false;   // (NaN from a degenerate triangle propagates, as in the reference)
    // centroid test of stress.cu:527 for the sign of sin theta
    const double dtx = (a1x - a4x) / 3.0, dty = (a1y - a4y) / 3.0, dtz = (a1z - a4z) / 3.0;
    const double sgn = ((xix - zex) * dtx + (xiy - zey) * dty + (xiz - zez) * dtz) >= 0.0 ? 1.0 : -1.0;
    const double rs = rsqrt(cost2);
    const double sint = sgn * cost2 * rs;
    double c0 = 1.0, s0 = 0.0;
    if (a.cs0) {
        const double2 cs = __ldg(&a.cs0[(long long)e1 * 3 + s]);
        c0 = cs.x; s0 = cs.y;
    }
    const double beta = sgn * a.coef * (sint * c0 - cost * s0) * rs;
    const double b11 = -beta * cost * (ixi * ixi), b12 = beta * ixi * ize, b22 = -beta * cost * (ize * ize);
    f[0][0] = b11 * (xiy * -a23z - xiz * -a23y) + b12 * (zey * -a23z - zez * -a23y);
    f[0][1] = b11 * (xiz * -a23x - xix * -a23z) + b12 * (zez * -a23x - zex * -a23z);
    f[0][2] = b11 * (xix * -a23y - xiy * -a23x) + b12 * (zex * -a23y - zey * -a23x);
    f[1][0] = 0.5 * (b11 * (xiy * -a31z - xiz * -a31y) + b22 * (zey * a34z - zez * a34y)
                     + b12 * ((xiy * a34z - xiz * a34y) + (zey * -a31z - zez * -a31y)));
    f[1][1] = 0.5 * (b11 * (xiz * -a31x - xix * -a31z) + b22 * (zez * a34x - zex * a34z)
                     + b12 * ((xiz * a34x - xix * a34z) + (zez * -a31x - zex * -a31z)));
    f[1][2] = 0.5 * (b11 * (xix * -a31y - xiy * -a31x) + b22 * (zex * a34y - zey * a34x)
                     + b12 * ((xix * a34y - xiy * a34x) + (zex * -a31y - zey * -a31x)));
    f[2][0] = 0.5 * (b11 * (xiy * a21z - xiz * a21y) + b22 * (zey * -a24z - zez * -a24y)
                     + b12 * ((xiy * -a24z - xiz * -a24y) + (zey * a21z - zez * a21y)));
    f[2][1] = 0.5 * (b11 * (xiz * a21x - xix * a21z) + b22 * (zez * -a24x - zex * -a24z)
                     + b12 * ((xiz * -a24x - xix * -a24z) + (zez * a21x - zex * a21z)));
    f[2][2] = 0.5 * (b11 * (xix * a21y - xiy * a21x) + b22 * (zex * -a24y - zey * -a24x)
                     + b12 * ((xix * -a24y - xiy * -a24x) + (zex * a21y - zey * a21x)));
    return true;
}

// pass 1: every visit (cell, e1, s) once, its three vertex forces into a record
__global__ void __launch_bounds__(BEND_THREADS)
bend_visit_kernel(const BendArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;   // (cell * E + e1) * 3 + s
    if (t >= (long long)a.ncell * a.E * 3) return;
    const int cell = (int)(t / (3LL * a.E)), r = (int)(t - 3LL * a.E * cell), e1 = r / 3, s = r - 3 * e1;
    const long long vb = (long long)cell * a.V;
    const double *xs = a.X + vb, *ys = a.X + a.nv + vb, *zs = a.X + 2 * a.nv + vb;
    BendArgs ac = a;
    if (ac.cs0) ac.cs0 += (long long)cell * a.E * 3;
    const int4 q = __ldg(&a.visit[3 * e1 + s]);
    double f[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    if (q.x >= 0) visit_forces(ac, xs, ys, zs, e1, s, q, f);
    double *rec = a.rec + 9 * t;
#pragma unroll
    for (int k = 0; k < 9; k++) rec[k] = f[k / 3][k % 3];
}

// pass 2: each vertex adds its shares of the visits of its incident elements,
// in incidence-list order (deterministic, no atomics)
__global__ void __launch_bounds__(BEND_THREADS)
bend_gather_kernel(const BendArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.nv) return;
    const int cell = (int)(t / a.V), i = (int)(t - (long long)cell * a.V);
    const double *rc = a.rec + 27LL * a.E * cell;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    const int k0 = __ldg(&a.v2e_off[i]), k1e = __ldg(&a.v2e_off[i + 1]);
    for (int k = k0; k < k1e; k++) {
        const int e1 = v2e_elem(__ldg(&a.v2e[k]));
#pragma unroll 1
        for (int s = 0; s < 3; s++) {
            const int4 q = __ldg(&a.visit[3 * e1 + s]);
            if (q.x < 0) continue;
            const int role = i == q.x ? 0 : (i == q.y ? 1 : 2);
            const double *f = rc + 9 * (3 * e1 + s) + 3 * role;
            fx += f[0]; fy += f[1]; fz += f[2];
        }
    }
    a.Fv[t] += (float)fx;
    a.Fv[a.nv + t] += (float)fy;
    a.Fv[2 * a.nv + t] += (float)fz;
}

void launch_bend(const BendArgs &a, cudaStream_t s)
{
    if (a.nv <= 0) return;
    const long long nvis = (long long)a.ncell * a.E * 3;
    bend_visit_kernel<<<(unsigned)((nvis + BEND_THREADS - 1) / BEND_THREADS), BEND_THREADS, 0, s>>>(a);
    bend_gather_kernel<<<(unsigned)((a.nv + BEND_THREADS - 1) / BEND_THREADS), BEND_THREADS, 0, s>>>(a);
}

}  // namespace rbc
