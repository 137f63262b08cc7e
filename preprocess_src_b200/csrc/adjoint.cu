// adjoint.cu -- reverse sweep of one step: the discrete adjoint of this
// library's forward step.
//
// Step t maps the state (g_t, X_t, Xd_t) -- populations, corrected positions
// (cel->x), positions before the correction (fem->xd) -- to the next one:
//   Fv     = membrane(Xd_t; C)             Skalak loads, mass-matrix solve, q2f
//   F      = spread(X_t, Fv)               4-point delta over the lattice
//   g_t+1, u = collide(pull(g_t), F; P, B) BGK + Guo forcing, velocity u
//   Xa     = advect(X_t, u)                RK4 in the frozen field
//   Xd_t+1 = Xa,   X_t+1 = volume_correction(Xa)
// The kernels below take the adjoints of a stage's outputs and return those of
// its inputs.  Nonlinear pointwise maps -- the collision of one node, the
// Skalak loads of one element, the normal / area / volume of one triangle --
// are written once as templates on the scalar type; a forward-mode dual number
// (value plus one derivative) seeded on one input at a time gives one column
// of their Jacobian, which is contracted with the output adjoint.  The linear
// global operators are transposed explicitly: pull streaming with half-way
// bounce-back becomes a gather of the downstream nodes' adjoints; spreading
// and interpolation are each other's transpose (plus the derivative of the
// delta weights with respect to the vertex position); RK4 runs its stages
// backwards; the mass-matrix solve M q = b (M symmetric) is reversed with the
// same Chebyshev solver; the volume correction's iterations are replayed and
// reversed one by one.
#include "rbc_internal.cuh"

namespace rbc {

// ---- forward-mode dual numbers -------------------------------------------

using ::sqrt;   // the plain overloads next to the dual one below

template <typename R> struct Dual {
    R v, d;
    __device__ Dual() : v(0), d(0) {}
    __device__ Dual(R x) : v(x), d(0) {}
    __device__ Dual(R x, R dx) : v(x), d(dx) {}
};
template <typename R> __device__ __forceinline__ Dual<R> operator+(Dual<R> a, Dual<R> b) { return Dual<R>(a.v + b.v, a.d + b.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator-(Dual<R> a, Dual<R> b) { return Dual<R>(a.v - b.v, a.d - b.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator-(Dual<R> a) { return Dual<R>(-a.v, -a.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator*(Dual<R> a, Dual<R> b) { return Dual<R>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator/(Dual<R> a, Dual<R> b) {
    const R q = a.v / b.v;
    return Dual<R>(q, (a.d - q * b.d) / b.v);
}
template <typename R> __device__ __forceinline__ Dual<R> operator+(Dual<R> a, R b) { return Dual<R>(a.v + b, a.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator+(R a, Dual<R> b) { return Dual<R>(a + b.v, b.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator-(Dual<R> a, R b) { return Dual<R>(a.v - b, a.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator-(R a, Dual<R> b) { return Dual<R>(a - b.v, -b.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator*(Dual<R> a, R b) { return Dual<R>(a.v * b, a.d * b); }
template <typename R> __device__ __forceinline__ Dual<R> operator*(R a, Dual<R> b) { return Dual<R>(a * b.v, a * b.d); }
template <typename R> __device__ __forceinline__ Dual<R> operator/(Dual<R> a, R b) { return Dual<R>(a.v / b, a.d / b); }
template <typename R> __device__ __forceinline__ Dual<R> operator/(R a, Dual<R> b) {
    const R q = a / b.v;
    return Dual<R>(q, -q * b.d / b.v);
}
template <typename R> __device__ __forceinline__ Dual<R> &operator+=(Dual<R> &a, Dual<R> b) { a = a + b; return a; }
template <typename R> __device__ __forceinline__ Dual<R> &operator-=(Dual<R> &a, Dual<R> b) { a = a - b; return a; }
template <typename R> __device__ __forceinline__ Dual<R> sqrt(Dual<R> a) {
    const R s = sqrt(a.v);
    return Dual<R>(s, a.d / (R(2) * s));
}

template <typename R>
__device__ __forceinline__ R block_sum_r(R v, R *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    R s = 0;
    for (int k = 0; k < nw; k++) s += red[k];
    return s;
}

// ---- collide-stream ----------------------------------------------------------

// The collision of one node as lbm.cu computes it (collision_terms +
// post_collision), generic in the scalar type.  g: pulled populations (f - w);
// (fx, fy, fz): spread force; pd: drive P of the step; Bc: B.  post: the
// post-collision populations; u: the velocity with the half-force shift (what
// the interpolation reads).
template <typename T, typename R>
__device__ __forceinline__ void collide_generic(const T (&g)[Q], T fx, T fy, T fz, T pd, T Bc, R omega, R Cr,
                                                T (&post)[Q], T (&u)[3])
{
    T drho = T(R(0)), jx = T(R(0)), jy = T(R(0)), jz = T(R(0));
#pragma unroll
    for (int q = 0; q < Q; q++) {
        drho += g[q];
        if (ex(q) == 1) jx += g[q]; else if (ex(q) == -1) jx -= g[q];
        if (ey(q) == 1) jy += g[q]; else if (ey(q) == -1) jy -= g[q];
        if (ez(q) == 1) jz += g[q]; else if (ez(q) == -1) jz -= g[q];
    }
    const T r = drho + R(1);
    const T Gx = r * Bc * fx, Gy = r * Bc * fy, Gz = r * (pd + Bc * fz);
    const T inv = R(1) / (r * Cr);
    u[0] = (jx + Gx) * inv; u[1] = (jy + Gy) * inv; u[2] = (jz + Gz) * inv;
    const R fo = (R(1) - R(0.5) * omega) * R(2), om1 = R(1) - omega;
    const T usq = (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]) * (R(-1.5) * Cr * Cr);
    const T uG = (u[0] * Gx + u[1] * Gy + u[2] * Gz) * (R(3) * Cr);
    const T A = (drho + r * usq) * omega - uG * fo;
    const T B = r * (R(3) * Cr * omega), C = r * (R(4.5) * Cr * Cr * omega);
    const R D = R(3) * fo, E = R(9) * Cr * fo;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        T eu = T(R(0)), eG = T(R(0));
        if (ex(q) == 1) { eu += u[0]; eG += Gx; } else if (ex(q) == -1) { eu -= u[0]; eG -= Gx; }
        if (ey(q) == 1) { eu += u[1]; eG += Gy; } else if (ey(q) == -1) { eu -= u[1]; eG -= Gy; }
        if (ez(q) == 1) { eu += u[2]; eG += Gz; } else if (ez(q) == -1) { eu -= u[2]; eG -= Gz; }
        post[q] = g[q] * om1 + (A + eu * (B + C * eu + eG * E) + eG * D) * R(wq(q));
    }
}

constexpr int LBM_ADJ_THREADS = 128;

// Adjoint of the collision at every fluid node.  gin: g_t (the populations the
// forward step pulled from); F: the spread force of the step; gbar_out:
// adjoint of g_t+1; ubar: adjoint of the velocity field ([n] float4, .w
// unused).  Writes the adjoint of the pulled populations (gbar_pre) and of the
// force (Fbar, 0 off the fluid), and adds dfac * d/dP and d/dB to pbar[0..1].
__global__ void __launch_bounds__(LBM_ADJ_THREADS)
lbm_adjoint_kernel(const LbmAdjArgs a, int nx, int ny, int nzc, long long nint)
{
    __shared__ double red[2][LBM_ADJ_THREADS / 32];
    const int plane = nx * ny;
    const int xy = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    double dP = 0.0, dB = 0.0;
    if (xy < plane) {
        const long long zb0 = (long long)z * plane, idx = zb0 + xy;
        const uint32_t m = __ldg(&a.mask2d[xy]);
        if (m & MASK_FLUID) {
            const long long zbm = (z == 0) ? (long long)(nzc - 1) * plane : zb0 - plane;
            const long long zbp = (z == nzc - 1) ? 0 : zb0 + plane;
            float g[Q], ob[Q];
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const long long src = ((ez(q) == 1) ? zbm : (ez(q) == -1) ? zbp : zb0) + xy - ex(q) - nx * ey(q);
                g[q] = ((m >> q) & 1u) ? a.gin[(long long)opp(q) * nint + idx] : a.gin[(long long)q * nint + src];
                ob[q] = a.gbar_out[(long long)q * nint + idx];
            }
            const float f3[3] = {a.Fx[idx], a.Fy[idx], a.Fz[idx]};
            const float4 ub = a.ubar[idx];
            // one Jacobian column per input: 19 populations, 3 force components, P, B
#pragma unroll 1
            for (int k = 0; k < Q + 5; k++) {
                Dual<float> gd[Q], post[Q], u[3];
#pragma unroll
                for (int q = 0; q < Q; q++) gd[q] = Dual<float>(g[q], k == q ? 1.f : 0.f);
                const Dual<float> fx(f3[0], k == Q ? 1.f : 0.f), fy(f3[1], k == Q + 1 ? 1.f : 0.f),
                    fz(f3[2], k == Q + 2 ? 1.f : 0.f), dp(a.pd, k == Q + 3 ? 1.f : 0.f), db(a.Bc, k == Q + 4 ? 1.f : 0.f);
                collide_generic<Dual<float>, float>(gd, fx, fy, fz, dp, db, a.omega, a.Cr, post, u);
                float s = u[0].d * ub.x + u[1].d * ub.y + u[2].d * ub.z;
#pragma unroll
                for (int q = 0; q < Q; q++) s += post[q].d * ob[q];
                if (k < Q) a.gbar_pre[(long long)k * nint + idx] = s;
                else if (k == Q) a.Fbar[idx] = s;
                else if (k == Q + 1) a.Fbar[nint + idx] = s;
                else if (k == Q + 2) a.Fbar[2 * nint + idx] = s;
                else if (k == Q + 3) dP = s;
                else dB = s;
            }
        } else {
            a.Fbar[idx] = 0.f; a.Fbar[nint + idx] = 0.f; a.Fbar[2 * nint + idx] = 0.f;
        }
    }
    // parameter adjoints: block sums in FP64, one atomic per block
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        dP += __shfl_xor_sync(0xffffffffu, dP, o);
        dB += __shfl_xor_sync(0xffffffffu, dB, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { red[0][wid] = dP; red[1][wid] = dB; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sp = 0.0, sb = 0.0;
        for (int w = 0; w < LBM_ADJ_THREADS / 32; w++) { sp += red[0][w]; sb += red[1][w]; }
        atomicAdd(&a.pbar[0], a.dfac * sp);
        atomicAdd(&a.pbar[1], sb);
    }
}

// Transpose of the pull.  Population q of fluid node j is read by node
// j + e_q (direction q; that node's source j is fluid, so it does not bounce
// back there) when j + e_q is fluid, and by node j itself in direction opp q
// when j's opp-q source is a wall (half-way bounce-back).  Populations of wall
// nodes are never read.
__global__ void lbm_pull_transpose_kernel(const float *__restrict__ gbar_pre, const uint32_t *__restrict__ mask2d,
                                          float *__restrict__ gbar_in, int nx, int ny, int nzc, long long nint)
{
    const int plane = nx * ny;
    const int xy = blockIdx.x * blockDim.x + threadIdx.x;
    if (xy >= plane) return;
    const int z = blockIdx.y;
    const long long zb0 = (long long)z * plane, idx = zb0 + xy;
    const uint32_t m = __ldg(&mask2d[xy]);
    const bool fluid = (m & MASK_FLUID) != 0;
    const long long zbm = (z == 0) ? (long long)(nzc - 1) * plane : zb0 - plane;
    const long long zbp = (z == nzc - 1) ? 0 : zb0 + plane;
#pragma unroll
    for (int q = 0; q < Q; q++) {
        float v = 0.f;
        if (fluid) {
            const int xyn = xy + ex(q) + nx * ey(q);   // inside the lattice: fluid is never on its edge
            if (__ldg(&mask2d[xyn]) & MASK_FLUID)
                v += gbar_pre[(long long)q * nint + ((ez(q) == 1) ? zbp : (ez(q) == -1) ? zbm : zb0) + xyn];
            if ((m >> opp(q)) & 1u) v += gbar_pre[(long long)opp(q) * nint + idx];
        }
        gbar_in[(long long)q * nint + idx] = v;
    }
}

// ---- delta stencil with position derivatives ------------------------------

// delta4 (rbc_internal.cuh) in FP64 with d/df of each weight.  With
// s = sin(pi f / 2), c = cos(pi f / 2): w = (1 - s, 1 + c, 1 + s, 1 - c) / 4,
// dw/df = (pi / 8) (-c, -s, c, s).
__device__ __forceinline__ void delta4_d(double f, double w[4], double dw[4]) {
    double s, c;
    sincospi(0.5 * f, &s, &c);
    const double k = 0.125 * 3.14159265358979323846;
    w[0] = 0.25 * (1.0 - s); w[1] = 0.25 * (1.0 + c); w[2] = 0.25 * (1.0 + s); w[3] = 0.25 * (1.0 - c);
    dw[0] = -k * c; dw[1] = -k * s; dw[2] = k * c; dw[3] = k * s;
}

struct Stencil {
    int ix0, iy0, iz0;            // first node on each axis (z in the raw frame of the position)
    double wx[4], wy[4], wz[4];   // weights
    double dx[4], dy[4], dz[4];   // d weight / d position
};

__device__ __forceinline__ void stencil_at(const Geom &g, double px, double py, double pz, Stencil &s) {
    const double lx = lat_x(g, px), ly = lat_y(g, py), lz = lat_z(g, pz);
    const double flx = floor(lx), fly = floor(ly), flz = floor(lz);
    s.ix0 = (int)flx - 1; s.iy0 = (int)fly - 1; s.iz0 = (int)flz - 1;
    delta4_d(lx - flx, s.wx, s.dx); delta4_d(ly - fly, s.wy, s.dy); delta4_d(lz - flz, s.wz, s.dz);
#pragma unroll
    for (int k = 0; k < 4; k++) { s.dx[k] *= g.inv_dx; s.dy[k] *= g.inv_dx; s.dz[k] *= g.inv_dx; }
}

// a lattice coordinate the stencil arithmetic can take (as in ibm.cu)
__device__ __forceinline__ bool sane_pos(const Geom &g, double px, double py, double pz) {
    return fabs(lat_x(g, px)) < 16777216.0 && fabs(lat_y(g, py)) < 16777216.0 && fabs(lat_z(g, pz)) < 16777216.0;
}

// ---- interpolation + RK4, reversed -----------------------------------------

// Velocity of the frozen field at p as the forward advection interpolates it
// (stencil nodes beyond the two BUFF planes or outside x, y contribute nothing).
__device__ __forceinline__ void interp(const Geom &g, const float4 *__restrict__ uvr, double px, double py, double pz,
                                       double u[3]) {
    Stencil s;
    stencil_at(g, px, py, pz, s);
    u[0] = u[1] = u[2] = 0.0;
    for (int c = 0; c < 4; c++) {
        const int iz = s.iz0 + c;
        if (iz < -2 || iz >= g.nzc + 2) continue;
        const long long zb = (long long)wrap_z(iz, g.nzc) * g.plane;
        for (int b = 0; b < 4; b++) {
            const int gy = s.iy0 + b;
            if (gy < 0 || gy >= g.ny) continue;
            for (int a = 0; a < 4; a++) {
                const int gx = s.ix0 + a;
                if (gx < 0 || gx >= g.nx) continue;
                const float4 q = __ldg(&uvr[zb + gx + (long long)g.nx * gy]);
                const double w = s.wx[a] * s.wy[b] * s.wz[c];
                u[0] += w * q.x; u[1] += w * q.y; u[2] += w * q.z;
            }
        }
    }
}

// Adjoint of one interpolation at p with output adjoint kb: adds w_n kb to
// the velocity adjoint of each stencil node and returns in pb the position
// adjoint, sum_n (d w_n / d p) (u_n . kb).
__device__ __forceinline__ void interp_adjoint(const Geom &g, const float4 *__restrict__ uvr, float *__restrict__ ubar,
                                               double px, double py, double pz, const double kb[3], double pb[3]) {
    Stencil s;
    stencil_at(g, px, py, pz, s);
    pb[0] = pb[1] = pb[2] = 0.0;
    for (int c = 0; c < 4; c++) {
        const int iz = s.iz0 + c;
        if (iz < -2 || iz >= g.nzc + 2) continue;
        const long long zb = (long long)wrap_z(iz, g.nzc) * g.plane;
        for (int b = 0; b < 4; b++) {
            const int gy = s.iy0 + b;
            if (gy < 0 || gy >= g.ny) continue;
            for (int a = 0; a < 4; a++) {
                const int gx = s.ix0 + a;
                if (gx < 0 || gx >= g.nx) continue;
                const long long n = zb + gx + (long long)g.nx * gy;
                const float4 q = __ldg(&uvr[n]);
                const double w = s.wx[a] * s.wy[b] * s.wz[c];
                atomicAdd(&ubar[4 * n + 0], (float)(w * kb[0]));
                atomicAdd(&ubar[4 * n + 1], (float)(w * kb[1]));
                atomicAdd(&ubar[4 * n + 2], (float)(w * kb[2]));
                const double uk = q.x * kb[0] + q.y * kb[1] + q.z * kb[2];
                pb[0] += s.dx[a] * s.wy[b] * s.wz[c] * uk;
                pb[1] += s.wx[a] * s.dy[b] * s.wz[c] * uk;
                pb[2] += s.wx[a] * s.wy[b] * s.dz[c] * uk;
            }
        }
    }
}

// One thread per vertex.  xa_bar: adjoint of the advected positions; writes
// X_bar (adjoint of X_t through the advection, overwritten) and adds to ubar.
// The periodic wrap of the result in x and z is a translation (derivative 1).
__global__ void advect_adjoint_kernel(const Geom g, const double *__restrict__ X, const float4 *__restrict__ uvr,
                                      const double *__restrict__ xa_bar, double *__restrict__ X_bar,
                                      float *__restrict__ ubar, long long nv, double dtM, int *__restrict__ flags)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    double p[4][3], k[4][3];
    p[0][0] = X[v]; p[0][1] = X[nv + v]; p[0][2] = X[2 * nv + v];
    if (!sane_pos(g, p[0][0], p[0][1], p[0][2])) {
        atomicOr(flags, RBC_FLAG_NONFINITE);
        X_bar[v] = X_bar[nv + v] = X_bar[2 * nv + v] = 0.0;
        return;
    }
    const double hs[4] = {0.0, 0.5 * dtM, 0.5 * dtM, dtM};   // stage offsets (ibm.cu:474-498)
    interp(g, uvr, p[0][0], p[0][1], p[0][2], k[0]);
    for (int s = 1; s < 4; s++) {
        // the forward adds the FP32 stage velocity to the FP64 position
        for (int c = 0; c < 3; c++) p[s][c] = p[0][c] + (double)(float)k[s - 1][c] * hs[s];
        interp(g, uvr, p[s][0], p[s][1], p[s][2], k[s]);
    }
    double xb[3], kb[4][3];
    for (int c = 0; c < 3; c++) {
        const double a = xa_bar[(long long)c * nv + v];
        xb[c] = a;   // Xa = X + dt (k1 + 2 k2 + 2 k3 + k4) / 6
        kb[0][c] = a * dtM / 6.0; kb[1][c] = a * dtM / 3.0; kb[2][c] = a * dtM / 3.0; kb[3][c] = a * dtM / 6.0;
    }
    for (int s = 3; s >= 0; s--) {
        double pb[3];
        interp_adjoint(g, uvr, ubar, p[s][0], p[s][1], p[s][2], kb[s], pb);
        for (int c = 0; c < 3; c++) {
            xb[c] += pb[c];
            if (s > 0) kb[s - 1][c] += hs[s] * pb[c];   // p_s = X + h_s k_s-1
        }
    }
    for (int c = 0; c < 3; c++) X_bar[(long long)c * nv + v] = xb[c];
}

// ---- spreading, reversed --------------------------------------------------

// F(n) = sum_v w_n(X_v) Fv_v / dx^3 over fluid columns, stencil planes beyond
// the BUFF planes of the vertex's raw frame dropped (ibm.cu:107-110).  One
// thread per vertex: Fv_bar = sum_n w_n Fbar(n) / dx^3 (overwritten) and
// X_bar += sum_n (d w_n / d X) (Fv . Fbar(n)) / dx^3.
__global__ void spread_adjoint_kernel(const Geom g, const double *__restrict__ X, const float *__restrict__ Fv,
                                      const float *__restrict__ Fbar, const uint32_t *__restrict__ mask2d,
                                      double *__restrict__ Fv_bar, double *__restrict__ X_bar, long long nv)
{
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const double px = X[v], py = X[nv + v], pz = X[2 * nv + v];
    double fb[3] = {0.0, 0.0, 0.0}, pb[3] = {0.0, 0.0, 0.0};
    if (sane_pos(g, px, py, pz)) {
        const double wscale = 1.0 / (g.dx * g.dx * g.dx);
        Stencil s;
        stencil_at(g, px, py, pz, s);
        const double f[3] = {Fv[v], Fv[nv + v], Fv[2 * nv + v]};
        for (int c = 0; c < 4; c++) {
            const int iz = s.iz0 + c;
            if (iz < -2 || iz >= g.nzc + 2) continue;
            const long long zb = (long long)wrap_z(iz, g.nzc) * g.plane;
            for (int b = 0; b < 4; b++) {
                const int gy = s.iy0 + b;
                if (gy < 0 || gy >= g.ny) continue;
                for (int a = 0; a < 4; a++) {
                    const int gx = s.ix0 + a;
                    if (gx < 0 || gx >= g.nx) continue;
                    if (!(__ldg(&mask2d[gx + g.nx * gy]) & MASK_FLUID)) continue;
                    const long long n = zb + gx + (long long)g.nx * gy;
                    const double F0 = Fbar[n], F1 = Fbar[g.nint + n], F2 = Fbar[2 * g.nint + n];
                    const double w = s.wx[a] * s.wy[b] * s.wz[c] * wscale;
                    fb[0] += w * F0; fb[1] += w * F1; fb[2] += w * F2;
                    const double fF = (f[0] * F0 + f[1] * F1 + f[2] * F2) * wscale;
                    pb[0] += s.dx[a] * s.wy[b] * s.wz[c] * fF;
                    pb[1] += s.wx[a] * s.dy[b] * s.wz[c] * fF;
                    pb[2] += s.wx[a] * s.wy[b] * s.dz[c] * fF;
                }
            }
        }
    }
    for (int c = 0; c < 3; c++) {
        Fv_bar[(long long)c * nv + v] = fb[c];
        X_bar[(long long)c * nv + v] += pb[c];
    }
}

// ---- membrane, reversed -----------------------------------------------------

// The Skalak loads of one element as membrane.cu's element pass computes them:
// edge vectors e1 = x_b - x_a, e2 = x_c - x_a, reference metric (G11, G12,
// G22, 1 / det G), C -> loads on vertices b and c (vertex a gets minus their
// sum) and gab = twice the area.
template <typename T>
__device__ __forceinline__ void element_loads(const T (&e1)[3], const T (&e2)[3], double G11, double G12, double G22,
                                              double idG, T C, double rgs, int law, T (&bB)[3], T (&bC)[3], T &gab)
{
    const T g11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
    const T g12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
    const T g22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
    const T d11 = g11 - G11, d12 = g12 - G12, d22 = g22 - G22;
    const double n00 = G22 * idG, n01 = -G12 * idG, n11 = G11 * idG, detn = idG;
    const T det = g11 * g22 - g12 * g12;
    const T idet = 1.0 / det;
    const T i1 = d11 * n00 + d12 * (2.0 * n01) + d22 * n11;
    const T i2 = (d22 * G11 + d11 * G22 - d12 * (2.0 * G12) + d11 * d22 - d12 * d12) * detn;
    const T js = sqrt(i2 + 1.0);
    const T jsm1 = i2 / (js + 1.0);
    T al, be;
    if (law == RBC_LAW_SKALAK) {
        al = (i1 * rgs + (rgs - 1.0) - jsm1) / js;
        be = C * i2 * js - jsm1;
    } else {
        const T js3 = js * js * js;
        al = ((rgs - 1.0) - jsm1) / js;
        be = (jsm1 * (js * js + js + 1.0) - (rgs - 1.0)) / js3;
    }
    const T gi00 = g22 * idet, gi01 = -g12 * idet, gi11 = g11 * idet;
    const T p00 = d11 * n00 + d12 * n01, p01 = d12 * n00 + d22 * n01;
    const T p10 = d11 * n01 + d12 * n11, p11 = d12 * n01 + d22 * n11;
    const T t00 = al * n00 + be * gi00 + (p00 * gi00 + p01 * gi01);
    const T t01 = al * n01 + be * gi01 + ((p00 * gi01 + p01 * gi11) + (p10 * gi00 + p11 * gi01)) * 0.5;
    const T t11 = al * n11 + be * gi11 + (p10 * gi01 + p11 * gi11);
    gab = sqrt(det);
    const T h = gab * 0.5;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        bB[c] = h * (t00 * e1[c] + t01 * e2[c]);
        bC[c] = h * (t01 * e1[c] + t11 * e2[c]);
    }
}

__device__ __forceinline__ double mimage_d(double d, double L) {
    if (d > L * 0.5) d -= L; else if (d < -L * 0.5) d += L;
    return d;
}

// edge vectors of local element e of the cell whose vertices start at vb
// (minimum image in x and z per edge, as the forward)
__device__ __forceinline__ void edges_of(const MembraneAdjArgs &a, long long vb, int e, double (&e1)[3], double (&e2)[3],
                                         int &ia, int &ib, int &ic) {
    ia = __ldg(&a.tri[3 * e]); ib = __ldg(&a.tri[3 * e + 1]); ic = __ldg(&a.tri[3 * e + 2]);
    const double *xs = a.Xd + vb, *ys = a.Xd + a.nv + vb, *zs = a.Xd + 2 * a.nv + vb;
    e1[0] = mimage_d(xs[ib] - xs[ia], a.LX); e1[1] = ys[ib] - ys[ia]; e1[2] = mimage_d(zs[ib] - zs[ia], a.LZ);
    e2[0] = mimage_d(xs[ic] - xs[ia], a.LX); e2[1] = ys[ic] - ys[ia]; e2[2] = mimage_d(zs[ic] - zs[ia], a.LZ);
}

constexpr int MEM_ADJ_THREADS = 1024;

// One CTA per cell.  Fv: the membrane forces of the step (forward output);
// Fv_bar: their adjoint.  The forward solves M q = b (b = element loads
// gathered per vertex, M the P1 mass matrix) and sets Fv = -q ds (ds = one-ring
// area / 3).  Reverse: q_bar = -ds Fv_bar, ds_bar = -q . Fv_bar,
// lambda = M^-1 q_bar (Chebyshev on D^-1 M as the forward: with M symmetric the
// transpose of the polynomial solve is the same polynomial solve), b_bar =
// lambda, M_bar = -lambda q^T.  Per element the adjoints of (load on b, load on
// c, gab) are contracted with the Jacobian of element_loads (seven dual
// passes: e1, e2, C) and the edge adjoints gathered to the vertices.  Writes
// Xd_bar (overwritten) and adds dL/dC to cbar.
template <int VPT>
__global__ void __launch_bounds__(MEM_ADJ_THREADS, 1)
membrane_adjoint_kernel(const MembraneAdjArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[32];
    const int V = a.V, E = a.E, tid = threadIdx.x, T = blockDim.x;
    float4 *dbuf = reinterpret_cast<float4 *>(smem);                    // [2][V]
    float *coef = reinterpret_cast<float *>(smem + 32 * (size_t)V);     // [6][V]
    int16_t *snbr = reinterpret_cast<int16_t *>(smem + 56 * (size_t)V); // [6][V]
    const int cell = blockIdx.x;
    const long long vb = (long long)cell * V, eb = (long long)cell * E, nv = a.nv;
    double *er = a.scratch + eb * 7;   // per element: gab, then the adjoints of e1 and e2
    for (int k = tid; k < 6 * V; k += T) snbr[k] = a.nbr[k];
    for (int e = tid; e < E; e += T) {
        double e1[3], e2[3];
        int ia, ib, ic;
        edges_of(a, vb, e, e1, e2, ia, ib, ic);
        const double g11 = e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2];
        const double g12 = e1[0] * e2[0] + e1[1] * e2[1] + e1[2] * e2[2];
        const double g22 = e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2];
        er[7 * e] = sqrt(g11 * g22 - g12 * g12);
    }
    __syncthreads();
    // rows of D^-1 M, q, ds_bar and the scaled right-hand side D^-1 q_bar
    float q[VPT][3], rhs[VPT][3], dsb[VPT];
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
        dsb[m] = 0.f;
        for (int c = 0; c < 3; c++) { q[m][c] = 0.f; rhs[m][c] = 0.f; }
        if (i >= V) continue;
        double off[6] = {0, 0, 0, 0, 0, 0}, dg = 0.0, s = 0.0;
        for (int k = __ldg(&a.v2e_off[i]); k < __ldg(&a.v2e_off[i + 1]); k++) {
            const int pk = __ldg(&a.v2e[k]);
            const double ga = er[7 * v2e_elem(pk)];
            dg += ga / 12.0;
            off[v2e_sa(pk)] += ga / 24.0;
            off[v2e_sb(pk)] += ga / 24.0;
            s += ga / 6.0;
        }
        for (int t = 0; t < 6; t++) coef[t * V + i] = (float)(off[t] / dg);
        double d = 0.0;
        for (int c = 0; c < 3; c++) {
            const double fv = a.Fv[(long long)c * nv + vb + i], fb = a.Fv_bar[(long long)c * nv + vb + i];
            const double qc = -fv / s;
            q[m][c] = (float)qc;
            d -= qc * fb;
            rhs[m][c] = (float)(-s * fb / dg);
        }
        dsb[m] = (float)d;
    }
    __syncthreads();
    // lambda = M^-1 q_bar: Chebyshev on D^-1 M with the forward's bounds [1/2, 2]
    const float theta = 1.25f, delta = 0.75f, sigma = theta / delta;
    float x[VPT][3], r[VPT][3], dd[VPT][3];
    float rho = 1.0f / sigma;
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
        for (int c = 0; c < 3; c++) { x[m][c] = 0.f; r[m][c] = rhs[m][c]; dd[m][c] = rhs[m][c] / theta; }
        if (i < V) dbuf[i] = make_float4(dd[m][0], dd[m][1], dd[m][2], 0.f);
    }
    __syncthreads();
    for (int it = 0; it < a.niter; it++) {
        const float4 *cur = dbuf + (it & 1) * V;
        float4 *nxt = dbuf + ((it + 1) & 1) * V;
        const float rho_n = 1.0f / (2.0f * sigma - rho);
        const float c1 = rho_n * rho, c2 = 2.0f * rho_n / delta;
#pragma unroll
        for (int m = 0; m < VPT; m++) {
            const int i = tid + m * T;
            if (i >= V) continue;
            float ad0 = dd[m][0], ad1 = dd[m][1], ad2 = dd[m][2];
            for (int s = 0; s < 6; s++) {
                const int j = snbr[s * V + i];
                if (j >= 0) {
                    const float w = coef[s * V + i];
                    const float4 dj = cur[j];
                    ad0 += w * dj.x; ad1 += w * dj.y; ad2 += w * dj.z;
                }
            }
            x[m][0] += dd[m][0]; x[m][1] += dd[m][1]; x[m][2] += dd[m][2];
            r[m][0] -= ad0; r[m][1] -= ad1; r[m][2] -= ad2;
            for (int c = 0; c < 3; c++) dd[m][c] = c1 * dd[m][c] + c2 * r[m][c];
            nxt[i] = make_float4(dd[m][0], dd[m][1], dd[m][2], 0.f);
        }
        rho = rho_n;
        __syncthreads();
    }
    // lambda, q and ds_bar of every vertex to shared memory (the solve's buffers are free)
    float4 *slam = dbuf, *sq = dbuf + V;
    float *sdsb = coef;
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
        if (i >= V) continue;
        slam[i] = make_float4(x[m][0], x[m][1], x[m][2], 0.f);
        sq[i] = make_float4(q[m][0], q[m][1], q[m][2], 0.f);
        sdsb[i] = dsb[m];
    }
    __syncthreads();
    double cb = 0.0;
    for (int e = tid; e < E; e += T) {
        double e1[3], e2[3];
        int ia, ib, ic;
        edges_of(a, vb, e, e1, e2, ia, ib, ic);
        const float4 la = slam[ia], lb = slam[ib], lc = slam[ic], qa = sq[ia], qb = sq[ib], qc = sq[ic];
        auto dotf = [](float4 u, float4 w) { return (double)u.x * w.x + (double)u.y * w.y + (double)u.z * w.z; };
        // M = sum_e gab (1 + delta_ij) / 24 over the element's vertex pairs; ds_i = sum_e gab / 6
        const double mdiag = -(dotf(la, qa) + dotf(lb, qb) + dotf(lc, qc));
        const double moff = -(dotf(la, qb) + dotf(lb, qa) + dotf(la, qc) + dotf(lc, qa) + dotf(lb, qc) + dotf(lc, qb));
        const double gb = mdiag / 12.0 + moff / 24.0 + ((double)sdsb[ia] + sdsb[ib] + sdsb[ic]) / 6.0;
        const double bBb[3] = {(double)lb.x - la.x, (double)lb.y - la.y, (double)lb.z - la.z};
        const double bCb[3] = {(double)lc.x - la.x, (double)lc.y - la.y, (double)lc.z - la.z};
        const double4 G = a.gref[eb + e];
        double res[7];
#pragma unroll 1
        for (int k = 0; k < 7; k++) {
            Dual<double> d1[3], d2[3], oB[3], oC[3], og;
            for (int c = 0; c < 3; c++) {
                d1[c] = Dual<double>(e1[c], k == c ? 1.0 : 0.0);
                d2[c] = Dual<double>(e2[c], k == 3 + c ? 1.0 : 0.0);
            }
            const Dual<double> Cd(a.C, k == 6 ? 1.0 : 0.0);
            element_loads<Dual<double>>(d1, d2, G.x, G.y, G.z, G.w, Cd, a.rgs, a.law, oB, oC, og);
            double s = og.d * gb;
            for (int c = 0; c < 3; c++) s += oB[c].d * bBb[c] + oC[c].d * bCb[c];
            res[k] = s;
        }
        for (int k = 0; k < 6; k++) er[7 * e + 1 + k] = res[k];
        cb += res[6];
    }
    cb = block_sum_r(cb, red);
    if (tid == 0) atomicAdd(a.cbar, cb);
    __syncthreads();
    // edge adjoints to the vertices: e1 = x_b - x_a, e2 = x_c - x_a
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
        if (i >= V) continue;
        double xb[3] = {0.0, 0.0, 0.0};
        for (int k = __ldg(&a.v2e_off[i]); k < __ldg(&a.v2e_off[i + 1]); k++) {
            const int pk = __ldg(&a.v2e[k]);
            const double *rec = er + 7 * v2e_elem(pk);
            const int en = v2e_en(pk);
            for (int c = 0; c < 3; c++) {
                if (en == 0) xb[c] -= rec[1 + c] + rec[4 + c];
                else if (en == 1) xb[c] += rec[1 + c];
                else xb[c] += rec[4 + c];
            }
        }
        for (int c = 0; c < 3; c++) a.Xd_bar[(long long)c * nv + vb + i] = xb[c];
    }
}

// ---- volume correction, reversed ------------------------------------------

// Normal, area and volume contribution of one triangle as volume.cu's
// ele_normal computes them, generic in the scalar type.
template <typename T>
__device__ __forceinline__ void tri_geom(const T (&pa)[3], const T (&pb)[3], const T (&pc)[3], T (&n)[3], T &dS, T &vt)
{
    const T v1x = pb[0] - pa[0], v1y = pb[1] - pa[1], v1z = pb[2] - pa[2];
    const T v2x = pc[0] - pa[0], v2y = pc[1] - pa[1], v2z = pc[2] - pa[2];
    const T c0 = v1y * v2z - v1z * v2y, c1 = v1z * v2x - v1x * v2z, c2 = v1x * v2y - v1y * v2x;
    const T nc = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    n[0] = c0 / nc; n[1] = c1 / nc; n[2] = c2 / nc;
    dS = nc / 2.0;
    const T rx = (pa[0] + pb[0] + pc[0]) / 3.0, ry = (pa[1] + pb[1] + pc[1]) / 3.0, rz = (pa[2] + pb[2] + pc[2]) / 3.0;
    vt = (rx * n[0] + ry * n[1] + rz * n[2]) * dS / 3.0;
}

constexpr int VC_ADJ_THREADS = 1024;
constexpr double VC_COEFF = 0.1;     // COEFF_VOL_CHANGE (volume_correction.cu:14)
constexpr double VC_TOL = 1.0e-3;    // percent (volume_correction.cu:15)

// One CTA per cell.  Replays the forward correction of the positions Xa (the
// same unwrap about gx, the same iterations: while |V - V0| / V0 * 100 >= tol,
// every vertex moves by s n_v with s = -0.3 (V - V0) / A and n_v the mean of
// its elements' unit normals), storing the positions before each move, then
// reverses the moves: for a move x' = x + s(x) n(x),
//   x_bar += s (dn/dx)^T x'_bar + (ds/dx)^T (sum_v n_v . x'_bar_v)
// with ds/dx = -0.3 (dV/dx / A - (V - V0) / A^2 dA/dx); all three are sums
// over triangles, differentiated per triangle with dual numbers (nine passes).
// The final z wrap is a translation.  Writes Xa_bar = (reversed X_bar) + Xd_bar.
__global__ void __launch_bounds__(VC_ADJ_THREADS, 1)
volume_adjoint_kernel(const Geom g, const VolumeAdjArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ double red[32];
    double *p = reinterpret_cast<double *>(smem);   // [3][V] positions
    double *pb = p + 3 * (size_t)a.V;               // [3][V] position adjoints
    const int V = a.V, E = a.E, tid = threadIdx.x, T = blockDim.x, cell = blockIdx.x, N = a.ncell;
    const long long vb = (long long)cell * V, nv = a.nv;
    double *hist = a.hist + (long long)cell * a.kmax * 3 * V;   // positions before each move
    double *er = a.escr + (long long)cell * E * 9;              // per triangle: adjoints of its 3 vertices
    const double gz = a.gx[2 * N + cell];
    for (int v = tid; v < V; v += T) {
        p[v] = a.Xa[vb + v];
        p[V + v] = a.Xa[nv + vb + v];
        double z = a.Xa[2 * nv + vb + v];
        const double dz = z - gz;
        if (dz > g.LZ * 0.5) z -= g.LZ; else if (dz < -g.LZ * 0.5) z += g.LZ;
        p[2 * V + v] = z;
        for (int c = 0; c < 3; c++) pb[c * V + v] = a.X_bar[(long long)c * nv + vb + v];
    }
    __syncthreads();
    auto tri_at = [&](const double *P, int e, double (&A)[3], double (&B)[3], double (&Cc)[3]) {
        const int ia = __ldg(&a.tri[3 * e]), ib = __ldg(&a.tri[3 * e + 1]), ic = __ldg(&a.tri[3 * e + 2]);
        for (int c = 0; c < 3; c++) { A[c] = P[c * V + ia]; B[c] = P[c * V + ib]; Cc[c] = P[c * V + ic]; }
    };
    auto vol_area = [&](const double *P, double &vol, double &area) {
        double sv = 0.0, sa = 0.0;
        for (int e = tid; e < E; e += T) {
            double A[3], B[3], Cc[3], n[3], dS, vt;
            tri_at(P, e, A, B, Cc);
            tri_geom<double>(A, B, Cc, n, dS, vt);
            sv += vt; sa += dS;
        }
        vol = block_sum_r(sv, red);
        area = block_sum_r(sa, red);
    };
    auto mean_normal = [&](const double *P, int v, double (&nn)[3]) {
        const int k0 = __ldg(&a.v2e_off[v]), k1 = __ldg(&a.v2e_off[v + 1]), nne = k1 - k0;
        nn[0] = nn[1] = nn[2] = 0.0;
        for (int k = k0; k < k1; k++) {
            double A[3], B[3], Cc[3], n[3], dS, vt;
            tri_at(P, v2e_elem(__ldg(&a.v2e[k])), A, B, Cc);
            tri_geom<double>(A, B, Cc, n, dS, vt);
            for (int c = 0; c < 3; c++) nn[c] += n[c] / nne;
        }
    };
    // forward replay
    const double V0 = a.vol0[cell];
    int moves = 0;
    for (int it = 1;; it++) {
        double vol, area;
        vol_area(p, vol, area);
        if (fabs(vol - V0) / V0 * 100.0 < VC_TOL) break;
        if (moves >= a.kmax || it >= 1000) {   // more moves than the history holds: reverse only those recorded
            if (tid == 0) atomicOr(a.status, 1);
            break;
        }
        for (int k = tid; k < 3 * V; k += T) hist[(long long)moves * 3 * V + k] = p[k];
        const double s = -18.0 * (vol - V0) / area / 6.0 * VC_COEFF;
        double disp[4][3];
        for (int m = 0; m < 4; m++) {
            const int v = tid + m * T;
            if (v >= V) continue;
            double nn[3];
            mean_normal(p, v, nn);
            for (int c = 0; c < 3; c++) disp[m][c] = s * nn[c];
        }
        __syncthreads();
        for (int m = 0; m < 4; m++) {
            const int v = tid + m * T;
            if (v >= V) continue;
            for (int c = 0; c < 3; c++) p[c * V + v] += disp[m][c];
        }
        __syncthreads();
        moves++;
    }
    // reverse the moves
    for (int j = moves - 1; j >= 0; j--) {
        const double *P = hist + (long long)j * 3 * V;
        double vol, area;
        vol_area(P, vol, area);
        const double s = -18.0 * (vol - V0) / area / 6.0 * VC_COEFF;
        double w = 0.0;
        for (int v = tid; v < V; v += T) {
            double nn[3];
            mean_normal(P, v, nn);
            w += nn[0] * pb[v] + nn[1] * pb[V + v] + nn[2] * pb[2 * V + v];
        }
        w = block_sum_r(w, red);
        const double al = -0.3 * w / area, be = 0.3 * w * (vol - V0) / (area * area);
        for (int e = tid; e < E; e += T) {
            const int id[3] = {__ldg(&a.tri[3 * e]), __ldg(&a.tri[3 * e + 1]), __ldg(&a.tri[3 * e + 2])};
            double W[3] = {0.0, 0.0, 0.0}, x0[3][3];
            for (int t = 0; t < 3; t++) {
                const int u = id[t];
                const double inv = 1.0 / (double)(__ldg(&a.v2e_off[u + 1]) - __ldg(&a.v2e_off[u]));
                for (int c = 0; c < 3; c++) { W[c] += pb[c * V + u] * inv; x0[t][c] = P[c * V + u]; }
            }
#pragma unroll 1
            for (int k = 0; k < 9; k++) {
                Dual<double> A[3], B[3], Cc[3], n[3], dS, vt;
                for (int c = 0; c < 3; c++) {
                    A[c] = Dual<double>(x0[0][c], k == c ? 1.0 : 0.0);
                    B[c] = Dual<double>(x0[1][c], k == 3 + c ? 1.0 : 0.0);
                    Cc[c] = Dual<double>(x0[2][c], k == 6 + c ? 1.0 : 0.0);
                }
                tri_geom<Dual<double>>(A, B, Cc, n, dS, vt);
                er[9 * e + k] = s * (n[0].d * W[0] + n[1].d * W[1] + n[2].d * W[2]) + al * vt.d + be * dS.d;
            }
        }
        __syncthreads();
        for (int v = tid; v < V; v += T) {
            for (int k = __ldg(&a.v2e_off[v]); k < __ldg(&a.v2e_off[v + 1]); k++) {
                const int pk = __ldg(&a.v2e[k]);
                const double *rec = er + 9 * v2e_elem(pk) + 3 * v2e_en(pk);
                for (int c = 0; c < 3; c++) pb[c * V + v] += rec[c];
            }
        }
        __syncthreads();
    }
    for (int v = tid; v < V; v += T)
        for (int c = 0; c < 3; c++)
            a.Xa_bar[(long long)c * nv + vb + v] = pb[c * V + v] + a.Xd_bar[(long long)c * nv + vb + v];
}

// ---- launchers ----------------------------------------------------------------

void launch_lbm_adjoint(const Geom &g, const LbmAdjArgs &a, cudaStream_t s)
{
    const dim3 grid((unsigned)((g.plane + LBM_ADJ_THREADS - 1) / LBM_ADJ_THREADS), (unsigned)g.nzc);
    lbm_adjoint_kernel<<<grid, LBM_ADJ_THREADS, 0, s>>>(a, g.nx, g.ny, g.nzc, g.nint);
    const dim3 grid2((unsigned)((g.plane + 255) / 256), (unsigned)g.nzc);
    lbm_pull_transpose_kernel<<<grid2, 256, 0, s>>>(a.gbar_pre, a.mask2d, a.gbar_in, g.nx, g.ny, g.nzc, g.nint);
}

void launch_advect_adjoint(const Geom &g, const double *X, const float4 *uvr, const double *xa_bar, double *X_bar,
                           float *ubar, long long nv, double dtM, int *flags, cudaStream_t s)
{
    if (nv <= 0) return;
    advect_adjoint_kernel<<<(unsigned)((nv + 127) / 128), 128, 0, s>>>(g, X, uvr, xa_bar, X_bar, ubar, nv, dtM, flags);
}

void launch_spread_adjoint(const Geom &g, const double *X, const float *Fv, const float *Fbar, const uint32_t *mask2d,
                           double *Fv_bar, double *X_bar, long long nv, cudaStream_t s)
{
    if (nv <= 0) return;
    spread_adjoint_kernel<<<(unsigned)((nv + 127) / 128), 128, 0, s>>>(g, X, Fv, Fbar, mask2d, Fv_bar, X_bar, nv);
}

int volume_adjoint_smem_bytes(int V) { return 48 * V; }

cudaError_t adjoint_setup(int optin)
{
    const void *ks[] = {(const void *)membrane_adjoint_kernel<1>, (const void *)membrane_adjoint_kernel<2>,
                        (const void *)membrane_adjoint_kernel<3>, (const void *)membrane_adjoint_kernel<4>,
                        (const void *)volume_adjoint_kernel};
    for (const void *k : ks) {
        cudaFuncAttributes fa{};
        cudaError_t e = cudaFuncGetAttributes(&fa, k);
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void launch_membrane_adjoint(const MembraneAdjArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    const int vpt = (a.V + MEM_ADJ_THREADS - 1) / MEM_ADJ_THREADS;
    const int T = (((a.V + vpt - 1) / vpt) + 31) / 32 * 32;
    const size_t smem = (size_t)membrane_smem_bytes(a.V);
    switch (vpt) {
    case 1: membrane_adjoint_kernel<1><<<a.ncell, T, smem, s>>>(a); break;
    case 2: membrane_adjoint_kernel<2><<<a.ncell, T, smem, s>>>(a); break;
    case 3: membrane_adjoint_kernel<3><<<a.ncell, T, smem, s>>>(a); break;
    default: membrane_adjoint_kernel<4><<<a.ncell, T, smem, s>>>(a); break;
    }
}

void launch_volume_adjoint(const Geom &g, const VolumeAdjArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    volume_adjoint_kernel<<<a.ncell, VC_ADJ_THREADS, volume_adjoint_smem_bytes(a.V), s>>>(g, a);
}

}  // namespace rbc
