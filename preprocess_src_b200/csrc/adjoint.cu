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
// its inputs.  The collision of one node is differentiated by hand in reverse
// mode, and pull streaming with half-way bounce-back, which reads every fluid
// slot exactly once, is reversed as a conflict-free push in the same kernel.
// The Skalak loads of one element and the normal / area / volume of one
// triangle are written once as templates on the scalar type; a forward-mode
// dual number (value plus one derivative) seeded on one input at a time gives
// one column of their Jacobian, which is contracted with the output adjoint.
// Spreading and interpolation are each other's transpose (plus the derivative
// of the delta weights with respect to the vertex position); RK4 runs its
// stages backwards; the mass-matrix solve M q = b (M symmetric) is reversed
// with the same Chebyshev solver; the volume correction's iterations are
// replayed and reversed one by one.
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

constexpr int LBM_ADJ_THREADS = 128;

// Adjoint of collide-stream at every fluid node, written out in reverse mode.
// The forward (lbm.cu) pulls g_q from node i - e_q (or its own opp-q slot
// across a wall link), forms drho = sum g, j = sum e g, r = 1 + drho,
// G = (r B fx, r B fy, r (pd + B fz)), u = (j + G) / (r Cr) and stores
//   post_q = (1 - om) g_q + w_q (A + eu_q (Bq + Cq eu_q + E eG_q) + D eG_q)
// with eu_q = e_q . u, eG_q = e_q . G, A = om (drho + r usq) - fo uG,
// usq = -1.5 Cr^2 u.u, uG = 3 Cr u.G, Bq = 3 Cr om r, Cq = 4.5 Cr^2 om r,
// D = 3 fo, E = 9 Cr fo, fo = 2 - om.  From the adjoints of post (gbar_out at
// the node) and of u (ubar) the chain rule, taken back through these lines,
// gives those of g, F, pd and B.  The pulled populations' adjoints go back to
// the slots they were pulled from: the pull reads every fluid slot exactly
// once (slot q of node j by node j + e_q when that node is fluid, else by j
// itself through its opp-q wall link), so the reverse is a conflict-free push
// and every fluid slot of gbar_in is written once.  Wall slots are never
// read.  dfac * dL/dpd and dL/dB are added to pbar[0..1].
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
            float g[Q];
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const long long src = ((ez(q) == 1) ? zbm : (ez(q) == -1) ? zbp : zb0) + xy - ex(q) - nx * ey(q);
                g[q] = ((m >> q) & 1u) ? a.gin[(long long)opp(q) * nint + idx] : a.gin[(long long)q * nint + src];
            }
            const float fx = a.Fx[idx], fy = a.Fy[idx], fz = a.Fz[idx];
            const float om = a.omega, Cr = a.Cr, Bc = a.Bc, pd = __ldg(a.pd);
            // forward
            float drho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
            for (int q = 0; q < Q; q++) {
                drho += g[q];
                if (ex(q)) jx += ex(q) * g[q];
                if (ey(q)) jy += ey(q) * g[q];
                if (ez(q)) jz += ez(q) * g[q];
            }
            const float r = 1.0f + drho;
            const float Gx = r * Bc * fx, Gy = r * Bc * fy, Gz = r * (pd + Bc * fz);
            const float inv = 1.0f / (r * Cr);
            const float ux = (jx + Gx) * inv, uy = (jy + Gy) * inv, uz = (jz + Gz) * inv;
            const float fo = (1.0f - 0.5f * om) * 2.0f;
            const float usq = -1.5f * Cr * Cr * (ux * ux + uy * uy + uz * uz);
            const float Bq = 3.0f * Cr * om * r, Cq = 4.5f * Cr * Cr * om * r, D = 3.0f * fo, E = 9.0f * Cr * fo;
            // reverse: post_q
            const float4 ub = a.ubar[idx];
            float ob[Q];
            float Ab = 0.f, Bb = 0.f, Cb = 0.f;
            float uxb = ub.x, uyb = ub.y, uzb = ub.z, Gxb = 0.f, Gyb = 0.f, Gzb = 0.f;
#pragma unroll
            for (int q = 0; q < Q; q++) {
                ob[q] = a.gbar_out[(long long)q * nint + idx];
                const float W = wq(q) * ob[q];
                const float eu = ex(q) * ux + ey(q) * uy + ez(q) * uz;
                const float eG = ex(q) * Gx + ey(q) * Gy + ez(q) * Gz;
                Ab += W; Bb += W * eu; Cb += W * eu * eu;
                const float eub = W * (Bq + 2.0f * Cq * eu + E * eG), eGb = W * (E * eu + D);
                if (ex(q)) { uxb += ex(q) * eub; Gxb += ex(q) * eGb; }
                if (ey(q)) { uyb += ey(q) * eub; Gyb += ey(q) * eGb; }
                if (ez(q)) { uzb += ez(q) * eub; Gzb += ez(q) * eGb; }
            }
            // A, Bq, Cq
            float drhob = om * Ab;
            float rb = om * usq * Ab + 3.0f * Cr * om * Bb + 4.5f * Cr * Cr * om * Cb;
            const float ku = -3.0f * Cr * Cr * (om * r * Ab), kG = 3.0f * Cr * (-fo * Ab);
            uxb += ku * ux + kG * Gx; uyb += ku * uy + kG * Gy; uzb += ku * uz + kG * Gz;
            Gxb += kG * ux; Gyb += kG * uy; Gzb += kG * uz;
            // u = (j + G) / (r Cr)
            const float jxb = uxb * inv, jyb = uyb * inv, jzb = uzb * inv;
            Gxb += jxb; Gyb += jyb; Gzb += jzb;
            rb -= (uxb * ux + uyb * uy + uzb * uz) / r;
            // G
            rb += Bc * (Gxb * fx + Gyb * fy) + Gzb * (pd + Bc * fz);
            a.Fbar[idx] = Gxb * r * Bc; a.Fbar[nint + idx] = Gyb * r * Bc; a.Fbar[2 * nint + idx] = Gzb * r * Bc;
            dP = (double)(Gzb * r);
            dB = (double)(r * (Gxb * fx + Gyb * fy + Gzb * fz));
            drhob += rb;
            const float om1 = 1.0f - om;
#pragma unroll
            for (int q = 0; q < Q; q++) {
                const float gb = om1 * ob[q] + drhob + ex(q) * jxb + ey(q) * jyb + ez(q) * jzb;
                const long long src = ((ez(q) == 1) ? zbm : (ez(q) == -1) ? zbp : zb0) + xy - ex(q) - nx * ey(q);
                if ((m >> q) & 1u) a.gbar_in[(long long)opp(q) * nint + idx] = gb;
                else a.gbar_in[(long long)q * nint + src] = gb;
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
        atomicAdd(&a.pbar[0], __ldg(a.dfac) * sp);
        atomicAdd(&a.pbar[1], sb);
    }
}

// ---- delta stencil with position derivatives ------------------------------

// One warp per vertex for the interpolation and spreading adjoints: lane l
// owns the stencil nodes k = l and l + 32 of the 64 (k = a + 4 b + 16 c with
// x offset a, y offset b, z plane c from the node below the position minus 1).
// delta4 (rbc_internal.cuh) weights in FP64 with their derivatives: with
// s = sin(pi f / 2), c = cos(pi f / 2), w = (1 - s, 1 + c, 1 + s, 1 - c) / 4
// and dw/df = (pi / 8) (-c, -s, c, s).
__device__ __forceinline__ void delta_w(int k, double s, double c, double &w, double &dw)
{
    const double pi8 = 0.125 * 3.14159265358979323846;
    w = k == 0 ? 0.25 * (1.0 - s) : k == 1 ? 0.25 * (1.0 + c) : k == 2 ? 0.25 * (1.0 + s) : 0.25 * (1.0 - c);
    dw = k == 0 ? -pi8 * c : k == 1 ? -pi8 * s : k == 2 ? pi8 * c : pi8 * s;
}

struct LaneStencil {
    long long n[2];     // lattice index of the lane's two nodes, -1 = dropped
    double w[2];        // weights
    double dw[2][3];    // d weight / d position
};

// The lane's two nodes of the stencil at p.  Nodes outside x, y or beyond the
// two BUFF planes of the position's own z frame are dropped, as in the forward
// spread (ibm.cu:107-110) and interpolation (ibm.cu:453-455).
__device__ __forceinline__ void lane_stencil(const Geom &g, double px, double py, double pz, int lane, LaneStencil &s)
{
    const double lx = lat_x(g, px), ly = lat_y(g, py), lz = lat_z(g, pz);
    const double flx = floor(lx), fly = floor(ly), flz = floor(lz);
    double sx, cx, sy, cy, sz, cz;
    sincospi(0.5 * (lx - flx), &sx, &cx);
    sincospi(0.5 * (ly - fly), &sy, &cy);
    sincospi(0.5 * (lz - flz), &sz, &cz);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int k = lane + 32 * h, a = k & 3, b = (k >> 2) & 3, c = k >> 4;
        const int gx = (int)flx - 1 + a, gy = (int)fly - 1 + b, iz = (int)flz - 1 + c;
        const bool in = gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && iz >= -2 && iz < g.nzc + 2;
        s.n[h] = in ? (long long)wrap_z(iz, g.nzc) * g.plane + gx + (long long)g.nx * gy : -1LL;
        double wa, da, wb, db, wc, dc;
        delta_w(a, sx, cx, wa, da);
        delta_w(b, sy, cy, wb, db);
        delta_w(c, sz, cz, wc, dc);
        s.w[h] = wa * wb * wc;
        s.dw[h][0] = da * wb * wc * g.inv_dx;
        s.dw[h][1] = wa * db * wc * g.inv_dx;
        s.dw[h][2] = wa * wb * dc * g.inv_dx;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;   // the butterfly leaves the same sum in every lane
}

// a lattice coordinate the stencil arithmetic can take (as in ibm.cu)
__device__ __forceinline__ bool sane_pos(const Geom &g, double px, double py, double pz) {
    return fabs(lat_x(g, px)) < 16777216.0 && fabs(lat_y(g, py)) < 16777216.0 && fabs(lat_z(g, pz)) < 16777216.0;
}

// ---- interpolation + RK4, reversed -----------------------------------------

constexpr int VTX_ADJ_THREADS = 128;   // four vertices per CTA, one warp each

// Velocity of the frozen field at p as the forward advection interpolates it
// (every lane returns the same sum).
__device__ __forceinline__ void warp_interp(const Geom &g, const float4 *__restrict__ uvr, const double p[3], int lane,
                                            double u[3]) {
    LaneStencil s;
    lane_stencil(g, p[0], p[1], p[2], lane, s);
    double u0 = 0.0, u1 = 0.0, u2 = 0.0;
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (s.n[h] >= 0) {
            const float4 q = __ldg(&uvr[s.n[h]]);
            u0 += s.w[h] * q.x; u1 += s.w[h] * q.y; u2 += s.w[h] * q.z;
        }
    u[0] = warp_sum(u0); u[1] = warp_sum(u1); u[2] = warp_sum(u2);
}

// Adjoint of one interpolation at p with output adjoint kb: adds w_n kb to
// the velocity adjoint of each stencil node; returns in pb (every lane) the
// position adjoint sum_n (d w_n / d p) (u_n . kb).
__device__ __forceinline__ void warp_interp_adjoint(const Geom &g, const float4 *__restrict__ uvr,
                                                    float *__restrict__ ubar, const double p[3], const double kb[3],
                                                    int lane, double pb[3]) {
    LaneStencil s;
    lane_stencil(g, p[0], p[1], p[2], lane, s);
    double b0 = 0.0, b1 = 0.0, b2 = 0.0;
#pragma unroll
    for (int h = 0; h < 2; h++)
        if (s.n[h] >= 0) {
            const long long n = s.n[h];
            const float4 q = __ldg(&uvr[n]);
            atomicAdd(&ubar[4 * n + 0], (float)(s.w[h] * kb[0]));
            atomicAdd(&ubar[4 * n + 1], (float)(s.w[h] * kb[1]));
            atomicAdd(&ubar[4 * n + 2], (float)(s.w[h] * kb[2]));
            const double uk = q.x * kb[0] + q.y * kb[1] + q.z * kb[2];
            b0 += s.dw[h][0] * uk; b1 += s.dw[h][1] * uk; b2 += s.dw[h][2] * uk;
        }
    pb[0] = warp_sum(b0); pb[1] = warp_sum(b1); pb[2] = warp_sum(b2);
}

// One warp per vertex.  xa_bar: adjoint of the advected positions; writes
// X_bar (adjoint of X_t through the advection, overwritten) and adds to ubar.
// The periodic wrap of the result in x and z is a translation (derivative 1).
__global__ void __launch_bounds__(VTX_ADJ_THREADS)
advect_adjoint_kernel(const Geom g, const double *__restrict__ X, const float4 *__restrict__ uvr,
                      const double *__restrict__ xa_bar, double *__restrict__ X_bar, float *__restrict__ ubar,
                      long long nv, double dtM, int *__restrict__ flags)
{
    const long long v = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (v >= nv) return;   // uniform over the warp
    double p[4][3], k[3][3];
    p[0][0] = X[v]; p[0][1] = X[nv + v]; p[0][2] = X[2 * nv + v];
    if (!sane_pos(g, p[0][0], p[0][1], p[0][2])) {
        if (lane == 0) {
            atomicOr(flags, RBC_FLAG_NONFINITE);
            X_bar[v] = X_bar[nv + v] = X_bar[2 * nv + v] = 0.0;
        }
        return;
    }
    const double hs[4] = {0.0, 0.5 * dtM, 0.5 * dtM, dtM};   // stage offsets (ibm.cu:474-498)
    for (int s = 0; s < 3; s++) {
        warp_interp(g, uvr, p[s], lane, k[s]);
        // the forward adds the FP32 stage velocity to the FP64 position
        for (int c = 0; c < 3; c++) p[s + 1][c] = p[0][c] + (double)(float)k[s][c] * hs[s + 1];
    }
    double xb[3], kb[4][3];
    for (int c = 0; c < 3; c++) {
        const double a = xa_bar[(long long)c * nv + v];
        xb[c] = a;   // Xa = X + dt (k1 + 2 k2 + 2 k3 + k4) / 6
        kb[0][c] = a * dtM / 6.0; kb[1][c] = a * dtM / 3.0; kb[2][c] = a * dtM / 3.0; kb[3][c] = a * dtM / 6.0;
    }
    for (int s = 3; s >= 0; s--) {
        double pb[3];
        warp_interp_adjoint(g, uvr, ubar, p[s], kb[s], lane, pb);
        for (int c = 0; c < 3; c++) {
            xb[c] += pb[c];
            if (s > 0) kb[s - 1][c] += hs[s] * pb[c];   // p_s = X + h_s k_s-1
        }
    }
    if (lane < 3) X_bar[(long long)lane * nv + v] = xb[lane];
}

// ---- spreading, reversed --------------------------------------------------

// F(n) = sum_v w_n(X_v) Fv_v / dx^3 over fluid columns.  One warp per vertex:
// Fv_bar = sum_n w_n Fbar(n) / dx^3 (overwritten) and
// X_bar += sum_n (d w_n / d X) (Fv . Fbar(n)) / dx^3.
__global__ void __launch_bounds__(VTX_ADJ_THREADS)
spread_adjoint_kernel(const Geom g, const double *__restrict__ X, const float *__restrict__ Fv,
                      const float *__restrict__ Fbar, const uint32_t *__restrict__ mask2d,
                      double *__restrict__ Fv_bar, double *__restrict__ X_bar, long long nv)
{
    const long long v = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (v >= nv) return;   // uniform over the warp
    const double p[3] = {X[v], X[nv + v], X[2 * nv + v]};
    double fb[3] = {0.0, 0.0, 0.0}, pb[3] = {0.0, 0.0, 0.0};
    if (sane_pos(g, p[0], p[1], p[2])) {
        const double wscale = 1.0 / (g.dx * g.dx * g.dx);
        const double f[3] = {Fv[v], Fv[nv + v], Fv[2 * nv + v]};
        LaneStencil s;
        lane_stencil(g, p[0], p[1], p[2], lane, s);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const long long n = s.n[h];
            if (n < 0 || !(__ldg(&mask2d[n % g.plane]) & MASK_FLUID)) continue;
            const double F0 = Fbar[n], F1 = Fbar[g.nint + n], F2 = Fbar[2 * g.nint + n];
            const double w = s.w[h] * wscale;
            fb[0] += w * F0; fb[1] += w * F1; fb[2] += w * F2;
            const double fF = (f[0] * F0 + f[1] * F1 + f[2] * F2) * wscale;
            pb[0] += s.dw[h][0] * fF; pb[1] += s.dw[h][1] * fF; pb[2] += s.dw[h][2] * fF;
        }
    }
    for (int c = 0; c < 3; c++) { fb[c] = warp_sum(fb[c]); pb[c] = warp_sum(pb[c]); }
    if (lane < 3) {
        Fv_bar[(long long)lane * nv + v] = fb[lane];
        X_bar[(long long)lane * nv + v] += pb[lane];
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

// The forward solves M q = b per cell (b = element loads gathered per vertex,
// M the P1 mass matrix) and sets Fv = -q ds (ds = one-ring area / 3).  Its
// reverse, from Fv_bar: q_bar = -ds Fv_bar, ds_bar = -q . Fv_bar,
// lambda = M^-1 q_bar (Chebyshev on D^-1 M as the forward: with M symmetric
// the transpose of the polynomial solve is the same polynomial solve),
// b_bar = lambda, M_bar = -lambda q^T.  Three kernels: the per-cell solve,
// one thread per element for the element Jacobians, one thread per vertex
// for the gather.

// One CTA per cell: element areas (scratch[7 e]), rows of D^-1 M, q, ds_bar,
// and lambda; writes lam, qv, dsb per vertex.
template <int VPT>
__global__ void __launch_bounds__(MEM_ADJ_THREADS, 1)
membrane_adjoint_solve_kernel(const MembraneAdjArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    const int V = a.V, E = a.E, tid = threadIdx.x, T = blockDim.x;
    float4 *dbuf = reinterpret_cast<float4 *>(smem);                    // [2][V]
    float *coef = reinterpret_cast<float *>(smem + 32 * (size_t)V);     // [6][V]
    int16_t *snbr = reinterpret_cast<int16_t *>(smem + 56 * (size_t)V); // [6][V]
    const int cell = blockIdx.x;
    const long long vb = (long long)cell * V, eb = (long long)cell * E, nv = a.nv;
    double *er = a.scratch + eb * 7;
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
#pragma unroll
    for (int m = 0; m < VPT; m++) {
        const int i = tid + m * T;
        if (i >= V) continue;
        a.lam[vb + i] = make_float4(x[m][0], x[m][1], x[m][2], 0.f);
        a.qv[vb + i] = make_float4(q[m][0], q[m][1], q[m][2], 0.f);
        a.dsb[vb + i] = dsb[m];
    }
}

constexpr int MEM_ADJ_ELEM_THREADS = 128;

// One thread per element of any cell: the adjoints of (load on b, load on c,
// gab) from lambda, q and ds_bar of the element's vertices, contracted with
// the Jacobian of element_loads (seven dual passes: e1, e2, C).  Writes the
// edge adjoints to scratch[7 e + 1 .. 6] and adds dL/dC to cbar.
__global__ void __launch_bounds__(MEM_ADJ_ELEM_THREADS)
membrane_adjoint_element_kernel(const MembraneAdjArgs a)
{
    __shared__ double red[MEM_ADJ_ELEM_THREADS / 32];
    const long long eg = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double cb = 0.0;
    if (eg < a.ne) {
        const int cell = (int)(eg / a.E), e = (int)(eg - (long long)cell * a.E);
        const long long vb = (long long)cell * a.V;
        double e1[3], e2[3];
        int ia, ib, ic;
        edges_of(a, vb, e, e1, e2, ia, ib, ic);
        const float4 la = a.lam[vb + ia], lb = a.lam[vb + ib], lc = a.lam[vb + ic];
        const float4 qa = a.qv[vb + ia], qb = a.qv[vb + ib], qc = a.qv[vb + ic];
        auto dotf = [](float4 u, float4 w) { return (double)u.x * w.x + (double)u.y * w.y + (double)u.z * w.z; };
        // M = sum_e gab (1 + delta_ij) / 24 over the element's vertex pairs; ds_i = sum_e gab / 6
        const double mdiag = -(dotf(la, qa) + dotf(lb, qb) + dotf(lc, qc));
        const double moff = -(dotf(la, qb) + dotf(lb, qa) + dotf(la, qc) + dotf(lc, qa) + dotf(lb, qc) + dotf(lc, qb));
        const double gb = mdiag / 12.0 + moff / 24.0 + ((double)a.dsb[vb + ia] + a.dsb[vb + ib] + a.dsb[vb + ic]) / 6.0;
        const double bBb[3] = {(double)lb.x - la.x, (double)lb.y - la.y, (double)lb.z - la.z};
        const double bCb[3] = {(double)lc.x - la.x, (double)lc.y - la.y, (double)lc.z - la.z};
        const double4 G = a.gref[eg];
        double *er = a.scratch + 7 * eg;
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
            if (k < 6) er[1 + k] = s; else cb = s;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cb += __shfl_xor_sync(0xffffffffu, cb, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = cb;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < MEM_ADJ_ELEM_THREADS / 32; w++) s += red[w];
        atomicAdd(a.cbar, s);
    }
}

// One thread per vertex of any cell: edge adjoints to the vertices
// (e1 = x_b - x_a, e2 = x_c - x_a); writes Xd_bar.
__global__ void membrane_adjoint_vertex_kernel(const MembraneAdjArgs a)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.nv) return;
    const int cell = (int)(t / a.V), i = (int)(t - (long long)cell * a.V);
    const double *er = a.scratch + 7 * ((long long)cell * a.E);
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
    for (int c = 0; c < 3; c++) a.Xd_bar[(long long)c * a.nv + t] = xb[c];
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
    auto vol_area = [&](const double *P, double &vol, double &area) {   // as volume.cu measures them
        double sv = 0.0, sa = 0.0;
        for (int e = tid; e < E; e += T) {
            double A[3], B[3], Cc[3];
            tri_at(P, e, A, B, Cc);
            tri_measure(A, B, Cc, sv, sa);
        }
        vol = block_sum_r(sv, red) / 18.0;
        area = block_sum_r(sa, red) / 2.0;
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
}

static unsigned warp_blocks(long long nv) {
    return (unsigned)((nv * 32 + VTX_ADJ_THREADS - 1) / VTX_ADJ_THREADS);
}

void launch_advect_adjoint(const Geom &g, const double *X, const float4 *uvr, const double *xa_bar, double *X_bar,
                           float *ubar, long long nv, double dtM, int *flags, cudaStream_t s)
{
    if (nv <= 0) return;
    advect_adjoint_kernel<<<warp_blocks(nv), VTX_ADJ_THREADS, 0, s>>>(g, X, uvr, xa_bar, X_bar, ubar, nv, dtM, flags);
}

void launch_spread_adjoint(const Geom &g, const double *X, const float *Fv, const float *Fbar, const uint32_t *mask2d,
                           double *Fv_bar, double *X_bar, long long nv, cudaStream_t s)
{
    if (nv <= 0) return;
    spread_adjoint_kernel<<<warp_blocks(nv), VTX_ADJ_THREADS, 0, s>>>(g, X, Fv, Fbar, mask2d, Fv_bar, X_bar, nv);
}

int volume_adjoint_smem_bytes(int V) { return 48 * V; }

cudaError_t adjoint_setup(int optin)
{
    const void *ks[] = {(const void *)membrane_adjoint_solve_kernel<1>, (const void *)membrane_adjoint_solve_kernel<2>,
                        (const void *)membrane_adjoint_solve_kernel<3>, (const void *)membrane_adjoint_solve_kernel<4>,
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
    case 1: membrane_adjoint_solve_kernel<1><<<a.ncell, T, smem, s>>>(a); break;
    case 2: membrane_adjoint_solve_kernel<2><<<a.ncell, T, smem, s>>>(a); break;
    case 3: membrane_adjoint_solve_kernel<3><<<a.ncell, T, smem, s>>>(a); break;
    default: membrane_adjoint_solve_kernel<4><<<a.ncell, T, smem, s>>>(a); break;
    }
    membrane_adjoint_element_kernel<<<(unsigned)((a.ne + MEM_ADJ_ELEM_THREADS - 1) / MEM_ADJ_ELEM_THREADS),
                                      MEM_ADJ_ELEM_THREADS, 0, s>>>(a);
    membrane_adjoint_vertex_kernel<<<(unsigned)((a.nv + 127) / 128), 128, 0, s>>>(a);
}

void launch_volume_adjoint(const Geom &g, const VolumeAdjArgs &a, cudaStream_t s)
{
    if (a.ncell <= 0) return;
    volume_adjoint_kernel<<<a.ncell, VC_ADJ_THREADS, volume_adjoint_smem_bytes(a.V), s>>>(g, a);
}

}  // namespace rbc
