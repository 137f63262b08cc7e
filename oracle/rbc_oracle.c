/*
 * rbc_oracle.c -- FP64 CPU oracle for the coupled fluid-membrane step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see rbc_oracle.h).  Each function
 * restates the reference's algorithm on the reference's own layout and cites
 * the reference file:line it follows.  OpenMP parallelises loops whose
 * iterations are independent; loops with scattered accumulation (the IB
 * spread) run sequentially so results are deterministic.
 */
#define _DEFAULT_SOURCE   /* M_PI */
#include "rbc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* D3Q19 velocity set in the reference's slot order (lbm.cu:1038-1047):
 * ___ p__ m__ _p_ _m_ __p __m pp_ mm_ mp_ pm_ _pp _mm _mp _pm p_p m_m p_m m_p */
static const int EX[ORC_Q] = {0, 1,-1, 0, 0, 0, 0, 1,-1,-1, 1, 0, 0, 0, 0, 1,-1, 1,-1};
static const int EY[ORC_Q] = {0, 0, 0, 1,-1, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1, 0, 0, 0, 0};
static const int EZ[ORC_Q] = {0, 0, 0, 0, 0, 1,-1, 0, 0, 0, 0, 1,-1, 1,-1, 1,-1,-1, 1};
static const int OPP[ORC_Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7,10, 9,12,11,14,13,16,15,18,17};
static const double WQ[ORC_Q] = {1.0/3.0,
    1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0, 1.0/18.0,
    1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0,
    1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0, 1.0/36.0};

#define COEFF_VOL_CHANGE 0.1   /* volume_correction.cu:14 */
#define VC_EPS           1.0e-03 /* volume_correction.cu:15 (percent) */
#define VC_ITRMAX        1000  /* volume_correction.cu:487 */

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

static inline double min_image(double d, double L)
{
    /* stress.cu:63-72: one shift by L when |d| > L/2 */
    if (d > L * 0.5) d -= L; else if (d < -L * 0.5) d += L;
    return d;
}

/* ------------------------------------------------------------------------ */
/* Setup                                                                     */
/* ------------------------------------------------------------------------ */

/* init2.cu:12-42 */
static void add_nlink(int na, int nb, int *nln, int *ln)
{
    int flag = 0;
    for (int i = 0; i < nln[na]; i++) if (nb == ln[7 * na + i]) flag = 1;
    if (flag == 0) { ln[7 * na + nln[na]] = nb; nln[na]++; }
}

/* init2.cu:45-63 */
static void add_elink(int ni, int ei, int *nle, int *le)
{
    le[6 * ni + nle[ni]] = ei;
    nle[ni]++;
}

/* init2.cu:66-89 */
static int checklink(int na, int nb, const int *nln, const int *ln)
{
    int flag = 0;
    for (int i = 0; i < nln[na]; i++) if (nb == ln[7 * na + i]) flag = 1;
    return flag;
}

/* init2.cu:92-166: order each one-ring counter-clockwise about the outward
 * direction (vertex minus cell centroid). */
static int sort_link_spring(const double *x, const int *nln, int *ln, int vertex, int ic)
{
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int j = 0; j < vertex; j++) {
        int jid = ic * vertex + j;
        gx += x[3 * jid + 0]; gy += x[3 * jid + 1]; gz += x[3 * jid + 2];
    }
    gx /= vertex; gy /= vertex; gz /= vertex;

    for (int j = 0; j < vertex; j++) {
        int jid = ic * vertex + j, n = 0, lns[7];
        lns[0] = ln[7 * jid + 0];
        for (int k = 1; k < nln[jid]; k++) {
            int na = lns[k - 1];
            double va[3] = {x[3*na+0] - x[3*jid+0], x[3*na+1] - x[3*jid+1], x[3*na+2] - x[3*jid+2]};
            for (int l = 0; l < nln[jid]; l++) {
                int nb = ln[7 * jid + l];
                if (na == nb) continue;
                if (checklink(na, nb, nln, ln) == 1) {
                    double vb[3] = {x[3*nb+0] - x[3*jid+0], x[3*nb+1] - x[3*jid+1], x[3*nb+2] - x[3*jid+2]};
                    double c[3] = {va[1]*vb[2] - va[2]*vb[1], va[2]*vb[0] - va[0]*vb[2], va[0]*vb[1] - va[1]*vb[0]};
                    double inpro = c[0] * (x[3*jid+0] - gx) + c[1] * (x[3*jid+1] - gy) + c[2] * (x[3*jid+2] - gz);
                    if (inpro > 0) { lns[k] = nb; n++; }
                }
            }
        }
        if (n + 1 != nln[jid]) return 3;
        for (int k = 0; k < nln[jid]; k++) ln[7 * jid + k] = lns[k];
    }
    return 0;
}

/* init2.cu:169-203: append the vertex itself and sort ascending. */
static void sort_link_order(const int *nln, int *lo, int vertex, int ic)
{
    for (int j = 0; j < vertex; j++) {
        int jid = ic * vertex + j;
        lo[7 * jid + nln[jid]] = jid;
        for (int k = 0; k < nln[jid] + 1; k++)
            for (int l = nln[jid]; l > k; l--)
                if (lo[7*jid + l - 1] > lo[7*jid + l]) {
                    int tmp = lo[7*jid + l]; lo[7*jid + l] = lo[7*jid + l - 1]; lo[7*jid + l - 1] = tmp;
                }
    }
}

/* init2.cu:206-255 */
static void set_contravariant(const double *xr, double *n, const int *ele, int cln, int element)
{
    for (int ic = 0; ic < cln; ic++)
        for (int e = 0; e < element; e++) {
            int eid = ic * element + e;
            int ea = ele[3*eid+0], eb = ele[3*eid+1], ec = ele[3*eid+2];
            double v1[3], v2[3];
            for (int j = 0; j < 3; j++) { v1[j] = xr[3*eb+j] - xr[3*ea+j]; v2[j] = xr[3*ec+j] - xr[3*ea+j]; }
            double lv1 = v1[0]*v1[0] + v1[1]*v1[1] + v1[2]*v1[2];
            double lv2 = v2[0]*v2[0] + v2[1]*v2[1] + v2[2]*v2[2];
            double inv12 = v1[0]*v2[0] + v1[1]*v2[1] + v1[2]*v2[2];
            double dv12 = lv1 * lv2 - inv12 * inv12;
            n[4*eid+0] = lv2 / dv12;  n[4*eid+1] = -inv12 / dv12;
            n[4*eid+2] = -inv12 / dv12; n[4*eid+3] = lv1 / dv12;
        }
}

/* init2.cu:258-400 (fem_init, RBC branch) */
/* init1.cu:755-795: cel->ec, the elements sharing an edge with each element,
 * in increasing element order (the reference scans all elements of the cell) */
static void edge_neighbours(const orc_params *p, orc_state *s)
{
    const long ne = (long)p->ncell * p->element;
    for (long e1 = 0; e1 < ne; e1++) {
        long nb[3] = {-1, -1, -1};
        int cnt = 0;
        for (int a = 0; a < 3; a++) {
            const int ia = s->ele[e1*3 + a], ib = s->ele[e1*3 + (a + 1) % 3];
            for (int k = 0; k < s->nle[ia]; k++) {
                const long e2 = s->le[ia*6 + k];
                if (e2 == e1) continue;
                if (s->ele[e2*3] == ib || s->ele[e2*3+1] == ib || s->ele[e2*3+2] == ib) {
                    if (cnt < 3) nb[cnt++] = e2;
                    break;
                }
            }
        }
        for (int x = 0; x < cnt; x++)   /* increasing element order */
            for (int y = x + 1; y < cnt; y++)
                if (nb[y] < nb[x]) { long t = nb[x]; nb[x] = nb[y]; nb[y] = t; }
        for (int k = 0; k < 3; k++) s->ec[e1*3 + k] = (int)(k < cnt ? nb[k] : e1);
    }
}

int orc_fem_init(const orc_params *p, orc_state *s)
{
    int V = p->vertex, E = p->element, N = p->ncell;
    int n_edge = V + E - 2;
    memset(s->nln, 0, sizeof(int) * (size_t)N * V);
    memset(s->ln, 0, sizeof(int) * (size_t)N * V * 7);
    memset(s->lo, 0, sizeof(int) * (size_t)N * V * 7);
    memset(s->nle, 0, sizeof(int) * (size_t)N * V);
    memset(s->le, 0, sizeof(int) * (size_t)N * V * 6);
    for (int i = 0; i < N; i++) {
        for (int e = 0; e < E; e++) {
            int eid = i * E + e;
            int ea = s->ele[3*eid+0], eb = s->ele[3*eid+1], ec = s->ele[3*eid+2];
            add_nlink(ea, eb, s->nln, s->ln); add_nlink(ea, ec, s->nln, s->ln);
            add_nlink(eb, ec, s->nln, s->ln); add_nlink(eb, ea, s->nln, s->ln);
            add_nlink(ec, ea, s->nln, s->ln); add_nlink(ec, eb, s->nln, s->ln);
            add_elink(ea, eid, s->nle, s->le); add_elink(eb, eid, s->nle, s->le);
            add_elink(ec, eid, s->nle, s->le);
        }
        int checker = 0;
        for (int j = 0; j < V; j++) checker += s->nln[i * V + j];
        if (checker != 2 * n_edge) return 3;
        for (int j = 0; j < V; j++) {
            int jid = i * V + j;
            for (int k = 0; k < s->nln[jid]; k++) s->lo[7*jid + k] = s->ln[7*jid + k];
        }
        if (sort_link_spring(s->xd, s->nln, s->ln, V, i) != 0) return 3;
        sort_link_order(s->nln, s->lo, V, i);
    }
    set_contravariant(s->xd, s->nd, s->ele, N, E);
    if (s->ec) edge_neighbours(p, s);
    return 0;
}

/* init1.cu:413-434 with td = 1, u = 0 (CapsuleCHANNELFLOW branch 399-407) */
void orc_flu_init(const orc_params *p, orc_state *s)
{
    long n = (long)p->nx * p->ny * p->nz, plane = (long)p->nx * p->ny;
    double LY = (double)(p->ny - 4) * p->dx, Cr = p->Cr, Cr2 = Cr * Cr;
    for (long i = 0; i < n; i++) {
        double tw = 0.0;
        if (p->flow == 1 && p->flowstart == 0) {
            long iy = (i % plane) / p->nx;
            tw = p->walls == 0 ? p->sr * (-LY / 2.0 - 1.5 * p->dx + (double)iy * p->dx)
                               : p->sr * (-1.5 * p->dx + (double)iy * p->dx);
        }
        double uvw = -1.5 * tw * tw * Cr2;
        for (int q = 0; q < ORC_Q; q++) {
            double eu = EZ[q] * tw;
            s->fn[i*ORC_Q + q] = WQ[q] * (1.0 + 3.0 * eu * Cr + 4.5 * eu * eu * Cr2 + uvw);
            s->fm[i*ORC_Q + q] = 0.0;
        }
        s->dn[i] = 1.0; s->un[i] = 0.0; s->vn[i] = 0.0; s->wn[i] = tw;
        s->dm[i] = 1.0; s->um[i] = 0.0; s->vm[i] = 0.0; s->wm[i] = tw;
        s->fx[i] = 0.0; s->fy[i] = 0.0; s->fz[i] = 0.0;
    }
}

/* ------------------------------------------------------------------------ */
/* Membrane: stress.cu                                                       */
/* ------------------------------------------------------------------------ */

/* stress.cu:29-121 (principal-tension diagnostics tp omitted) */
void orc_calc_tension(const orc_params *p, orc_state *s)
{
    long ne = (long)p->ncell * p->element;
    const double *x = s->xd, *n = s->nd;
#pragma omp parallel for schedule(static)
    for (long j = 0; j < ne; j++) {
        int ea = s->ele[3*j+0], eb = s->ele[3*j+1], ec = s->ele[3*j+2];
        double v1d[3], v2d[3];
        for (int i = 0; i < 3; i++) {
            v1d[i] = x[3*eb + i] - x[3*ea + i];
            v2d[i] = x[3*ec + i] - x[3*ea + i];
            if (i == 0) { v1d[i] = min_image(v1d[i], p->LX); v2d[i] = min_image(v2d[i], p->LX); }
            else if (i == 2) { v1d[i] = min_image(v1d[i], p->LZ); v2d[i] = min_image(v2d[i], p->LZ); }
        }
        double lv1d = sqrt(v1d[0]*v1d[0] + v1d[1]*v1d[1] + v1d[2]*v1d[2]);
        double lv2d = sqrt(v2d[0]*v2d[0] + v2d[1]*v2d[1] + v2d[2]*v2d[2]);
        double inv12d = v1d[0]*v2d[0] + v1d[1]*v2d[1] + v1d[2]*v2d[2];
        double dv12d = (lv1d*lv1d) * (lv2d*lv2d) - inv12d * inv12d;
        double dn12 = n[4*j+0] * n[4*j+3] - n[4*j+1] * n[4*j+2];
        s->rg[j] = sqrt(dv12d);
        double vd[4] = {lv1d*lv1d, inv12d, inv12d, lv2d*lv2d};
        double ndf[4] = {vd[3]/dv12d, -vd[1]/dv12d, -vd[2]/dv12d, vd[0]/dv12d};
        double i1 = n[4*j+0]*vd[0] + n[4*j+1]*vd[1] + n[4*j+2]*vd[2] + n[4*j+3]*vd[3] - 2.0;
        double i2 = dv12d * dn12 - 1.0;
        double js = sqrt(i2 + 1.0);
        const double rgs = s->crg ? s->crg[j / p->element] : p->rgs;
        for (int i = 0; i < 4; i++) {
            if (p->law == 0)
                s->t[4*j + i] = rgs * (i1 + 1.0) / js * n[4*j + i] + (p->C * i2 - 1.0) * js * ndf[i];
            else
                s->t[4*j + i] = rgs * (n[4*j + i] / js - ndf[i] * js / (i2 + 1.0) / (i2 + 1.0));
        }
    }
}

/* matrix_solver.cu:266-277 (spmv_ell) */
static void spmv_ell(const int *ptr, const int *index, const double *value,
                     const double *in, double *out, int n)
{
    for (int tid = 0; tid < n; tid++) {
        double sum = 0.0;
        for (int i = 0; i < ptr[tid]; i++) { int jj = i * n + tid; sum += value[jj] * in[index[jj]]; }
        out[tid] = sum;
    }
}

static double dot(const double *a, const double *b, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* matrix_solver.cu:279-377 (bicgstab); dot_product.cu sums are plain sums here */
static int bicgstab(const int *ptr, const int *index, const double *value, double *x, const double *b,
                    double *ra, double *r, double *pp, double *m, double *nn, int n,
                    double residual, int itrmax, int *iters)
{
    double err, alfa = 1.0, beta = 0.0, omeg = 1.0;
    double r_dot_ra = 0.0, r_dot_ra_old;
    int iter;
    memset(ra, 0, sizeof(double) * n); memset(r, 0, sizeof(double) * n);
    memset(pp, 0, sizeof(double) * n); memset(m, 0, sizeof(double) * n);
    memset(nn, 0, sizeof(double) * n);
    spmv_ell(ptr, index, value, x, r, n);
    for (int i = 0; i < n; i++) { double t = b[i] - r[i]; r[i] = t; ra[i] = t; pp[i] = t; }
    double b_dot_b = dot(b, b, n);
    for (iter = 0; iter < itrmax; iter++) {
        r_dot_ra_old = r_dot_ra;
        r_dot_ra = dot(r, ra, n);
        if (r_dot_ra == 0) { *iters = iter; return 1; }
        if (iter > 0) {
            beta = (r_dot_ra / r_dot_ra_old) * (alfa / omeg);
            for (int i = 0; i < n; i++) pp[i] = r[i] + beta * (pp[i] - omeg * m[i]);
        }
        spmv_ell(ptr, index, value, pp, m, n);
        alfa = r_dot_ra / dot(m, ra, n);
        for (int i = 0; i < n; i++) r[i] = r[i] - alfa * m[i];
        spmv_ell(ptr, index, value, r, nn, n);
        omeg = dot(r, nn, n) / dot(nn, nn, n);
        for (int i = 0; i < n; i++) { x[i] = x[i] + alfa * pp[i] + omeg * r[i]; r[i] = r[i] - omeg * nn[i]; }
        err = sqrt(dot(r, r, n) / b_dot_b);
        if (err < residual) break;
    }
    *iters = iter;
    if (iter >= itrmax) return 2;
    return 0;
}

/* stress.cu:306-373 (calc_load) with initialize (124-143), set_matrix_component
 * (146-179), set_matrix_coefficient (182-272) and substitute_load (275-303). */
int orc_calc_load(const orc_params *p, orc_state *s)
{
    int V = p->vertex, mn = p->mn, N = p->ncell, flag_all = 0, maxit = 0;
    static const double f[3][2] = {{-1.0, -1.0}, {1.0, 0.0}, {0.0, 1.0}};
#pragma omp parallel for schedule(dynamic, 1) reduction(|:flag_all) reduction(max:maxit)
    for (int cid = 0; cid < N; cid++) {
        int *ptr = (int *)calloc(mn, sizeof(int));
        int *index = (int *)calloc((size_t)mn * 7, sizeof(int));
        double *value = (double *)calloc((size_t)mn * 7, sizeof(double));
        double *qc = (double *)calloc(mn, sizeof(double));
        double *bc = (double *)calloc(mn, sizeof(double));
        double *w = (double *)calloc((size_t)mn * 5, sizeof(double));
        for (int j = 0; j < mn; j++) {
            int node = j / 3, d = j % 3, jj = node + cid * V;
            if (node < V) {
                ptr[j] = s->nln[jj] + 1;
                for (int i = 0; i < s->nln[jj] + 1; i++)
                    index[i * mn + j] = 3 * (s->lo[7*jj + i] - cid * V) + d;
            } else {
                ptr[j] = 1;
                index[0 * mn + j] = j;
            }
        }
        for (int j = 0; j < mn; j++) {
            int node = j / 3, d = j % 3, jj = node + cid * V;
            if (node >= V) continue;
            int n = s->nln[jj], oa = 0, ob = 0, oc = 0, order = 0, en = 0;
            double tb = 0.0, tvalue[7] = {0.0};
            for (int i = 0; i < n; i++) {
                int element = s->le[6*jj + i];
                double gab = s->rg[element];
                int ea = s->ele[3*element+0], eb = s->ele[3*element+1], ec = s->ele[3*element+2];
                for (int k = 0; k < n + 1; k++) {
                    if (ea == s->lo[7*jj + k]) oa = k;
                    if (eb == s->lo[7*jj + k]) ob = k;
                    if (ec == s->lo[7*jj + k]) oc = k;
                    if (jj == s->lo[7*jj + k]) order = k;
                }
                if (ea == jj) { tvalue[oa] += gab / 12.0; en = 0; } else tvalue[oa] += gab / 24.0;
                if (eb == jj) { tvalue[ob] += gab / 12.0; en = 1; } else tvalue[ob] += gab / 24.0;
                if (ec == jj) { tvalue[oc] += gab / 12.0; en = 2; } else tvalue[oc] += gab / 24.0;
                double vd[2] = {s->xd[3*eb + d] - s->xd[3*ea + d], s->xd[3*ec + d] - s->xd[3*ea + d]};
                if (d == 0) { vd[0] = min_image(vd[0], p->LX); vd[1] = min_image(vd[1], p->LX); }
                else if (d == 2) { vd[0] = min_image(vd[0], p->LZ); vd[1] = min_image(vd[1], p->LZ); }
                for (int k = 0; k < 4; k++) {
                    int alpha = k / 2, beta = k % 2;
                    tb += gab * s->t[4*element + k] * (vd[alpha] * f[en][beta] + vd[beta] * f[en][alpha]) / 4.0;
                }
            }
            double jacobi = tvalue[order];
            for (int k = 0; k < 7; k++) value[k * mn + j] = tvalue[k] / jacobi;
            bc[j] = tb / jacobi;
        }
        int iters = 0;
        int flag = bicgstab(ptr, index, value, qc, bc, w, w + mn, w + 2*mn, w + 3*mn, w + 4*mn, mn,
                            p->residual, p->itrmax, &iters);
        if (flag != 0) flag_all |= flag;
        if (iters > maxit) maxit = iters;
        /* substitute_load: qd[j + 3 cid V] = qc[j]; entries j >= 3V spill into the
         * next cell's slice and are overwritten by it (stress.cu:292-300). */
        for (int j = 0; j < 3 * V; j++) s->qd[j + 3 * cid * V] = qc[j];
        free(ptr); free(index); free(value); free(qc); free(bc); free(w);
    }
    s->bicg_iters = maxit;
    return flag_all;
}

/* stress.cu:376-445 (q2f) */
void orc_q2f(const orc_params *p, orc_state *s)
{
    long nv = (long)p->ncell * p->vertex;
    const double *x = s->xd;
#pragma omp parallel for schedule(static)
    for (long jid = 0; jid < nv; jid++) {
        long j1 = jid;
        double x1 = x[j1*3+0], y1 = x[j1*3+1], z1 = x[j1*3+2], ds = 0.0;
        for (int k = 0; k < s->nln[j1]; k++) {
            int j2 = s->ln[j1*7 + k], j3 = s->ln[j1*7 + (k+1) % s->nln[j1]];
            double xx1 = min_image(x[j2*3+0] - x1, p->LX), yy1 = x[j2*3+1] - y1, zz1 = min_image(x[j2*3+2] - z1, p->LZ);
            double xx2 = min_image(x[j3*3+0] - x1, p->LX), yy2 = x[j3*3+1] - y1, zz2 = min_image(x[j3*3+2] - z1, p->LZ);
            double nvx = -(yy1*zz2 - zz1*yy2), nvy = -(zz1*xx2 - xx1*zz2), nvz = -(xx1*yy2 - yy1*xx2);
            ds += sqrt(nvx*nvx + nvy*nvy + nvz*nvz) / 2.0 / 3.0;
        }
        s->cfx[jid] = -1.0 * s->qd[jid*3+0] * ds;
        s->cfy[jid] = -1.0 * s->qd[jid*3+1] * ds;
        s->cfz[jid] = -1.0 * s->qd[jid*3+2] * ds;
    }
}

/* The four vertices of element e1's visit of its k-th edge neighbour e2
 * (cel->ec order): the shared edge (k2, k3) in e1's winding, e1's third
 * vertex k1 and e2's vertex k4 off the edge (stress.cu:490-502).  Returns 0
 * when e1 has no k-th neighbour. */
static int bend_quad(const orc_state *s, long e1, int k, int q[4])
{
    const long e2 = s->ec[e1*3 + k];
    const int i[3] = {s->ele[e1*3], s->ele[e1*3+1], s->ele[e1*3+2]};
    const int j[3] = {s->ele[e2*3], s->ele[e2*3+1], s->ele[e2*3+2]};
    for (int a = 0; a < 3; a++) {
        const int ia = i[a], ib = i[(a + 1) % 3];
        int has_a = -1, has_b = -1;
        for (int b = 0; b < 3; b++) { if (j[b] == ia) has_a = b; if (j[b] == ib) has_b = b; }
        if (e2 != e1 && has_a >= 0 && has_b >= 0) {
            q[0] = i[(a + 2) % 3]; q[1] = ia; q[2] = ib; q[3] = j[3 - has_a - has_b];
            return 1;
        }
    }
    return 0;
}

/* init1.cu:797-848 (init3.cu:313-364 for white cells): cos and sin of each
 * visit's dihedral angle on the current positions, the sign of sin from the
 * centroid test, 1 - cos^2 clamped at 0.  The reference computes these from
 * the initial shape and then overwrites them with c0 = 1, s0 = 0
 * (init1.cu:849-850); this keeps them (spontaneous angles of the reference
 * shape).  Positions are minimum images about k1, the same for an unwrapped
 * initial shape. */
void orc_bend_reference(const orc_params *p, orc_state *s)
{
    const long ne = (long)p->ncell * p->element;
    for (long e1 = 0; e1 < ne; e1++)
        for (int k = 0; k < 3; k++) {
            int q[4];
            s->c0[e1*3 + k] = 1.0;
            s->s0[e1*3 + k] = 0.0;
            if (!bend_quad(s, e1, k, q)) continue;
            double ax[4], ay[4], az[4];
            for (int v = 0; v < 4; v++) {
                ax[v] = s->x[q[0]] + min_image(s->x[q[v]] - s->x[q[0]], p->LX);
                ay[v] = s->y[q[v]];
                az[v] = s->z[q[0]] + min_image(s->z[q[v]] - s->z[q[0]], p->LZ);
            }
            const double a21x = ax[1] - ax[0], a31x = ax[2] - ax[0], a34x = ax[2] - ax[3], a24x = ax[1] - ax[3];
            const double a21y = ay[1] - ay[0], a31y = ay[2] - ay[0], a34y = ay[2] - ay[3], a24y = ay[1] - ay[3];
            const double a21z = az[1] - az[0], a31z = az[2] - az[0], a34z = az[2] - az[3], a24z = az[1] - az[3];
            const double xix = a21y*a31z - a21z*a31y, xiy = a21z*a31x - a21x*a31z, xiz = a21x*a31y - a21y*a31x;
            const double zex = a34y*a24z - a34z*a24y, zey = a34z*a24x - a34x*a24z, zez = a34x*a24y - a34y*a24x;
            const double cost = (xix*zex + xiy*zey + xiz*zez) / sqrt(xix*xix + xiy*xiy + xiz*xiz)
                              / sqrt(zex*zex + zey*zey + zez*zez);
            double cost2 = 1.0 - cost * cost;
            if (cost2 < 0.0) cost2 = 0.0;
            const double t = (xix - zex) * (ax[0] - ax[3]) + (xiy - zey) * (ay[0] - ay[3]) + (xiz - zez) * (az[0] - az[3]);
            s->c0[e1*3 + k] = cost;
            s->s0[e1*3 + k] = t >= 0.0 ? sqrt(cost2) : -sqrt(cost2);
        }
}

/* stress.cu:448-578.  For every element e1 and each of its edge neighbours
 * (bend_quad): xi and ze are the two triangle normals with positions taken
 * as minimum images about k1; pairs with sin^2 < 1e-6 are skipped; beta =
 * (2/sqrt 3) BR sgn (sin c0 - cos s0) / |sin| with the spontaneous angle
 * (c0, s0) of the visit, (1, 0) as init1.cu:849-850 leaves it unless
 * s->c0 / s->s0 hold others; k1 receives the whole force of the pair, k2 and
 * k3 half of theirs (e2's visit of the same pair adds the rest). */
void orc_bend(const orc_params *p, orc_state *s)
{
    if (p->br == 0.0 && !s->cbr) return;
    const long ne = (long)p->ncell * p->element;
    const double eps = 1.0e-6;
    for (long e1 = 0; e1 < ne; e1++) {
        const double br = s->cbr ? s->cbr[e1 / p->element] : p->br;
        if (br == 0.0) continue;
        for (int k = 0; k < 3; k++) {
            int q[4];
            if (!bend_quad(s, e1, k, q)) continue;
            const int k1 = q[0], k2 = q[1], k3 = q[2], k4 = q[3];
            const double cost0 = s->c0 ? s->c0[e1*3 + k] : 1.0, sint0 = s->s0 ? s->s0[e1*3 + k] : 0.0;
            double a1x = s->x[k1], a2x = s->x[k2], a3x = s->x[k3], a4x = s->x[k4];
            double a1y = s->y[k1], a2y = s->y[k2], a3y = s->y[k3], a4y = s->y[k4];
            double a1z = s->z[k1], a2z = s->z[k2], a3z = s->z[k3], a4z = s->z[k4];
            a2x = a1x + min_image(a2x - a1x, p->LX); a3x = a1x + min_image(a3x - a1x, p->LX); a4x = a1x + min_image(a4x - a1x, p->LX);
            a2z = a1z + min_image(a2z - a1z, p->LZ); a3z = a1z + min_image(a3z - a1z, p->LZ); a4z = a1z + min_image(a4z - a1z, p->LZ);
            const double a21x = a2x - a1x, a31x = a3x - a1x, a34x = a3x - a4x, a24x = a2x - a4x, a23x = a2x - a3x;
            const double a21y = a2y - a1y, a31y = a3y - a1y, a34y = a3y - a4y, a24y = a2y - a4y, a23y = a2y - a3y;
            const double a21z = a2z - a1z, a31z = a3z - a1z, a34z = a3z - a4z, a24z = a2z - a4z, a23z = a2z - a3z;
            const double xix = a21y*a31z - a21z*a31y, xiy = a21z*a31x - a21x*a31z, xiz = a21x*a31y - a21y*a31x;
            const double zex = a34y*a24z - a34z*a24y, zey = a34z*a24x - a34x*a24z, zez = a34x*a24y - a34y*a24x;
            const double t1x = (a1x + a2x + a3x) / 3.0, t2x = (a4x + a2x + a3x) / 3.0;
            const double t1y = (a1y + a2y + a3y) / 3.0, t2y = (a4y + a2y + a3y) / 3.0;
            const double t1z = (a1z + a2z + a3z) / 3.0, t2z = (a4z + a2z + a3z) / 3.0;
            const double nxi = sqrt(xix*xix + xiy*xiy + xiz*xiz), nze = sqrt(zex*zex + zey*zey + zez*zez);
            const double cost = (xix*zex + xiy*zey + xiz*zez) / nxi / nze;
            const double cost2 = 1.0 - cost * cost;
            if (cost2 < eps) continue;
            const double sgn = ((xix-zex)*(t1x-t2x) + (xiy-zey)*(t1y-t2y) + (xiz-zez)*(t1z-t2z)) >= 0.0 ? 1.0 : -1.0;
            const double sint = sgn * sqrt(cost2);
            const double beta = sgn * 2.0 / sqrt(3.0) * br * (sint * cost0 - cost * sint0) / sqrt(cost2);
            const double b11 = -beta * cost / (nxi * nxi), b12 = beta / nxi / nze, b22 = -beta * cost / (nze * nze);
            s->cfx[k1] += b11*(xiy*-a23z - xiz*-a23y) + b12*(zey*-a23z - zez*-a23y);
            s->cfy[k1] += b11*(xiz*-a23x - xix*-a23z) + b12*(zez*-a23x - zex*-a23z);
            s->cfz[k1] += b11*(xix*-a23y - xiy*-a23x) + b12*(zex*-a23y - zey*-a23x);
            s->cfx[k2] += 0.5 * (b11*(xiy*-a31z - xiz*-a31y) + b22*(zey*a34z - zez*a34y) + b12*((xiy*a34z - xiz*a34y) + (zey*-a31z - zez*-a31y)));
            s->cfy[k2] += 0.5 * (b11*(xiz*-a31x - xix*-a31z) + b22*(zez*a34x - zex*a34z) + b12*((xiz*a34x - xix*a34z) + (zez*-a31x - zex*-a31z)));
            s->cfz[k2] += 0.5 * (b11*(xix*-a31y - xiy*-a31x) + b22*(zex*a34y - zey*a34x) + b12*((xix*a34y - xiy*a34x) + (zex*-a31y - zey*-a31x)));
            s->cfx[k3] += 0.5 * (b11*(xiy*a21z - xiz*a21y) + b22*(zey*-a24z - zez*-a24y) + b12*((xiy*-a24z - xiz*-a24y) + (zey*a21z - zez*a21y)));
            s->cfy[k3] += 0.5 * (b11*(xiz*a21x - xix*a21z) + b22*(zez*-a24x - zex*-a24z) + b12*((xiz*-a24x - xix*-a24z) + (zez*a21x - zex*a21z)));
            s->cfz[k3] += 0.5 * (b11*(xix*a21y - xiy*a21x) + b22*(zex*-a24y - zey*-a24x) + b12*((xix*-a24y - xiy*-a24x) + (zex*a21y - zey*a21x)));
        }
    }
}

/* stress.cu:580-659 */
int orc_stress(const orc_params *p, orc_state *s)
{
    orc_calc_tension(p, s);
    int flag = orc_calc_load(p, s);
    orc_q2f(p, s);
    orc_bend(p, s);
    return flag;
}

/* ------------------------------------------------------------------------ */
/* Immersed boundary: ibm.cu                                                 */
/* ------------------------------------------------------------------------ */

/* ibm.cu:299-369: ibm_st1a (27-52), ibm_st1b (55-131), ibm_st1c (214-296,
 * CapsuleCHANNELFLOW: fold the z BUFF planes) */
void orc_ibm_st1(const orc_params *p, orc_state *s)
{
    int nx = p->nx, ny = p->ny, nz = p->nz;
    long n = (long)nx * ny * nz, nv = (long)p->ncell * p->vertex;
    double dx = p->dx;
    memset(s->fx, 0, sizeof(double) * n);
    memset(s->fy, 0, sizeof(double) * n);
    memset(s->fz, 0, sizeof(double) * n);
    for (long jid = 0; jid < nv; jid++) {
        double xtr = s->x[jid] + (double)(nx - 1) * dx / 2.0;
        double ytr = s->y[jid] + (double)(ny - 1) * dx / 2.0;
        double ztr = s->z[jid] + (double)(nz - 1) * dx / 2.0;
        int x1 = (int)floor(xtr / dx) - 1, x2 = (int)ceil(xtr / dx) + 1;
        int y1 = (int)floor(ytr / dx) - 1, y2 = (int)ceil(ytr / dx) + 1;
        int z1 = (int)floor(ztr / dx) - 1, z2 = (int)ceil(ztr / dx) + 1;
        for (int iz = z1; iz <= z2; iz++)
            for (int iy = y1; iy <= y2; iy++)
                for (int ix = x1; ix <= x2; ix++) {
                    if (ix < 0 || ix >= nx || iy < 0 || iy >= ny || iz < 0 || iz >= nz) continue;
                    long i = ix + (long)nx * iy + (long)nx * ny * iz;
                    double xx = fabs((double)ix * dx - xtr), yy = fabs((double)iy * dx - ytr), zz = fabs((double)iz * dx - ztr);
                    double xcos = 1.0 + cos(M_PI * xx / (2.0 * dx));
                    double ycos = 1.0 + cos(M_PI * yy / (2.0 * dx));
                    double zcos = 1.0 + cos(M_PI * zz / (2.0 * dx));
                    double dlt = xcos * ycos * zcos / (64.0 * dx * dx * dx);
                    s->fx[i] += dlt * s->cfx[jid];
                    s->fy[i] += dlt * s->cfy[jid];
                    s->fz[i] += dlt * s->cfz[jid];
                }
    }
    long plane = (long)nx * ny, shift = plane * (nz - 4), xs = nx - 4;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        if (s->bc[i] != ORC_COMP) continue;
        long iz = i / plane, ix = (i % plane) % nx;
        /* every COMP node adds the spread force its BUFF images received (ibm.cu:239-294);
         * the images are not modified, so the order of the adds does not matter */
        long img[8];
        int k = 0;
        if (iz <= 3) img[k++] = i + shift;
        if (iz >= nz - 4) img[k++] = i - shift;
        if (p->flow == 1) {
            if (ix <= 3) img[k++] = i + xs;
            if (ix >= nx - 4) img[k++] = i - xs;
            if (ix <= 3 && iz <= 3) img[k++] = i + xs + shift;
            if (ix >= nx - 4 && iz <= 3) img[k++] = i - xs + shift;
            if (ix <= 3 && iz >= nz - 4) img[k++] = i + xs - shift;
            if (ix >= nx - 4 && iz >= nz - 4) img[k++] = i - xs - shift;
        }
        for (int t = 0; t < k; t++) { s->fx[i] += s->fx[img[t]]; s->fy[i] += s->fy[img[t]]; s->fz[i] += s->fz[img[t]]; }
    }
}

static int orc_M(const orc_params *p) { return p->M > 0 ? p->M : 1; }
static int orc_rk(const orc_params *p) { return p->rk_order > 0 ? p->rk_order : 4; }

/* The interpolated velocity at (xr, yr, zr) (ibm.cu:444-482).  The RUNGE_KUTTA
 * == 4 branch works in physical units (xtr / dx, cos(pi |ix dx - xtr| / 2 dx));
 * the 2 and 1 branches (ibm.cu:522-556, 579-612) leave dx out (xtr = xr + (nx -
 * 1) / 2, cos(pi |ix - xtr| / 2)), the same for dx = 1.  Both visit the 4 x 4 x 4
 * nodes of nonzero weight (a node at distance 2 has weight 0). */
static void interp_velocity(const orc_params *p, const orc_state *s, int with_dx, double xr, double yr, double zr,
                            double *ur, double *vr, double *wr)
{
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const double dx = with_dx ? p->dx : 1.0;
    double u = 0.0, v = 0.0, w = 0.0;
    const double xtr = xr + (double)(nx - 1) * dx / 2.0;
    const double ytr = yr + (double)(ny - 1) * dx / 2.0;
    const double ztr = zr + (double)(nz - 1) * dx / 2.0;
    const int x1 = (int)floor(xtr / dx) - 1, x2 = (int)ceil(xtr / dx) + 1;
    const int y1 = (int)floor(ytr / dx) - 1, y2 = (int)ceil(ytr / dx) + 1;
    const int z1 = (int)floor(ztr / dx) - 1, z2 = (int)ceil(ztr / dx) + 1;
    for (int iz = z1; iz <= z2; iz++)
        for (int iy = y1; iy <= y2; iy++)
            for (int ix = x1; ix <= x2; ix++) {
                if (ix < 0 || ix >= nx || iy < 0 || iy >= ny || iz < 0 || iz >= nz) continue;
                long i = ix + (long)nx * iy + (long)nx * ny * iz;
                double xx = fabs((double)ix * dx - xtr), yy = fabs((double)iy * dx - ytr), zz = fabs((double)iz * dx - ztr);
                double dlt = (1.0 + cos(M_PI * xx / (2.0 * dx))) * (1.0 + cos(M_PI * yy / (2.0 * dx)))
                           * (1.0 + cos(M_PI * zz / (2.0 * dx))) / 64.0;
                u += dlt * s->um[i]; v += dlt * s->vm[i]; w += dlt * s->wm[i];
            }
    *ur = u; *vr = v; *wr = w;
}

/* ibm.cu:372-639 (ibm_st2a): RUNGE_KUTTA 4 (ibm.cu:430-517), 2 (518-574) or 1
 * (575-617) stages over the averaged lattice velocity, then x += u M dt with the
 * periodic wrap (ibm.cu:625-632) */
void orc_ibm_st2(const orc_params *p, orc_state *s)
{
    long nv = (long)p->ncell * p->vertex;
    double dt = p->dt;
    const double Md = (double)orc_M(p);
    const int rk = orc_rk(p);
#pragma omp parallel for schedule(static)
    for (long jid = 0; jid < nv; jid++) {
        double xn = s->x[jid], yn = s->y[jid], zn = s->z[jid];
        double um, vm, wm;
        if (rk == 4) {
            double xr = xn, yr = yn, zr = zn, uk[4][3];
            for (int k = 0; k < 4; k++) {
                interp_velocity(p, s, 1, xr, yr, zr, &uk[k][0], &uk[k][1], &uk[k][2]);
                double h = (k < 2) ? Md * dt / 2.0 : Md * dt;
                xr = xn + uk[k][0] * h; yr = yn + uk[k][1] * h; zr = zn + uk[k][2] * h;
            }
            um = (uk[0][0] + 2.0 * uk[1][0] + 2.0 * uk[2][0] + uk[3][0]) / 6.0;
            vm = (uk[0][1] + 2.0 * uk[1][1] + 2.0 * uk[2][1] + uk[3][1]) / 6.0;
            wm = (uk[0][2] + 2.0 * uk[1][2] + 2.0 * uk[2][2] + uk[3][2]) / 6.0;
        } else if (rk == 2) {
            double u1, v1, w1, u2, v2, w2;
            interp_velocity(p, s, 0, xn, yn, zn, &u1, &v1, &w1);
            /* ibm.cu:560-562: the second stage at x + u1 M (no dt) */
            interp_velocity(p, s, 0, xn + u1 * Md, yn + v1 * Md, zn + w1 * Md, &u2, &v2, &w2);
            um = (u1 + u2) / 2.0; vm = (v1 + v2) / 2.0; wm = (w1 + w2) / 2.0;
        } else {
            interp_velocity(p, s, 0, xn, yn, zn, &um, &vm, &wm);
        }
        double xr = xn + um * Md * dt, yr = yn + vm * Md * dt, zr = zn + wm * Md * dt;
        if (xr < p->xmin) xr += p->LX;
        if (xr > p->xmax) xr -= p->LX;
        if (zr < p->zmin) zr += p->LZ;
        if (zr > p->zmax) zr -= p->LZ;
        s->u[jid] = um; s->x[jid] = xr; s->xd[jid*3 + 0] = xr;
        s->v[jid] = vm; s->y[jid] = yr; s->xd[jid*3 + 1] = yr;
        s->w[jid] = wm; s->z[jid] = zr; s->xd[jid*3 + 2] = zr;
    }
}

/* ------------------------------------------------------------------------ */
/* Lattice Boltzmann: lbm.cu                                                 */
/* ------------------------------------------------------------------------ */

/* lbm.cu:983-1313 (lbm_CapsuleCHANNELFLOW) + 1378-1432 (BUFF copy) +
 * 1435-1460 (the sums of the M sub-steps divided by M) + pointer swap (1575).  omega = 1 / (3 (1 +
 * (LAMBDA1 - 1) vf) Df + 1/2) with Df = (tau - 1/2) / 3 (lbm.cu:1131); with
 * LAMBDA1 = 1 that is 1 / tau, used as such. */
void orc_lbm_d3q19(const orc_params *p, orc_state *s)
{
    int nx = p->nx, ny = p->ny, nz = p->nz, iter = s->iter;
    long n = (long)nx * ny * nz, plane = (long)nx * ny, shift = plane * (nz - 4);
    double Cr = p->Cr, Cr2 = Cr * Cr, P = p->P, B = p->B;
    double t = p->dt * (double)iter;
    double wi = (iter > p->flowstart) ? 1.0 + 0.5 * sin(M_PI * t / p->freq) : 0.0;
    const double om0 = 1.0 / p->tau, Df = (p->tau - 0.5) / 3.0;
    const int visc = p->lambda1 != 1.0 && s->vf;
    const int Ms = orc_M(p);
    const double *fn = s->fn; double *fm = s->fm;
    const int *bc = s->bc;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        if (bc[i] != ORC_COMP) continue;
        double f[ORC_Q];
        for (int q = 0; q < ORC_Q; q++) f[q] = fn[i * ORC_Q + q];
        double tfx = s->fx[i], tfy = s->fy[i], tfz = s->fz[i];
        double td = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
        for (int q = 0; q < ORC_Q; q++) { td += f[q]; jx += EX[q] * f[q]; jy += EY[q] * f[q]; jz += EZ[q] * f[q]; }
        double tu = (jx + td * P * 0.0 + td * B * tfx) / (td * Cr);
        double tv = (jy + td * P * 0.0 + td * B * tfy) / (td * Cr);
        double tw = (jz + td * P * wi + td * B * tfz) / (td * Cr);
        s->dn[i] = td; s->un[i] = tu; s->vn[i] = tv; s->wn[i] = tw;
        /* lbm.cu:1097-1102, 1122-1126: the sums restart at the first of every M steps */
        if ((iter - 1) % Ms == 0) { s->dm[i] = 0.0; s->um[i] = 0.0; s->vm[i] = 0.0; s->wm[i] = 0.0; }
        s->dm[i] += td; s->um[i] += tu; s->vm[i] += tv; s->wm[i] += tw;
        const double om = visc ? 1.0 / (3.0 * (1.0 + (p->lambda1 - 1.0) * s->vf[i]) * Df + 0.5) : om0;
        double om1 = 1.0 - om, om2 = (1.0 - om / 2.0) * 2.0 * td * P, om3 = (1.0 - om / 2.0) * 2.0 * td * B;
        double uvw = -1.5 * (tu*tu + tv*tv + tw*tw) * Cr2;
        double gP[3] = {0.0, 0.0, wi}, gB[3] = {tfx, tfy, tfz}, uu[3] = {tu, tv, tw};
        for (int q = 0; q < ORC_Q; q++) {
            double e[3] = {EX[q], EY[q], EZ[q]};
            double eu = e[0]*tu + e[1]*tv + e[2]*tw;
            double feq = WQ[q] * td * (1.0 + 3.0 * eu * Cr + 4.5 * eu * eu * Cr2 + uvw);
            double sP = 0.0, sB = 0.0;
            for (int d = 0; d < 3; d++) {
                double c = 3.0 * (e[d] - uu[d] * Cr) + 9.0 * Cr * eu * e[d];
                sP += c * gP[d]; sB += c * gB[d];
            }
            f[q] = om1 * f[q] + om * feq + om2 * WQ[q] * sP + om3 * WQ[q] * sB;
        }
        if (p->flow == 1) {
            /* lbm.cu:754-826, 922-978: x and z periodic through the COMP range, half-way
             * bounce-back at the y walls, which move along z (sra = 0 before FLOWSTART) */
            long iz = i / plane, iy = (i % plane) / nx, ix = (i % plane) % nx;
            double sra = (iter < p->flowstart) ? 0.0 : p->sr, LY = (double)(ny - 4) * p->dx;
            double utop = p->walls == 0 ? sra * LY / 2.0 : sra * LY, ubot = p->walls == 0 ? -sra * LY / 2.0 : 0.0;
            for (int q = 0; q < ORC_Q; q++) {
                long jx = ix + EX[q], jy = iy + EY[q], jz = iz + EZ[q];
                if (jx > nx - 3) jx -= nx - 4; else if (jx < 2) jx += nx - 4;
                if (jz > nz - 3) jz -= nz - 4; else if (jz < 2) jz += nz - 4;
                if (jy > ny - 3 || jy < 2) {
                    double uw = jy > ny - 3 ? utop : ubot;
                    fm[i * ORC_Q + OPP[q]] = f[q] - 6.0 * WQ[q] * td * Cr * EZ[q] * uw;
                } else {
                    fm[(jx + (long)nx * jy + plane * jz) * ORC_Q + q] = f[q];
                }
            }
            continue;
        }
        /* push streaming with half-way bounce-back (lbm.cu:1050-1094, 1272-1310) */
        for (int q = 0; q < ORC_Q; q++) {
            long d = i + EX[q] + (long)nx * EY[q] + plane * EZ[q];
            long j;
            if (q == 0) j = i * ORC_Q;
            else if (q == 5 || q == 6) {
                if (bc[d] == ORC_BUFF) d -= EZ[q] * shift;
                j = d * ORC_Q + q;
            } else if (EZ[q] == 0) {
                j = (bc[d] == ORC_WALL) ? i * ORC_Q + OPP[q] : d * ORC_Q + q;
            } else {
                if (bc[d] == ORC_WALL) j = i * ORC_Q + OPP[q];
                else { if (bc[d] == ORC_BUFF) d -= EZ[q] * shift; j = d * ORC_Q + q; }
            }
            fm[j] = f[q];
        }
    }
    if (p->flow == 0 && p->tube_r > 0.0) {
        /* lbm_cylinder.cu:116-231: every half-way bounced population of a link that crosses the
         * circle x^2 + y^2 = R^2 at fraction t of the link is replaced by a linear interpolation
         * (BounceBackLinearInterpolation_DEV, lbm_cylinder.cu:61-87) of itself (f1), the
         * population streamed into the node along the link's direction (f2) and the one the
         * node streamed to its opposite neighbour (f3).  The reference list is built once from
         * the bc map (SetDistanceFromWall_GPU); the links are z-invariant, so it is recomputed. */
        const double R = p->tube_r, dxl = p->dx;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++) {
            if (bc[i] != ORC_COMP) continue;
            long iz = i / plane, iy = (i % plane) / nx, ix = (i % plane) % nx;
            const double xi = (ix - (nx - 1) / 2.0) * dxl, yi = (iy - (ny - 1) / 2.0) * dxl;   /* init1.cu:223-224 */
            for (int q = 1; q < ORC_Q; q++) {
                long j = i + EX[q] + (long)nx * EY[q] + plane * EZ[q];
                if (bc[j] != ORC_WALL) continue;
                double ddx = EX[q] * dxl, ddy = EY[q] * dxl;
                double a = ddx * ddx + ddy * ddy;
                double Det = (xi * ddx + yi * ddy) * (xi * ddx + yi * ddy) - a * (xi * xi + yi * yi - R * R);
                if (Det < 0.0) continue;
                double t1 = (-xi * ddx - yi * ddy + sqrt(Det)) / a, t2 = (-xi * ddx - yi * ddy - sqrt(Det)) / a, t;
                if (t1 > 0.0 && t1 < 1.0) t = t1; else if (t2 > 0.0 && t2 < 1.0) t = t2; else continue;
                int o = OPP[q];
                long jj = i + EX[o] + (long)nx * EY[o] + plane * EZ[o];
                if (bc[jj] == ORC_BUFF) jj = i + EX[o] + (long)nx * EY[o] - plane * EZ[o] * (nz - 5);
                double f1 = fm[i * ORC_Q + o], f2 = fm[i * ORC_Q + q], f3 = fm[jj * ORC_Q + o], f;
                if (t < 0.5) f = 2.0 * t * f1 + (1.0 - 2.0 * t) * f2;
                else f = 1.0 / (2.0 * t) * f1 + (2.0 * t - 1.0) / (2.0 * t) * f3;
                fm[i * ORC_Q + o] = f;
            }
        }
    }
    /* lbm.cu:1378-1432: BUFF planes take their periodic images */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        if (bc[i] != ORC_BUFF) continue;
        long iz = i / plane, i2 = i;
        if (iz <= 1) i2 += shift;
        if (iz >= nz - 2) i2 -= shift;
        if (p->flow == 1) {   /* lbm.cu:1316-1374: x BUFF columns too */
            long ix = (i % plane) % nx;
            if (ix <= 1) i2 += nx - 4;
            if (ix >= nx - 2) i2 -= nx - 4;
        }
        s->dn[i] = s->dn[i2]; s->un[i] = s->un[i2]; s->vn[i] = s->vn[i2]; s->wn[i] = s->wn[i2];
        s->dm[i] = s->dm[i2]; s->um[i] = s->um[i2]; s->vm[i] = s->vm[i2]; s->wm[i] = s->wm[i2];
    }
    /* lbm.cu:1545-1548, 1435-1460: at the last of every M steps the velocity sums
     * become averages (every node, as lbm_AVERAGE does) */
    if (iter % Ms == 0) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++) { s->um[i] /= (double)Ms; s->vm[i] /= (double)Ms; s->wm[i] /= (double)Ms; }
    }
    /* lbm.cu:1575 swaps the buffers */
    double *tmp = s->fn; s->fn = s->fm; s->fm = tmp;
}

/* ------------------------------------------------------------------------ */
/* Volume fraction: thincwlic.cu, fronttrack.cu, matrix_solver.cu            */
/* ------------------------------------------------------------------------ */

/* thincwlic.cu:12-106 (normal3d_st1, normal3d_st2): n2, the vf gradient at the
 * cell corner below-left of every node with ix, iy, iz >= 1, and n1, the
 * average of the eight corner gradients around every interior node */
static void vof_normals(const orc_params *p, const double *vf, double *n1[3], double *n2[3])
{
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const long n = (long)nx * ny * nz, pl = (long)nx * ny;
    const double dx = p->dx;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        const long iz = i / pl, iy = i / nx - ny * iz, ix = i - nx * iy - pl * iz;
        if (ix == 0 || iy == 0 || iz == 0) continue;
        n2[0][i] = 0.25 / dx * (vf[i] - vf[i-1] + vf[i-nx] - vf[i-1-nx] + vf[i-pl] - vf[i-1-pl] + vf[i-nx-pl] - vf[i-1-nx-pl]);
        n2[1][i] = 0.25 / dx * (vf[i] - vf[i-nx] + vf[i-1] - vf[i-1-nx] + vf[i-pl] - vf[i-nx-pl] + vf[i-1-pl] - vf[i-1-nx-pl]);
        n2[2][i] = 0.25 / dx * (vf[i] - vf[i-pl] + vf[i-1] - vf[i-1-pl] + vf[i-nx] - vf[i-nx-pl] + vf[i-1-nx] - vf[i-1-nx-pl]);
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        const long iz = i / pl, iy = i / nx - ny * iz, ix = i - nx * iy - pl * iz;
        if (ix == 0 || iy == 0 || iz == 0 || ix == nx - 1 || iy == ny - 1 || iz == nz - 1) continue;
        for (int d = 0; d < 3; d++) {
            const double *m = n2[d];
            n1[d][i] = 0.125 * (m[i] + m[i+pl] + m[i+1] + m[i+1+pl] + m[i+nx] + m[i+nx+pl] + m[i+1+nx] + m[i+1+nx+pl]);
        }
    }
}

void orc_thinc_wlic(const orc_params *p, orc_state *s)
{
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const long n = (long)nx * ny * nz, pl = (long)nx * ny, shift = pl * (nz - 4);
    const double dx = p->dx, dt = p->dt, beta = 2.0;
    double *buf = (double *)calloc((size_t)n * 7, sizeof(double));
    double *n1[3] = {buf, buf + n, buf + 2 * n}, *n2[3] = {buf + 3 * n, buf + 4 * n, buf + 5 * n}, *flux = buf + 6 * n;
    double *vf = s->vf;
    const int *bc = s->bc;
    const double *u[3] = {s->um, s->vm, s->wm};
    const double Mt = (double)orc_M(p);   /* thincwlic.cu:179-207: the flux over M steps */
    for (int idr = 0; idr < 3; idr++) {
        vof_normals(p, vf, n1, n2);
        const long acs = idr == 0 ? 1 : idr == 1 ? nx : pl;
        /* wlic1d4md_st1 (thincwlic.cu:108-238): the flux through the face between
         * i - acs and i, THINC in the upwind node weighted by its normal's share
         * along the sweep (WLIC), plain upwind in full or empty nodes */
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++) {
            flux[i] = 0.0;
            const long iz = i / pl, iy = i / nx - ny * iz, ix = i - nx * iy - pl * iz;
            if (ix == 0 || iy == 0 || iz == 0) continue;
            if (ix == 1 || iy == 1 || iz == 1) continue;
            if (ix == nx - 1 || iy == ny - 1 || iz == nz - 1) continue;
            const double up = u[idr][i], um = u[idr][i - acs], uc = (up + um) / 2.0;
            int isgn;
            long ii;
            if (uc <= 0.0) { isgn = 0; ii = i; } else { isgn = 1; ii = i - acs; }
            const double nn = fabs(n1[0][ii]) + fabs(n1[1][ii]) + fabs(n1[2][ii]);
            double f;
            if (vf[ii] >= 1.0 - 1.0e-6 || vf[ii] <= 1.0e-6) f = vf[ii] * uc * Mt * dt;
            else if (nn <= 1.0e-6) f = vf[ii] * uc * Mt * dt;
            else {
                /* the reference's three assignments of ib leave ii - acs (ii's z index is >= 1) */
                const long ib = ii - acs;
                const double alpha = vf[ib] <= vf[ii + acs] ? 1.0 : -1.0;
                const double a1 = expf(beta * (2.0 * vf[ii] - 1.0) / alpha);
                const double a3 = expf(beta);
                const double xc = 0.5 / beta * log((a3 * a3 - a1 * a3) / (a1 * a3 - 1.0));
                const double a4 = coshf(beta * ((double)isgn - uc * Mt * dt / dx - xc));
                const double a5 = coshf(beta * ((double)isgn - xc));
                f = 0.5 * (uc * Mt * dt - alpha * dx / beta * log(a4 / a5));
                const double weight = fabs(n1[idr][ii]) / nn;
                f = f * weight + vf[ii] * uc * Mt * dt * (1.0 - weight);
            }
            if (bc[i] == ORC_WALL || bc[i - acs] == ORC_WALL) f = 0.0;
            flux[i] = f;
        }
        /* wlic1d4md_st2 (thincwlic.cu:241-272) */
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++)
            if (bc[i] == ORC_COMP) vf[i] = vf[i] - (flux[i + acs] - flux[i]) / dx;
        /* wlic1d4md_st3 (thincwlic.cu:275-313): BUFF nodes take their periodic
         * images, WALL nodes 0 */
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; i++) {
            if (bc[i] == ORC_COMP) continue;
            if (bc[i] == ORC_BUFF) {
                const long iz = i / pl, ix = (i % pl) % nx;
                long i2 = i;
                if (p->flow == 1) {
                    if (ix <= 1) i2 += nx - 4;
                    if (ix >= nx - 2) i2 -= nx - 4;
                }
                if (iz <= 1) i2 += shift;
                if (iz >= nz - 2) i2 -= shift;
                vf[i] = vf[i2];
            } else if (bc[i] == ORC_WALL) {
                vf[i] = 0.0;
            }
        }
    }
    free(buf);
}

static long pow2_at_least(long n)
{
    long m = 1;
    while (m < n) m *= 2;
    return m;
}

int orc_front_tracking(const orc_params *p, orc_state *s)
{
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const long n = (long)nx * ny * nz, pl = (long)nx * ny, mn = pow2_at_least(n);
    const long ne = (long)p->ncell * p->element;
    const double dx = p->dx, LX = p->LX, LZ = p->LZ;
    const int *bc = s->bc;
    if (p->ncell == 0) {   /* nothing to track (the reference's solve would divide by |b| = 0) */
        memset(s->vf, 0, sizeof(double) * (size_t)n);
        return 0;
    }
    double *g[3], *dg = (double *)calloc((size_t)mn * 7, sizeof(double));
    g[0] = dg + mn; g[1] = dg + 2 * mn; g[2] = dg + 3 * mn;
    double *b = dg + 4 * mn, *x = dg + 5 * mn, *r = dg + 6 * mn;
    /* front_tracking_source2 (fronttrack.cu:351-455): every triangle spreads
     * its inward normal times its area with the 4-point cosine delta around
     * its centroid; nodes outside the lattice are dropped.  Serial, so the sums
     * run in element order. */
    for (long e = 0; e < ne; e++) {
        const int j1 = s->ele[3*e], j2 = s->ele[3*e+1], j3 = s->ele[3*e+2];
        double tx1 = s->x[j1], tx2 = s->x[j2], tx3 = s->x[j3];
        double ty1 = s->y[j1], ty2 = s->y[j2], ty3 = s->y[j3];
        double tz1 = s->z[j1], tz2 = s->z[j2], tz3 = s->z[j3];
        double xx1 = tx2 - tx1, yy1 = ty2 - ty1, zz1 = tz2 - tz1;
        if (xx1 > LX * 0.5) { xx1 -= LX; tx1 += LX; } else if (xx1 < -LX * 0.5) { xx1 += LX; tx2 += LX; }
        if (zz1 > LZ * 0.5) { zz1 -= LZ; tz1 += LZ; } else if (zz1 < -LZ * 0.5) { zz1 += LZ; tz2 += LZ; }
        double xx2 = tx3 - tx1, yy2 = ty3 - ty1, zz2 = tz3 - tz1;
        if (xx2 > LX * 0.5) { xx2 -= LX; tx1 += LX; } else if (xx2 < -LX * 0.5) { xx2 += LX; tx3 += LX; }
        if (zz2 > LZ * 0.5) { zz2 -= LZ; tz1 += LZ; } else if (zz2 < -LZ * 0.5) { zz2 += LZ; tz3 += LZ; }
        const double xg = (tx1 + tx2 + tx3) / 3.0, yg = (ty1 + ty2 + ty3) / 3.0, zg = (tz1 + tz2 + tz3) / 3.0;
        const double xtr = xg + (double)(nx - 1) * dx / 2.0, ytr = yg + (double)(ny - 1) * dx / 2.0,
                     ztr = zg + (double)(nz - 1) * dx / 2.0;
        const int x1 = (int)floor(xtr / dx) - 1, x2 = (int)ceil(xtr / dx) + 1;
        const int y1 = (int)floor(ytr / dx) - 1, y2 = (int)ceil(ytr / dx) + 1;
        const int z1 = (int)floor(ztr / dx) - 1, z2 = (int)ceil(ztr / dx) + 1;
        double nvx = -(yy1 * zz2 - zz1 * yy2), nvy = -(zz1 * xx2 - xx1 * zz2), nvz = -(xx1 * yy2 - yy1 * xx2);
        const double nn = sqrt(nvx * nvx + nvy * nvy + nvz * nvz), ds = nn / 2.0;
        nvx /= nn; nvy /= nn; nvz /= nn;
        for (int iz = z1; iz <= z2; iz++)
            for (int iy = y1; iy <= y2; iy++)
                for (int ix = x1; ix <= x2; ix++) {
                    if (ix < 0 || ix >= nx || iy < 0 || iy >= ny || iz < 0 || iz >= nz) continue;
                    const long i = ix + (long)nx * iy + pl * iz;
                    const double xx = (double)ix * dx - xtr, yy = (double)iy * dx - ytr, zz = (double)iz * dx - ztr;
                    const double xcos = 1.0 + cos(M_PI * xx / (2.0 * dx)), ycos = 1.0 + cos(M_PI * yy / (2.0 * dx)),
                                 zcos = 1.0 + cos(M_PI * zz / (2.0 * dx));
                    const double dlt = xcos * ycos * zcos / (64.0 * dx * dx * dx);
                    g[0][i] += dlt * nvx * ds;
                    g[1][i] += dlt * nvy * ds;
                    g[2][i] += dlt * nvz * ds;
                }
    }
    /* front_tracking_source3 (fronttrack.cu:458-537): COMP nodes within two
     * planes (columns) of a periodic end add their BUFF images and copy the sum
     * back to them */
    for (long i = 0; i < n; i++) {
        if (bc[i] != ORC_COMP) continue;
        const long iz = i / pl, iy = i / nx - ny * iz, ix = i - nx * iy - pl * iz;
        long im[3] = {-1, -1, -1};
        const long sz = pl * (nz - 4), sx = nx - 4;
        if (p->flow == 1) {
            const long dxs = ix <= 3 ? sx : (ix >= nx - 4 ? -sx : 0), dzs = iz <= 3 ? sz : (iz >= nz - 4 ? -sz : 0);
            if (dxs && dzs) { im[0] = i + dxs; im[1] = i + dzs; im[2] = i + dxs + dzs; }
            else if (dxs) im[0] = i + dxs;
            else if (dzs) im[0] = i + dzs;
        } else {
            if (iz <= 3) im[0] = i + sz; else if (iz >= nz - 4) im[0] = i - sz;
        }
        for (int d = 0; d < 3; d++) {
            for (int k = 0; k < 3; k++) if (im[k] >= 0) g[d][i] += g[d][im[k]];
            for (int k = 0; k < 3; k++) if (im[k] >= 0) g[d][im[k]] = g[d][i];
        }
    }
    /* front_tracking_source4 (fronttrack.cu:540-583): divergence on COMP nodes;
     * jacobi_source: b = dg / diagonal (-6 / dx^2 on COMP rows, 1 elsewhere) */
    for (long i = 0; i < n; i++) {
        if (bc[i] != ORC_COMP) continue;
        const double d = (g[0][i+1] - g[0][i-1] + g[1][i+nx] - g[1][i-nx] + g[2][i+pl] - g[2][i-pl]) / (2.0 * dx);
        b[i] = d / (-6.0 / (dx * dx));
    }
    /* the matrix of front_tracking_matrix (fronttrack.cu:27-238) after
     * jacobi_matrix: COMP rows the 7-point Laplacian over -6/dx^2 (neighbours
     * (1/dx^2) / (-6/dx^2), diagonal 1); BUFF rows x_i - x_image = 0; WALL and
     * padding rows x_i = 0 */
    const double off = (1.0 / (dx * dx)) / (-6.0 / (dx * dx));
    double bb = 0.0;
    for (long i = 0; i < mn; i++) bb += b[i] * b[i];
    int result = -1;
    for (int cnt = 0; cnt <= 10 && result < 0; cnt++) {
        for (long i = 0; i < mn; i++) { x[i] = (double)cnt; r[i] = 0.0; }   /* front_tracking_solution */
        int iter;
        for (iter = 0; iter < p->vof_itrmax; iter++) {
            for (int color = 0; color < 2; color++) {   /* redblacksor_1, redblacksor_2 */
                for (long t = 0; t < mn; t++) {
                    long par;
                    if (t < n) { const long iz = t / pl, iy = t / nx - ny * iz, ix = t - nx * iy - pl * iz; par = ix + iy + iz; }
                    else par = t;
                    if (par % 2 != color) continue;
                    double sum;
                    if (t >= n || bc[t] == ORC_WALL) sum = 1.0 * x[t];
                    else if (bc[t] == ORC_COMP) {
                        sum = 0.0;
                        sum += off * x[t - pl]; sum += off * x[t - nx]; sum += off * x[t - 1]; sum += 1.0 * x[t];
                        sum += off * x[t + 1]; sum += off * x[t + nx]; sum += off * x[t + pl];
                    } else {   /* BUFF: the image of fronttrack.cu:104-124 / 146-150 */
                        const long iz = t / pl, ix = (t % pl) % nx;
                        long img = t;
                        if (p->flow == 1) {
                            if (ix <= 1) img += nx - 4; else if (ix >= nx - 2) img -= nx - 4;
                        }
                        if (iz <= 1) img += pl * (nz - 4); else if (iz >= nz - 2) img -= pl * (nz - 4);
                        sum = 0.0;
                        if (t < img) { sum += 1.0 * x[t]; sum += -1.0 * x[img]; }
                        else { sum += -1.0 * x[img]; sum += 1.0 * x[t]; }
                    }
                    r[t] = b[t] - sum;
                    x[t] += 1.3 * r[t];
                }
            }
            double rr = 0.0;
            for (long i = 0; i < mn; i++) rr += r[i] * r[i];
            if (sqrt(rr / bb) < p->vof_residual) break;
        }
        if (iter < p->vof_itrmax) result = iter + 1;
    }
    s->vof_iters = result;
    if (result > 0) memcpy(s->vf, x, sizeof(double) * (size_t)n);
    free(dg);
    return result;
}

/* ------------------------------------------------------------------------ */
/* Volume correction: volume_correction.cu                                   */
/* ------------------------------------------------------------------------ */

/* volume_correction.cu:138-200 (CalcEleNormal_GPU) + 246-281 (CalcVolume) */
static void calc_ele_normal(const orc_params *p, const orc_state *s, double *normal, double *dS, double *vtmp)
{
    long ne = (long)p->ncell * p->element;
#pragma omp parallel for schedule(static)
    for (long e = 0; e < ne; e++) {
        int na = s->ele[3*e+0], nb = s->ele[3*e+1], nc = s->ele[3*e+2];
        double v1[3] = {s->x[nb] - s->x[na], s->y[nb] - s->y[na], s->z[nb] - s->z[na]};
        double v2[3] = {s->x[nc] - s->x[na], s->y[nc] - s->y[na], s->z[nc] - s->z[na]};
        double c[3] = {v1[1]*v2[2] - v1[2]*v2[1], v1[2]*v2[0] - v1[0]*v2[2], v1[0]*v2[1] - v1[1]*v2[0]};
        double nc_ = sqrt(c[0]*c[0] + c[1]*c[1] + c[2]*c[2]);
        normal[3*e+0] = c[0] / nc_; normal[3*e+1] = c[1] / nc_; normal[3*e+2] = c[2] / nc_;
        dS[e] = nc_ / 2.0;
        double r[3] = {(s->x[na] + s->x[nb] + s->x[nc]) / 3.0, (s->y[na] + s->y[nb] + s->y[nc]) / 3.0,
                       (s->z[na] + s->z[nb] + s->z[nc]) / 3.0};
        vtmp[e] = 1.0 / 3.0 * (r[0]*normal[3*e+0] + r[1]*normal[3*e+1] + r[2]*normal[3*e+2]) * dS[e];
    }
}

void orc_calc_volume(const orc_params *p, const orc_state *s, double *volume, double *area)
{
    long ne = (long)p->ncell * p->element;
    double *normal = (double *)malloc(sizeof(double) * 3 * ne);
    double *dS = (double *)malloc(sizeof(double) * ne), *vtmp = (double *)malloc(sizeof(double) * ne);
    calc_ele_normal(p, s, normal, dS, vtmp);
    for (int c = 0; c < p->ncell; c++) {
        double V = 0.0, A = 0.0;
        for (int e = 0; e < p->element; e++) { V += vtmp[c * p->element + e]; A += dS[c * p->element + e]; }
        volume[c] = V; area[c] = A;
    }
    free(normal); free(dS); free(vtmp);
}

/* volume_correction.cu:310-352 (CalcCenter, channel branch) */
static void calc_center(const orc_params *p, orc_state *s)
{
    int V = p->vertex;
    for (int c = 0; c < p->ncell; c++) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int j = 0; j < V; j++) { sx += s->x[c*V + j]; sy += s->y[c*V + j]; sz += s->z[c*V + j]; }
        s->gx[3*c+0] = sx / (double)V; s->gx[3*c+1] = sy / (double)V; s->gx[3*c+2] = sz / (double)V;
        if (p->flow == 1) {   /* volume_correction.cu:319-325 */
            if (s->gx[3*c+0] < p->xmin) s->gx[3*c+0] += p->LX;
            else if (s->gx[3*c+0] > p->xmax) s->gx[3*c+0] -= p->LX;
        }
        if (s->gx[3*c+2] < p->zmin) s->gx[3*c+2] += p->LZ;
        else if (s->gx[3*c+2] > p->zmax) s->gx[3*c+2] -= p->LZ;
    }
}

/* volume_correction.cu:427-450 */
void orc_volume_init(const orc_params *p, orc_state *s)
{
    double *area = (double *)malloc(sizeof(double) * p->ncell);
    orc_calc_volume(p, s, s->volume0, area);
    free(area);
    calc_center(p, s);
}

/* volume_correction.cu:453-524 (RBC branch) with CapsulePeriodicBefore/After
 * (28-94), CalcLambda1 (378-399) and VolumeCorrection_GPU (97-135). */
int orc_volume_correction(const orc_params *p, orc_state *s)
{
    int N = p->ncell, V = p->vertex;
    long nv = (long)N * V, ne = (long)N * p->element;
    double *normal = (double *)malloc(sizeof(double) * 3 * ne);
    double *dS = (double *)malloc(sizeof(double) * ne), *vtmp = (double *)malloc(sizeof(double) * ne);
    double *volume = (double *)malloc(sizeof(double) * N), *area = (double *)malloc(sizeof(double) * N);
    double *lambda = (double *)malloc(sizeof(double) * N);
    int *conv = (int *)calloc(N, sizeof(int));
    /* CapsulePeriodicBefore: z unwrap about the stored centroid */
    for (int c = 0; c < N; c++)
        for (int j = 0; j < V; j++) {
            long id = (long)c * V + j;
            double dz = s->z[id] - s->gx[3*c+2];
            if (dz > p->LZ * 0.5) s->z[id] -= p->LZ; else if (dz < -p->LZ * 0.5) s->z[id] += p->LZ;
            if (p->flow == 1) {   /* volume_correction.cu:48-57 */
                double dxx = s->x[id] - s->gx[3*c+0];
                if (dxx > p->LX * 0.5) s->x[id] -= p->LX; else if (dxx < -p->LX * 0.5) s->x[id] += p->LX;
            }
        }
    int iter = 0, all_converged;
    do {
        calc_ele_normal(p, s, normal, dS, vtmp);
        for (int c = 0; c < N; c++) {
            double Vs = 0.0, As = 0.0;
            for (int e = 0; e < p->element; e++) { Vs += vtmp[(long)c * p->element + e]; As += dS[(long)c * p->element + e]; }
            volume[c] = Vs; area[c] = As;
        }
        all_converged = 1;
        for (int c = 0; c < N; c++) {
            double dV = fabs(volume[c] - s->volume0[c]) / s->volume0[c] * 100.0;
            if (dV < VC_EPS) { lambda[c] = 0.0; conv[c] = 1; }
            else lambda[c] = 18.0 * (volume[c] - s->volume0[c]) / area[c];
            all_converged &= conv[c];
        }
#pragma omp parallel for schedule(static)
        for (long id = 0; id < nv; id++) {
            int c = (int)(id / V), nne = s->nle[id];
            double nn[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < nne; k++) {
                int e = s->le[6*id + k];
                nn[0] += normal[3*e+0] / nne; nn[1] += normal[3*e+1] / nne; nn[2] += normal[3*e+2] / nne;
            }
            s->x[id] += -lambda[c] / 6.0 * nn[0] * COEFF_VOL_CHANGE;
            s->y[id] += -lambda[c] / 6.0 * nn[1] * COEFF_VOL_CHANGE;
            s->z[id] += -lambda[c] / 6.0 * nn[2] * COEFF_VOL_CHANGE;
        }
        iter++;
    } while (!all_converged && iter < VC_ITRMAX);
    calc_center(p, s);
    /* CapsulePeriodicAfter */
    for (long id = 0; id < nv; id++) {
        if (p->flow == 1) {   /* volume_correction.cu:88-91 */
            if (s->x[id] < p->xmin) s->x[id] += p->LX;
            else if (s->x[id] > p->xmax) s->x[id] -= p->LX;
        }
        if (s->z[id] < p->zmin) s->z[id] += p->LZ;
        else if (s->z[id] > p->zmax) s->z[id] -= p->LZ;
    }
    free(normal); free(dS); free(vtmp); free(volume); free(area); free(lambda); free(conv);
    if (iter >= VC_ITRMAX) return -1;
    return iter - 1;
}

/* main.cu:73-110 (no adhesion: CYTOADHESION = false): the membrane and the
 * spread at the first of every M steps ((iter - 1) % M == 0), the advection,
 * THINC/WLIC and the volume correction at the last (iter % M == 0), front
 * tracking every vof_k steps when vof_k > 0 */
int orc_step(const orc_params *p, orc_state *s, int nsteps)
{
    const int Ms = orc_M(p);
    for (int k = 0; k < nsteps; k++) {
        s->iter++;
        const int first = (s->iter - 1) % Ms == 0, last = s->iter % Ms == 0;
        if (p->ncell > 0 && first) {
            int flag = orc_stress(p, s);
            if (flag != 0) return 4;          /* error(4) in stress.cu:366 */
            orc_ibm_st1(p, s);
        }
        orc_lbm_d3q19(p, s);
        if (p->ncell > 0 && last) orc_ibm_st2(p, s);
        if (p->vof_k > 0 && s->vf) {
            if (last) orc_thinc_wlic(p, s);
            if (s->iter % p->vof_k == 0 && orc_front_tracking(p, s) < 0) return 6;   /* error(5) */
        }
        if (p->ncell > 0 && last && orc_volume_correction(p, s) < 0) return 5;
    }
    return 0;
}
