// ref_files.cu -- the reference's restart and output files.
//
// Byte layouts of etc.cu for a run with red cells (N_R), white cells (N_W)
// or both, no cytoadhesion, written and read with this library's state:
//   restart.bin  (output_data etc.cu:738-781, restart_file etc.cu:164-270)
//     int iter, int fnum, double fn[n*19], dm[n], um[n], vm[n], wm[n], vf[n],
//     vf2[n]; then per population (red, then white): double x[N*V], y[N*V],
//     z[N*V], rx[N], ry[N], rz[N], u[N*V], v[N*V], w[N*V], qi[N*mn], tp[N*E*2]
//   cell%04d.bin (etc.cu:566-600)
//     per population: int N, V, E, double x, y, z, u, v, w [N*V], qi[N*V*3],
//     tp[N*E*2], int ele[N*E*3] (vertex ids within the population)
//   prof%04d.bin (etc.cu:547-560)
//     int iter, double dm, um, vm, wm, vf, vf2 [n], int bc[n]
//   center.dat   (OutputCapsuleCenter / InputCapsuleCenter, etc.cu:110-160)
//     one line per cell, red cells then white cells, each numbered from 0:
//     "%d %e %e %e \n" (cell, cel->gx[3c + 0..2] or cel->gx_w)
// n = nx * ny * nz counts the BUFF planes.  vf and vf2 are the red and white
// cells' volume fractions when they are tracked (vof_k > 0), else flu_init's 0;
// rx, ry, rz are never set by the reference: written as 0, ignored when read.
// qi and tp are the output-interval averages of the load and the principal
// tensions (rbc_set_output_interval; 0 when no interval is set).  The
// populations of non-COMP nodes are never read by the reference's step: they
// keep flu_init's rest equilibrium w_q or 0 as its two population buffers
// swap, so they are written as w_q after an even number of steps and 0 after
// an odd one, as a reference run from iteration 0 holds them.
#include "rbc_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

using namespace rbc;

namespace {

struct Pop {   // one cell population: 0 red cells (cel->x), 1 white cells (cel->x_w)
    int N = 0, V = 0, E = 0, mn = 0;
    long long nv = 0, ne = 0;
};

struct Dims {
    int nx = 0, ny = 0, nz = 0;
    long long n = 0;
    Pop pop[2];
};

int dims_of(rbc_handle *h, Dims &d)
{
    int nzp = 0, N = 0, V = 0, E = 0;
    int rc = rbc_dims(h, &d.nx, &d.ny, &nzp, &N, &V, &E);
    if (rc) return rc;
    d.nz = nzp + 4;
    d.n = (long long)d.nx * d.ny * d.nz;
    for (int k = 0; k < 2; k++) {
        Pop &p = d.pop[k];
        group_sizes(h, k, &p.N, &p.V, &p.E);
        p.nv = (long long)p.N * p.V;
        p.ne = (long long)p.N * p.E;
        p.mn = p.N > 0 ? reference_mn(p.V) : 0;
    }
    return RBC_OK;
}

int export_pop(rbc_handle *h, int k, double *x, double *y, double *z, double *u, double *v, double *w, double *gx)
{
    return k == 0 ? rbc_export_ref_cells(h, x, y, z, nullptr, u, v, w, nullptr, nullptr, nullptr, gx)
                  : rbc_export_ref_wbc(h, x, y, z, nullptr, u, v, w, nullptr, nullptr, nullptr, gx);
}

int import_pop(rbc_handle *h, int k, const double *x, const double *y, const double *z, const double *xd,
               const double *gx)
{
    return k == 0 ? rbc_import_ref_cells(h, x, y, z, xd, nullptr, nullptr, gx)
                  : rbc_import_ref_wbc(h, x, y, z, xd, nullptr, nullptr, gx);
}

// cel->x, y, z, u, v, w of one population and its fem->qi [N mn] and fem->tp [2 N E]
struct PopState {
    std::vector<double> cx, qi, tp;
};

int pop_state(rbc_handle *h, const Pop &p, int k, PopState &st)
{
    st.cx.resize((size_t)p.nv * 6);
    st.qi.resize((size_t)p.N * p.mn);
    st.tp.resize((size_t)p.ne * 2);
    double *x = st.cx.data();
    int rc = export_pop(h, k, x, x + p.nv, x + 2 * p.nv, x + 3 * p.nv, x + 4 * p.nv, x + 5 * p.nv, nullptr);
    return rc ? rc : output_averages(h, k, st.qi.data(), st.tp.data(), false);
}

struct File {
    FILE *f = nullptr;
    explicit File(const char *path, const char *mode) : f(std::fopen(path, mode)) {}
    ~File() { if (f) std::fclose(f); }
};

template <typename T>
bool put(FILE *f, const T *p, size_t count) { return std::fwrite(p, sizeof(T), count, f) == count; }
template <typename T>
bool get(FILE *f, T *p, size_t count) { return std::fread(p, sizeof(T), count, f) == count; }

int io_error(rbc_handle *h, const char *what, const char *path)
{
    set_handle_error(h, std::string(what) + ": " + (path ? path : "(null)"));
    return RBC_ERR_ARG;
}

// the lattice in the reference's layout with non-COMP populations as the reference holds them
// ltc->vf, vf2 [2][n]: the tracked volume fractions, or 0
int vof_of(rbc_handle *h, const Dims &d, std::vector<double> &vf)
{
    vf.assign((size_t)d.n * 2, 0.0);
    if (rbc_export_ref_vof(h, vf.data(), vf.data() + d.n) == RBC_OK) return RBC_OK;
    set_handle_error(h, "");   // not tracked: zeros
    return RBC_OK;
}

int lattice_of(rbc_handle *h, const Dims &d, std::vector<double> &fn, std::vector<double> &mac, std::vector<int> &bc)
{
    fn.resize((size_t)d.n * Q);
    mac.resize((size_t)d.n * 4);
    bc.resize((size_t)d.n);
    int rc = rbc_export_ref_lattice(h, fn.data(), mac.data(), mac.data() + d.n, mac.data() + 2 * d.n, mac.data() + 3 * d.n);
    if (rc) return rc;
    if ((rc = reference_bc(h, bc.data()))) return rc;
    int iter = 0;
    rbc_get_iter(h, &iter);
    for (long long i = 0; i < d.n; i++)
        if (bc[i] != RBC_COMP)
            for (int q = 0; q < Q; q++) fn[(size_t)i * Q + q] = (iter % 2 == 0) ? wqd(q) : 0.0;
    return RBC_OK;
}

}  // namespace

extern "C" {

int rbc_write_restart(rbc_handle *h, const char *path, int fnum)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    std::vector<double> fn, mac;
    std::vector<int> bc;
    if ((rc = lattice_of(h, d, fn, mac, bc))) return rc;
    std::vector<double> vf;
    if ((rc = vof_of(h, d, vf))) return rc;
    std::vector<double> zeros((size_t)std::max<long long>({d.n, d.pop[0].N, d.pop[1].N}), 0.0);
    PopState st[2];
    for (int k = 0; k < 2; k++)
        if (d.pop[k].N > 0 && (rc = pop_state(h, d.pop[k], k, st[k]))) return rc;
    int iter = 0;
    rbc_get_iter(h, &iter);
    File f(path, "wb");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    bool ok = put(f.f, &iter, 1) && put(f.f, &fnum, 1) && put(f.f, fn.data(), fn.size())
           && put(f.f, mac.data(), mac.size())          // dm, um, vm, wm
           && put(f.f, vf.data(), 2 * d.n);             // vf, vf2
    for (int k = 0; k < 2 && ok; k++) {
        const Pop &p = d.pop[k];
        if (p.N == 0) continue;
        const double *x = st[k].cx.data();
        ok = put(f.f, x, 3 * p.nv)                       // x, y, z
          && put(f.f, zeros.data(), p.N) && put(f.f, zeros.data(), p.N) && put(f.f, zeros.data(), p.N)   // rx, ry, rz
          && put(f.f, x + 3 * p.nv, 3 * p.nv)            // u, v, w
          && put(f.f, st[k].qi.data(), st[k].qi.size()) && put(f.f, st[k].tp.data(), st[k].tp.size());
    }
    return ok ? RBC_OK : io_error(h, "write failed", path);
}

int rbc_read_restart(rbc_handle *h, const char *path, int *fnum)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    File f(path, "rb");
    if (!f.f) return io_error(h, "cannot open for reading", path);
    int iter = 0, fn_ = 0;
    std::vector<double> fn((size_t)d.n * Q), skip((size_t)d.n * 6);
    bool ok = get(f.f, &iter, 1) && get(f.f, &fn_, 1) && get(f.f, fn.data(), fn.size())
           && get(f.f, skip.data(), skip.size());     // dm, um, vm, wm, vf, vf2
    PopState st[2];
    for (int k = 0; k < 2 && ok; k++) {
        const Pop &p = d.pop[k];
        if (p.N == 0) continue;
        st[k].cx.resize((size_t)p.nv * 6);
        st[k].qi.resize((size_t)p.N * p.mn);
        st[k].tp.resize((size_t)p.ne * 2);
        std::vector<double> r((size_t)p.N * 3);
        double *x = st[k].cx.data();
        ok = get(f.f, x, 3 * p.nv) && get(f.f, r.data(), r.size()) && get(f.f, x + 3 * p.nv, 3 * p.nv)
          && get(f.f, st[k].qi.data(), st[k].qi.size()) && get(f.f, st[k].tp.data(), st[k].tp.size());
    }
    if (!ok) return io_error(h, "restart file too short for this lattice and these cells", path);
    if (std::fgetc(f.f) != EOF) return io_error(h, "restart file longer than this lattice and these cells", path);
    if (fn_ > 100) { iter = 0; fn_ = 0; }   // etc.cu:205
    if ((rc = rbc_import_ref_lattice(h, fn.data()))) return rc;
    // the density and velocity sums (etc.cu:277-280): what the advection reads
    // when the file ends inside a sub-cycle, and what the next write repeats
    if ((rc = import_macro(h, skip.data(), skip.data() + d.n, skip.data() + 2 * d.n, skip.data() + 3 * d.n))) return rc;
    // the file holds no IB force: the reference resumes with the ltc->fx of its
    // set-up, 0 (init1.cu:394-409, 923), which matters only for a file written
    // inside a sub-cycle
    if ((rc = clear_force(h))) return rc;
    // the volume fractions when tracked (etc.cu:213-214, 281-282); else unused
    if (rbc_import_ref_vof(h, skip.data() + 4 * d.n, skip.data() + 5 * d.n) != RBC_OK) set_handle_error(h, "");
    for (int k = 0; k < 2; k++) {
        const Pop &p = d.pop[k];
        if (p.N == 0) continue;
        // fem->x (hence fem->xd) is set from cel->x (etc.cu:256-274); the vertex velocities (the
        // last advection's, which the next one overwrites) are kept for the next file write
        const double *x = st[k].cx.data(), *y = x + p.nv, *z = y + p.nv;
        std::vector<double> xd((size_t)p.nv * 3);
        for (long long j = 0; j < p.nv; j++) { xd[3 * j] = x[j]; xd[3 * j + 1] = y[j]; xd[3 * j + 2] = z[j]; }
        if ((rc = import_pop(h, k, x, y, z, xd.data(), nullptr))) return rc;
        if ((rc = import_vertex_velocity(h, k, x + 3 * p.nv, x + 4 * p.nv, x + 5 * p.nv))) return rc;
        if ((rc = output_averages(h, k, st[k].qi.data(), st[k].tp.data(), true))) return rc;
    }
    if ((rc = rbc_set_iter(h, iter))) return rc;
    if (fnum) *fnum = fn_;
    return RBC_OK;
}

int rbc_write_cell_file(rbc_handle *h, const char *path)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    if (d.pop[0].N == 0 && d.pop[1].N == 0) return RBC_ERR_STATE;
    PopState st[2];
    std::vector<int> ele[2];
    for (int k = 0; k < 2; k++) {
        const Pop &p = d.pop[k];
        if (p.N == 0) continue;
        if ((rc = pop_state(h, p, k, st[k]))) return rc;
        ele[k].resize((size_t)p.ne * 3);
        if ((rc = reference_ele(h, k, ele[k].data()))) return rc;
    }
    File f(path, "wb");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    bool ok = true;
    for (int k = 0; k < 2 && ok; k++) {
        const Pop &p = d.pop[k];
        if (p.N == 0) continue;
        ok = put(f.f, &p.N, 1) && put(f.f, &p.V, 1) && put(f.f, &p.E, 1) && put(f.f, st[k].cx.data(), 6 * p.nv)
          && put(f.f, st[k].qi.data(), 3 * p.nv) && put(f.f, st[k].tp.data(), st[k].tp.size())
          && put(f.f, ele[k].data(), ele[k].size());
    }
    return ok ? RBC_OK : io_error(h, "write failed", path);
}

int rbc_write_prof_file(rbc_handle *h, const char *path)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    std::vector<double> fn, mac;
    std::vector<int> bc;
    if ((rc = lattice_of(h, d, fn, mac, bc))) return rc;
    std::vector<double> vf;
    if ((rc = vof_of(h, d, vf))) return rc;
    int iter = 0;
    rbc_get_iter(h, &iter);
    File f(path, "wb");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    const bool ok = put(f.f, &iter, 1) && put(f.f, mac.data(), mac.size()) && put(f.f, vf.data(), 2 * d.n)
                 && put(f.f, bc.data(), bc.size());
    return ok ? RBC_OK : io_error(h, "write failed", path);
}

int rbc_write_center_file(rbc_handle *h, const char *path)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    std::vector<double> gx[2];
    for (int k = 0; k < 2; k++) {
        gx[k].resize((size_t)d.pop[k].N * 3 + 1);
        if (d.pop[k].N > 0 && (rc = export_pop(h, k, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, gx[k].data())))
            return rc;
    }
    File f(path, "w");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    for (int k = 0; k < 2; k++)
        for (int c = 0; c < d.pop[k].N; c++)
            if (std::fprintf(f.f, "%d %e %e %e \n", c, gx[k][3 * c], gx[k][3 * c + 1], gx[k][3 * c + 2]) < 0)
                return io_error(h, "write failed", path);
    return RBC_OK;
}

int rbc_read_center_file(rbc_handle *h, const char *path)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    if (d.pop[0].N == 0 && d.pop[1].N == 0) return RBC_ERR_STATE;
    File f(path, "r");
    if (!f.f) return io_error(h, "cannot open for reading", path);
    std::vector<double> gx[2];
    for (int k = 0; k < 2; k++) {
        gx[k].resize((size_t)d.pop[k].N * 3);
        for (int c = 0; c < d.pop[k].N; c++)
            if (std::fscanf(f.f, "%*d %lf %lf %lf", &gx[k][3 * c], &gx[k][3 * c + 1], &gx[k][3 * c + 2]) != 3)
                return io_error(h, "center file has fewer lines than cells", path);
    }
    for (int k = 0; k < 2; k++)
        if (d.pop[k].N > 0 && (rc = import_pop(h, k, nullptr, nullptr, nullptr, nullptr, gx[k].data()))) return rc;
    return RBC_OK;
}

}  // extern "C"
