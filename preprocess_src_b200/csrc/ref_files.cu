// ref_files.cu -- the reference's restart and output files.
//
// Byte layouts of etc.cu for a red-cell run (N_R > 0, N_W = 0, no
// cytoadhesion), written and read with this library's state:
//   restart.bin  (output_data etc.cu:738-766, restart_file etc.cu:164-270)
//     int iter, int fnum, double fn[n*19], dm[n], um[n], vm[n], wm[n], vf[n],
//     vf2[n]; then for cells: double x[N*V], y[N*V], z[N*V], rx[N], ry[N],
//     rz[N], u[N*V], v[N*V], w[N*V], qi[N*mn], tp[N*E*2]
//   cell%04d.bin (etc.cu:566-590)
//     int N, V, E, double x, y, z, u, v, w [N*V], qi[N*V*3], tp[N*E*2],
//     int ele[N*E*3] (global vertex ids)
//   prof%04d.bin (etc.cu:547-560)
//     int iter, double dm, um, vm, wm, vf, vf2 [n], int bc[n]
//   center.dat   (OutputCapsuleCenter / InputCapsuleCenter, etc.cu:110-160)
//     one line per cell: "%d %e %e %e \n" (cell, cel->gx[3c + 0..2])
// n = nx * ny * nz counts the BUFF planes.  vf and vf2 (the VOF indicator,
// used only with a viscosity contrast) stay at flu_init's 0, and rx, ry, rz are
// never set by the reference; both are written as 0 and ignored when read.
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

struct Dims {
    int nx = 0, ny = 0, nz = 0, N = 0, V = 0, E = 0, mn = 0;
    long long n = 0, nv = 0, ne = 0;
};

int dims_of(rbc_handle *h, Dims &d)
{
    int nzp = 0;
    int rc = rbc_dims(h, &d.nx, &d.ny, &nzp, &d.N, &d.V, &d.E);
    if (rc) return rc;
    d.nz = nzp + 4;
    d.n = (long long)d.nx * d.ny * d.nz;
    d.nv = (long long)d.N * d.V;
    d.ne = (long long)d.N * d.E;
    d.mn = d.N > 0 ? reference_mn(d.V) : 0;
    return RBC_OK;
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
    std::vector<double> zeros((size_t)std::max<long long>(d.n, d.N), 0.0);
    std::vector<double> cx, qi, tp;
    if (d.N > 0) {
        cx.resize((size_t)d.nv * 6);
        double *x = cx.data(), *y = x + d.nv, *z = y + d.nv, *u = z + d.nv, *v = u + d.nv, *w = v + d.nv;
        if ((rc = rbc_export_ref_cells(h, x, y, z, nullptr, u, v, w, nullptr, nullptr, nullptr, nullptr))) return rc;
        qi.resize((size_t)d.N * d.mn);
        tp.resize((size_t)d.ne * 2);
        if ((rc = output_averages(h, qi.data(), tp.data(), false))) return rc;
    }
    int iter = 0;
    rbc_get_iter(h, &iter);
    File f(path, "wb");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    bool ok = put(f.f, &iter, 1) && put(f.f, &fnum, 1) && put(f.f, fn.data(), fn.size())
           && put(f.f, mac.data(), mac.size())          // dm, um, vm, wm
           && put(f.f, zeros.data(), d.n) && put(f.f, zeros.data(), d.n);   // vf, vf2
    if (ok && d.N > 0) {
        const double *x = cx.data();
        ok = put(f.f, x, 3 * d.nv)                       // x, y, z
          && put(f.f, zeros.data(), d.N) && put(f.f, zeros.data(), d.N) && put(f.f, zeros.data(), d.N)   // rx, ry, rz
          && put(f.f, x + 3 * d.nv, 3 * d.nv)            // u, v, w
          && put(f.f, qi.data(), qi.size()) && put(f.f, tp.data(), tp.size());
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
           && get(f.f, skip.data(), skip.size());     // dm, um, vm, wm, vf, vf2: recomputed by the step / unused
    std::vector<double> cx, qi, tp;
    if (ok && d.N > 0) {
        cx.resize((size_t)d.nv * 6);
        std::vector<double> r((size_t)d.N * 3);
        qi.resize((size_t)d.N * d.mn);
        tp.resize((size_t)d.ne * 2);
        ok = get(f.f, cx.data(), 3 * d.nv) && get(f.f, r.data(), r.size()) && get(f.f, cx.data() + 3 * d.nv, 3 * d.nv)
          && get(f.f, qi.data(), qi.size()) && get(f.f, tp.data(), tp.size());
    }
    if (!ok) return io_error(h, "restart file too short for this lattice and these cells", path);
    if (std::fgetc(f.f) != EOF) return io_error(h, "restart file longer than this lattice and these cells", path);
    if (fn_ > 100) { iter = 0; fn_ = 0; }   // etc.cu:205
    if ((rc = rbc_import_ref_lattice(h, fn.data()))) return rc;
    if (d.N > 0) {
        // fem->x (hence fem->xd) is set from cel->x (etc.cu:248-255); the vertex velocities are the
        // next advection's output and are not needed to step
        const double *x = cx.data(), *y = x + d.nv, *z = y + d.nv;
        std::vector<double> xd((size_t)d.nv * 3);
        for (long long j = 0; j < d.nv; j++) { xd[3 * j] = x[j]; xd[3 * j + 1] = y[j]; xd[3 * j + 2] = z[j]; }
        if ((rc = rbc_import_ref_cells(h, x, y, z, xd.data(), nullptr, nullptr, nullptr))) return rc;
        if ((rc = output_averages(h, qi.data(), tp.data(), true))) return rc;
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
    if (d.N == 0) return RBC_ERR_STATE;
    std::vector<double> cx((size_t)d.nv * 6), qi((size_t)d.N * d.mn), tp((size_t)d.ne * 2);
    double *x = cx.data();
    if ((rc = rbc_export_ref_cells(h, x, x + d.nv, x + 2 * d.nv, nullptr, x + 3 * d.nv, x + 4 * d.nv, x + 5 * d.nv,
                                   nullptr, nullptr, nullptr, nullptr))) return rc;
    if ((rc = output_averages(h, qi.data(), tp.data(), false))) return rc;
    std::vector<int> ele((size_t)d.ne * 3);
    if ((rc = reference_ele(h, ele.data()))) return rc;
    File f(path, "wb");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    const bool ok = put(f.f, &d.N, 1) && put(f.f, &d.V, 1) && put(f.f, &d.E, 1) && put(f.f, x, 6 * d.nv)
                 && put(f.f, qi.data(), 3 * d.nv) && put(f.f, tp.data(), tp.size()) && put(f.f, ele.data(), ele.size());
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
    std::vector<double> zeros((size_t)d.n, 0.0);
    int iter = 0;
    rbc_get_iter(h, &iter);
    File f(path, "wb");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    const bool ok = put(f.f, &iter, 1) && put(f.f, mac.data(), mac.size()) && put(f.f, zeros.data(), d.n)
                 && put(f.f, zeros.data(), d.n) && put(f.f, bc.data(), bc.size());
    return ok ? RBC_OK : io_error(h, "write failed", path);
}

int rbc_write_center_file(rbc_handle *h, const char *path)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    std::vector<double> gx((size_t)d.N * 3 + 1);
    if (d.N > 0 && (rc = rbc_export_ref_cells(h, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                              nullptr, nullptr, nullptr, gx.data()))) return rc;
    File f(path, "w");
    if (!f.f) return io_error(h, "cannot open for writing", path);
    for (int c = 0; c < d.N; c++)
        if (std::fprintf(f.f, "%d %e %e %e \n", c, gx[3 * c], gx[3 * c + 1], gx[3 * c + 2]) < 0)
            return io_error(h, "write failed", path);
    return RBC_OK;
}

int rbc_read_center_file(rbc_handle *h, const char *path)
{
    if (!h || !path) return RBC_ERR_ARG;
    Dims d;
    int rc = dims_of(h, d);
    if (rc) return rc;
    if (d.N == 0) return RBC_ERR_STATE;
    File f(path, "r");
    if (!f.f) return io_error(h, "cannot open for reading", path);
    std::vector<double> gx((size_t)d.N * 3);
    for (int c = 0; c < d.N; c++)
        if (std::fscanf(f.f, "%*d %lf %lf %lf", &gx[3 * c], &gx[3 * c + 1], &gx[3 * c + 2]) != 3)
            return io_error(h, "center file has fewer lines than cells", path);
    return rbc_import_ref_cells(h, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, gx.data());
}

}  // extern "C"
