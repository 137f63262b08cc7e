// rbc_abi.cu -- host side of the C ABI declared in include/rbc_step.h.
//
// Owns the device state of one simulation and sequences the step kernels on
// one CUDA stream.  rbc_step replays CUDA graphs of one step (two graphs, one
// per population-buffer parity, since the buffers ping-pong); the reference
// instead launches each module with a blocking
// cudaThreadSynchronize() and host round trips inside the membrane solve and
// the volume correction (main.cu:73-110).
#include "rbc_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <map>
#include <new>
#include <numeric>
#include <string>
#include <vector>

using namespace rbc;

namespace {

thread_local std::string g_create_error;

constexpr int DEFAULT_SOLVER_ITERS = 16;  // Chebyshev error factor <= 2 * 3^-16 ~ 4.6e-8 (FP32 solve)

}  // namespace

namespace rbc {
// text returned by rbc_last_error(NULL), for entry points that take no handle
void set_last_error(const std::string &msg) { g_create_error = msg; }
}

struct AdjointState;
void adjoint_free(AdjointState *a);

// One cell population: the red cells (the reference's cel->x ..., fem->...) or
// the white cells (cel->x_w ..., fem->..._w, init3.cu), each with its own mesh
// shared by its cells, tension normalisation rg (1 for red cells, GSw / GS for
// white ones) and bending modulus.
struct CellGroup {
    int ncell = 0, V = 0, E = 0;
    long long nv = 0, ne = 0;
    double rgs = 1.0, br = 0.0;
    double *X = nullptr, *Xd = nullptr;
    double4 *gref = nullptr;
    void *erec = nullptr;   // membrane element records, [ne][3] 4-vectors of float or double
    float *U = nullptr, *Fv = nullptr;
    int *tri = nullptr, *v2e_off = nullptr, *v2e = nullptr;
    int16_t *nbr = nullptr;
    int16_t *nbrp = nullptr;  // neighbours by solve position ([6][V]) and the vertex at each position ([V])
    int *vord = nullptr;
    int4 *visit = nullptr;   // bending visits [E][3], allocated when BR != 0
    double2 *cs0 = nullptr;  // spontaneous angle (cos, sin) per visit [ncell][E][3] (bend_spont), else none
    double *bend_rec = nullptr;   // bending visit records [ncell][E][3][9], allocated when BR != 0
    double *vol0 = nullptr, *gx = nullptr, *vol_out = nullptr, *area_out = nullptr, *cen_out = nullptr;
    int *patch_off = nullptr, *patch_vtx = nullptr, *patch_stride = nullptr;
    int npatch = 1;
    int mn = 0;                                       // the reference's per-cell vector length (expand2pow2(3 V))
    double *qi_acc = nullptr, *tp_acc = nullptr;      // output-interval averages [ncell][mn], [ne][2]
    double *vf = nullptr;                             // volume fraction [nint] (ltc->vf, vf2), VOF only
};

struct rbc_handle {
    rbc_params p{};
    Geom geo{};
    // cell populations: cg[0] red cells, cg[1] white cells (rbc_add_wbc)
    CellGroup cg[2];
    int ngroups = 1;
    // the red cells under the names the single-population code uses (the handle is never copied)
    int &ncell = cg[0].ncell, &V = cg[0].V, &E = cg[0].E;
    long long &nv = cg[0].nv, &ne = cg[0].ne;
    double *&X = cg[0].X, *&Xd = cg[0].Xd;
    double4 *&gref = cg[0].gref;
    float *&U = cg[0].U, *&Fv = cg[0].Fv;
    int *&tri = cg[0].tri, *&v2e_off = cg[0].v2e_off, *&v2e = cg[0].v2e;
    int16_t *&nbr = cg[0].nbr;
    double *&vol0 = cg[0].vol0, *&gx = cg[0].gx;
    long long nref_nodes = 0;
    cudaStream_t stream = nullptr;
    // lattice
    void *g[2] = {nullptr, nullptr};
    int cur = 0;
    size_t gbytes = 0;
    float4 *uvr = nullptr;
    long long *Fint = nullptr;                        // IB force, fixed point [3][nint] (ForceField)
    uint32_t *Fbits = nullptr;                        // its occupancy words [nzc][wpp]
    uint32_t *mask2d = nullptr;
    int *tube_links = nullptr; float *tube_frac = nullptr; int ntube = 0;   // interpolated wall links (circular tube)
    // device scalars: iter, flags, vc_max, vc_last, front-tracking sweeps of populations 0 and 1
    int *d_int = nullptr;
    // volume fraction scratch (vof_k > 0): THINC sweep buffers, indicator gradient / CG vectors,
    // right-hand side, CG block partials
    double *vof_s1 = nullptr, *vof_s2 = nullptr, *vof_G = nullptr, *vof_b = nullptr, *vof_partial = nullptr;
    MgHierarchy vof_mg;                               // multigrid levels of the front-tracking solve
    float *d_drive = nullptr;                          // [3]: drive P * factor, then the walls' z velocities
    // host<->reference staging
    void *staging = nullptr;
    size_t staging_bytes = 0;
    // lattice import: IMPORT_SLOTS chunks of imp_planes reference planes in a ring, then the two
    // periodic edge planes; a copy and a conversion event per slot (allocated on first use)
    double *imp_ring = nullptr;
    int imp_planes = 0;
    cudaEvent_t imp_copied[4] = {}, imp_freed[4] = {};
    int iter = 0;
    // the IB force field may hold nonzero values: a spread not yet cleared (a
    // stage call, or a sub-cycled step ended before the last step of its M)
    bool force_pending = false;
    // CUDA graphs of one step starting from population buffer 0 / 1, in three
    // forms (StepForm): the whole step; the step without its volume
    // correction; the step without its correction but with the previous
    // step's correction beside its membrane pass
    // (and three more, StepForm STEP_SUB_*, for the first, middle and last of
    // M sub-cycled steps), with the kernels each launches
    cudaGraphExec_t graph[6][2] = {};
    int graph_kernels[6] = {};
    cudaStream_t side = nullptr;                      // second branch of the pipelined graphs (capture only)
    cudaEvent_t fork = nullptr, join = nullptr;
    // split membrane pass: the first full wave's spread beside the last wave's membrane (capture only)
    cudaStream_t side2 = nullptr;
    cudaEvent_t wave_done = nullptr, spread_done = nullptr;
    // the force reset beside the advection (capture only; on side2, idle by then)
    cudaEvent_t lbm_done = nullptr, reset_done = nullptr;
    int sms = 0;                                      // multiprocessors of the device
    int prio_high = 0;                                // greatest stream priority of the device
    long long launches = 0;
    float scale = 1.0f, inv_scale = 1.0f;
    std::string err;
    int device = 0;
    AdjointState *adj = nullptr;                      // checkpoints and buffers of the adjoint, on first use
    int fileoutput = 0;                               // FILEOUTPUT of the qi / tp averages; 0 = not accumulated
    int lbm_planes = 0;                               // RBC_SHAPE_LBM_PLANES (0 = automatic)
    // the volume correction that ended the last rbc_step left every population's
    // volume, area (vol_out, area_out) and centroid (gx) of the current state
    bool metrics_valid = false;
    double *metrics_host = nullptr;                   // pinned staging of one population's metrics [5][ncell]
    size_t metrics_host_n = 0;

    int kernels_per_step() const {
        int k = 2 + (ntube > 0 ? 1 : 0) + (has_cells() ? 1 : 0);   // step_begin, lbm (+ tube bounce-back, force reset)
        if (ngroups == 1 && cg[0].br == 0.0 && fileoutput == 0 && sms > 0 && cg[0].ncell > sms && cg[0].ncell % sms)
            k += 2;                        // the membrane pass and the spread in two launches each
        for (int g = 0; g < ngroups; g++) {
            const CellGroup &c = cg[g];
            if (c.ncell == 0) continue;
            k += 4 + (c.br != 0.0 ? 2 : 0) + (fileoutput > 0 ? 2 : 0);   // membrane, spread, advect, volume
            if (c.vf) k += 3;                                            // THINC/WLIC sweeps
        }
        return k;
    }
    ForceField force() const { return ForceField{Fint, Fbits, force_words_per_plane(geo.plane)}; }
    size_t force_bit_bytes() const { return sizeof(uint32_t) * (size_t)geo.nzc * force_words_per_plane(geo.plane); }
    bool has_cells() const {
        for (int g = 0; g < ngroups; g++) if (cg[g].ncell > 0) return true;
        return false;
    }
    int *d_iter() { return d_int; }
    int *d_flags() { return d_int + 1; }
    int *d_vcmax() { return d_int + 2; }
    int *d_vclast() { return d_int + 3; }
    int *d_vofit() { return d_int + 4; }
    bool vof() const { return p.vof_k > 0; }
};

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            h->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
            return RBC_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

// Entry points that may change the device state drop the record that the
// cells' metrics on the device are those of the current state; read-only
// entry points keep it.
#define RBC_DEVICE_GUARD(h)                                                            \
    do {                                                                               \
        if (cudaSetDevice((h)->device) != cudaSuccess) return RBC_ERR_CUDA;            \
        (h)->metrics_valid = false;                                                    \
    } while (0)
#define RBC_DEVICE_GUARD_RO(h)                                                         \
    do {                                                                               \
        if (cudaSetDevice((h)->device) != cudaSuccess) return RBC_ERR_CUDA;            \
    } while (0)

#define CK_LAUNCH()                                                                    \
    do {                                                                               \
        cudaError_t e_ = cudaGetLastError();                                           \
        if (e_ != cudaSuccess) {                                                       \
            h->err = std::string("kernel launch: ") + cudaGetErrorString(e_);          \
            return RBC_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

namespace {

int fail(rbc_handle *h, int code, const std::string &msg)
{
    if (h) h->err = msg; else g_create_error = msg;
    return code;
}

template <typename T>
int dalloc(rbc_handle *h, T **p, size_t count)
{
    CK(cudaMalloc((void **)p, sizeof(T) * (count ? count : 1)));
    return RBC_OK;
}

int ensure_staging(rbc_handle *h, size_t bytes)
{
    if (h->staging_bytes >= bytes) return RBC_OK;
    if (h->staging) { CK(cudaFree(h->staging)); h->staging = nullptr; h->staging_bytes = 0; }
    CK(cudaMalloc(&h->staging, bytes));
    h->staging_bytes = bytes;
    return RBC_OK;
}

// the step-begin arguments of the handle (the adjoint adds where to keep the drive)
StepBeginArgs step_begin_args(rbc_handle *h);
WallVel wall_velocities(const rbc_handle *h, int step);

double drive_factor(const rbc_params &p, int iter)
{
    // lbm.cu:1030-1035
    return (iter > p.flowstart) ? 1.0 + 0.5 * std::sin(M_PI * p.dt * (double)iter / p.freq) : 0.0;
}

StepBeginArgs step_begin_args(rbc_handle *h)
{
    StepBeginArgs a{};
    a.iter = h->d_iter(); a.drive = h->d_drive;
    a.P = h->p.P; a.freq = h->p.freq; a.dt = h->p.dt; a.flowstart = h->p.flowstart;
    if (h->p.flow == RBC_FLOW_SHEAR) {
        a.wall = h->d_drive + 1;
        a.sr = h->p.sr; a.LY = (double)(h->p.ny - 4) * h->p.dx; a.walls = h->p.walls;
    }
    return a;
}

// the walls' z velocities in step `step` as step_begin_kernel sets them (lbm.cu:752, 946-964)
WallVel wall_velocities(const rbc_handle *h, int step)
{
    WallVel w{0.0, 0.0, h->p.Cr};
    if (h->p.flow != RBC_FLOW_SHEAR) return w;
    const double sra = step < h->p.flowstart ? 0.0 : h->p.sr, LY = (double)(h->p.ny - 4) * h->p.dx;
    w.top = (double)(float)(h->p.walls == RBC_WALLS_BOTH ? sra * LY / 2.0 : sra * LY);
    w.bot = (double)(float)(h->p.walls == RBC_WALLS_BOTH ? -sra * LY / 2.0 : 0.0);
    return w;
}

// Link tables of the shared local connectivity (init2.cu:258-400): neighbour
// lists (the vertices add_nlink collects, kept in the membrane solve's order
// below), vertex -> element lists in element order (add_elink), the
// reference's link-count check, and the packed incidence entries used by the
// membrane and volume kernels.
int build_topology(rbc_handle *h, const CellGroup &c, const int *tri, std::vector<int> &off, std::vector<int> &packed,
                   std::vector<int16_t> &nbr6, std::vector<int16_t> &nbrp6, std::vector<int> &vord)
{
    const int V = c.V, E = c.E;
    std::vector<std::vector<int>> nl(V), el(V);
    auto add = [&](int a, int b) {
        for (int x : nl[a]) if (x == b) return;
        nl[a].push_back(b);
    };
    for (int e = 0; e < E; e++) {
        const int a = tri[3 * e], b = tri[3 * e + 1], c = tri[3 * e + 2];
        if (a < 0 || a >= V || b < 0 || b >= V || c < 0 || c >= V || a == b || b == c || a == c)
            return fail(h, RBC_ERR_TOPOLOGY, "triangle " + std::to_string(e) + " has invalid vertex ids");
        add(a, b); add(a, c); add(b, c); add(b, a); add(c, a); add(c, b);
        el[a].push_back(e); el[b].push_back(e); el[c].push_back(e);
    }
    long long links = 0;
    for (int i = 0; i < V; i++) {
        links += (long long)nl[i].size();
        if (nl[i].size() > 6 || el[i].size() > 6)
            return fail(h, RBC_ERR_TOPOLOGY, "vertex " + std::to_string(i) + " has valence above 6 (the reference's link tables hold 6)");
        if (nl[i].size() != el[i].size() || nl[i].size() < 3)
            return fail(h, RBC_ERR_TOPOLOGY, "mesh is not a closed manifold at vertex " + std::to_string(i));
    }
    if (links != 2LL * (V + E - 2))   // init2.cu:369-370
        return fail(h, RBC_ERR_TOPOLOGY, "link count check failed (closed genus-0 mesh expected)");
    // Solve order of the membrane kernel: breadth first from a vertex of least
    // valence, each vertex's unvisited neighbours in the order of their
    // valence, so the positions run ring by ring around the surface; each
    // neighbour list is then sorted by position.  Consecutive positions (the
    // lanes of a warp) then gather neighbours at nearby positions in every slot,
    // which spreads their shared-memory loads over the banks.
    vord.clear();
    {
        std::vector<int> pos(V, -1);
        for (int root = 0; root < V; root++) {
            if (pos[root] >= 0) continue;
            int best = root;
            for (int i = root; i < V; i++) if (pos[i] < 0 && nl[i].size() < nl[best].size()) best = i;
            size_t head = vord.size();
            pos[best] = (int)vord.size(); vord.push_back(best);
            while (head < vord.size()) {
                const int u = vord[head++];
                std::vector<int> nx;
                for (int x : nl[u]) if (pos[x] < 0) nx.push_back(x);
                std::stable_sort(nx.begin(), nx.end(), [&](int a, int b) { return nl[a].size() < nl[b].size(); });
                for (int x : nx) { pos[x] = (int)vord.size(); vord.push_back(x); }
            }
        }
        for (int i = 0; i < V; i++)
            std::sort(nl[i].begin(), nl[i].end(), [&](int a, int b) { return pos[a] < pos[b]; });
        nbrp6.assign((size_t)6 * V, (int16_t)-1);
        for (int p = 0; p < V; p++)
            for (size_t s = 0; s < nl[vord[p]].size(); s++) nbrp6[s * V + p] = (int16_t)pos[nl[vord[p]][s]];
    }
    off.assign(V + 1, 0);
    packed.clear();
    nbr6.assign((size_t)6 * V, (int16_t)-1);
    for (int i = 0; i < V; i++) {
        off[i] = (int)packed.size();
        for (size_t s = 0; s < nl[i].size(); s++) nbr6[s * V + i] = (int16_t)nl[i][s];
        for (int e : el[i]) {
            int en = (tri[3 * e] == i) ? 0 : (tri[3 * e + 1] == i ? 1 : 2);
            const int o1 = tri[3 * e + (en + 1) % 3], o2 = tri[3 * e + (en + 2) % 3];
            int sa = -1, sb = -1;
            for (size_t s = 0; s < nl[i].size(); s++) {
                if (nl[i][s] == o1) sa = (int)s;
                if (nl[i][s] == o2) sb = (int)s;
            }
            if (sa < 0 || sb < 0) return fail(h, RBC_ERR_TOPOLOGY, "inconsistent incidence");
            packed.push_back((int)((unsigned)e | ((unsigned)en << 24) | ((unsigned)sa << 26) | ((unsigned)sb << 29)));
        }
    }
    off[V] = (int)packed.size();
    return RBC_OK;
}

// The reference metric of set_contravariant (init2.cu:206-255) on the AoS
// reference shape, kept in covariant form G [ne] with 1 / det G (the kernel forms n = G^-1)
void reference_metric(const CellGroup &g, const int *tri, const double *xr, std::vector<double4> &gref)
{
    const long long ne = g.ne;
    gref.assign(ne, make_double4(0, 0, 0, 0));
    for (int c = 0; c < g.ncell; c++)
        for (int e = 0; e < g.E; e++) {
            const long long a = (long long)c * g.V + tri[3 * e], b = (long long)c * g.V + tri[3 * e + 1],
                            cc = (long long)c * g.V + tri[3 * e + 2];
            double v1[3], v2[3];
            for (int j = 0; j < 3; j++) { v1[j] = xr[3 * b + j] - xr[3 * a + j]; v2[j] = xr[3 * cc + j] - xr[3 * a + j]; }
            const double lv1 = v1[0] * v1[0] + v1[1] * v1[1] + v1[2] * v1[2];
            const double lv2 = v2[0] * v2[0] + v2[1] * v2[1] + v2[2] * v2[2];
            const double inv12 = v1[0] * v2[0] + v1[1] * v2[1] + v1[2] * v2[2];
            const long long id = (long long)c * g.E + e;
            gref[id] = make_double4(lv1, inv12, lv2, 1.0 / (lv1 * lv2 - inv12 * inv12));
        }
}

// volume_init (volume_correction.cu:427-450): V0 and the wrapped centroid
void initial_volume(const rbc_handle *h, const CellGroup &g, const int *tri, const double *xr, std::vector<double> &vol0,
                    std::vector<double> &gx)
{
    const int N = g.ncell, V = g.V;
    vol0.assign(N, 0.0);
    gx.assign(3 * N, 0.0);
    for (int c = 0; c < N; c++) {
        double vs = 0.0;
        for (int e = 0; e < g.E; e++) {
            const double *pa = xr + 3 * ((long long)c * V + tri[3 * e]);
            const double *pb = xr + 3 * ((long long)c * V + tri[3 * e + 1]);
            const double *pc = xr + 3 * ((long long)c * V + tri[3 * e + 2]);
            const double v1[3] = {pb[0] - pa[0], pb[1] - pa[1], pb[2] - pa[2]};
            const double v2[3] = {pc[0] - pa[0], pc[1] - pa[1], pc[2] - pa[2]};
            const double cr[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2], v1[0] * v2[1] - v1[1] * v2[0]};
            const double nn = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
            const double dS = nn / 2.0;
            const double r[3] = {(pa[0] + pb[0] + pc[0]) / 3.0, (pa[1] + pb[1] + pc[1]) / 3.0, (pa[2] + pb[2] + pc[2]) / 3.0};
            vs += 1.0 / 3.0 * (r[0] * cr[0] / nn + r[1] * cr[1] / nn + r[2] * cr[2] / nn) * dS;
        }
        vol0[c] = vs;
        double s[3] = {0, 0, 0};
        for (int j = 0; j < V; j++)
            for (int k = 0; k < 3; k++) s[k] += xr[3 * ((long long)c * V + j) + k];
        for (int k = 0; k < 3; k++) s[k] /= (double)V;
        if (s[2] < h->p.zmin) s[2] += h->p.LZ; else if (s[2] > h->p.zmax) s[2] -= h->p.LZ;
        if (h->p.flow == RBC_FLOW_SHEAR) { if (s[0] < h->p.xmin) s[0] += h->p.LX; else if (s[0] > h->p.xmax) s[0] -= h->p.LX; }
        gx[c] = s[0]; gx[N + c] = s[1]; gx[2 * N + c] = s[2];
    }
}

// Surface patches for the spread kernel: recursive coordinate bisection of the
// first cell's initial vertex positions (split along the widest axis at the
// median until a patch has at most 512 vertices).  The same vertex sets serve
// every cell, since all cells share the mesh and a compact patch of the surface
// stays compact as the membrane moves.  Also a lane stride per patch, near
// 0.618 of its size and coprime with it, that scatters neighbours across lanes.
void surface_patches(int V, const double *xr, std::vector<int> &off, std::vector<int> &vtx, std::vector<int> &stride)
{
    vtx.resize(V);
    for (int i = 0; i < V; i++) vtx[i] = i;
    off.assign(1, 0);
    std::vector<std::pair<int, int>> stack{{0, V}};
    std::vector<std::pair<int, int>> leaves;
    while (!stack.empty()) {
        auto [b, e] = stack.back();
        stack.pop_back();
        if (e - b <= MAX_PATCH_VERTICES) { leaves.push_back({b, e}); continue; }
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int k = b; k < e; k++)
            for (int d = 0; d < 3; d++) { lo[d] = std::min(lo[d], xr[3 * vtx[k] + d]); hi[d] = std::max(hi[d], xr[3 * vtx[k] + d]); }
        int ax = 0;
        for (int d = 1; d < 3; d++) if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
        const int mid = b + (e - b) / 2;
        std::nth_element(vtx.begin() + b, vtx.begin() + mid, vtx.begin() + e,
                         [&](int i, int j) { return xr[3 * i + ax] < xr[3 * j + ax]; });
        stack.push_back({mid, e});
        stack.push_back({b, mid});
    }
    std::sort(leaves.begin(), leaves.end());
    stride.clear();
    for (auto [b, e] : leaves) {
        off.push_back(e);
        const int n = e - b;
        int s = std::max(1, (int)(0.6180339887 * n)) | 1;
        while (std::gcd(s, n) != 1) s += 2;
        stride.push_back(s);
    }
}

// Edge-neighbour visits of fourpoint_bend (stress.cu:448-578, cel->ec from
// init1.cu:755-795): for element e1, its edge neighbours in increasing
// element order; per neighbour e2 across e1's edge (k2 -> k3 in e1's
// winding), k1 = e1's third vertex and k4 = e2's vertex off the edge.
void bend_visits(int V, int E, const int *tri, std::vector<int4> &visit)
{
    std::vector<std::vector<int>> el(V);
    for (int e = 0; e < E; e++) for (int a = 0; a < 3; a++) el[tri[3 * e + a]].push_back(e);
    visit.assign((size_t)3 * E, make_int4(-1, -1, -1, -1));
    for (int e1 = 0; e1 < E; e1++) {
        std::vector<int4> found;   // (e2, k1, k2, k3) ... packed below
        std::vector<std::pair<int, int4>> nb;
        for (int a = 0; a < 3; a++) {
            const int ia = tri[3 * e1 + a], ib = tri[3 * e1 + (a + 1) % 3], ic = tri[3 * e1 + (a + 2) % 3];
            for (int e2 : el[ia]) {
                if (e2 == e1) continue;
                int hb = -1, ha = -1;
                for (int b = 0; b < 3; b++) { if (tri[3 * e2 + b] == ib) hb = b; if (tri[3 * e2 + b] == ia) ha = b; }
                if (ha < 0 || hb < 0) continue;
                nb.push_back({e2, make_int4(ic, ia, ib, tri[3 * e2 + (3 - ha - hb)])});
                break;
            }
        }
        std::sort(nb.begin(), nb.end(), [](const std::pair<int, int4> &x, const std::pair<int, int4> &y) { return x.first < y.first; });
        for (size_t k = 0; k < nb.size() && k < 3; k++) visit[(size_t)3 * e1 + k] = nb[k].second;
    }
}

// init1.cu:797-848 (init3.cu:313-364 for white cells) without the override
// of 849-850: cos and sin of every visit's dihedral angle on the initial
// shape xr (AoS [3 ncell V]), the sign of sin from the centroid test, 1 - cos^2
// clamped at 0; positions as minimum images about k1 like the bending kernel.
void spontaneous_angles(const rbc_params &p, const CellGroup &c, const double *xr, const std::vector<int4> &visit,
                        std::vector<double2> &cs0)
{
    auto mi = [](double d, double L) { return d > L * 0.5 ? d - L : (d < -L * 0.5 ? d + L : d); };
    cs0.assign((size_t)c.ncell * c.E * 3, make_double2(1.0, 0.0));
    for (int cell = 0; cell < c.ncell; cell++) {
        const double *x = xr + (size_t)3 * cell * c.V;
        for (size_t k = 0; k < (size_t)3 * c.E; k++) {
            const int4 q = visit[k];
            if (q.x < 0) continue;
            const int id[4] = {q.x, q.y, q.z, q.w};
            double a[4][3];
            for (int v = 0; v < 4; v++) {
                a[v][0] = x[3 * q.x] + mi(x[3 * id[v]] - x[3 * q.x], p.LX);
                a[v][1] = x[3 * id[v] + 1];
                a[v][2] = x[3 * q.x + 2] + mi(x[3 * id[v] + 2] - x[3 * q.x + 2], p.LZ);
            }
            double r21[3], r31[3], r34[3], r24[3], xi[3], ze[3];
            for (int d = 0; d < 3; d++) {
                r21[d] = a[1][d] - a[0][d]; r31[d] = a[2][d] - a[0][d];
                r34[d] = a[2][d] - a[3][d]; r24[d] = a[1][d] - a[3][d];
            }
            for (int d = 0; d < 3; d++) {
                const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
                xi[d] = r21[d1] * r31[d2] - r21[d2] * r31[d1];
                ze[d] = r34[d1] * r24[d2] - r34[d2] * r24[d1];
            }
            const double cost = (xi[0] * ze[0] + xi[1] * ze[1] + xi[2] * ze[2])
                              / std::sqrt(xi[0] * xi[0] + xi[1] * xi[1] + xi[2] * xi[2])
                              / std::sqrt(ze[0] * ze[0] + ze[1] * ze[1] + ze[2] * ze[2]);
            const double cost2 = std::max(1.0 - cost * cost, 0.0);
            double t = 0.0;   // (xi - ze) . (t1 - t2), t1 - t2 = (x1 - x4) / 3
            for (int d = 0; d < 3; d++) t += (xi[d] - ze[d]) * (a[0][d] - a[3][d]) / 3.0;
            cs0[(size_t)cell * c.E * 3 + k] = make_double2(cost, t >= 0.0 ? std::sqrt(cost2) : -std::sqrt(cost2));
        }
    }
}

int check_params(const rbc_params *p)
{
    if (!p) return fail(nullptr, RBC_ERR_ARG, "params is NULL");
    if (p->nx < 3 || p->ny < 3 || p->nz < 9)
        return fail(nullptr, RBC_ERR_ARG, "lattice too small (nx, ny >= 3, nz >= 9 including the 4 BUFF planes)");
    if ((long long)p->nx * p->ny > (1LL << 30) || (long long)p->nx * p->ny * p->nz > (1LL << 40))
        return fail(nullptr, RBC_ERR_ARG, "lattice too large");
    if (!(p->dx > 0) || !(p->dt > 0) || !(p->tau > 0.5) || !(p->Cr > 0))
        return fail(nullptr, RBC_ERR_ARG, "dx, dt, Cr must be > 0 and tau > 1/2");
    if (!(p->LX > 0) || !(p->LZ > 0)) return fail(nullptr, RBC_ERR_ARG, "LX and LZ must be > 0");
    if (p->M < 1) return fail(nullptr, RBC_ERR_ARG, "M must be >= 1");
    if (p->rk_order != 1 && p->rk_order != 2 && p->rk_order != 4)
        return fail(nullptr, RBC_ERR_ARG, "rk_order must be 1, 2 or 4 (RUNGE_KUTTA)");
    // the reference's RUNGE_KUTTA 2 and 1 branches interpolate in lattice units
    // without dx and take the midpoint at x + u M without dt (ibm.cu:522-562),
    // the RUNGE_KUTTA 4 form only for dx = dt = 1
    if (p->rk_order != 4 && (p->dx != 1.0 || p->dt != 1.0))
        return fail(nullptr, RBC_ERR_UNSUPPORTED, "RUNGE_KUTTA 1 and 2 need dx = dt = 1");
    if (!std::isfinite(p->br)) return fail(nullptr, RBC_ERR_ARG, "BR must be finite");
    if (p->bend_spont != 0 && p->bend_spont != 1) return fail(nullptr, RBC_ERR_ARG, "bend_spont must be 0 or 1");
    if (p->vof_k < 0) return fail(nullptr, RBC_ERR_ARG, "vof_k must be >= 0");
    if (!(p->lambda1 > 0.0) || !std::isfinite(p->lambda1)) return fail(nullptr, RBC_ERR_ARG, "lambda1 must be > 0");
    if (p->vof_k > 0 && (!(p->vof_residual > 0.0) || p->vof_itrmax < 1))
        return fail(nullptr, RBC_ERR_ARG, "vof_residual must be > 0 and vof_itrmax >= 1");
    if (p->vof_k > 0 && p->M != 1) return fail(nullptr, RBC_ERR_UNSUPPORTED, "VOF with M = 1 only");
    if (p->storage != RBC_STORE_F32 && p->storage != RBC_STORE_F16) return fail(nullptr, RBC_ERR_ARG, "unknown storage");
    if (p->law != RBC_LAW_SKALAK && p->law != RBC_LAW_NEOHOOKEAN) return fail(nullptr, RBC_ERR_ARG, "unknown law");
    if (p->solver_iters < 0 || p->solver_iters > 200) return fail(nullptr, RBC_ERR_ARG, "solver_iters out of range");
    if (p->flow != RBC_FLOW_CHANNEL && p->flow != RBC_FLOW_SHEAR) return fail(nullptr, RBC_ERR_ARG, "unknown flow mode");
    if (!(p->tube_r >= 0.0) || !std::isfinite(p->tube_r)) return fail(nullptr, RBC_ERR_ARG, "tube_r must be >= 0");
    if (p->tube_r > 0.0 && p->flow != RBC_FLOW_CHANNEL) return fail(nullptr, RBC_ERR_ARG, "tube_r applies to the channel mode");
    if (p->flow == RBC_FLOW_SHEAR) {
        if (p->walls != RBC_WALLS_BOTH && p->walls != RBC_WALLS_TOP) return fail(nullptr, RBC_ERR_ARG, "unknown wall motion");
        if (!std::isfinite(p->sr)) return fail(nullptr, RBC_ERR_ARG, "shear rate must be finite");
        if (p->P != 0.0) return fail(nullptr, RBC_ERR_ARG, "the shear mode has no body-force drive (P must be 0, lbm.cu:706-980)");
        if (p->nx < 8 || p->ny < 6) return fail(nullptr, RBC_ERR_ARG, "shear mode: nx >= 8 (4 periodic columns + 4 BUFF), ny >= 6");
    }
    return RBC_OK;
}

// Shear mode (CapsuleSHEARFLOW, init1.cu:133-187): the bc map must be COMP inside
// the box, BUFF in the two x and z layers of each end between the walls and WALL
// in the two rows beyond each y wall.  The internal columns are the periodic x
// range (BUFF columns stripped); fluid rows are y = 2 .. ny - 3, the walls are
// half a node beyond them and move along z.
int build_mask_shear(const rbc_params *p, const int *bc, std::vector<uint32_t> &mask)
{
    const int nx = p->nx, ny = p->ny, nz = p->nz, nxi = nx - 4;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                const bool rowf = y >= 2 && y < ny - 2, inx = x >= 2 && x < nx - 2, inz = z >= 2 && z < nz - 2;
                const int want = !rowf ? RBC_WALL : (inx && inz) ? RBC_COMP : RBC_BUFF;
                if (bc[((long long)z * ny + y) * nx + x] != want)
                    return fail(nullptr, RBC_ERR_ARG, "bc: not the shear-flow box (COMP inside, BUFF x/z layers, WALL rows beyond y)");
            }
    mask.assign((size_t)nxi * ny, 0u);
    for (int y = 2; y < ny - 2; y++)
        for (int x = 0; x < nxi; x++) {
            uint32_t m = MASK_FLUID;
            for (int q = 1; q < Q; q++) {
                const int sy = y - ey(q);
                if (sy < 2 || sy >= ny - 2) m |= (1u << q);
            }
            if (x == 0) m |= MASK_XLO;
            if (x == nxi - 1) m |= MASK_XHI;
            if (y == ny - 3) m |= MASK_TOPW;
            else if (y == 2) m |= MASK_BOTW;
            mask[(size_t)y * nxi + x] = m;
        }
    return RBC_OK;
}

// SetDistanceFromWall_GPU (lbm_cylinder.cu:116-183): every wall link of a fluid
// column (pull direction p, wall at i - e_p) that crosses the circle
// x^2 + y^2 = R^2 of the cross-section, with the fraction t in (0, 1) of the
// link i -> i - e_p at the crossing.  Links are z-invariant: one list per plane.
void tube_links(const rbc_params *p, const std::vector<uint32_t> &mask, std::vector<int> &links, std::vector<float> &frac)
{
    const int nx = p->nx, ny = p->ny;
    const long long plane = (long long)nx * ny;
    const double R = p->tube_r, dx = p->dx;
    links.clear();
    frac.clear();
    for (long long xy = 0; xy < plane; xy++) {
        const uint32_t m = mask[xy];
        if (!(m & MASK_FLUID)) continue;
        const int ix = (int)(xy % nx), iy = (int)(xy / nx);
        const double xi = (ix - (nx - 1) / 2.0) * dx, yi = (iy - (ny - 1) / 2.0) * dx;   // init1.cu:223-224
        for (int q = 1; q < Q; q++) {
            if (!((m >> q) & 1u) || ((m >> opp(q)) & 1u)) continue;   // a wall on both sides: half-way
            const double ddx = -ex(q) * dx, ddy = -ey(q) * dx, a = ddx * ddx + ddy * ddy;
            if (a == 0.0) continue;
            const double b = xi * ddx + yi * ddy, det = b * b - a * (xi * xi + yi * yi - R * R);
            if (det < 0.0) continue;
            const double t1 = (-b + std::sqrt(det)) / a, t2 = (-b - std::sqrt(det)) / a;
            double t;
            if (t1 > 0.0 && t1 < 1.0) t = t1; else if (t2 > 0.0 && t2 < 1.0) t = t2; else continue;
            links.push_back((int)(xy * 32 + q));
            frac.push_back((float)t);
        }
    }
}

// Wall mask of one z plane from the reference bc map; checks z invariance.
int build_mask(const rbc_params *p, const int *bc, std::vector<uint32_t> &mask)
{
    if (p->flow == RBC_FLOW_SHEAR) return build_mask_shear(p, bc, mask);
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const long long plane = (long long)nx * ny;
    mask.assign(plane, 0u);
    std::vector<char> fluid(plane, 0);
    for (long long xy = 0; xy < plane; xy++) {
        const int t = bc[2 * plane + xy];
        if (t != RBC_COMP && t != RBC_WALL)
            return fail(nullptr, RBC_ERR_ARG, "bc: first COMP plane (z = 2) holds a value other than COMP/WALL");
        fluid[xy] = (t == RBC_COMP);
        for (int z = 2; z < nz - 2; z++)
            if (bc[z * plane + xy] != t)
                return fail(nullptr, RBC_ERR_UNSUPPORTED, "bc: wall pattern must be the same in every COMP plane");
        const int want = fluid[xy] ? RBC_BUFF : RBC_WALL;
        for (int z : {0, 1, nz - 2, nz - 1})
            if (bc[z * plane + xy] != want)
                return fail(nullptr, RBC_ERR_ARG, "bc: BUFF planes must be BUFF over fluid columns and WALL elsewhere");
        const int x = (int)(xy % nx), y = (int)(xy / nx);
        if (fluid[xy] && (x == 0 || y == 0 || x == nx - 1 || y == ny - 1))
            return fail(nullptr, RBC_ERR_ARG, "bc: fluid node on the lattice edge (walls must enclose the channel)");
    }
    for (long long xy = 0; xy < plane; xy++) {
        if (!fluid[xy]) continue;
        const int x = (int)(xy % nx), y = (int)(xy / nx);
        uint32_t m = MASK_FLUID;
        for (int q = 1; q < Q; q++) {
            const int sx = x - ex(q), sy = y - ey(q);
            if (!fluid[sx + (long long)nx * sy]) m |= (1u << q);
        }
        mask[xy] = m;
    }
    return RBC_OK;
}

void free_group(CellGroup &c)
{
    void *cp[] = {c.X, c.Xd, c.gref, c.erec, c.U, c.Fv, c.tri, c.v2e_off, c.v2e, c.nbr, c.nbrp, c.vord, c.visit, c.cs0, c.patch_off,
                  c.patch_vtx, c.patch_stride, c.vol0, c.gx, c.vol_out, c.area_out, c.cen_out, c.qi_acc, c.tp_acc,
                  c.vf, c.bend_rec};
    for (void *q : cp) if (q) cudaFree(q);
    c = CellGroup{};
}

void free_all(rbc_handle *h)
{
    if (!h) return;
    for (auto &form : h->graph)
        for (cudaGraphExec_t g : form) if (g) cudaGraphExecDestroy(g);
    if (h->fork) cudaEventDestroy(h->fork);
    if (h->join) cudaEventDestroy(h->join);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->metrics_host) cudaFreeHost(h->metrics_host);
    if (h->wave_done) cudaEventDestroy(h->wave_done);
    if (h->spread_done) cudaEventDestroy(h->spread_done);
    if (h->lbm_done) cudaEventDestroy(h->lbm_done);
    if (h->reset_done) cudaEventDestroy(h->reset_done);
    if (h->side2) cudaStreamDestroy(h->side2);
    for (int k = 0; k < 4; k++) {
        if (h->imp_copied[k]) cudaEventDestroy(h->imp_copied[k]);
        if (h->imp_freed[k]) cudaEventDestroy(h->imp_freed[k]);
    }
    void *ptrs[] = {h->g[0], h->g[1], h->uvr, h->Fint, h->Fbits, h->mask2d, h->tube_links, h->tube_frac,
                    h->d_int, h->d_drive, h->staging, h->vof_s1, h->vof_s2, h->vof_G, h->vof_b, h->vof_partial,
                    h->imp_ring};
    for (void *q : ptrs) if (q) cudaFree(q);
    for (CellGroup &c : h->cg) free_group(c);
    vof_mg_free(h->vof_mg);
    adjoint_free(h->adj);
    h->adj = nullptr;
    if (h->stream) cudaStreamDestroy(h->stream);
}

// ---- stage launches -------------------------------------------------------

// the membrane pass (stress.cu:580-660) of cells [c0, c1) of population g: the
// kernel indexes cells from the pointers it is given, so a range is an offset
int launch_membrane_range(rbc_handle *h, CellGroup &g, int c0, int c1, cudaStream_t st)
{
    const size_t rec_bytes = (h->p.membrane_fp64 ? sizeof(double4) : sizeof(float4)) * 3;
    MembraneArgs a{};
    a.Xd = g.Xd + (size_t)c0 * g.V; a.nv = g.nv; a.ne = g.ne; a.gref = g.gref + (size_t)c0 * g.E;
    a.erec = (char *)g.erec + (size_t)c0 * g.E * rec_bytes;
    a.tri = g.tri; a.v2e_off = g.v2e_off; a.v2e = g.v2e; a.nbr = g.nbr; a.nbrp = g.nbrp; a.vord = g.vord; a.Fv = g.Fv + (size_t)c0 * g.V;
    a.V = g.V; a.E = g.E; a.ncell = c1 - c0;
    a.C = h->p.C; a.rgs = g.rgs; a.law = h->p.law; a.LX = h->p.LX; a.LZ = h->p.LZ;
    a.niter = h->p.solver_iters > 0 ? h->p.solver_iters : DEFAULT_SOLVER_ITERS;
    a.flags = h->d_flags();
    a.priority = h->prio_high;
    launch_membrane(a, h->p.membrane_fp64 != 0, st);
    h->launches++;
    CK_LAUNCH();
    return RBC_OK;
}

// the spread (ibm.cu:299-369) of cells [c0, c1) of population g
int launch_spread_range(rbc_handle *h, CellGroup &g, int c0, int c1, cudaStream_t st)
{
    SpreadArgs a{};
    a.X = g.X + (size_t)c0 * g.V; a.nv = g.nv; a.V = g.V; a.ncell = c1 - c0; a.Fv = g.Fv + (size_t)c0 * g.V;
    a.patch_off = g.patch_off; a.patch_vtx = g.patch_vtx; a.patch_stride = g.patch_stride;
    a.npatch = g.npatch;
    a.F = h->force(); a.mask2d = h->mask2d; a.flags = h->d_flags();
    launch_spread(h->geo, a, st);
    h->launches++;
    CK_LAUNCH();
    return RBC_OK;
}

// Cells in the full waves of the membrane kernel (one CTA per cell and per
// multiprocessor) when splitting off the last partial wave pays: one
// population, no bending and no output averages (both read all the forces
// of the step), more cells than multiprocessors.  0 = no split.
int membrane_wave_split(const rbc_handle *h)
{
    const CellGroup &g = h->cg[0];
    if (h->ngroups != 1 || g.br != 0.0 || h->fileoutput > 0 || h->sms <= 0 || g.ncell <= h->sms) return 0;
    const int full = (g.ncell / h->sms) * h->sms;
    return full < g.ncell ? full : 0;
}

// the membrane kernel's arguments for population g
MembraneArgs membrane_args(rbc_handle *h, CellGroup &g)
{
    MembraneArgs a{};
    a.Xd = g.Xd; a.nv = g.nv; a.ne = g.ne; a.gref = g.gref; a.erec = g.erec;
    a.tri = g.tri; a.v2e_off = g.v2e_off; a.v2e = g.v2e; a.nbr = g.nbr; a.nbrp = g.nbrp; a.vord = g.vord; a.Fv = g.Fv;
    a.V = g.V; a.E = g.E; a.ncell = g.ncell;
    a.C = h->p.C; a.rgs = g.rgs; a.law = h->p.law; a.LX = h->p.LX; a.LZ = h->p.LZ;
    a.niter = h->p.solver_iters > 0 ? h->p.solver_iters : DEFAULT_SOLVER_ITERS;
    a.flags = h->d_flags();
    a.priority = h->prio_high;
    return a;
}

// stress() (stress.cu:580-660) for every cell population
int launch_stress(rbc_handle *h)
{
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (g.ncell == 0) continue;
        const MembraneArgs a = membrane_args(h, g);
        launch_membrane(a, h->p.membrane_fp64 != 0, h->stream);
        h->launches++;
        CK_LAUNCH();
        if (h->fileoutput > 0) {   // calc_tension's tp and substitute_load's qi (stress.cu:101-118, 280-300)
            AccumArgs c{};
            c.Xd = g.Xd; c.Fv = g.Fv; c.gref = g.gref; c.tri = g.tri; c.v2e_off = g.v2e_off; c.v2e = g.v2e;
            c.iter = h->d_iter(); c.qi = g.qi_acc; c.tp = g.tp_acc; c.nv = g.nv; c.ne = g.ne;
            c.V = g.V; c.E = g.E; c.ncell = g.ncell; c.fileoutput = h->fileoutput; c.M = h->p.M;
            c.C = h->p.C; c.LX = h->p.LX; c.LZ = h->p.LZ;
            launch_output_accum(c, h->stream);
            h->launches += 2;
            CK_LAUNCH();
        }
    }
    return RBC_OK;
}

// The force reset after the collide-stream kernel read the field: zero the
// forces of the nodes whose occupancy bit is set, then the bits, so the next
// spread starts from zero.  Right after the read the field's set lines are
// still in L2 (a reset before the next step's spread, with those lines
// evicted by the rest of the step, took 14 us on the dense suspension).
int launch_force_reset_stage(rbc_handle *h, cudaStream_t st)
{
    if (!h->has_cells()) return RBC_OK;   // nothing spreads: the field stays zero
    launch_force_reset(h->geo, h->force(), st);
    h->launches++;
    CK_LAUNCH();
    return RBC_OK;
}

// the spread kernel's arguments for population g
SpreadArgs spread_args(rbc_handle *h, CellGroup &g)
{
    SpreadArgs a{};
    a.X = g.X; a.nv = g.nv; a.V = g.V; a.ncell = g.ncell; a.Fv = g.Fv;
    a.patch_off = g.patch_off; a.patch_vtx = g.patch_vtx; a.patch_stride = g.patch_stride;
    a.npatch = g.npatch;
    a.F = h->force(); a.mask2d = h->mask2d; a.flags = h->d_flags();
    return a;
}

// ibm_st1's spreading (ibm.cu:299-369) of every population into the same force field
int launch_spread_stage(rbc_handle *h)
{
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (g.ncell == 0) continue;
        const SpreadArgs a = spread_args(h, g);
        launch_spread(h->geo, a, h->stream);
        h->launches++;
        CK_LAUNCH();
    }
    return RBC_OK;
}

// fourpoint_bend (stress.cu:621-623, 650-652) on cel->x, added to the membrane forces
int launch_bend_stage(rbc_handle *h)
{
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (g.ncell == 0 || g.br == 0.0) continue;
        BendArgs a{};
        a.X = g.X; a.nv = g.nv; a.V = g.V; a.E = g.E; a.v2e_off = g.v2e_off; a.v2e = g.v2e; a.visit = g.visit;
        a.cs0 = g.cs0; a.ncell = g.ncell; a.rec = g.bend_rec;
        a.LX = h->p.LX; a.LZ = h->p.LZ; a.coef = 2.0 / std::sqrt(3.0) * g.br; a.Fv = g.Fv;
        launch_bend(a, h->stream);
        h->launches += 2;   // the visit and gather passes
        CK_LAUNCH();
    }
    return RBC_OK;
}

// the collide-stream kernel's arguments from population buffer cur
LbmArgs lbm_args(rbc_handle *h, int cur, int acc = LBM_ACC_WRITE)
{
    LbmArgs a{};
    a.acc = acc; a.Mf = (float)h->p.M;
    a.gin = h->g[cur]; a.gout = h->g[1 - cur];
    a.uvr = h->uvr;
    a.F = h->force(); a.mask2d = h->mask2d; a.drive = h->d_drive; a.iter = h->d_iter();
    a.wall = h->p.flow == RBC_FLOW_SHEAR ? h->d_drive + 1 : nullptr;
    a.omega = (float)(1.0 / h->p.tau); a.Cr = (float)h->p.Cr; a.Bc = (float)h->p.B;
    a.scale = h->scale; a.inv_scale = h->inv_scale;
    a.planes = h->lbm_planes;
    // the red cells' volume fraction sets omega (lbm.cu:1131; ltc->vf2 of the white cells does not)
    a.vf = (h->p.lambda1 != 1.0 && h->cg[0].vf) ? h->cg[0].vf : nullptr;
    a.lm1 = (float)(h->p.lambda1 - 1.0);
    a.df3 = (float)(h->p.tau - 0.5);   // 3 Df, tau = 3 Df + 1/2
    return a;
}

// the collide-stream launch (+ the tube's bounce-back) and, with reset, the
// force reset after it; acc: the velocity sums of a sub-cycled step (LBM_ACC_*)
int launch_lbm_stage(rbc_handle *h, bool reset = true, int acc = LBM_ACC_WRITE)
{
    LbmArgs a = lbm_args(h, h->cur, acc);
    launch_lbm(h->geo, h->p.storage, a, h->stream);
    h->launches++;
    CK_LAUNCH();
    if (h->ntube > 0) {   // circular tube: lbm_BounceBack_GPU (lbm_cylinder.cu:190-231) after the stream
        launch_tube_bounce(h->geo, h->p.storage, h->g[1 - h->cur], h->tube_links, h->tube_frac, h->ntube,
                           h->inv_scale, h->scale, h->stream);
        h->launches++;
        CK_LAUNCH();
    }
    h->cur ^= 1;
    return reset ? launch_force_reset_stage(h, h->stream) : RBC_OK;
}

// the advection kernel's arguments for population g
AdvectArgs advect_args(rbc_handle *h, CellGroup &g)
{
    AdvectArgs a{};
    a.X = g.X; a.Xd = g.Xd; a.U = g.U; a.uvr = h->uvr; a.nv = g.nv;
    a.V = g.V; a.ncell = g.ncell; a.patch_off = g.patch_off; a.patch_vtx = g.patch_vtx; a.npatch = g.npatch;
    a.dtM = h->p.dt * h->p.M; a.rk = h->p.rk_order; a.flags = h->d_flags();
    return a;
}

// ibm_st2 (ibm.cu:642-694) for every population
int launch_advect_stage(rbc_handle *h)
{
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (g.ncell == 0) continue;
        const AdvectArgs a = advect_args(h, g);
        launch_advect(h->geo, a, h->stream);
        h->launches++;
        CK_LAUNCH();
    }
    return RBC_OK;
}

// thinc_wlic (thincwlic.cu:316-420) of every population's volume fraction
int launch_thinc_stage(rbc_handle *h)
{
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (!g.vf || g.ncell == 0) continue;
        launch_thinc_wlic(h->geo, g.vf, h->vof_s1, h->vof_s2, h->uvr, h->mask2d, h->p.dt * h->p.M, h->stream);
        h->launches += 3;
        CK_LAUNCH();
    }
    return RBC_OK;
}

// front_tracking (fronttrack.cu:628-944) of every population into its volume fraction
int launch_front_tracking_stage(rbc_handle *h)
{
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (!g.vf || g.ncell == 0) continue;
        FrontArgs a{};
        a.X = g.X; a.nv = g.nv; a.tri = g.tri; a.V = g.V; a.E = g.E; a.ncell = g.ncell; a.mask2d = h->mask2d;
        a.G = h->vof_G; a.b = h->vof_b; a.vf = g.vf; a.partial = h->vof_partial; a.mg = &h->vof_mg;
        a.tol = h->p.vof_residual; a.itrmax = h->p.vof_itrmax; a.iters = h->d_vofit() + k; a.flags = h->d_flags();
        CK(launch_front_tracking(h->geo, a, h->stream));
        h->launches += 3;
        CK_LAUNCH();
    }
    return RBC_OK;
}

// volume fraction storage of population g and the shared scratch, and vof_init
// (init1.cu:1094-1120): front tracking of the initial cells (synchronous)
int vof_init_group(rbc_handle *h, CellGroup &g)
{
    const size_t n = (size_t)h->geo.nint;
    if (h->geo.nint >= (1LL << 31)) return fail(h, RBC_ERR_UNSUPPORTED, "the volume fraction needs fewer than 2^31 nodes");
    if (!h->vof_s1) {
        CK(cudaMalloc(&h->vof_s1, 8 * n));
        CK(cudaMalloc(&h->vof_s2, 8 * n));
        CK(cudaMalloc(&h->vof_G, 8 * 3 * n));
        CK(cudaMalloc(&h->vof_b, 8 * n));
        CK(cudaMalloc(&h->vof_partial, 8 * 4 * (size_t)std::max(vof_cg_blocks(), 1)));
        std::vector<uint32_t> mask((size_t)h->geo.plane);
        CK(cudaMemcpy(mask.data(), h->mask2d, 4 * mask.size(), cudaMemcpyDeviceToHost));
        CK(vof_mg_build(h->geo, mask.data(), h->vof_mg));
    }
    if (!g.vf) {
        CK(cudaMalloc(&g.vf, 8 * n));
        CK(cudaMemset(g.vf, 0, 8 * n));   // flu_init's vf = 0 (init1.cu:396-411)
    }
    if (g.ncell == 0) return RBC_OK;
    FrontArgs a{};
    a.X = g.X; a.nv = g.nv; a.tri = g.tri; a.V = g.V; a.E = g.E; a.ncell = g.ncell; a.mask2d = h->mask2d;
    a.G = h->vof_G; a.b = h->vof_b; a.vf = g.vf; a.partial = h->vof_partial; a.mg = &h->vof_mg;
    a.tol = h->p.vof_residual; a.itrmax = h->p.vof_itrmax; a.iters = h->d_vofit() + (&g == &h->cg[1] ? 1 : 0);
    a.flags = h->d_flags();
    CK(launch_front_tracking(h->geo, a, h->stream));
    h->launches += 3;
    CK(cudaStreamSynchronize(h->stream));
    return RBC_OK;
}

VolumeArgs volume_args(rbc_handle *h, CellGroup &g, int correct)
{
    VolumeArgs a{};
    a.X = g.X; a.nv = g.nv; a.tri = g.tri; a.v2e_off = g.v2e_off; a.v2e = g.v2e;
    a.vol0 = g.vol0; a.gx = g.gx; a.vol_out = g.vol_out; a.area_out = g.area_out; a.cen_out = g.cen_out;
    a.V = g.V; a.E = g.E; a.ncell = g.ncell;
    a.flags = h->d_flags(); a.vc_max = h->d_vcmax(); a.vc_last = h->d_vclast();
    a.correct = correct;
    return a;
}

// volume_correction (volume_correction.cu:453-524, both populations) on stream st
int launch_volume_stage(rbc_handle *h, cudaStream_t st)
{
    if (!h->has_cells()) return RBC_OK;
    CK(cudaMemsetAsync(h->d_vclast(), 0, sizeof(int), st));
    for (int k = 0; k < h->ngroups; k++) {
        if (h->cg[k].ncell == 0) continue;
        launch_volume(h->geo, volume_args(h, h->cg[k], 1), st);
        h->launches++;
        CK_LAUNCH();
    }
    return RBC_OK;
}

enum StepForm { STEP_WHOLE = 0, STEP_BODY = 1, STEP_PIPELINED = 2, STEP_SUB_FIRST = 3, STEP_SUB_MID = 4,
                STEP_SUB_LAST = 5 };

// Sub-cycling (M > 1, main.cu:78-106): step iter runs the membrane pass and
// the spread when (iter - 1) % M == 0 and the advection, THINC/WLIC and the
// volume correction when iter % M == 0; the force field persists over the M
// collide-streams between them, and the velocity they store is summed, then
// averaged at the last (lbm.cu:1097-1126, 1435-1460).
StepForm sub_form(const rbc_handle *h, int iter)
{
    const int M = h->p.M, ph = (iter - 1) % M;
    return ph == 0 ? STEP_SUB_FIRST : ph == M - 1 ? STEP_SUB_LAST : STEP_SUB_MID;
}
int lbm_acc(StepForm f)
{
    return f == STEP_SUB_MID ? LBM_ACC_ADD : f == STEP_SUB_LAST ? LBM_ACC_AVERAGE : LBM_ACC_WRITE;
}

// one step (main.cu:73-110 with M = 1); the device increments iter.
// STEP_BODY leaves out the step's volume correction; STEP_PIPELINED also runs
// the previous step's correction on a second branch beside step_begin +
// membrane (the membrane pass reads fem->xd, which the correction does not
// touch; the correction writes cel->x, which the spread reads, so the
// branches join before the spread).
//
// With more cells than multiprocessors the membrane kernel (one cell per
// multiprocessor) runs in full waves and a last partial one that leaves most
// multiprocessors idle.  Then the full waves run as one launch and the last
// wave as a second, high-priority launch, while a third branch spreads the
// full waves' cells beside it: each cell's spread needs only its own forces,
// and the spread adds integer fixed-point values, so the order of the two
// spreads does not change the force field.
int enqueue_step(rbc_handle *h, StepForm form = STEP_WHOLE)
{
    int rc;
    const bool pipelined = form == STEP_PIPELINED;
    const bool sub = form >= STEP_SUB_FIRST;
    const bool first = !sub || form == STEP_SUB_FIRST, last = !sub || form == STEP_SUB_LAST;
    if (pipelined) {
        CK(cudaEventRecord(h->fork, h->stream));
        CK(cudaStreamWaitEvent(h->side, h->fork, 0));
        if ((rc = launch_volume_stage(h, h->side))) return rc;
        CK(cudaEventRecord(h->join, h->side));
    }
    launch_step_begin(step_begin_args(h), h->stream);
    h->launches++;
    CK_LAUNCH();
    const int split = first ? membrane_wave_split(h) : 0;
    if (!first) {
        // a middle or last sub-cycled step: the cycle's force is in the field
    } else if (split > 0) {
        CellGroup &g = h->cg[0];
        if ((rc = launch_membrane_range(h, g, 0, split, h->stream))) return rc;
        CK(cudaEventRecord(h->wave_done, h->stream));
        if ((rc = launch_membrane_range(h, g, split, g.ncell, h->stream))) return rc;
        CK(cudaStreamWaitEvent(h->side2, h->wave_done, 0));
        if (pipelined) CK(cudaStreamWaitEvent(h->side2, h->join, 0));   // the spread reads cel->x
        if ((rc = launch_spread_range(h, g, 0, split, h->side2))) return rc;
        CK(cudaEventRecord(h->spread_done, h->side2));
        if (pipelined) CK(cudaStreamWaitEvent(h->stream, h->join, 0));
        if ((rc = launch_spread_range(h, g, split, g.ncell, h->stream))) return rc;
        CK(cudaStreamWaitEvent(h->stream, h->spread_done, 0));
    } else {
        if ((rc = launch_stress(h))) return rc;
        if (pipelined) CK(cudaStreamWaitEvent(h->stream, h->join, 0));
        if ((rc = launch_bend_stage(h))) return rc;   // reads cel->x, after the correction
        if ((rc = launch_spread_stage(h))) return rc;
    }
    // the force reset runs beside the advection (which reads neither the
    // field nor its bits) and joins before the step ends
    if ((rc = launch_lbm_stage(h, false, lbm_acc(form)))) return rc;
    if (!last) return RBC_OK;
    CK(cudaEventRecord(h->lbm_done, h->stream));
    CK(cudaStreamWaitEvent(h->side2, h->lbm_done, 0));
    if ((rc = launch_force_reset_stage(h, h->side2))) return rc;
    CK(cudaEventRecord(h->reset_done, h->side2));
    if ((rc = launch_advect_stage(h))) return rc;
    if ((rc = launch_thinc_stage(h))) return rc;   // main.cu:94-95
    if ((form == STEP_WHOLE || form == STEP_SUB_LAST) && (rc = launch_volume_stage(h, h->stream))) return rc;
    CK(cudaStreamWaitEvent(h->stream, h->reset_done, 0));
    return RBC_OK;
}

// CUDA graph of one step starting from population buffer c (the step flips
// the buffers, so two graphs alternate)
// one step of the given form starting from population buffer c, captured
// from the handle's stream into *out (not instantiated)
int capture_step(rbc_handle *h, int c, StepForm form, cudaGraph_t *out)
{
    *out = nullptr;
    const long long launches0 = h->launches;
    const int cur0 = h->cur;
    h->cur = c;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(h, form);
    cudaError_t e = cudaStreamEndCapture(h->stream, out);
    h->graph_kernels[form] = (int)(h->launches - launches0);
    h->launches = launches0;
    h->cur = cur0;
    if (rc != RBC_OK) { if (*out) cudaGraphDestroy(*out); *out = nullptr; return rc; }
    if (e != cudaSuccess) { h->err = std::string("graph capture: ") + cudaGetErrorString(e); return RBC_ERR_CUDA; }
    return RBC_OK;
}

int build_graph(rbc_handle *h, int c, StepForm form)
{
    cudaGraph_t graph = nullptr;
    int rc = capture_step(h, c, form, &graph);
    if (rc != RBC_OK) return rc;
    cudaError_t e;
    cudaGraphExec_t &exec = h->graph[form][c];
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { exec = nullptr; h->err = std::string("graph instantiate: ") + cudaGetErrorString(e); return RBC_ERR_CUDA; }
    return RBC_OK;
}

int prepare_steps(rbc_handle *h)
{
    // a step that spreads starts from a zero field; a middle or last sub-cycled
    // step uses the field its cycle's first step spread
    const bool spreads = h->p.M == 1 || (h->iter % h->p.M) == 0;
    if (h->force_pending && spreads) {
        CK(cudaMemsetAsync(h->Fint, 0, 24 * h->geo.nint, h->stream));
        CK(cudaMemsetAsync(h->Fbits, 0, h->force_bit_bytes(), h->stream));
        h->force_pending = false;
    }
    // the device counter follows the host's prc->iter mirror
    CK(cudaMemcpyAsync(h->d_iter(), &h->iter, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    return RBC_OK;
}

}  // namespace

// ---- batches of independent simulations -----------------------------------

struct rbc_batch {
    std::vector<rbc_handle *> h;
    std::vector<int> base_cur;          // each handle's buffer parity when the graphs were built
    std::vector<cudaEvent_t> ready;     // one per handle: its pending work, before a batch step
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int parity = 0;                     // graph[parity] advances every handle by one step
    int chain = 1;                      // simulations per dependency chain in the batch graph
    std::string err;
    // Fused form: every stage of all simulations in one launch (FusedLaunch).
    // Used when the simulations share what selects the kernels' code (storage,
    // flow mode, membrane precision, vertices per cell) and have none of the
    // stages a fused step leaves out (white cells, bending, output averages,
    // the volume fraction, the circular tube); else each simulation's step is a
    // child graph of the batch graph.
    int use_fused = 1;                  // rbc_batch_set_form: 1 fused when possible, 0 child graphs
    bool fused = false;                 // the graphs are the fused form
    int lbm_threads = 256, lbm_planes = 0, mem_vpt = 0;   // fused launch shapes (0: as one simulation)
    void *fmem = nullptr;               // device: descriptors [2][n], block offsets [2][FSTAGES][n + 1]
    long long launches = 0;             // fused kernel launches
};

namespace {

#define CKB(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            b->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
            return RBC_ERR_CUDA;                                                       \
        }                                                                              \
    } while (0)

void batch_free_graphs(rbc_batch *b)
{
    for (cudaGraphExec_t &g : b->graph) { if (g) cudaGraphExecDestroy(g); g = nullptr; }
    if (b->fmem) { cudaFree(b->fmem); b->fmem = nullptr; }
    b->fused = false;
}

// stages of a fused step, in order
enum { FS_CLEAR, FS_MEMBRANE, FS_SPREAD, FS_LBM, FS_ADVECT, FS_VOLUME, FSTAGES };
constexpr int FUSED_KERNELS_PER_STEP = FSTAGES + 1;   // + step begin

// why the batch's simulations cannot run as one fused step ("" = they can)
std::string fused_obstacle(const rbc_batch *b)
{
    const rbc_handle *h0 = b->h[0];
    int V = 0;
    for (size_t i = 0; i < b->h.size(); i++) {
        const rbc_handle *h = b->h[i];
        const std::string who = "simulation " + std::to_string(i) + ": ";
        if (h->p.storage != h0->p.storage || h->p.flow != h0->p.flow || h->p.membrane_fp64 != h0->p.membrane_fp64)
            return who + "storage, flow mode and membrane precision differ";
        if (h->ngroups > 1) return who + "white cells";
        if (h->cg[0].br != 0.0) return who + "bending (BR != 0)";
        if (h->fileoutput > 0) return who + "output-interval averages";
        if (h->vof()) return who + "volume fraction";
        if (h->ntube > 0) return who + "circular tube";
        if (h->p.rk_order != 4) return who + "RUNGE_KUTTA != 4";
        if (h->cg[0].ncell > 0) {
            if (V && h->cg[0].V != V) return who + "another number of vertices per cell";
            V = h->cg[0].V;
        }
    }
    return "";
}

// The fused graphs: descriptors of every simulation for both buffer
// parities, block offsets of every stage, and one graph per parity of
// step begin, membrane, spread, collide-stream, force reset, advection and
// volume correction launches.
int batch_build_fused(rbc_batch *b)
{
    const int n = (int)b->h.size();
    rbc_handle *h0 = b->h[0];
    int V = 0;
    bool off32 = true;
    for (rbc_handle *h : b->h) {
        if (h->cg[0].ncell > 0) V = h->cg[0].V;
        off32 = off32 && (long long)Q * h->geo.nint < (1LL << 31);
    }
    const int vpt = b->mem_vpt > 0 ? b->mem_vpt : (V > 0 ? membrane_default_vpt(V) : 1);
    const int tpb = b->lbm_threads;
    std::vector<DomainArgs> dom(2 * (size_t)n);
    std::vector<int> boff(2 * (size_t)FSTAGES * (n + 1), 0);
    int nblocks[FSTAGES] = {};
    for (int k = 0; k < 2; k++) {
        int acc[FSTAGES] = {};
        for (int i = 0; i < n; i++) {
            rbc_handle *h = b->h[i];
            CellGroup &g = h->cg[0];
            DomainArgs &D = dom[(size_t)k * n + i];
            D.g = h->geo;
            D.sb = step_begin_args(h);
            D.sb.vc_last = h->d_vclast();   // the memset before a one-simulation volume stage
            D.F = h->force();
            D.mem = membrane_args(h, g);
            D.spread = spread_args(h, g);
            D.lbm = lbm_args(h, b->base_cur[i] ^ k);
            D.adv = advect_args(h, g);
            D.vol = volume_args(h, g, 1);
            int zpt = b->lbm_planes > 0 ? b->lbm_planes : (h->p.storage == RBC_STORE_F16 ? 4 : 2);
            zpt = std::min(zpt, h->geo.nzc);
            D.lbm_bx = (int)((h->geo.plane + tpb - 1) / tpb);
            D.lbm_gy = (h->geo.nzc + zpt - 1) / zpt;
            const long long words = (long long)h->geo.nzc * D.F.wpp;
            constexpr int words_per_block = FUSED_CLEAR_THREADS;   // a warp per 32 words
            const long long cnt[FSTAGES] = {(words + words_per_block - 1) / words_per_block, g.ncell,
                                            (long long)g.ncell * g.npatch, (long long)D.lbm_bx * D.lbm_gy,
                                            (long long)g.ncell * g.npatch, g.ncell};
            for (int st = 0; st < FSTAGES; st++) {
                boff[((size_t)k * FSTAGES + st) * (n + 1) + i] = acc[st];
                if ((long long)acc[st] + cnt[st] >= (1LL << 31)) {
                    b->err = "fused batch: more than 2^31 blocks in one stage";
                    return RBC_ERR_UNSUPPORTED;
                }
                acc[st] += (int)cnt[st];
            }
        }
        for (int st = 0; st < FSTAGES; st++) {
            boff[((size_t)k * FSTAGES + st) * (n + 1) + n] = acc[st];
            nblocks[st] = acc[st];
        }
    }
    const size_t dbytes = sizeof(DomainArgs) * dom.size(), obytes = sizeof(int) * boff.size();
    CKB(cudaMalloc(&b->fmem, dbytes + obytes));
    DomainArgs *d_dom = (DomainArgs *)b->fmem;
    int *d_boff = (int *)((char *)b->fmem + dbytes);
    CKB(cudaMemcpy(d_dom, dom.data(), dbytes, cudaMemcpyHostToDevice));
    CKB(cudaMemcpy(d_boff, boff.data(), obytes, cudaMemcpyHostToDevice));
    const bool fp64 = h0->p.membrane_fp64 != 0, xper = h0->geo.xper != 0;
    for (int k = 0; k < 2; k++) {
        FusedLaunch f[FSTAGES];
        for (int st = 0; st < FSTAGES; st++)
            f[st] = FusedLaunch{d_dom + (size_t)k * n, d_boff + ((size_t)k * FSTAGES + st) * (n + 1), n, nblocks[st]};
        cudaGraph_t graph = nullptr;
        CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        launch_step_begin_fused(f[FS_CLEAR], b->stream);
        launch_membrane_fused(f[FS_MEMBRANE], fp64, V, vpt, b->stream);
        launch_spread_fused(f[FS_SPREAD], xper, b->stream);
        launch_lbm_fused(f[FS_LBM], h0->p.storage, off32, tpb, b->stream);
        launch_clear_bits_fused(f[FS_CLEAR], b->stream);   // the force reset after the read
        launch_advect_fused(f[FS_ADVECT], xper, b->stream);
        launch_volume_fused(f[FS_VOLUME], V, b->stream);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (le != cudaSuccess || e != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            b->err = std::string("fused batch capture: ") + cudaGetErrorString(le != cudaSuccess ? le : e);
            return RBC_ERR_CUDA;
        }
        const cudaError_t ei = cudaGraphInstantiate(&b->graph[k], graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) { b->graph[k] = nullptr; b->err = std::string("fused batch instantiate: ") + cudaGetErrorString(ei); return RBC_ERR_CUDA; }
    }
    b->fused = true;
    return RBC_OK;
}

// The batch graph for parity k: every simulation's whole step (from buffer
// base_cur ^ k) as a child graph; simulations i and i + 1 of the same chain
// (i / chain equal) run one after the other, chains run concurrently.
int batch_build(rbc_batch *b)
{
    batch_free_graphs(b);
    const int n = (int)b->h.size();
    for (int i = 0; i < n; i++) b->base_cur[i] = b->h[i]->cur;
    b->parity = 0;
    if (b->use_fused && fused_obstacle(b).empty()) {
        const int rc = batch_build_fused(b);
        if (rc != RBC_OK) batch_free_graphs(b);
        return rc;
    }
    for (int k = 0; k < 2; k++) {
        cudaGraph_t g = nullptr;
        CKB(cudaGraphCreate(&g, 0));
        cudaGraphNode_t prev = nullptr;
        int rc = RBC_OK;
        for (int i = 0; i < n && rc == RBC_OK; i++) {
            cudaGraph_t child = nullptr;
            rc = capture_step(b->h[i], b->base_cur[i] ^ k, STEP_WHOLE, &child);
            if (rc != RBC_OK) { b->err = "simulation " + std::to_string(i) + ": " + b->h[i]->err; break; }
            cudaGraphNode_t node = nullptr;
            const bool chained = i % b->chain != 0;
            const cudaError_t e = cudaGraphAddChildGraphNode(&node, g, chained ? &prev : nullptr, chained ? 1 : 0, child);
            cudaGraphDestroy(child);
            if (e != cudaSuccess) { b->err = std::string("batch graph: ") + cudaGetErrorString(e); rc = RBC_ERR_CUDA; }
            prev = node;
        }
        cudaError_t e = cudaSuccess;
        if (rc == RBC_OK) e = cudaGraphInstantiate(&b->graph[k], g, 0);
        cudaGraphDestroy(g);
        if (rc != RBC_OK) return rc;
        if (e != cudaSuccess) {
            b->graph[k] = nullptr;
            b->err = std::string("batch graph instantiate: ") + cudaGetErrorString(e);
            return RBC_ERR_CUDA;
        }
    }
    return RBC_OK;
}

// Host-side setup of one cell population from its mesh (init2.cu:258-400,
// volume_correction.cu:427-450): link tables, reference metric, V0 and
// centroids, surface patches, bending visits.
struct GroupPrep {
    std::vector<int> off, packed, poff, pvtx, pstride;
    std::vector<int16_t> nbr6, nbrp6;
    std::vector<int> vord;
    std::vector<double> vol0, gx, xs;
    std::vector<double4> gref;
    std::vector<int4> visit;
    std::vector<double2> cs0;
};

int prepare_group(rbc_handle *h, CellGroup &c, const rbc_mesh *mesh, GroupPrep &pp)
{
    c.ncell = mesh->ncell; c.V = mesh->vertex; c.E = mesh->element;
    c.nv = (long long)c.ncell * c.V; c.ne = (long long)c.ncell * c.E;
    int rc = build_topology(h, c, mesh->tri, pp.off, pp.packed, pp.nbr6, pp.nbrp6, pp.vord);
    if (rc) return rc;
    surface_patches(c.V, mesh->xr, pp.poff, pp.pvtx, pp.pstride);
    c.npatch = (int)pp.poff.size() - 1;
    reference_metric(c, mesh->tri, mesh->xr, pp.gref);
    initial_volume(h, c, mesh->tri, mesh->xr, pp.vol0, pp.gx);
    pp.xs.resize(3 * c.nv);
    for (long long j = 0; j < c.nv; j++)
        for (int k = 0; k < 3; k++) pp.xs[k * c.nv + j] = mesh->xr[3 * j + k];
    if (c.br != 0.0) bend_visits(c.V, c.E, mesh->tri, pp.visit);
    if (c.br != 0.0 && h->p.bend_spont) spontaneous_angles(h->p, c, mesh->xr, pp.visit, pp.cs0);
    return RBC_OK;
}

// device arrays of one cell population
int upload_group(rbc_handle *h, CellGroup &c, const rbc_mesh *mesh, const GroupPrep &pp)
{
    int rc;
#define TRYG(x) do { if ((rc = (x))) return rc; } while (0)
    TRYG(dalloc(h, &c.X, 3 * c.nv)); TRYG(dalloc(h, &c.Xd, 3 * c.nv)); TRYG(dalloc(h, &c.gref, c.ne));
    CK(cudaMalloc(&c.erec, (size_t)c.ne * 12 * (h->p.membrane_fp64 ? sizeof(double) : sizeof(float))));
    TRYG(dalloc(h, &c.U, 3 * c.nv)); TRYG(dalloc(h, &c.Fv, 3 * c.nv));
    TRYG(dalloc(h, &c.tri, 3 * c.E)); TRYG(dalloc(h, &c.v2e_off, c.V + 1)); TRYG(dalloc(h, &c.v2e, pp.packed.size()));
    TRYG(dalloc(h, &c.nbr, 6 * c.V)); TRYG(dalloc(h, &c.nbrp, 6 * c.V)); TRYG(dalloc(h, &c.vord, c.V));
    if (!pp.visit.empty()) {
        TRYG(dalloc(h, &c.visit, pp.visit.size()));
        CK(cudaMemcpy(c.visit, pp.visit.data(), sizeof(int4) * pp.visit.size(), cudaMemcpyHostToDevice));
        TRYG(dalloc(h, &c.bend_rec, (size_t)c.ncell * c.E * 27));
    }
    if (!pp.cs0.empty()) {
        TRYG(dalloc(h, &c.cs0, pp.cs0.size()));
        CK(cudaMemcpy(c.cs0, pp.cs0.data(), sizeof(double2) * pp.cs0.size(), cudaMemcpyHostToDevice));
    }
    TRYG(dalloc(h, &c.patch_off, pp.poff.size())); TRYG(dalloc(h, &c.patch_vtx, pp.pvtx.size()));
    TRYG(dalloc(h, &c.patch_stride, pp.pstride.size()));
    TRYG(dalloc(h, &c.vol0, c.ncell)); TRYG(dalloc(h, &c.gx, 3 * c.ncell));
    TRYG(dalloc(h, &c.vol_out, c.ncell)); TRYG(dalloc(h, &c.area_out, c.ncell)); TRYG(dalloc(h, &c.cen_out, 3 * c.ncell));
#undef TRYG
    CK(cudaMemcpy(c.X, pp.xs.data(), 8 * 3 * c.nv, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.Xd, pp.xs.data(), 8 * 3 * c.nv, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.gref, pp.gref.data(), sizeof(double4) * c.ne, cudaMemcpyHostToDevice));
    CK(cudaMemset(c.U, 0, 4 * 3 * c.nv));
    CK(cudaMemset(c.Fv, 0, 4 * 3 * c.nv));
    CK(cudaMemcpy(c.tri, mesh->tri, 4 * 3 * c.E, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.v2e_off, pp.off.data(), 4 * (c.V + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.v2e, pp.packed.data(), 4 * pp.packed.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.nbr, pp.nbr6.data(), 2 * 6 * c.V, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.nbrp, pp.nbrp6.data(), 2 * 6 * c.V, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.vord, pp.vord.data(), 4 * c.V, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.patch_off, pp.poff.data(), 4 * pp.poff.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.patch_vtx, pp.pvtx.data(), 4 * pp.pvtx.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.patch_stride, pp.pstride.data(), 4 * pp.pstride.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.vol0, pp.vol0.data(), 8 * c.ncell, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.gx, pp.gx.data(), 8 * 3 * c.ncell, cudaMemcpyHostToDevice));
    return RBC_OK;
}

// volume, area, centroid of the cells of population g (synchronous): the values
// the step's volume correction left when the state is that step's, else a
// launch of the volume kernel in measuring mode
int group_metrics(rbc_handle *h, CellGroup &g, double *volume, double *area, double *centroid)
{
    if (g.ncell == 0) return fail(h, RBC_ERR_STATE, "no cells in this population");
    const int N = g.ncell;
    const double *cen = g.gx;
    if (!h->metrics_valid) {
        launch_volume(h->geo, volume_args(h, g, 0), h->stream);
        h->launches++;
        CK_LAUNCH();
        cen = g.cen_out;
    }
    if (h->metrics_host_n < (size_t)N) {
        if (h->metrics_host) { CK(cudaFreeHost(h->metrics_host)); h->metrics_host = nullptr; h->metrics_host_n = 0; }
        CK(cudaMallocHost(&h->metrics_host, 8 * 5 * (size_t)N));
        h->metrics_host_n = N;
    }
    double *t = h->metrics_host;
    CK(cudaMemcpyAsync(t, g.vol_out, 8 * N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(t + N, g.area_out, 8 * N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(t + 2 * N, cen, 8 * 3 * N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < N; c++) {
        if (volume) volume[c] = t[c];
        if (area) area[c] = t[N + c];
        if (centroid) for (int k = 0; k < 3; k++) centroid[3 * c + k] = t[(2 + k) * N + c];
    }
    return RBC_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char *rbc_last_error(const rbc_handle *h)
{
    return h ? h->err.c_str() : g_create_error.c_str();
}

constexpr int IMPORT_SLOTS = 4;
constexpr size_t IMPORT_CHUNK_BYTES = size_t(16) << 20;

// reference planes per import chunk: about IMPORT_CHUNK_BYTES, at most the whole lattice
static int import_chunk_planes(const Geom &g)
{
    const size_t plane_bytes = sizeof(double) * (size_t)g.nxr * g.ny * Q;
    return std::max(1, std::min(g.nzc, (int)(IMPORT_CHUNK_BYTES / plane_bytes)));
}

// the import ring (IMPORT_SLOTS chunks and the two edge planes) and its events
static int ensure_import_ring(rbc_handle *h)
{
    const Geom &g = h->geo;
    const int P = import_chunk_planes(g);
    if (h->imp_ring && h->imp_planes == P) return RBC_OK;
    const size_t plane_bytes = sizeof(double) * (size_t)g.nxr * g.ny * Q;
    if (h->imp_ring) { CK(cudaFree(h->imp_ring)); h->imp_ring = nullptr; }
    CK(cudaMalloc(&h->imp_ring, plane_bytes * (size_t)(IMPORT_SLOTS * P + 2)));
    h->imp_planes = P;
    for (int k = 0; k < IMPORT_SLOTS; k++) {
        if (!h->imp_copied[k]) CK(cudaEventCreateWithFlags(&h->imp_copied[k], cudaEventDisableTiming));
        if (!h->imp_freed[k]) CK(cudaEventCreateWithFlags(&h->imp_freed[k], cudaEventDisableTiming));
    }
    return RBC_OK;
}

static int import_lattice_pipelined(rbc_handle *h, const double *fn, const WallVel &w);
static cudaError_t cell_io_setup();
static int ensure_cell_staging(rbc_handle *h, const CellGroup &G);

int rbc_create(const rbc_params *p, const rbc_mesh *mesh, const int *bc, rbc_handle **out)
{
    g_create_error.clear();
    if (!out) return fail(nullptr, RBC_ERR_ARG, "out is NULL");
    *out = nullptr;
    int rc = check_params(p);
    if (rc) return rc;
    if (!bc) return fail(nullptr, RBC_ERR_ARG, "bc is NULL");
    std::vector<uint32_t> mask;
    if ((rc = build_mask(p, bc, mask))) return rc;
    const bool cells = mesh && mesh->ncell > 0;
    if (cells) {
        if (mesh->vertex < 4 || mesh->element < 4 || !mesh->tri || !mesh->xr)
            return fail(nullptr, RBC_ERR_ARG, "mesh needs vertex, element >= 4, tri and xr");
        if (membrane_smem_bytes(mesh->vertex) > 227 * 1024 || mesh->vertex > 4096)
            return fail(nullptr, RBC_ERR_UNSUPPORTED, "more vertices per cell than one CTA holds (max 3874)");
        if (mesh->element >= (1 << 24)) return fail(nullptr, RBC_ERR_UNSUPPORTED, "too many elements per cell");
    }
    rbc_handle *h = new (std::nothrow) rbc_handle();
    if (!h) return fail(nullptr, RBC_ERR_ARG, "out of host memory");
    h->p = *p;
    if (h->p.solver_iters == 0) h->p.solver_iters = DEFAULT_SOLVER_ITERS;
    Geom &g = h->geo;
    const bool shear = p->flow == RBC_FLOW_SHEAR;
    g.nxr = p->nx; g.xb = shear ? 2 : 0; g.xper = shear ? 1 : 0;
    g.nx = p->nx - 2 * g.xb; g.ny = p->ny; g.nzr = p->nz; g.nzc = p->nz - 4;
    g.plane = (long long)g.nx * p->ny; g.nint = g.plane * g.nzc;
    g.dx = p->dx;
    g.inv_dx = 1.0 / p->dx;
    g.xoff = (double)(p->nx - 1) * p->dx / 2.0;
    g.yoff = (double)(p->ny - 1) * p->dx / 2.0;
    g.zoff = (double)(p->nz - 1) * p->dx / 2.0;
    g.LX = p->LX; g.LZ = p->LZ; g.xmin = p->xmin; g.xmax = p->xmax; g.zmin = p->zmin; g.zmax = p->zmax;
    h->nref_nodes = (long long)g.nxr * g.ny * g.nzr;
    if (p->storage == RBC_STORE_F16) { h->scale = F16_SCALE; h->inv_scale = 1.0f / F16_SCALE; }

    auto bail = [&](int code) {
        g_create_error = h->err;
        free_all(h);
        delete h;
        return code;
    };
#define TRY(x) do { int r_ = (x); if (r_) return bail(r_); } while (0)
    // host-side setup first, so argument and mesh errors are reported without a GPU
    GroupPrep prep;
    h->cg[0].rgs = p->rgs;
    h->cg[0].br = p->br;
    if (cells) TRY(prepare_group(h, h->cg[0], mesh, prep));
    {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            h->err = "no CUDA device";
            return bail(RBC_ERR_NO_DEVICE);
        }
        h->device = p->device >= 0 ? p->device : 0;
        if (h->device >= ndev) { h->err = "device ordinal out of range"; return bail(RBC_ERR_ARG); }
        if (cudaSetDevice(h->device) != cudaSuccess) { h->err = "cudaSetDevice failed"; return bail(RBC_ERR_CUDA); }
    }
    {
        int mem_max = 0;
        int e = setup_kernel_attributes(&mem_max);
        if (!e) e = (int)lattice_io_setup();
        if (!e) e = (int)cell_io_setup();
        if (e) { h->err = std::string("kernel attributes: ") + cudaGetErrorString((cudaError_t)e); return bail(RBC_ERR_CUDA); }
        if (cells && membrane_smem_bytes(mesh->vertex) > mem_max) {
            h->err = "more vertices per cell than one CTA's shared memory holds";
            return bail(RBC_ERR_UNSUPPORTED);
        }
    }
    {
        int lo = 0, hi = 0;
        if (cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess ||
            cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaStreamCreateWithFlags(&h->side2, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->wave_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->spread_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->lbm_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->reset_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess) {
            h->err = "stream creation failed";
            return bail(RBC_ERR_CUDA);
        }
        h->prio_high = hi;   // numerically lowest value = greatest priority
    }
    const size_t esz = p->storage == RBC_STORE_F16 ? 2 : 4;
    h->gbytes = esz * (size_t)Q * (size_t)g.nint;
    if (cudaMalloc(&h->g[0], h->gbytes) != cudaSuccess || cudaMalloc(&h->g[1], h->gbytes) != cudaSuccess) {
        h->err = "out of device memory for the populations";
        return bail(RBC_ERR_CUDA);
    }
    TRY(dalloc(h, &h->uvr, g.nint)); TRY(dalloc(h, &h->Fint, 3 * g.nint));
    TRY(dalloc(h, &h->Fbits, h->force_bit_bytes() / sizeof(uint32_t))); TRY(dalloc(h, &h->mask2d, g.plane));
    TRY(dalloc(h, &h->d_int, 6)); TRY(dalloc(h, &h->d_drive, 3));
    if (cudaMemset(h->g[0], 0, h->gbytes) != cudaSuccess || cudaMemset(h->g[1], 0, h->gbytes) != cudaSuccess ||
        cudaMemset(h->Fint, 0, 24 * g.nint) != cudaSuccess || cudaMemset(h->Fbits, 0, h->force_bit_bytes()) != cudaSuccess ||
        cudaMemset(h->d_int, 0, 6 * sizeof(int)) != cudaSuccess || cudaMemset(h->d_drive, 0, 3 * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(h->mask2d, mask.data(), 4 * g.plane, cudaMemcpyHostToDevice) != cudaSuccess) {
        h->err = "device initialisation failed";
        return bail(RBC_ERR_CUDA);
    }
    launch_fill_f4(h->uvr, g.nint, make_float4(0.f, 0.f, 0.f, 1.f), h->stream);
    if (p->tube_r > 0.0) {
        std::vector<int> links;
        std::vector<float> frac;
        tube_links(p, mask, links, frac);
        h->ntube = (int)links.size();
        TRY(dalloc(h, &h->tube_links, links.size()));
        TRY(dalloc(h, &h->tube_frac, frac.size()));
        if (!links.empty() &&
            (cudaMemcpy(h->tube_links, links.data(), 4 * links.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemcpy(h->tube_frac, frac.data(), 4 * frac.size(), cudaMemcpyHostToDevice) != cudaSuccess)) {
            h->err = "device initialisation failed";
            return bail(RBC_ERR_CUDA);
        }
    }
    if (shear && p->flowstart == 0) {
        // flu_init's linear profile between the walls (init1.cu:367-381), as reference-layout
        // populations imported for the first step
        const double LY = (double)(p->ny - 4) * p->dx, Cr = p->Cr;
        const long long pr = (long long)p->nx * p->ny;
        std::vector<double> fn((size_t)h->nref_nodes * Q);
        std::vector<float4> uv((size_t)g.nint);
        auto tw_of = [&](int iy) {
            return p->walls == RBC_WALLS_BOTH ? p->sr * (-LY / 2.0 - 1.5 * p->dx + iy * p->dx)
                                              : p->sr * (-1.5 * p->dx + iy * p->dx);
        };
        for (long long i = 0; i < h->nref_nodes; i++) {
            const double tw = tw_of((int)((i % pr) / p->nx)), uvw = -1.5 * tw * tw * Cr * Cr;
            for (int q = 0; q < Q; q++) {
                const double eu = ez(q) * tw;
                fn[(size_t)i * Q + q] = wqd(q) * (1.0 + 3.0 * eu * Cr + 4.5 * eu * eu * Cr * Cr + uvw);
            }
        }
        for (long long i = 0; i < g.nint; i++) {
            const int y = (int)((i % g.plane) / g.nx);
            uv[(size_t)i] = (y >= 2 && y < g.ny - 2) ? make_float4(0.f, 0.f, (float)tw_of(y), 1.f) : make_float4(0.f, 0.f, 0.f, 1.f);
        }
        if (cudaMemcpy(h->uvr, uv.data(), 16 * uv.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            import_lattice_pipelined(h, fn.data(), wall_velocities(h, 1)) != RBC_OK) {
            h->err = "initial shear profile upload failed";
            return bail(RBC_ERR_CUDA);
        }
    }

    if (cells) TRY(upload_group(h, h->cg[0], mesh, prep));
    if (p->vof_k > 0) TRY(vof_init_group(h, h->cg[0]));
    // buffers of the reference-layout imports and exports, allocated here rather than in the first
    // call: the cells' layout conversions, and the lattice import's ring where the ring is a
    // bounded part of the lattice (more chunks than slots; smaller lattices allocate it on use)
    if (cells) TRY(ensure_cell_staging(h, h->cg[0]));
    if ((g.nzc + import_chunk_planes(g) - 1) / import_chunk_planes(g) > IMPORT_SLOTS) TRY(ensure_import_ring(h));
    if (cudaStreamSynchronize(h->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        h->err = "initialisation kernels failed";
        return bail(RBC_ERR_CUDA);
    }
#undef TRY
    *out = h;
    return RBC_OK;
}

int rbc_destroy(rbc_handle *h)
{
    if (!h) return RBC_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return RBC_OK;
}

// Reference fn (host, AoS FP64, all nzc + 4 planes) -> population buffer g[cur], as a pipeline:
// the copy stream brings chunks of IMPORT_CHUNK_BYTES into a ring of IMPORT_SLOTS slots while the
// main stream converts each internal slab once the chunk after it has arrived (a slab reads one
// plane of each neighbouring chunk).  The BUFF planes are not copied; the periodic images of the
// first and last planes come from two edge planes copied first.  Returns after the conversion.
static int import_lattice_pipelined(rbc_handle *h, const double *fn, const WallVel &w)
{
    const Geom &g = h->geo;
    const long long plane_vals = (long long)g.nxr * g.ny * Q;
    const size_t plane_bytes = sizeof(double) * (size_t)plane_vals;
    int rc = ensure_import_ring(h);
    if (rc) return rc;
    const int P = h->imp_planes;
    const ImportPlanes src{h->imp_ring, h->imp_ring + (long long)IMPORT_SLOTS * P * plane_vals, IMPORT_SLOTS * P,
                           plane_vals};
    cudaStream_t cs = h->side, ks = h->stream;
    // internal plane z is reference plane z + 2
    auto ref_plane = [&](int z) { return fn + (long long)(z + 2) * plane_vals; };
    const int nch = (g.nzc + P - 1) / P;
    // the copy stream starts after the main stream's earlier work (it may still read the ring)
    CK(cudaEventRecord(h->imp_freed[0], ks));
    CK(cudaStreamWaitEvent(cs, h->imp_freed[0], 0));
    CK(cudaMemcpyAsync((double *)src.edge, ref_plane(g.nzc - 1), plane_bytes, cudaMemcpyHostToDevice, cs));
    CK(cudaMemcpyAsync((double *)src.edge + plane_vals, ref_plane(0), plane_bytes, cudaMemcpyHostToDevice, cs));
    auto convert = [&](int j) {
        launch_import_lattice(g, h->p.storage, src, h->g[h->cur], h->mask2d, h->scale, w, j * P,
                              std::min(g.nzc, (j + 1) * P), ks);
        h->launches++;
    };
    for (int c = 0; c < nch; c++) {
        const int slot = c % IMPORT_SLOTS;
        // chunk c - IMPORT_SLOTS, in this slot, was last read by slab c - IMPORT_SLOTS + 1
        if (c >= IMPORT_SLOTS) CK(cudaStreamWaitEvent(cs, h->imp_freed[slot], 0));
        const int planes = std::min(P, g.nzc - c * P);
        CK(cudaMemcpyAsync(h->imp_ring + (long long)slot * P * plane_vals, ref_plane(c * P), plane_bytes * planes,
                           cudaMemcpyHostToDevice, cs));
        CK(cudaEventRecord(h->imp_copied[slot], cs));
        if (c >= 1) {
            CK(cudaStreamWaitEvent(ks, h->imp_copied[slot], 0));
            convert(c - 1);
            CK_LAUNCH();
            if (c >= 2) CK(cudaEventRecord(h->imp_freed[(c - 2) % IMPORT_SLOTS], ks));
        }
    }
    CK(cudaStreamWaitEvent(ks, h->imp_copied[(nch - 1) % IMPORT_SLOTS], 0));
    convert(nch - 1);
    CK_LAUNCH();
    CK(cudaStreamSynchronize(ks));
    return RBC_OK;
}

int rbc_import_ref_lattice(rbc_handle *h, const double *fn)
{
    if (!h || !fn) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    return import_lattice_pipelined(h, fn, wall_velocities(h, h->iter + 1));
}

int rbc_export_ref_lattice(rbc_handle *h, double *fn, double *dn, double *un, double *vn, double *wn)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    const bool macro = dn || un || vn || wn;
    if (!fn && !macro) return RBC_OK;
    const size_t n = (size_t)h->nref_nodes;
    int rc = ensure_staging(h, sizeof(double) * n * (fn ? (Q + 4) : 4));
    if (rc) return rc;
    double *sfn = (double *)h->staging;
    double *smac = fn ? sfn + Q * n : sfn;
    launch_export_lattice(h->geo, h->p.storage, h->g[h->cur], h->mask2d, h->uvr, h->inv_scale,
                          fn ? sfn : nullptr, macro ? smac : nullptr, smac + n, smac + 2 * n, smac + 3 * n, wall_velocities(h, h->iter + 1), h->stream);
    h->launches++;
    CK_LAUNCH();
    if (fn) CK(cudaMemcpyAsync(fn, sfn, sizeof(double) * Q * n, cudaMemcpyDeviceToHost, h->stream));
    if (dn) CK(cudaMemcpyAsync(dn, smac, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (un) CK(cudaMemcpyAsync(un, smac + n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (vn) CK(cudaMemcpyAsync(vn, smac + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (wn) CK(cudaMemcpyAsync(wn, smac + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return RBC_OK;
}

int rbc_export_ref_force(rbc_handle *h, double *fx, double *fy, double *fz)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    const size_t n = (size_t)h->nref_nodes;
    int rc = ensure_staging(h, sizeof(double) * 3 * n);
    if (rc) return rc;
    double *s = (double *)h->staging;
    launch_export_force(h->geo, h->Fint, h->mask2d, s, h->stream);
    h->launches++;
    CK_LAUNCH();
    if (fx) CK(cudaMemcpyAsync(fx, s, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (fy) CK(cudaMemcpyAsync(fy, s + n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (fz) CK(cudaMemcpyAsync(fz, s + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return RBC_OK;
}

// Reference cell layouts <-> the handle's, converted on the device: the host
// only copies the caller's arrays.  The metric conversion rounds each product,
// the difference and each quotient separately, as the host expression
// n00 * n11 - n01 * n01 with no contraction would (explicit _rn intrinsics: the
// device compiler would otherwise fuse the products into a multiply-add).
__global__ void import_metric_kernel(const double *__restrict__ nd, double4 *__restrict__ gref, long long ne)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const double n00 = nd[4 * e], n01 = nd[4 * e + 1], n11 = nd[4 * e + 3];
    const double det = __dsub_rn(__dmul_rn(n00, n11), __dmul_rn(n01, n01));
    // G = n^-1, 1 / det G = det n
    gref[e] = make_double4(__ddiv_rn(n11, det), __ddiv_rn(-n01, det), __ddiv_rn(n00, det), det);
}

// [n][3] (AoS, the reference's fem->xd and cel->gx) <-> [3][n] (the handle's)
__global__ void aos3_to_soa_kernel(const double *__restrict__ in, double *__restrict__ out, long long n)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    out[j] = in[3 * j]; out[n + j] = in[3 * j + 1]; out[2 * n + j] = in[3 * j + 2];
}

__global__ void soa3_to_aos_kernel(const double *__restrict__ in, double *__restrict__ out, long long n)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    out[3 * j] = in[j]; out[3 * j + 1] = in[n + j]; out[3 * j + 2] = in[2 * n + j];
}

__global__ void f32_to_f64_kernel(const float *__restrict__ in, double *__restrict__ out, long long n)
{
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) out[j] = (double)in[j];
}

static unsigned blocks_for(long long n) { return (unsigned)((n + 255) / 256); }

// load the layout kernels now (lazy module loading would load each in its first call)
static cudaError_t cell_io_setup()
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)import_metric_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)aos3_to_soa_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)soa3_to_aos_kernel);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, (const void *)f32_to_f64_kernel);
    return e;
}

// staging of the cell imports ([nv][3] + [ne][4] + [N][3] doubles) and exports ([nv][3] + 6 [nv] + [N][3])
static size_t cell_staging_bytes(const CellGroup &G)
{
    const size_t nv = (size_t)G.nv, ne = (size_t)G.ne, N = (size_t)G.ncell;
    return sizeof(double) * (std::max(3 * nv + 4 * ne, 9 * nv) + 3 * N);
}

static int ensure_cell_staging(rbc_handle *h, const CellGroup &G) { return ensure_staging(h, cell_staging_bytes(G)); }

static int import_cells(rbc_handle *h, CellGroup &G, const double *x, const double *y, const double *z,
                        const double *xd, const double *nd, const double *volume0, const double *gx)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    if (G.ncell == 0) return fail(h, RBC_ERR_STATE, "no cells in this population");
    const long long nv = G.nv, ne = G.ne;
    const int N = G.ncell;
    cudaStream_t s = h->stream;
    CK(cudaStreamSynchronize(s));
    // staging: xd [nv][3], nd [ne][4], gx [N][3]
    const size_t o_nd = 3 * (size_t)nv, o_gx = o_nd + 4 * (size_t)ne;
    if (xd || nd || gx) {
        const int rc = ensure_cell_staging(h, G);
        if (rc) return rc;
    }
    double *st = (double *)h->staging;
    if (x) CK(cudaMemcpyAsync(G.X, x, 8 * nv, cudaMemcpyHostToDevice, s));
    if (y) CK(cudaMemcpyAsync(G.X + nv, y, 8 * nv, cudaMemcpyHostToDevice, s));
    if (z) CK(cudaMemcpyAsync(G.X + 2 * nv, z, 8 * nv, cudaMemcpyHostToDevice, s));
    if (xd) {
        CK(cudaMemcpyAsync(st, xd, 8 * 3 * nv, cudaMemcpyHostToDevice, s));
        aos3_to_soa_kernel<<<blocks_for(nv), 256, 0, s>>>(st, G.Xd, nv);
        h->launches++;
        CK_LAUNCH();
    }
    if (nd) {
        CK(cudaMemcpyAsync(st + o_nd, nd, 8 * 4 * ne, cudaMemcpyHostToDevice, s));
        import_metric_kernel<<<blocks_for(ne), 256, 0, s>>>(st + o_nd, G.gref, ne);
        h->launches++;
        CK_LAUNCH();
    }
    if (volume0) CK(cudaMemcpyAsync(G.vol0, volume0, 8 * N, cudaMemcpyHostToDevice, s));
    if (gx) {
        CK(cudaMemcpyAsync(st + o_gx, gx, 8 * 3 * N, cudaMemcpyHostToDevice, s));
        aos3_to_soa_kernel<<<blocks_for(N), 256, 0, s>>>(st + o_gx, G.gx, N);
        h->launches++;
        CK_LAUNCH();
    }
    CK(cudaStreamSynchronize(s));
    return RBC_OK;
}

int rbc_import_ref_cells(rbc_handle *h, const double *x, const double *y, const double *z,
                         const double *xd, const double *nd, const double *volume0, const double *gx)
{
    if (!h) return RBC_ERR_ARG;
    return import_cells(h, h->cg[0], x, y, z, xd, nd, volume0, gx);
}

int rbc_import_ref_vertex_force(rbc_handle *h, const double *fx, const double *fy, const double *fz)
{
    if (!h || !fx || !fy || !fz) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    if (h->ncell == 0) return fail(h, RBC_ERR_STATE, "handle has no cells");
    const long long nv = h->nv;
    std::vector<float> t(3 * nv);
    for (long long j = 0; j < nv; j++) { t[j] = (float)fx[j]; t[nv + j] = (float)fy[j]; t[2 * nv + j] = (float)fz[j]; }
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(h->Fv, t.data(), 4 * 3 * nv, cudaMemcpyHostToDevice));
    return RBC_OK;
}

static int export_cells(rbc_handle *h, CellGroup &G, double *x, double *y, double *z, double *xd,
                        double *u, double *v, double *w, double *fx, double *fy, double *fz, double *gxo)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    if (G.ncell == 0) return fail(h, RBC_ERR_STATE, "no cells in this population");
    const long long nv = G.nv;
    const int N = G.ncell;
    cudaStream_t s = h->stream;
    CK(cudaStreamSynchronize(s));
    double *outs[6] = {u, v, w, fx, fy, fz};
    const bool vel = u || v || w, frc = fx || fy || fz;
    // staging: xd [nv][3], u v w [3][nv], fx fy fz [3][nv], gx [N][3]
    const size_t o_u = 3 * (size_t)nv, o_f = o_u + 3 * (size_t)nv, o_gx = o_f + 3 * (size_t)nv;
    if (xd || vel || frc || gxo) {
        const int rc = ensure_cell_staging(h, G);
        if (rc) return rc;
    }
    double *st = (double *)h->staging;
    if (xd) {
        soa3_to_aos_kernel<<<blocks_for(nv), 256, 0, s>>>(G.Xd, st, nv);
        h->launches++;
        CK_LAUNCH();
    }
    if (vel) {
        f32_to_f64_kernel<<<blocks_for(3 * nv), 256, 0, s>>>(G.U, st + o_u, 3 * nv);
        h->launches++;
        CK_LAUNCH();
    }
    if (frc) {
        f32_to_f64_kernel<<<blocks_for(3 * nv), 256, 0, s>>>(G.Fv, st + o_f, 3 * nv);
        h->launches++;
        CK_LAUNCH();
    }
    if (gxo) {
        soa3_to_aos_kernel<<<blocks_for(N), 256, 0, s>>>(G.gx, st + o_gx, N);
        h->launches++;
        CK_LAUNCH();
    }
    if (x) CK(cudaMemcpyAsync(x, G.X, 8 * nv, cudaMemcpyDeviceToHost, s));
    if (y) CK(cudaMemcpyAsync(y, G.X + nv, 8 * nv, cudaMemcpyDeviceToHost, s));
    if (z) CK(cudaMemcpyAsync(z, G.X + 2 * nv, 8 * nv, cudaMemcpyDeviceToHost, s));
    if (xd) CK(cudaMemcpyAsync(xd, st, 8 * 3 * nv, cudaMemcpyDeviceToHost, s));
    for (int k = 0; k < 6; k++)
        if (outs[k]) CK(cudaMemcpyAsync(outs[k], st + o_u + (size_t)k * nv, 8 * nv, cudaMemcpyDeviceToHost, s));
    if (gxo) CK(cudaMemcpyAsync(gxo, st + o_gx, 8 * 3 * N, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return RBC_OK;
}

int rbc_export_ref_cells(rbc_handle *h, double *x, double *y, double *z, double *xd,
                         double *u, double *v, double *w, double *fx, double *fy, double *fz, double *gxo)
{
    if (!h) return RBC_ERR_ARG;
    return export_cells(h, h->cg[0], x, y, z, xd, u, v, w, fx, fy, fz, gxo);
}

int rbc_set_iter(rbc_handle *h, int iter)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    CK(cudaStreamSynchronize(h->stream));
    h->iter = iter;
    // the drive and wall velocities of step `iter`, as step_begin leaves them (for stage calls)
    const WallVel w = wall_velocities(h, iter);
    const float dv[3] = {(float)(h->p.P * drive_factor(h->p, iter)), (float)w.top, (float)w.bot};
    CK(cudaMemcpy(h->d_iter(), &iter, sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(h->d_drive, dv, sizeof(dv), cudaMemcpyHostToDevice));
    return RBC_OK;
}

int rbc_get_iter(const rbc_handle *h, int *iter)
{
    if (!h || !iter) return RBC_ERR_ARG;
    *iter = h->iter;
    return RBC_OK;
}

int rbc_stress(rbc_handle *h)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    const int rc = launch_stress(h);
    return rc ? rc : launch_bend_stage(h);
}

int rbc_ibm_st1(rbc_handle *h)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    if (h->force_pending) {   // ibm_st1a: start from zero (ibm.cu:315-320)
        CK(cudaMemsetAsync(h->Fint, 0, 24 * h->geo.nint, h->stream));
        CK(cudaMemsetAsync(h->Fbits, 0, h->force_bit_bytes(), h->stream));
    }
    int rc = launch_spread_stage(h);
    if (rc) return rc;
    h->force_pending = true;
    return RBC_OK;
}

int rbc_lbm_d3q19(rbc_handle *h)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    // sub-cycled: the step h->iter's place among the M (as set by rbc_set_iter);
    // the force is cleared after the last
    const StepForm f = h->p.M == 1 ? STEP_WHOLE : sub_form(h, h->iter);
    const bool last = f == STEP_WHOLE || f == STEP_SUB_LAST;
    int rc = launch_lbm_stage(h, last, lbm_acc(f));
    if (rc) return rc;
    if (last) h->force_pending = false;   // the reset cleared the force
    return RBC_OK;
}

int rbc_ibm_st2(rbc_handle *h)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    return launch_advect_stage(h);
}

int rbc_thinc_wlic(rbc_handle *h)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    return launch_thinc_stage(h);
}

int rbc_front_tracking(rbc_handle *h, int *iters)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    int rc = launch_front_tracking_stage(h);
    if (rc || !iters) return rc;
    int v[2] = {0, 0};
    CK(cudaMemcpyAsync(v, h->d_vofit(), sizeof(v), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    iters[0] = v[0];
    return RBC_OK;
}

// ltc->vf / vf2 [nx*ny*nz] in the reference layout <-> the populations' internal fields
static int vof_transfer(rbc_handle *h, double *out0, double *out1, const double *in0, const double *in1)
{
    if (in0 || in1) RBC_DEVICE_GUARD(h); else RBC_DEVICE_GUARD_RO(h);
    if (!h->vof()) return fail(h, RBC_ERR_STATE, "the volume fraction is not tracked (vof_k = 0)");
    const Geom &g = h->geo;
    std::vector<uint32_t> mask((size_t)g.plane);
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(mask.data(), h->mask2d, 4 * mask.size(), cudaMemcpyDeviceToHost));
    std::vector<double> in((size_t)g.nint);
    const long long nref = (long long)g.nxr * g.ny * g.nzr;
    for (int k = 0; k < 2; k++) {
        double *out = k ? out1 : out0;
        const double *src = k ? in1 : in0;
        CellGroup &cgp = h->cg[k];
        if (!out && !src) continue;
        if (k >= h->ngroups || !cgp.vf) {   // no such population: its field is 0
            if (out) std::fill(out, out + nref, 0.0);
            continue;
        }
        if (out) {
            CK(cudaMemcpy(in.data(), cgp.vf, 8 * in.size(), cudaMemcpyDeviceToHost));
            for (int iz = 0; iz < g.nzr; iz++)
                for (int iy = 0; iy < g.ny; iy++)
                    for (int ix = 0; ix < g.nxr; ix++) {
                        int xi = ix - g.xb;
                        const bool in_x = xi >= 0 && xi < g.nx;
                        if (g.xper) xi = ((xi % g.nx) + g.nx) % g.nx;
                        const long long r = ((long long)iz * g.ny + iy) * g.nxr + ix;
                        if ((!in_x && !g.xper) || !(mask[(size_t)iy * g.nx + xi] & MASK_FLUID)) { out[r] = 0.0; continue; }
                        const int zc = (((iz - 2) % g.nzc) + g.nzc) % g.nzc;
                        out[r] = in[(size_t)zc * g.plane + (size_t)iy * g.nx + xi];
                    }
        } else {
            for (int zc = 0; zc < g.nzc; zc++)
                for (int iy = 0; iy < g.ny; iy++)
                    for (int xi = 0; xi < g.nx; xi++) {
                        const bool fl = (mask[(size_t)iy * g.nx + xi] & MASK_FLUID) != 0;
                        const long long r = ((long long)(zc + 2) * g.ny + iy) * g.nxr + xi + g.xb;
                        in[(size_t)zc * g.plane + (size_t)iy * g.nx + xi] = fl ? src[r] : 0.0;
                    }
            CK(cudaMemcpy(cgp.vf, in.data(), 8 * in.size(), cudaMemcpyHostToDevice));
        }
    }
    return RBC_OK;
}

int rbc_export_ref_vof(rbc_handle *h, double *vf, double *vf2)
{
    if (!h) return RBC_ERR_ARG;
    return vof_transfer(h, vf, vf2, nullptr, nullptr);
}

int rbc_import_ref_vof(rbc_handle *h, const double *vf, const double *vf2)
{
    if (!h) return RBC_ERR_ARG;
    return vof_transfer(h, nullptr, nullptr, vf, vf2);
}

int rbc_volume_correction(rbc_handle *h, int *iters)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    int rc = launch_volume_stage(h, h->stream);
    if (rc) return rc;
    if (iters) {
        int v = 0;
        if (h->has_cells()) {
            CK(cudaMemcpyAsync(&v, h->d_vclast(), sizeof(int), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
        *iters = v;
    }
    return RBC_OK;
}

int rbc_step(rbc_handle *h, int nsteps)
{
    if (!h || nsteps < 0) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    if (nsteps == 0) return RBC_OK;
    int rc;
    if ((rc = prepare_steps(h))) return rc;
    if (h->p.M > 1) {   // sub-cycled: each step's graph by its place among the M
        bool ended = false;
        for (int k = 0; k < nsteps; k++) {
            const StepForm f = sub_form(h, h->iter + k + 1);
            if (!h->graph[f][h->cur] && (rc = build_graph(h, h->cur, f))) return rc;
            CK(cudaGraphLaunch(h->graph[f][h->cur], h->stream));
            h->cur ^= 1;
            h->launches += h->graph_kernels[f];
            ended = f == STEP_SUB_LAST;
        }
        h->iter += nsteps;
        h->force_pending = h->iter % h->p.M != 0;   // the cycle's force stays for its remaining steps
        if (ended) h->metrics_valid = h->has_cells();
        return RBC_OK;
    }
    // one step, or no cells: whole steps.  Otherwise step 1 without its
    // correction, steps 2..n pipelined with the correction of the step before,
    // then the correction of step n: the same kernels in the same data order.
    // with the volume fraction, front tracking (main.cu:97-98) runs between the
    // step's graph and its volume correction, which the pipelined forms leave
    // to the next graph
    const bool pipe = (nsteps > 1 || h->vof()) && h->has_cells();
    for (int c = 0; c < 2; c++) {
        if (!h->graph[STEP_WHOLE][c] && (rc = build_graph(h, c, STEP_WHOLE))) return rc;
        if (pipe && !h->graph[STEP_BODY][c] && (rc = build_graph(h, c, STEP_BODY))) return rc;
        if (pipe && !h->graph[STEP_PIPELINED][c] && (rc = build_graph(h, c, STEP_PIPELINED))) return rc;
    }
    for (int k = 0; k < nsteps; k++) {
        const StepForm form = !pipe ? STEP_WHOLE : k == 0 ? STEP_BODY : STEP_PIPELINED;
        CK(cudaGraphLaunch(h->graph[form][h->cur], h->stream));
        h->cur ^= 1;
        h->launches += h->kernels_per_step();
        if (h->vof() && (h->iter + k + 1) % h->p.vof_k == 0 && (rc = launch_front_tracking_stage(h))) return rc;
    }
    if (pipe) {
        for (int k = 0; k < h->ngroups; k++)   // step n's corrections, counted with its step, are launched here
            h->launches -= h->cg[k].ncell > 0 ? 1 : 0;
        if ((rc = launch_volume_stage(h, h->stream))) return rc;
    }
    h->iter += nsteps;
    h->metrics_valid = h->has_cells();   // the last kernels of every population were its volume correction
    return RBC_OK;
}

int rbc_profile_steps(rbc_handle *h, int nsteps, double *kernel_ms)
{
    if (!h || nsteps < 0 || !kernel_ms) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    for (int k = 0; k < RBC_NUM_KERNELS; k++) kernel_ms[k] = 0.0;
    int rc;
    if ((rc = prepare_steps(h))) return rc;
    cudaEvent_t ev[RBC_NUM_KERNELS + 1];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    bool ended = false;
    for (int s = 0; s < nsteps && rc == RBC_OK; s++) {
        // the stages of this step's place among M sub-cycled steps (all of them for M = 1)
        const StepForm f = h->p.M == 1 ? STEP_WHOLE : sub_form(h, h->iter + s + 1);
        const bool first = f == STEP_WHOLE || f == STEP_SUB_FIRST, last = f == STEP_WHOLE || f == STEP_SUB_LAST;
        ended = last;
        cudaEventRecord(ev[0], h->stream);
        launch_step_begin(step_begin_args(h), h->stream);
        h->launches++;
        cudaEventRecord(ev[1], h->stream);
        if (!rc && first) rc = launch_stress(h);
        if (!rc && first) rc = launch_bend_stage(h);   // timed with the membrane pass
        cudaEventRecord(ev[2], h->stream);
        if (!rc && first) rc = launch_spread_stage(h);
        cudaEventRecord(ev[3], h->stream);
        if (!rc) rc = launch_lbm_stage(h, false, lbm_acc(f));
        cudaEventRecord(ev[4], h->stream);
        if (!rc && last) rc = launch_force_reset_stage(h, h->stream);
        cudaEventRecord(ev[5], h->stream);
        if (!rc && last) rc = launch_advect_stage(h);
        cudaEventRecord(ev[6], h->stream);
        if (!rc && last) rc = launch_thinc_stage(h);
        if (!rc && h->vof() && (h->iter + s + 1) % h->p.vof_k == 0) rc = launch_front_tracking_stage(h);
        cudaEventRecord(ev[7], h->stream);
        if (!rc && last) rc = launch_volume_stage(h, h->stream);
        cudaEventRecord(ev[8], h->stream);
        if (cudaEventSynchronize(ev[8]) != cudaSuccess) { rc = RBC_ERR_CUDA; h->err = "profiled step failed"; break; }
        for (int k = 0; k < RBC_NUM_KERNELS; k++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            kernel_ms[k] += ms;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    if (rc == RBC_OK) {
        h->iter += nsteps;
        h->force_pending = h->p.M > 1 && h->iter % h->p.M != 0;
    }
    if (ended || rc != RBC_OK) h->metrics_valid = rc == RBC_OK && nsteps > 0 && h->has_cells();
    return rc;
}

int rbc_get_stream(const rbc_handle *h, void **stream)
{
    if (!h || !stream) return RBC_ERR_ARG;
    *stream = (void *)h->stream;
    return RBC_OK;
}

int rbc_get_status(rbc_handle *h, int *flags, int *vc_iters_max)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    int v[4];
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(v, h->d_int, sizeof(v), cudaMemcpyDeviceToHost));
    if (flags) *flags = v[1];
    if (vc_iters_max) *vc_iters_max = v[2];
    CK(cudaMemset(h->d_flags(), 0, sizeof(int)));
    return RBC_OK;
}

int rbc_cell_metrics(rbc_handle *h, double *volume, double *area, double *centroid)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    if (h->ncell == 0) return fail(h, RBC_ERR_STATE, "handle has no cells");
    return group_metrics(h, h->cg[0], volume, area, centroid);
}

int rbc_cell_metrics_async(rbc_handle *h, double *out)
{
    if (!h || !out) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    CellGroup &g = h->cg[0];
    if (h->ncell == 0) return fail(h, RBC_ERR_STATE, "handle has no cells");
    const int N = g.ncell;
    const double *cen = g.gx;
    if (!h->metrics_valid) {   // as group_metrics: measure the current positions
        launch_volume(h->geo, volume_args(h, g, 0), h->stream);
        h->launches++;
        CK_LAUNCH();
        cen = g.cen_out;
    }
    CK(cudaMemcpyAsync(out, g.vol_out, 8 * (size_t)N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(out + N, g.area_out, 8 * (size_t)N, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(out + 2 * N, cen, 8 * 3 * (size_t)N, cudaMemcpyDeviceToHost, h->stream));
    return RBC_OK;
}

int rbc_synchronize(rbc_handle *h)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    CK(cudaStreamSynchronize(h->stream));
    return RBC_OK;
}

int rbc_launch_count(const rbc_handle *h, long long *count)
{
    if (!h || !count) return RBC_ERR_ARG;
    *count = h->launches;
    return RBC_OK;
}

int rbc_dims(const rbc_handle *h, int *nx, int *ny, int *nz_periodic, int *ncell, int *vertex, int *element)
{
    if (!h) return RBC_ERR_ARG;
    if (nx) *nx = h->geo.nxr;
    if (ny) *ny = h->geo.ny;
    if (nz_periodic) *nz_periodic = h->geo.nzc;
    if (ncell) *ncell = h->ncell;
    if (vertex) *vertex = h->V;
    if (element) *element = h->E;
    return RBC_OK;
}

// ---- batches ----------------------------------------------------------------

int rbc_batch_create(rbc_handle *const *handles, int n, rbc_batch **out)
{
    g_create_error.clear();
    if (!out) return fail(nullptr, RBC_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!handles || n <= 0) return fail(nullptr, RBC_ERR_ARG, "a batch needs at least one simulation");
    for (int i = 0; i < n; i++) {
        if (!handles[i]) return fail(nullptr, RBC_ERR_ARG, "simulation " + std::to_string(i) + " is NULL");
        if (handles[i]->device != handles[0]->device)
            return fail(nullptr, RBC_ERR_ARG, "all simulations of a batch must use the same device");
        for (int j = 0; j < i; j++)
            if (handles[j] == handles[i]) return fail(nullptr, RBC_ERR_ARG, "a simulation appears twice in the batch");
        if (handles[i]->vof())
            return fail(nullptr, RBC_ERR_UNSUPPORTED, "batched simulations do not track the volume fraction (needs vof_k = 0)");
        if (handles[i]->p.M != 1)
            return fail(nullptr, RBC_ERR_UNSUPPORTED, "batched simulations step with M = 1 (no sub-cycling)");
    }
    rbc_batch *b = new (std::nothrow) rbc_batch();
    if (!b) return fail(nullptr, RBC_ERR_ARG, "out of host memory");
    b->h.assign(handles, handles + n);
    b->base_cur.assign(n, 0);
    b->device = handles[0]->device;
    auto bail = [&](int code, const std::string &msg) {
        g_create_error = msg;
        rbc_batch_destroy(b);
        return code;
    };
    if (cudaSetDevice(b->device) != cudaSuccess) return bail(RBC_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
        return bail(RBC_ERR_CUDA, "stream creation failed");
    b->ready.assign(n, nullptr);
    for (int i = 0; i < n; i++)
        if (cudaEventCreateWithFlags(&b->ready[i], cudaEventDisableTiming) != cudaSuccess)
            return bail(RBC_ERR_CUDA, "event creation failed");
    *out = b;
    return RBC_OK;
}

int rbc_batch_destroy(rbc_batch *b)
{
    if (!b) return RBC_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_free_graphs(b);
    for (cudaEvent_t e : b->ready) if (e) cudaEventDestroy(e);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return RBC_OK;
}

const char *rbc_batch_last_error(const rbc_batch *b)
{
    return b ? b->err.c_str() : g_create_error.c_str();
}

int rbc_batch_set_chain(rbc_batch *b, int chain)
{
    if (!b || chain < 1) return RBC_ERR_ARG;
    if (chain != b->chain) { b->chain = chain; batch_free_graphs(b); }
    return RBC_OK;
}

int rbc_batch_get_chain(const rbc_batch *b, int *chain)
{
    if (!b || !chain) return RBC_ERR_ARG;
    *chain = b->chain;
    return RBC_OK;
}

int rbc_batch_step(rbc_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return RBC_ERR_ARG;
    if (nsteps == 0) return RBC_OK;
    CKB(cudaSetDevice(b->device));
    const int n = (int)b->h.size();
    // a simulation stepped on its own since the graphs were built has another buffer parity
    bool stale = !b->graph[0] || !b->graph[1];
    for (int i = 0; i < n && !stale; i++) stale = b->h[i]->cur != (b->base_cur[i] ^ b->parity);
    int rc;
    if (stale && (rc = batch_build(b))) return rc;
    for (int i = 0; i < n; i++) {
        rbc_handle *h = b->h[i];
        if ((rc = prepare_steps(h))) { b->err = "simulation " + std::to_string(i) + ": " + h->err; return rc; }
        CKB(cudaEventRecord(b->ready[i], h->stream));
        CKB(cudaStreamWaitEvent(b->stream, b->ready[i], 0));
    }
    for (int k = 0; k < nsteps; k++) {
        CKB(cudaGraphLaunch(b->graph[b->parity], b->stream));
        b->parity ^= 1;
    }
    CKB(cudaEventRecord(b->done, b->stream));
    if (b->fused) b->launches += (long long)FUSED_KERNELS_PER_STEP * nsteps;
    for (int i = 0; i < n; i++) {
        rbc_handle *h = b->h[i];
        if (nsteps & 1) h->cur ^= 1;
        h->iter += nsteps;
        if (!b->fused) {   // the batch graph ran each simulation's own step kernels
            h->launches += (long long)h->kernels_per_step() * nsteps;
            b->launches += (long long)h->kernels_per_step() * nsteps;
        }
        h->metrics_valid = h->has_cells();   // each simulation's step ends with its volume correction
        CKB(cudaStreamWaitEvent(h->stream, b->done, 0));
    }
    return RBC_OK;
}

int rbc_batch_get_stream(const rbc_batch *b, void **stream)
{
    if (!b || !stream) return RBC_ERR_ARG;
    *stream = (void *)b->stream;
    return RBC_OK;
}

int rbc_batch_synchronize(rbc_batch *b)
{
    if (!b) return RBC_ERR_ARG;
    CKB(cudaSetDevice(b->device));
    CKB(cudaStreamSynchronize(b->stream));
    return RBC_OK;
}

namespace {

// device time of steps_per_trial batch steps after one untimed step (which
// builds the graphs); -1 on an error
float batch_trial(rbc_batch *b, int steps_per_trial, cudaEvent_t t0, cudaEvent_t t1, int *rc)
{
    if ((*rc = rbc_batch_step(b, 1))) return -1.f;
    if (cudaEventRecord(t0, b->stream) != cudaSuccess) { *rc = RBC_ERR_CUDA; return -1.f; }
    if ((*rc = rbc_batch_step(b, steps_per_trial))) return -1.f;
    float ms = 0.f;
    if (cudaEventRecord(t1, b->stream) != cudaSuccess || cudaEventSynchronize(t1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, t0, t1) != cudaSuccess) { *rc = RBC_ERR_CUDA; return -1.f; }
    return ms;
}

}  // namespace

int rbc_batch_autotune(rbc_batch *b, int steps_per_trial, int *chain_out)
{
    if (!b || steps_per_trial < 1) return RBC_ERR_ARG;
    CKB(cudaSetDevice(b->device));
    const int n = (int)b->h.size();
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    CKB(cudaEventCreate(&t0));
    CKB(cudaEventCreate(&t1));
    int rc = RBC_OK;
    if (b->use_fused && fused_obstacle(b).empty()) {
        // fused form: the launch shapes, each tried for steps_per_trial steps --
        // collide-stream threads per block and planes per thread, membrane
        // vertices per thread (the one-simulation choice and the next larger)
        int V = 0;
        for (rbc_handle *h : b->h) if (h->cg[0].ncell > 0) V = h->cg[0].V;
        const int v0 = V > 0 ? membrane_default_vpt(V) : 1;
        int best[3] = {b->lbm_threads, b->lbm_planes, b->mem_vpt};
        float best_ms = -1.f;
        for (int tpb : {128, 256})
            for (int planes : {1, 2, 4})
                for (int vpt : {v0, std::min(v0 + 1, 4)}) {
                    if (vpt != v0 && vpt == std::min(v0 + 1, 4) && v0 == 4) continue;
                    b->lbm_threads = tpb; b->lbm_planes = planes; b->mem_vpt = vpt;
                    batch_free_graphs(b);
                    const float ms = batch_trial(b, steps_per_trial, t0, t1, &rc);
                    if (rc != RBC_OK) break;
                    if (best_ms < 0.f || ms < best_ms) { best_ms = ms; best[0] = tpb; best[1] = planes; best[2] = vpt; }
                }
        b->lbm_threads = best[0]; b->lbm_planes = best[1]; b->mem_vpt = best[2];
        batch_free_graphs(b);
    } else {
        // child graphs: the simulations per dependency chain
        int best = b->chain;
        float best_ms = 0.f;
        for (int chain = 1; chain <= n && rc == RBC_OK; chain *= 2) {
            if ((rc = rbc_batch_set_chain(b, chain))) break;
            const float ms = batch_trial(b, steps_per_trial, t0, t1, &rc);
            if (rc != RBC_OK) break;
            if (chain == 1 || ms < best_ms) { best_ms = ms; best = chain; }
            if (chain >= 64) break;   // longer chains only serialise more
        }
        if (rc == RBC_OK) rc = rbc_batch_set_chain(b, best);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != RBC_OK) return rc;
    if (chain_out) *chain_out = b->chain;
    return RBC_OK;
}

int rbc_batch_set_form(rbc_batch *b, int fused)
{
    if (!b || (fused != 0 && fused != 1)) return RBC_ERR_ARG;
    if (fused != b->use_fused) { b->use_fused = fused; batch_free_graphs(b); }
    return RBC_OK;
}

int rbc_batch_get_form(const rbc_batch *b, int *fused, const char **obstacle)
{
    if (!b) return RBC_ERR_ARG;
    static thread_local std::string why;
    why = fused_obstacle(b);
    if (fused) *fused = (b->use_fused && why.empty()) ? 1 : 0;
    if (obstacle) *obstacle = why.c_str();
    return RBC_OK;
}

int rbc_batch_set_shape(rbc_batch *b, int lbm_threads, int lbm_planes, int membrane_vpt)
{
    if (!b || (lbm_threads != 128 && lbm_threads != 256) || lbm_planes < 0 || lbm_planes > 8 ||
        membrane_vpt < 0 || membrane_vpt > 4) return RBC_ERR_ARG;
    if (membrane_vpt > 0) {   // the membrane block must fit its thread limit
        for (rbc_handle *h : b->h)
            if (h->cg[0].ncell > 0 && h->cg[0].V > 0 &&
                membrane_threads(h->cg[0].V, membrane_vpt) > (membrane_vpt >= 3 ? 896 : 1024))
                return RBC_ERR_ARG;
    }
    b->lbm_threads = lbm_threads; b->lbm_planes = lbm_planes; b->mem_vpt = membrane_vpt;
    batch_free_graphs(b);
    return RBC_OK;
}

int rbc_batch_get_shape(const rbc_batch *b, int *lbm_threads, int *lbm_planes, int *membrane_vpt)
{
    if (!b) return RBC_ERR_ARG;
    if (lbm_threads) *lbm_threads = b->lbm_threads;
    if (lbm_planes) *lbm_planes = b->lbm_planes;
    if (membrane_vpt) *membrane_vpt = b->mem_vpt;
    return RBC_OK;
}

int rbc_batch_launch_count(const rbc_batch *b, long long *count)
{
    if (!b || !count) return RBC_ERR_ARG;
    *count = b->launches;
    return RBC_OK;
}

}  // extern "C"

// ---- adjoint: checkpointed reverse sweep -----------------------------------
//
// rbc_adjoint_record runs the forward steps with the step graphs and keeps a
// checkpoint of the state (populations, cel->x, fem->xd, centroids, iter)
// every K steps, plus the state after the run.  rbc_adjoint_backward then
// takes the segments in reverse order: it restores a segment's checkpoint,
// recomputes the segment stage by stage while storing what the reverse stages
// read (populations, positions, membrane forces, lattice force, velocity
// field, positions before the correction, drive), and runs the adjoint
// kernels of adjoint.cu backwards through the segment.  Two segment stores
// alternate: the recomputation of segment s - 1 (handle stream) runs while
// segment s is reversed (adjoint stream), and each segment's recomputation
// and reversal are CUDA graphs, captured once per (store, buffer parity,
// length) and replayed.  Device memory: nsteps / K + 1 checkpoints
// (4 Q B per node + 48 B per vertex) and 2 K steps of stored stages
// (104 B per node + 84 B per vertex).

// Binomial checkpointing (rbc_adjoint_record_binomial): the run is cut into
// units of `unit` steps and reversed unit by unit under the schedule of
// binomial (revolve) checkpointing with S snapshot slots beside the initial
// state (A. Griewank, A. Walther, "Algorithm 799: revolve", ACM TOMS 26,
// 2000).  To reverse units [a, b) from the state at a (held in a slot) with s
// free slots: one unit is recorded and reversed at once; with no free slot,
// each unit t from b - 1 down is reached by restoring a and advancing t - a
// units; otherwise the state is advanced to m = a + N(s, r - 1), kept in a new
// slot, [m, b) is reversed with s - 1 slots, a is restored and [a, m) is
// reversed with s slots.  r is the least repetition count with N(s, r) >= b - a,
// where N(s, r) = C(s + r + 1, s + 1) is the most units that s free slots
// reverse when no unit is advanced more than r times, so every unit is
// advanced at most r times before its recording.
struct AdjAction { int op, arg; };
enum { ADJ_ADVANCE, ADJ_SNAP, ADJ_RESTORE, ADJ_RECORD, ADJ_REVERSE };

struct AdjointState {
    int K = 0, nseg_cap = 0, K_cap = 0;
    int nsteps = 0, nseg = 0;
    bool valid = false;
    // schedule: 0 = a checkpoint every K steps; 1 = binomial over units of K steps
    int mode = 0;
    int nunits = 0, snaps = 0, final_slot = 0;
    std::vector<AdjAction> plan;         // binomial: the backward sweep's actions
    long long advanced_units = 0;        // binomial: units advanced by the last backward sweep
    std::vector<int> ck_iter;            // iter at each checkpoint
    std::vector<void *> bufs;            // every allocation below, for adjoint_free
    // checkpoints [nseg + 1]
    float *ck_g = nullptr; double *ck_X = nullptr, *ck_Xd = nullptr, *ck_gx = nullptr;
    int *ck_itd = nullptr;               // the device iteration counter at each checkpoint
    // stored stages of two segments [2][K]
    float *sg = nullptr, *sF = nullptr, *sFv = nullptr, *sdrv = nullptr; float4 *suvr = nullptr;
    double *sX = nullptr, *sXd = nullptr, *sXa = nullptr, *sgx = nullptr, *sfac = nullptr;
    // adjoint state and scratch
    float *gbar[2] = {nullptr, nullptr}, *Fbar = nullptr; float4 *ubar = nullptr;
    float4 *lam = nullptr, *qv = nullptr; float *dsb = nullptr;
    double *Xbar = nullptr, *Xdbar = nullptr, *Xabar = nullptr, *Fvbar = nullptr;
    double *mscr = nullptr, *hist = nullptr, *escr = nullptr, *pbar = nullptr;
    int *status = nullptr;
    // outputs of the last recorded step (velocity field, vertex velocities and forces)
    float4 *fin_uvr = nullptr; float *fin_U = nullptr, *fin_Fv = nullptr;
    int kmax = 16;                       // volume-correction moves reversed per step
    // reverse stream, store events, graphs keyed by (kind, store, parity, length)
    cudaStream_t rev = nullptr;
    cudaEvent_t filled[2] = {nullptr, nullptr}, drained[2] = {nullptr, nullptr};
    std::map<long long, cudaGraphExec_t> graphs;
    std::map<long long, long long> graph_kernels;   // kernels each graph launches
};

void adjoint_drop_graphs(AdjointState *a)
{
    for (auto &kv : a->graphs) if (kv.second) cudaGraphExecDestroy(kv.second);
    a->graphs.clear();
    a->graph_kernels.clear();
}

void adjoint_free(AdjointState *a)
{
    if (!a) return;
    adjoint_drop_graphs(a);
    for (void *p : a->bufs) if (p) cudaFree(p);
    for (cudaEvent_t e : {a->filled[0], a->filled[1], a->drained[0], a->drained[1]}) if (e) cudaEventDestroy(e);
    if (a->rev) cudaStreamDestroy(a->rev);
    delete a;
}

namespace {

template <typename T>
int adj_alloc(rbc_handle *h, T **p, size_t count)
{
    CK(cudaMalloc((void **)p, sizeof(T) * (count ? count : 1)));
    h->adj->bufs.push_back((void *)*p);
    return RBC_OK;
}

// checkpoint and segment buffers for nseg segments of K steps
int adjoint_reserve(rbc_handle *h, int K, int nseg)
{
    if (!h->adj) h->adj = new (std::nothrow) AdjointState();
    if (!h->adj) return fail(h, RBC_ERR_CUDA, "out of host memory");
    AdjointState *a = h->adj;
    if (!a->rev) {
        CK(cudaStreamCreateWithFlags(&a->rev, cudaStreamNonBlocking));
        for (int b = 0; b < 2; b++) {
            CK(cudaEventCreateWithFlags(&a->filled[b], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&a->drained[b], cudaEventDisableTiming));
        }
    }
    if (a->K_cap >= K && a->nseg_cap >= nseg) return RBC_OK;
    adjoint_drop_graphs(a);
    for (void *p : a->bufs) if (p) cudaFree(p);
    a->bufs.clear();
    a->K_cap = a->nseg_cap = 0;
    const size_t n = (size_t)h->geo.nint, nq = (size_t)Q * n, nv3 = 3 * (size_t)h->nv, N3 = 3 * (size_t)h->ncell;
    const size_t nck = (size_t)nseg + 1, S = 2 * (size_t)K;
    int rc;
#define TRYA(x) do { if ((rc = (x))) { h->err = "adjoint: out of device memory (" #x ")"; return rc; } } while (0)
    TRYA(adj_alloc(h, &a->ck_g, nck * nq)); TRYA(adj_alloc(h, &a->ck_X, nck * nv3));
    TRYA(adj_alloc(h, &a->ck_Xd, nck * nv3)); TRYA(adj_alloc(h, &a->ck_gx, nck * N3));
    TRYA(adj_alloc(h, &a->ck_itd, nck));
    TRYA(adj_alloc(h, &a->sg, S * nq)); TRYA(adj_alloc(h, &a->sF, S * 3 * n)); TRYA(adj_alloc(h, &a->sFv, S * nv3));
    TRYA(adj_alloc(h, &a->suvr, S * n)); TRYA(adj_alloc(h, &a->sdrv, S)); TRYA(adj_alloc(h, &a->sfac, S));
    TRYA(adj_alloc(h, &a->sX, S * nv3)); TRYA(adj_alloc(h, &a->sXd, S * nv3)); TRYA(adj_alloc(h, &a->sXa, S * nv3));
    TRYA(adj_alloc(h, &a->sgx, S * N3));
    TRYA(adj_alloc(h, &a->gbar[0], nq)); TRYA(adj_alloc(h, &a->gbar[1], nq));
    TRYA(adj_alloc(h, &a->lam, h->nv)); TRYA(adj_alloc(h, &a->qv, h->nv)); TRYA(adj_alloc(h, &a->dsb, h->nv));
    TRYA(adj_alloc(h, &a->Fbar, 3 * n)); TRYA(adj_alloc(h, &a->ubar, n));
    TRYA(adj_alloc(h, &a->Xbar, nv3)); TRYA(adj_alloc(h, &a->Xdbar, nv3)); TRYA(adj_alloc(h, &a->Xabar, nv3));
    TRYA(adj_alloc(h, &a->Fvbar, nv3)); TRYA(adj_alloc(h, &a->mscr, 7 * (size_t)h->ne));
    TRYA(adj_alloc(h, &a->hist, (size_t)a->kmax * nv3)); TRYA(adj_alloc(h, &a->escr, 9 * (size_t)h->ne));
    TRYA(adj_alloc(h, &a->pbar, 4)); TRYA(adj_alloc(h, &a->status, 1));
    TRYA(adj_alloc(h, &a->fin_uvr, n)); TRYA(adj_alloc(h, &a->fin_U, nv3)); TRYA(adj_alloc(h, &a->fin_Fv, nv3));
#undef TRYA
    a->K_cap = K;
    a->nseg_cap = nseg;
    return RBC_OK;
}

int d2d(rbc_handle *h, void *dst, const void *src, size_t bytes, cudaStream_t st = nullptr)
{
    if (bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st ? st : h->stream));
    return RBC_OK;
}

// state <-> checkpoint k
int adjoint_save(rbc_handle *h, int k)
{
    AdjointState *a = h->adj;
    const size_t nq = (size_t)Q * h->geo.nint, nv3 = 3 * (size_t)h->nv, N3 = 3 * (size_t)h->ncell;
    int rc;
    if ((rc = d2d(h, a->ck_g + k * nq, h->g[h->cur], 4 * nq))) return rc;
    if ((rc = d2d(h, a->ck_X + k * nv3, h->X, 8 * nv3))) return rc;
    if ((rc = d2d(h, a->ck_Xd + k * nv3, h->Xd, 8 * nv3))) return rc;
    if ((rc = d2d(h, a->ck_gx + k * N3, h->gx, 8 * N3))) return rc;
    if ((rc = d2d(h, a->ck_itd + k, h->d_iter(), sizeof(int)))) return rc;
    a->ck_iter[k] = h->iter;
    return RBC_OK;
}

int adjoint_restore(rbc_handle *h, int k)
{
    AdjointState *a = h->adj;
    const size_t n = (size_t)h->geo.nint, nq = (size_t)Q * n, nv3 = 3 * (size_t)h->nv, N3 = 3 * (size_t)h->ncell;
    int rc;
    if ((rc = d2d(h, h->g[h->cur], a->ck_g + k * nq, 4 * nq))) return rc;
    if ((rc = d2d(h, h->X, a->ck_X + k * nv3, 8 * nv3))) return rc;
    if ((rc = d2d(h, h->Xd, a->ck_Xd + k * nv3, 8 * nv3))) return rc;
    if ((rc = d2d(h, h->gx, a->ck_gx + k * N3, 8 * N3))) return rc;
    CK(cudaMemsetAsync(h->Fint, 0, 24 * n, h->stream));
    CK(cudaMemsetAsync(h->Fbits, 0, h->force_bit_bytes(), h->stream));
    h->force_pending = false;
    h->iter = a->ck_iter[k];
    return d2d(h, h->d_iter(), a->ck_itd + k, sizeof(int));   // device to device: no host staging
}


// Enqueue the recomputation of len steps from the handle's state into store b
// (stream: the handle's).
int adjoint_enqueue_recompute_body(rbc_handle *h, int b, int len);

int adjoint_enqueue_recompute(rbc_handle *h, int b, int len)
{
    // the recomputation repeats past steps: it must not add to the output averages again
    const int f = h->fileoutput;
    h->fileoutput = 0;
    const int rc = adjoint_enqueue_recompute_body(h, b, len);
    h->fileoutput = f;
    return rc;
}

int adjoint_enqueue_recompute_body(rbc_handle *h, int b, int len)
{
    AdjointState *a = h->adj;
    const size_t n = (size_t)h->geo.nint, nq = (size_t)Q * n, nv3 = 3 * (size_t)h->nv, N3 = 3 * (size_t)h->ncell;
    int rc;
    for (int t = 0; t < len; t++) {
        const size_t k = (size_t)b * a->K + t;
        if ((rc = d2d(h, a->sg + k * nq, h->g[h->cur], 4 * nq))) return rc;
        if ((rc = d2d(h, a->sX + k * nv3, h->X, 8 * nv3))) return rc;
        if ((rc = d2d(h, a->sXd + k * nv3, h->Xd, 8 * nv3))) return rc;
        if ((rc = d2d(h, a->sgx + k * N3, h->gx, 8 * N3))) return rc;
        StepBeginArgs sb = step_begin_args(h);
        sb.drive_rec = a->sdrv + k;
        sb.factor_rec = a->sfac + k;
        launch_step_begin(sb, h->stream);
        h->launches++;
        CK_LAUNCH();
        if ((rc = launch_stress(h))) return rc;
        if ((rc = d2d(h, a->sFv + k * nv3, h->Fv, 4 * nv3))) return rc;
        if ((rc = launch_spread_stage(h))) return rc;
        launch_force_to_f32(h->geo, h->Fint, a->sF + k * 3 * n, h->stream);   // the force the collision reads
        h->launches++;
        CK_LAUNCH();
        if ((rc = launch_lbm_stage(h))) return rc;
        if ((rc = d2d(h, a->suvr + k * n, h->uvr, 16 * n))) return rc;
        if ((rc = launch_advect_stage(h))) return rc;
        if ((rc = d2d(h, a->sXa + k * nv3, h->Xd, 8 * nv3))) return rc;
        if ((rc = launch_volume_stage(h, h->stream))) return rc;
    }
    return RBC_OK;
}

// Enqueue the reverse of len steps stored in store b (stream: a->rev); the
// adjoint of the populations after them is in gbar[gb] and ends in
// gbar[gb ^ (len & 1)].
int adjoint_enqueue_reverse(rbc_handle *h, int b, int len, int gb)
{
    AdjointState *a = h->adj;
    const size_t n = (size_t)h->geo.nint, nq = (size_t)Q * n, nv3 = 3 * (size_t)h->nv, N3 = 3 * (size_t)h->ncell;
    const Geom &g = h->geo;
    cudaStream_t st = a->rev;
    for (int t = len - 1; t >= 0; t--) {
        const size_t k = (size_t)b * a->K + t;
        if (h->ncell > 0) {
            VolumeAdjArgs va{};
            va.Xa = a->sXa + k * nv3; va.gx = a->sgx + k * N3; va.vol0 = h->vol0;
            va.tri = h->tri; va.v2e_off = h->v2e_off; va.v2e = h->v2e;
            va.X_bar = a->Xbar; va.Xd_bar = a->Xdbar; va.Xa_bar = a->Xabar;
            va.hist = a->hist; va.escr = a->escr; va.status = a->status;
            va.nv = h->nv; va.V = h->V; va.E = h->E; va.ncell = h->ncell; va.kmax = a->kmax;
            launch_volume_adjoint(g, va, st);
            h->launches++;
            CK_LAUNCH();
        }
        CK(cudaMemsetAsync(a->ubar, 0, 16 * n, st));
        if (h->ncell > 0) {
            launch_advect_adjoint(g, a->sX + k * nv3, a->suvr + k * n, a->Xabar, a->Xbar, (float *)a->ubar, h->nv,
                                  h->p.dt * h->p.M, h->d_flags(), st);
            h->launches++;
            CK_LAUNCH();
        }
        LbmAdjArgs la{};
        la.gin = a->sg + k * nq;
        la.Fx = a->sF + k * 3 * n; la.Fy = la.Fx + n; la.Fz = la.Fx + 2 * n;
        la.mask2d = h->mask2d; la.gbar_out = a->gbar[gb]; la.ubar = a->ubar;
        la.gbar_in = a->gbar[gb ^ 1]; la.Fbar = a->Fbar; la.pbar = a->pbar;
        la.pd = a->sdrv + k; la.dfac = a->sfac + k;
        la.Bc = (float)h->p.B; la.omega = (float)(1.0 / h->p.tau); la.Cr = (float)h->p.Cr;
        launch_lbm_adjoint(g, la, st);
        h->launches++;
        CK_LAUNCH();
        gb ^= 1;
        if (h->ncell > 0) {
            launch_spread_adjoint(g, a->sX + k * nv3, a->sFv + k * nv3, a->Fbar, h->mask2d, a->Fvbar, a->Xbar, h->nv, st);
            h->launches++;
            CK_LAUNCH();
            MembraneAdjArgs ma{};
            ma.Xd = a->sXd + k * nv3; ma.nv = h->nv; ma.ne = h->ne; ma.gref = h->gref;
            ma.tri = h->tri; ma.v2e_off = h->v2e_off; ma.v2e = h->v2e; ma.nbr = h->nbr;
            ma.Fv = a->sFv + k * nv3; ma.Fv_bar = a->Fvbar; ma.Xd_bar = a->Xdbar; ma.scratch = a->mscr;
            ma.lam = a->lam; ma.qv = a->qv; ma.dsb = a->dsb;
            ma.cbar = a->pbar + 2;
            ma.V = h->V; ma.E = h->E; ma.ncell = h->ncell;
            ma.C = h->p.C; ma.rgs = h->cg[0].rgs; ma.law = h->p.law; ma.LX = h->p.LX; ma.LZ = h->p.LZ;
            ma.niter = h->p.solver_iters > 0 ? h->p.solver_iters : DEFAULT_SOLVER_ITERS;
            launch_membrane_adjoint(ma, st);
            h->launches += 3;   // the solve, element and vertex passes
            CK_LAUNCH();
        }
    }
    return RBC_OK;
}

// Launch (capturing on first use) the graph of a segment's recomputation
// (kind 0, on the handle stream, keyed by store and population buffer) or
// reversal (kind 1, on the adjoint stream, keyed by store and adjoint buffer).
int adjoint_launch_graph(rbc_handle *h, int kind, int b, int parity, int len)
{
    AdjointState *a = h->adj;
    const long long key = ((long long)len << 3) | (kind << 2) | (b << 1) | parity;
    cudaStream_t st = kind == 0 ? h->stream : a->rev;
    auto it = a->graphs.find(key);
    if (it == a->graphs.end()) {
        const long long launches0 = h->launches;
        const int cur0 = h->cur;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int rc = kind == 0 ? adjoint_enqueue_recompute(h, b, len) : adjoint_enqueue_reverse(h, b, len, parity);
        const cudaError_t e = cudaStreamEndCapture(st, &graph);
        const long long kernels = h->launches - launches0;   // the launches the capture recorded
        h->launches = launches0;
        h->cur = cur0;
        if (rc != RBC_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
        if (e != cudaSuccess) { h->err = std::string("adjoint graph capture: ") + cudaGetErrorString(e); return RBC_ERR_CUDA; }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ei != cudaSuccess) { h->err = std::string("adjoint graph instantiate: ") + cudaGetErrorString(ei); return RBC_ERR_CUDA; }
        it = a->graphs.emplace(key, exec).first;
        a->graph_kernels[key] = kernels;
    }
    CK(cudaGraphLaunch(it->second, st));
    h->launches += a->graph_kernels[key];
    if (kind == 0) {   // the recomputation advanced the handle
        if (len & 1) h->cur ^= 1;
        h->iter += len;
    }
    return RBC_OK;
}

// N(s, r) = C(s + r + 1, s + 1), saturated at 2^40
long long binomial_units(int s, int r)
{
    long double v = 1.0L;
    for (int i = 1; i <= s + 1; i++) {
        v = v * (long double)(r + i) / (long double)i;
        if (v > 1e12L) return 1LL << 40;
    }
    return (long long)(v + 0.5L);
}

// the actions that reverse units [a, b) when the state at a is the current
// one and is held in slot sa, with s free slots above sa
void binomial_plan(int a, int b, int s, int sa, std::vector<AdjAction> &out)
{
    const int n = b - a;
    if (n == 1) { out.push_back({ADJ_RECORD, a}); out.push_back({ADJ_REVERSE, a}); return; }
    if (s == 0) {
        for (int t = b - 1; t >= a; t--) {
            if (t != b - 1) out.push_back({ADJ_RESTORE, sa});
            if (t > a) out.push_back({ADJ_ADVANCE, t - a});
            out.push_back({ADJ_RECORD, t});
            out.push_back({ADJ_REVERSE, t});
        }
        return;
    }
    int r = 0;
    while (binomial_units(s, r) < n) r++;
    const int m = a + (int)binomial_units(s, r - 1);
    out.push_back({ADJ_ADVANCE, m - a});
    out.push_back({ADJ_SNAP, sa + 1});
    binomial_plan(m, b, s - 1, sa + 1, out);
    out.push_back({ADJ_RESTORE, sa});
    binomial_plan(a, m, s, sa, out);
}

int adjoint_supported(rbc_handle *h)
{
    if (h->p.storage != RBC_STORE_F32) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint needs FP32 population storage");
    if (h->cg[0].br != 0.0) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint does not cover bending (BR != 0)");
    if (h->ngroups > 1) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint covers one cell population (no white cells)");
    if (h->geo.nzc > 65535) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint handles at most 65535 periodic planes");
    if (h->p.flow != RBC_FLOW_CHANNEL) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint covers the channel mode only");
    if (h->ntube > 0) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint covers half-way bounce-back walls only (tube_r = 0)");
    if (h->vof()) return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint does not cover the volume fraction (needs vof_k = 0)");
    if (h->p.M != 1 || h->p.rk_order != 4)
        return fail(h, RBC_ERR_UNSUPPORTED, "the adjoint covers M = 1 and RUNGE_KUTTA = 4 only");
    return RBC_OK;
}

}  // namespace

extern "C" {

int rbc_adjoint_record(rbc_handle *h, int nsteps, int ckpt_every)
{
    if (!h || nsteps < 1 || ckpt_every < 1) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    int rc;
    if ((rc = adjoint_supported(h))) return rc;
    const int K = std::min(ckpt_every, nsteps), nseg = (nsteps + K - 1) / K;
    if ((rc = adjoint_reserve(h, K, nseg))) return rc;
    AdjointState *a = h->adj;
    if (a->K != K) adjoint_drop_graphs(a);   // the graphs index the stores by K
    a->valid = false;
    a->mode = 0;
    a->K = K; a->nsteps = nsteps; a->nseg = nseg;
    a->ck_iter.assign(nseg + 1, 0);
    CK(cudaStreamSynchronize(h->stream));
    // a spread force left by rbc_ibm_st1 belongs to no step of the run; the
    // device counter follows the host's
    if ((rc = prepare_steps(h))) return rc;
    for (int s = 0; s < nseg; s++) {
        if ((rc = adjoint_save(h, s))) return rc;
        if ((rc = rbc_step(h, std::min(K, nsteps - s * K)))) return rc;
    }
    if ((rc = adjoint_save(h, nseg))) return rc;
    const size_t nv3 = 3 * (size_t)h->nv;
    if ((rc = d2d(h, a->fin_uvr, h->uvr, 16 * (size_t)h->geo.nint))) return rc;
    if ((rc = d2d(h, a->fin_U, h->U, 4 * nv3))) return rc;
    if ((rc = d2d(h, a->fin_Fv, h->Fv, 4 * nv3))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    a->valid = true;
    return RBC_OK;
}

int rbc_adjoint_record_binomial(rbc_handle *h, int nsteps, int unit, int snaps)
{
    if (!h || nsteps < 1 || unit < 1 || snaps < 0) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    int rc;
    if ((rc = adjoint_supported(h))) return rc;
    const int K = std::min(unit, nsteps), U = (nsteps + K - 1) / K;
    const int S = std::min(snaps, U - 1);
    // slots 0 (the initial state) .. S, and S + 1 for the state after the run
    if ((rc = adjoint_reserve(h, K, S + 1))) return rc;
    AdjointState *a = h->adj;
    if (a->K != K) adjoint_drop_graphs(a);
    a->valid = false;
    a->mode = 1;
    a->K = K; a->nsteps = nsteps; a->nunits = U; a->snaps = S; a->final_slot = S + 1;
    a->ck_iter.assign(S + 2, 0);
    std::vector<AdjAction> full;
    binomial_plan(0, U, S, 0, full);
    CK(cudaStreamSynchronize(h->stream));
    if ((rc = prepare_steps(h))) return rc;
    // the forward run takes the snapshots the schedule takes before its first
    // recording, then runs to the end
    auto steps_of = [&](int u0, int u) { return std::min((long long)(u0 + u) * K, (long long)nsteps) - (long long)u0 * K; };
    if ((rc = adjoint_save(h, 0))) return rc;
    int pos = 0, last_snap = 0, snap_pos = 0;
    size_t i = 0;
    for (; i < full.size() && full[i].op != ADJ_RECORD; i++) {
        if (full[i].op == ADJ_ADVANCE) {
            if ((rc = rbc_step(h, (int)steps_of(pos, full[i].arg)))) return rc;
            pos += full[i].arg;
        } else {   // ADJ_SNAP
            if ((rc = adjoint_save(h, full[i].arg))) return rc;
            last_snap = full[i].arg;
            snap_pos = pos;
        }
    }
    if ((rc = rbc_step(h, (int)steps_of(pos, U - pos)))) return rc;
    if ((rc = adjoint_save(h, a->final_slot))) return rc;
    // the backward sweep restarts from the last snapshot, replays the advances
    // taken after it, then follows the schedule
    a->plan.clear();
    a->plan.push_back({ADJ_RESTORE, last_snap});
    for (size_t j = 0; j < i; j++) {
        if (full[j].op != ADJ_ADVANCE) continue;
        int before = 0;   // position before this advance
        for (size_t k2 = 0; k2 < j; k2++) if (full[k2].op == ADJ_ADVANCE) before += full[k2].arg;
        if (before >= snap_pos) a->plan.push_back(full[j]);
    }
    a->plan.insert(a->plan.end(), full.begin() + i, full.end());
    const size_t nv3 = 3 * (size_t)h->nv;
    if ((rc = d2d(h, a->fin_uvr, h->uvr, 16 * (size_t)h->geo.nint))) return rc;
    if ((rc = d2d(h, a->fin_U, h->U, 4 * nv3))) return rc;
    if ((rc = d2d(h, a->fin_Fv, h->Fv, 4 * nv3))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    a->valid = true;
    return RBC_OK;
}

int rbc_adjoint_binomial_plan(int units, int snaps, int *ops, int *args, int cap, int *len)
{
    if (units < 1 || snaps < 0 || !len || (cap > 0 && (!ops || !args))) return RBC_ERR_ARG;
    std::vector<AdjAction> plan;
    plan.push_back({ADJ_SNAP, 0});   // the initial state in slot 0
    binomial_plan(0, units, std::min(snaps, units - 1), 0, plan);
    *len = (int)plan.size();
    if ((int)plan.size() > cap) return cap > 0 ? RBC_ERR_ARG : RBC_OK;
    for (size_t i = 0; i < plan.size(); i++) { ops[i] = plan[i].op; args[i] = plan[i].arg; }
    return RBC_OK;
}

int rbc_adjoint_schedule(const rbc_handle *h, int *units, int *unit_steps, int *snapshots, long long *advances)
{
    if (!h || !h->adj || !h->adj->valid) return RBC_ERR_STATE;
    const AdjointState *a = h->adj;
    if (units) *units = a->mode == 1 ? a->nunits : a->nseg;
    if (unit_steps) *unit_steps = a->K;
    if (snapshots) *snapshots = a->mode == 1 ? a->snaps + 1 : a->nseg + 1;
    if (advances) {
        long long adv = 0;
        if (a->mode == 1)
            for (const AdjAction &x : a->plan) if (x.op == ADJ_ADVANCE) adv += x.arg;
        *advances = adv;
    }
    return RBC_OK;
}

int rbc_adjoint_backward(rbc_handle *h, const double *xbar, const double *ybar, const double *zbar,
                         double *grad, double *dx0, double *dy0, double *dz0, int *adj_flags, float *ms)
{
    if (!h || !grad) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    AdjointState *a = h->adj;
    if (!a || !a->valid) return fail(h, RBC_ERR_STATE, "rbc_adjoint_backward before rbc_adjoint_record");
    const long long nv = h->nv;
    const size_t n = (size_t)h->geo.nint, nq = (size_t)Q * n, nv3 = 3 * (size_t)nv;
    int rc;
    CK(cudaStreamSynchronize(h->stream));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // seeds: adjoint of the final cel->x; nothing depends on the final populations or fem->xd
    std::vector<double> seed(nv3, 0.0);
    const double *in[3] = {xbar, ybar, zbar};
    for (int c = 0; c < 3; c++) if (in[c]) std::copy(in[c], in[c] + nv, seed.begin() + c * nv);
    if (nv > 0) CK(cudaMemcpy(a->Xbar, seed.data(), 8 * nv3, cudaMemcpyHostToDevice));
    CK(cudaEventRecord(e0, h->stream));
    if (nv > 0) CK(cudaMemsetAsync(a->Xdbar, 0, 8 * nv3, h->stream));
    CK(cudaMemsetAsync(a->gbar[0], 0, 4 * nq, h->stream));
    CK(cudaMemsetAsync(a->pbar, 0, 4 * sizeof(double), h->stream));
    CK(cudaMemsetAsync(a->status, 0, sizeof(int), h->stream));
    // the adjoint stream starts after the initialisation; both stores start drained
    CK(cudaEventRecord(a->drained[0], h->stream));
    CK(cudaEventRecord(a->drained[1], h->stream));
    int gb = 0;
    if (a->mode == 1) {
        // binomial schedule: recordings alternate between the two stores, so the
        // recording of a unit (handle stream) runs while the unit recorded
        // before it is reversed (adjoint stream)
        auto unit_len = [&](int t) { return std::min(a->K, a->nsteps - t * a->K); };
        int pos = 0, nrec = 0, store = 0, last_store = 0;
        for (const AdjAction &x : a->plan) {
            switch (x.op) {
            case ADJ_RESTORE:
                if ((rc = adjoint_restore(h, x.arg))) return rc;
                pos = a->ck_iter[x.arg] - a->ck_iter[0];
                pos = pos / a->K;
                break;
            case ADJ_SNAP:
                if ((rc = adjoint_save(h, x.arg))) return rc;
                break;
            case ADJ_ADVANCE: {
                const int steps = std::min((pos + x.arg) * a->K, a->nsteps) - pos * a->K;
                if ((rc = rbc_step(h, steps))) return rc;
                pos += x.arg;
                break;
            }
            case ADJ_RECORD:
                store = nrec++ & 1;
                CK(cudaStreamWaitEvent(h->stream, a->drained[store], 0));
                if ((rc = adjoint_launch_graph(h, 0, store, h->cur, unit_len(x.arg)))) return rc;
                CK(cudaEventRecord(a->filled[store], h->stream));
                pos = x.arg + 1;
                last_store = store;
                break;
            case ADJ_REVERSE:
                CK(cudaStreamWaitEvent(a->rev, a->filled[last_store], 0));
                if ((rc = adjoint_launch_graph(h, 1, last_store, gb, unit_len(x.arg)))) return rc;
                gb ^= unit_len(x.arg) & 1;
                CK(cudaEventRecord(a->drained[last_store], a->rev));
                break;
            }
        }
        CK(cudaStreamWaitEvent(h->stream, a->drained[0], 0));
        CK(cudaStreamWaitEvent(h->stream, a->drained[1], 0));
    } else {
        auto seg_len = [&](int s) { return std::min(a->K, a->nsteps - s * a->K); };
        // segment s uses store (nseg - 1 - s) & 1
        if ((rc = adjoint_restore(h, a->nseg - 1))) return rc;
        if ((rc = adjoint_launch_graph(h, 0, 0, h->cur, seg_len(a->nseg - 1)))) return rc;
        CK(cudaEventRecord(a->filled[0], h->stream));
        for (int s = a->nseg - 1; s >= 0; s--) {
            const int b = (a->nseg - 1 - s) & 1;
            CK(cudaStreamWaitEvent(a->rev, a->filled[b], 0));
            if ((rc = adjoint_launch_graph(h, 1, b, gb, seg_len(s)))) return rc;
            gb ^= seg_len(s) & 1;
            CK(cudaEventRecord(a->drained[b], a->rev));
            if (s > 0) {   // recompute segment s - 1 into the other store while segment s is reversed
                CK(cudaStreamWaitEvent(h->stream, a->drained[b ^ 1], 0));
                if ((rc = adjoint_restore(h, s - 1))) return rc;
                if ((rc = adjoint_launch_graph(h, 0, b ^ 1, h->cur, seg_len(s - 1)))) return rc;
                CK(cudaEventRecord(a->filled[b ^ 1], h->stream));
            }
        }
        CK(cudaStreamWaitEvent(h->stream, a->drained[(a->nseg - 1) & 1], 0));
    }
    CK(cudaEventRecord(e1, h->stream));
    double pb[4];
    int st = 0;
    CK(cudaMemcpyAsync(pb, a->pbar, sizeof(pb), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(&st, a->status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    std::vector<double> x0(nv > 0 ? 2 * nv3 : 0);
    if (nv > 0 && (dx0 || dy0 || dz0)) {
        CK(cudaMemcpyAsync(x0.data(), a->Xbar, 8 * nv3, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(x0.data() + nv3, a->Xdbar, 8 * nv3, cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    grad[0] = pb[0]; grad[1] = pb[1]; grad[2] = pb[2];
    double *outs[3] = {dx0, dy0, dz0};
    for (int c = 0; c < 3; c++)
        if (outs[c]) for (long long j = 0; j < nv; j++) outs[c][j] = x0[c * nv + j] + x0[nv3 + c * nv + j];
    if (adj_flags) *adj_flags = st;
    if (ms) *ms = t;
    // leave the handle at the end of the recorded run
    if ((rc = adjoint_restore(h, a->mode == 1 ? a->final_slot : a->nseg))) return rc;
    if ((rc = d2d(h, h->uvr, a->fin_uvr, 16 * n))) return rc;
    if ((rc = d2d(h, h->U, a->fin_U, 4 * nv3))) return rc;
    if ((rc = d2d(h, h->Fv, a->fin_Fv, 4 * nv3))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return RBC_OK;
}

int rbc_set_coefficients(rbc_handle *h, double P, double B, double C)
{
    if (!h || !std::isfinite(P) || !std::isfinite(B) || !std::isfinite(C)) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    CK(cudaStreamSynchronize(h->stream));
    h->p.P = P; h->p.B = B; h->p.C = C;
    // the step graphs and the adjoint graphs hold the coefficients as kernel arguments
    for (auto &form : h->graph)
        for (cudaGraphExec_t &g : form) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    if (h->adj) {
        h->adj->valid = false;
        adjoint_drop_graphs(h->adj);
    }
    return RBC_OK;
}

int rbc_set_launch_shape(rbc_handle *h, int what, int value)
{
    if (!h) return RBC_ERR_ARG;
    if (what != RBC_SHAPE_LBM_PLANES) return fail(h, RBC_ERR_ARG, "unknown launch shape");
    if (value != 0 && value != 1 && value != 2 && value != 4 && value != 8)
        return fail(h, RBC_ERR_ARG, "RBC_SHAPE_LBM_PLANES takes 0 (automatic), 1, 2, 4 or 8");
    RBC_DEVICE_GUARD_RO(h);
    if (value == h->lbm_planes) return RBC_OK;
    CK(cudaStreamSynchronize(h->stream));
    h->lbm_planes = value;
    // the step graphs hold the launch configuration
    for (auto &form : h->graph)
        for (cudaGraphExec_t &g : form) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    if (h->adj) adjoint_drop_graphs(h->adj);
    return RBC_OK;
}

int rbc_get_launch_shape(const rbc_handle *h, int what, int *value)
{
    if (!h || !value || what != RBC_SHAPE_LBM_PLANES) return RBC_ERR_ARG;
    *value = h->lbm_planes;
    return RBC_OK;
}

}  // extern "C"

// ---- output-interval averages and the reference bc map (for ref_files.cu) ---

namespace rbc {

// expand2pow2 (etc.cu:425-446): the reference's per-cell vector length for 3 V values
int reference_mn(int V)
{
    int n = 3 * V, cnt = 0;
    while (n > 1) {
        if (n % 2 == 1) n += 1;
        n /= 2;
        cnt++;
    }
    return 1 << cnt;
}

// fem->qi [ncell * mn] and fem->tp [2 ne] of population `group` to (set = false)
// or from (set = true) host arrays; zeros when no output interval is set
int output_averages(rbc_handle *h, int group, double *qi, double *tp, bool set)
{
    RBC_DEVICE_GUARD(h);
    CellGroup &g = h->cg[group];
    const size_t nq = (size_t)g.ncell * reference_mn(g.V), nt = 2 * (size_t)g.ne;
    CK(cudaStreamSynchronize(h->stream));
    if (!g.qi_acc) {
        if (!set) {
            if (qi) std::fill(qi, qi + nq, 0.0);
            if (tp) std::fill(tp, tp + nt, 0.0);
        }
        return RBC_OK;
    }
    if (set) {
        if (qi) CK(cudaMemcpy(g.qi_acc, qi, 8 * nq, cudaMemcpyHostToDevice));
        if (tp) CK(cudaMemcpy(g.tp_acc, tp, 8 * nt, cudaMemcpyHostToDevice));
    } else {
        if (qi) CK(cudaMemcpy(qi, g.qi_acc, 8 * nq, cudaMemcpyDeviceToHost));
        if (tp) CK(cudaMemcpy(tp, g.tp_acc, 8 * nt, cudaMemcpyDeviceToHost));
    }
    return RBC_OK;
}

// The reference's bc map [nz][ny][nx] of this handle: WALL off the fluid
// columns, COMP on them in the periodic planes, BUFF in the two planes at
// each z end (the structure rbc_create accepted).
int reference_bc(rbc_handle *h, int *bc)
{
    RBC_DEVICE_GUARD(h);
    const Geom &g = h->geo;
    std::vector<uint32_t> mask(g.plane);
    CK(cudaMemcpy(mask.data(), h->mask2d, 4 * g.plane, cudaMemcpyDeviceToHost));
    const int nz = h->p.nz, nxr = g.nxr;
    const long long pr = (long long)nxr * g.ny;
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < g.ny; y++)
            for (int xr = 0; xr < nxr; xr++) {
                // x BUFF columns (shear mode) are periodic images of the internal columns
                const int x = g.xper ? ((xr - g.xb) % g.nx + g.nx) % g.nx : xr;
                const bool buff = z < 2 || z >= nz - 2 || xr < g.xb || xr >= nxr - g.xb;
                bc[z * pr + (long long)y * nxr + xr] = (mask[(size_t)y * g.nx + x] & MASK_FLUID) ? (buff ? RBC_BUFF : RBC_COMP) : RBC_WALL;
            }
    return RBC_OK;
}

// ltc->dmD, umD, vmD, wmD [nx*ny*nz] (reference layout, COMP nodes read) into
// the rho / u field the collide-stream stores (the cycle's sums with M > 1);
// other fluid nodes of the field are unused, wall columns hold rho 1, u 0 as
// the kernel leaves them
int import_macro(rbc_handle *h, const double *dm, const double *um, const double *vm, const double *wm)
{
    RBC_DEVICE_GUARD(h);
    const Geom &g = h->geo;
    std::vector<uint32_t> mask((size_t)g.plane);
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(mask.data(), h->mask2d, 4 * mask.size(), cudaMemcpyDeviceToHost));
    std::vector<float4> f((size_t)g.nint);
    for (int zc = 0; zc < g.nzc; zc++)
        for (int iy = 0; iy < g.ny; iy++)
            for (int xi = 0; xi < g.nx; xi++) {
                const size_t i = (size_t)zc * g.plane + (size_t)iy * g.nx + xi;
                if (!(mask[(size_t)iy * g.nx + xi] & MASK_FLUID)) { f[i] = make_float4(0.f, 0.f, 0.f, 1.f); continue; }
                const long long r = ((long long)(zc + 2) * g.ny + iy) * g.nxr + xi + g.xb;
                f[i] = make_float4((float)um[r], (float)vm[r], (float)wm[r], (float)dm[r]);
            }
    CK(cudaMemcpy(h->uvr, f.data(), sizeof(float4) * f.size(), cudaMemcpyHostToDevice));
    return RBC_OK;
}

// cel->u, v, w [ncell * vertex] of population `group` (the last advection's
// vertex velocities; FP32 in the handle)
int import_vertex_velocity(rbc_handle *h, int group, const double *u, const double *v, const double *w)
{
    RBC_DEVICE_GUARD(h);
    if (group >= h->ngroups) return RBC_OK;
    CellGroup &g = h->cg[group];
    if (g.nv == 0) return RBC_OK;
    std::vector<float> f(3 * (size_t)g.nv);
    for (long long j = 0; j < g.nv; j++) {
        f[j] = (float)u[j]; f[g.nv + j] = (float)v[j]; f[2 * g.nv + j] = (float)w[j];
    }
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpy(g.U, f.data(), 4 * f.size(), cudaMemcpyHostToDevice));
    return RBC_OK;
}

// a zero IB force field, as a freshly set-up reference lattice holds it
int clear_force(rbc_handle *h)
{
    RBC_DEVICE_GUARD(h);
    CK(cudaMemsetAsync(h->Fint, 0, 24 * h->geo.nint, h->stream));
    CK(cudaMemsetAsync(h->Fbits, 0, h->force_bit_bytes(), h->stream));
    h->force_pending = false;
    return RBC_OK;
}

int reference_ele(rbc_handle *h, int group, int *ele)
{
    RBC_DEVICE_GUARD(h);
    const CellGroup &g = h->cg[group];
    std::vector<int> tri(3 * (size_t)g.E);
    if (g.E > 0) CK(cudaMemcpy(tri.data(), g.tri, 4 * tri.size(), cudaMemcpyDeviceToHost));
    for (int c = 0; c < g.ncell; c++)
        for (size_t k = 0; k < tri.size(); k++) ele[(size_t)c * tri.size() + k] = tri[k] + c * g.V;
    return RBC_OK;
}

int group_sizes(const rbc_handle *h, int group, int *ncell, int *vertex, int *element)
{
    const CellGroup &g = h->cg[group];
    if (group >= h->ngroups) { *ncell = *vertex = *element = 0; return RBC_OK; }
    *ncell = g.ncell; *vertex = g.V; *element = g.E;
    return RBC_OK;
}

void set_handle_error(rbc_handle *h, const std::string &msg)
{
    if (h) h->err = msg; else g_create_error = msg;
}

}  // namespace rbc

extern "C" int rbc_set_output_interval(rbc_handle *h, int fileoutput)
{
    if (!h || fileoutput < 0) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    CK(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < h->ngroups; k++) {
        CellGroup &g = h->cg[k];
        if (fileoutput <= 0 || g.ncell == 0 || g.qi_acc) continue;
        g.mn = reference_mn(g.V);
        const size_t nq = (size_t)g.ncell * g.mn, nt = 2 * (size_t)g.ne;
        CK(cudaMalloc(&g.qi_acc, 8 * nq));
        CK(cudaMalloc(&g.tp_acc, 8 * nt));
        CK(cudaMemset(g.qi_acc, 0, 8 * nq));   // as fem_init leaves fem->qi (init2.cu:310)
        CK(cudaMemset(g.tp_acc, 0, 8 * nt));
    }
    if (fileoutput != h->fileoutput) {
        h->fileoutput = fileoutput;
        // the step graphs hold the accumulation launches (or not)
        for (auto &form : h->graph)
            for (cudaGraphExec_t &g : form) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    }
    return RBC_OK;
}

// ---- white cells (init3.cu) -------------------------------------------------

extern "C" {

int rbc_add_wbc(rbc_handle *h, const rbc_mesh *mesh, double rgs, double br)
{
    if (!h || !mesh || mesh->ncell <= 0) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD(h);
    if (h->ngroups > 1) return fail(h, RBC_ERR_STATE, "the white cells are already set");
    if (mesh->vertex < 4 || mesh->element < 4 || !mesh->tri || !mesh->xr)
        return fail(h, RBC_ERR_ARG, "mesh needs vertex, element >= 4, tri and xr");
    if (membrane_smem_bytes(mesh->vertex) > 227 * 1024 || mesh->vertex > 4096)
        return fail(h, RBC_ERR_UNSUPPORTED, "more vertices per cell than one CTA holds (max 3874)");
    if (mesh->element >= (1 << 24)) return fail(h, RBC_ERR_UNSUPPORTED, "too many elements per cell");
    if (!(rgs > 0.0) || !std::isfinite(rgs) || !std::isfinite(br)) return fail(h, RBC_ERR_ARG, "rgs must be > 0 and br finite");
    CK(cudaStreamSynchronize(h->stream));
    CellGroup &c = h->cg[1];
    c.rgs = rgs;
    c.br = br;
    GroupPrep prep;
    int rc = prepare_group(h, c, mesh, prep);
    if (!rc) rc = upload_group(h, c, mesh, prep);
    if (rc) {   // leave the handle with the red cells only
        free_group(c);
        return rc;
    }
    h->ngroups = 2;
    if (h->vof() && (rc = vof_init_group(h, c))) return rc;
    if (h->fileoutput > 0) {
        const int f = h->fileoutput;
        h->fileoutput = 0;
        if ((rc = rbc_set_output_interval(h, f))) return rc;
    }
    // the step graphs and the adjoint hold one population
    for (auto &form : h->graph)
        for (cudaGraphExec_t &g : form) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    if (h->adj) h->adj->valid = false;
    return RBC_OK;
}

int rbc_wbc_dims(const rbc_handle *h, int *ncell, int *vertex, int *element)
{
    if (!h) return RBC_ERR_ARG;
    int n = 0, v = 0, e = 0;
    group_sizes(h, 1, &n, &v, &e);
    if (ncell) *ncell = n;
    if (vertex) *vertex = v;
    if (element) *element = e;
    return RBC_OK;
}

int rbc_import_ref_wbc(rbc_handle *h, const double *x, const double *y, const double *z,
                       const double *xd, const double *nd, const double *volume0, const double *gx)
{
    if (!h) return RBC_ERR_ARG;
    if (h->ngroups < 2) return fail(h, RBC_ERR_STATE, "no white cells (rbc_add_wbc)");
    return import_cells(h, h->cg[1], x, y, z, xd, nd, volume0, gx);
}

int rbc_export_ref_wbc(rbc_handle *h, double *x, double *y, double *z, double *xd,
                       double *u, double *v, double *w, double *fx, double *fy, double *fz, double *gx)
{
    if (!h) return RBC_ERR_ARG;
    if (h->ngroups < 2) return fail(h, RBC_ERR_STATE, "no white cells (rbc_add_wbc)");
    return export_cells(h, h->cg[1], x, y, z, xd, u, v, w, fx, fy, fz, gx);
}

int rbc_wbc_metrics(rbc_handle *h, double *volume, double *area, double *centroid)
{
    if (!h) return RBC_ERR_ARG;
    RBC_DEVICE_GUARD_RO(h);
    if (h->ngroups < 2) return fail(h, RBC_ERR_STATE, "no white cells (rbc_add_wbc)");
    return group_metrics(h, h->cg[1], volume, area, centroid);
}

}  // extern "C"
