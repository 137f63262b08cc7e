/*
 * rbc_oracle.h -- FP64 CPU oracle for the coupled fluid-membrane step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: a plain-C restatement of the
 * reference's algorithm (enomoto-catallaxy/preProcess_src) that works on the
 * reference's own memory layout (AoS populations fn[i*19+q] with two BUFF planes
 * at each z end, SoA vertex arrays, AoS fem->xd, ELL mass matrix, BiCGSTAB).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it.  The product library never links or calls it.
 *
 * Parity pin: the reference ships no tests, fixtures or golden vectors.  This
 * oracle is pinned against the reference's own kernels, compiled from the
 * reference sources by oracle/ref_harness (see oracle/Makefile), through the
 * fixtures in tests/golden/.
 */
#ifndef RBC_ORACLE_H
#define RBC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Node types of the reference bc[] map.  The reference takes the values from
 * its (missing) def.h; the oracle, the product and the reference harness all use
 * these. */
#define ORC_COMP 0
#define ORC_BUFF 1
#define ORC_WALL 2

#define ORC_Q 19

typedef struct orc_params {
    /* lattice, reference frame: z is the periodic/flow axis, nz includes the
     * two BUFF planes at each end (init1.cu:207-210) */
    int nx, ny, nz;
    double dx, dt;
    double tau;          /* BGK relaxation time, tau = 3 Df + 1/2 (init1.cu:203) */
    double Cr;           /* Courant number macro Cr */
    double P;            /* body-force macro P: force density 2 rho P along z */
    double B;            /* IB-force macro B: force density 2 rho B F */
    int flowstart;       /* FLOWSTART: drive is zero for iter <= flowstart */
    double freq;         /* FREQ: drive factor 1 + 0.5 sin(pi t / FREQ) */
    /* membrane */
    double C;            /* Skalak area-dilation ratio */
    double rgs;          /* cel->rg (1.0 for RBCs): tension normalisation */
    int law;             /* 0 = SKALAK, 1 = NEOHOOKEAN (stress.cu:94-99) */
    double residual;     /* RESIDUAL: BiCGSTAB stopping rule */
    int itrmax;          /* ITRMAX */
    /* periodic lengths and extents (cdo->xmin ..., LX, LZ) */
    double LX, LZ;
    double xmin, xmax, zmin, zmax;
    /* cells */
    int ncell, vertex, element, mn;
    double br;           /* BR: bending modulus of fourpoint_bend (0 = no bending) */
    /* flow mode: 0 = CapsuleCHANNELFLOW (z periodic, drive P), 1 = CapsuleSHEARFLOW
     * (x and z periodic, y walls moving along z; init1.cu:133-187, lbm.cu:706-980) */
    int flow;
    double sr;           /* cdo->sr: shear rate (shear mode) */
    int walls;           /* 0: allwall (walls at -/+ sr LY / 2), 1: topwall (top at sr LY) */
    double tube_r;       /* > 0 (channel mode): interpolated bounce-back on the circle x^2 + y^2 = tube_r^2
                          * after streaming (lbm_cylinder.cu:116-231); 0: half-way bounce-back only */
    /* volume fraction of the cells (VOF): vof_k = K > 0 turns it on (CN != 0):
     * front tracking at setup (vof_init, init1.cu:1094-1120) and every K steps,
     * THINC/WLIC advection every step, omega = 1 / (3 (1 + (LAMBDA1 - 1) vf) Df
     * + 1/2) in the collision (lbm.cu:1131) */
    double lambda1;      /* LAMBDA1: viscosity ratio inside / outside the cells */
    int vof_k;           /* K: steps between front-tracking solves; 0 = no VOF (CN = 0) */
    double vof_residual; /* RESIDUAL of the front-tracking solve (matrix_solver.cu:112-216) */
    int vof_itrmax;      /* ITRMAX of that solve */
    /* sub-cycling and the advection's order (main.cu:78-106, ibm.cu:430-627):
     * the membrane and the spread run at the first of every M steps, the
     * advection and the volume correction at the last, and the advection moves
     * the vertices by the velocity averaged over the M steps (lbm.cu:1097-1126,
     * 1435-1460) times M dt; rk_order = RUNGE_KUTTA (1, 2 or 4).  0 means the
     * default (M = 1, RUNGE_KUTTA = 4). */
    int M;
    int rk_order;
} orc_params;

typedef struct orc_state {
    /* lattice: n = nx*ny*nz nodes */
    double *fn, *fm;                       /* [n*19] AoS; swapped by orc_lbm_d3q19 */
    double *dn, *un, *vn, *wn;             /* [n] */
    double *dm, *um, *vm, *wm;             /* [n] */
    double *fx, *fy, *fz;                  /* [n] spread force */
    int    *bc;                            /* [n] */
    /* cells: nv = ncell*vertex, ne = ncell*element */
    double *x, *y, *z;                     /* [nv] cel->x (post volume correction) */
    double *u, *v, *w;                     /* [nv] */
    double *cfx, *cfy, *cfz;               /* [nv] cel->fx */
    double *xd;                            /* [3*nv] fem->xd (AoS) */
    double *nd;                            /* [4*ne] reference contravariant metric */
    double *t, *rg;                        /* [4*ne], [ne] */
    double *qd;                            /* [ncell*mn] nodal load */
    int    *ele;                           /* [3*ne] global vertex ids */
    int    *nln, *ln, *lo;                 /* [nv], [7*nv], [7*nv] */
    int    *nle, *le;                      /* [nv], [6*nv] */
    double *volume0, *gx;                  /* [ncell], [3*ncell] */
    int    iter;                           /* prc->iter */
    int    bicg_iters;                     /* diagnostics: last solve's iterations */
    int    *ec;                            /* [3*ne] edge-neighbour elements (cel->ec) */
    /* [ncell] per-cell tension normalisation and bending modulus, or NULL for
     * p->rgs / p->br in every cell: a run with white cells as well (cel->rg_w
     * = GSw / GS, cel->br_w = BRw, init3.cu:91-92) on the same mesh */
    double *crg, *cbr;
    /* [3*ne] spontaneous angle (cos, sin) of each bending visit, or NULL for
     * (1, 0) as init1.cu:849-850 leaves it; orc_bend_reference fills them */
    double *c0, *s0;
    double *vf;                            /* [n] ltc->vf: volume fraction of the cells (VOF) */
    int    vof_iters;                      /* diagnostics: last front-tracking solve's sweeps */
} orc_state;

/* init2.cu:258-400 (fem_init): link tables and the reference metric from the
 * positions in s->xd.  Returns 0, or 3 as error(3) would. */
int  orc_fem_init(const orc_params *p, orc_state *s);
/* init1.cu:413-434 (flu_init): equilibrium at rho = 1, u = 0 (shear mode with
 * FLOWSTART = 0: u = (0, 0, w(y)) of the walls' linear profile, init1.cu:367-381). */
void orc_flu_init(const orc_params *p, orc_state *s);
/* volume_correction.cu:427-450 (volume_init). */
void orc_volume_init(const orc_params *p, orc_state *s);

/* stress.cu:580-659 (stress): calc_tension, calc_load (BiCGSTAB), q2f, then
 * fourpoint_bend when p->br != 0.
 * Returns 0, or the BiCGSTAB flag (1 breakdown, 2 no convergence). */
int  orc_stress(const orc_params *p, orc_state *s);
/* ibm.cu:299-369 (ibm_st1): zero, spread, periodic fold. */
void orc_ibm_st1(const orc_params *p, orc_state *s);
/* lbm.cu:1463-1579 (lbm_d3q19, CapsuleCHANNELFLOW branch). */
void orc_lbm_d3q19(const orc_params *p, orc_state *s);
/* ibm.cu:642-694 (ibm_st2): interpolate + RK4 advect. */
void orc_ibm_st2(const orc_params *p, orc_state *s);
/* volume_correction.cu:453-524.  Returns iterations - 1, or -1 when the
 * 1000-iteration cap is hit (the reference calls exit(1) there). */
int  orc_volume_correction(const orc_params *p, orc_state *s);

/* thincwlic.cu:316-420 (thinc_wlic, red cells): three directional THINC/WLIC
 * sweeps of s->vf with the step's velocity um, vm, wm. */
void orc_thinc_wlic(const orc_params *p, orc_state *s);
/* fronttrack.cu:628-700 (front_tracking, red cells): the indicator gradient
 * of the cell surfaces, its divergence, and the Poisson solve (red-black SOR,
 * matrix_solver.cu:112-216) into s->vf.  Returns the sweeps of the converged
 * attempt, or -1 when 10 attempts did not converge (the reference's error(5)). */
int  orc_front_tracking(const orc_params *p, orc_state *s);

/* main.cu:73-110: nsteps steps (sub-steps when M > 1).  Returns 0 or an error code. */
int  orc_step(const orc_params *p, orc_state *s, int nsteps);

/* Pieces used by the tests on their own. */
void orc_calc_tension(const orc_params *p, orc_state *s);
int  orc_calc_load(const orc_params *p, orc_state *s);
void orc_q2f(const orc_params *p, orc_state *s);
void orc_calc_volume(const orc_params *p, const orc_state *s, double *volume, double *area);
/* stress.cu:448-578 (fourpoint_bend): adds the dihedral bending forces of
 * every edge-neighbour pair to cel->fx/fy/fz (spontaneous angle 0, as
 * init1.cu:849-850 leaves it). */
void orc_bend(const orc_params *p, orc_state *s);
/* init1.cu:797-848 without the override of 849-850: s->c0 / s->s0 from the
 * current positions (the reference shape when called after orc_fem_init). */
void orc_bend_reference(const orc_params *p, orc_state *s);

int  orc_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
