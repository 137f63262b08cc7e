/*
 * rbc_step.h -- C ABI of the B200-native coupled fluid-membrane time step.
 *
 * One handle owns the device state of one simulation: a D3Q19 lattice stored
 * as pull-scheme SoA populations (f_i - w_i, FP32 or FP16), the Eulerian IB
 * force and velocity fields, and the red- and white-cell meshes (FP64 positions, shared
 * triangle connectivity, per-element reference metric).
 *
 * The step entry points replace the reference's step modules one for one and
 * keep their order and side effects (enomoto-catallaxy/preProcess_src):
 *
 *   rbc_stress             <- void stress(process*, domain*, cell*, fem*, lattice*)  stress.cu:580
 *   rbc_ibm_st1            <- void ibm_st1(domain*, lattice*, cell*)                 ibm.cu:299
 *   rbc_lbm_d3q19          <- void lbm_d3q19(process*, domain*, lattice*)            lbm.cu:1463
 *   rbc_ibm_st2            <- void ibm_st2(domain*, lattice*, cell*, fem*)           ibm.cu:642
 *   rbc_volume_correction  <- int  volume_correction(domain*, cell*, fem*)           volume_correction.cu:453
 *   rbc_step               <- the time loop of main.cu:73-110 (M = 1)
 *
 * The reference's setup that defines the step inputs (cdo_init bc map,
 * flu_init equilibrium, fem_init link tables and reference metric,
 * volume_init) happens in rbc_create; the rbc_import_ref_* / rbc_export_ref_*
 * calls move state in and out in the reference's own layouts (AoS FP64
 * populations fn[i*19+q] with BUFF planes, SoA cel->x/y/z, AoS fem->xd,
 * fem->nd[4*e+k]).
 *
 * Frame and units follow the reference's CapsuleCHANNELFLOW mode: the lattice
 * is nx * ny * nz nodes with x fastest, z is the periodic flow axis with two
 * BUFF planes at each end, node (ix,iy,iz) sits at physical position
 * (ix*dx - (nx-1)dx/2, iy*dx - (ny-1)dx/2, iz*dx - (nz-1)dx/2).  The wall and
 * fluid pattern must be the same in every z plane, as the reference's channel
 * builds it (init1.cu:219-234).
 *
 * Every call returns an int status (RBC_OK = 0).  Nothing calls exit().
 * All device work of a handle runs on one CUDA stream; calls are asynchronous
 * unless stated.  Calls on one handle must not be made from two host threads
 * at the same time.
 */
#ifndef RBC_STEP_H
#define RBC_STEP_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define RBC_OK                 0
#define RBC_ERR_ARG            1   /* bad argument or size */
#define RBC_ERR_CUDA           2   /* CUDA runtime error (see rbc_last_error) */
#define RBC_ERR_UNSUPPORTED    3   /* option outside the implemented scope */
#define RBC_ERR_TOPOLOGY       4   /* mesh link check failed (reference error(3), init2.cu:370) */
#define RBC_ERR_NOT_CONVERGED  5   /* volume correction hit 1000 iterations (reference exit(1)) */
#define RBC_ERR_NONFINITE      6   /* non-finite vertex position detected */
#define RBC_ERR_STATE          7   /* call out of order (e.g. no cells) */
#define RBC_ERR_NO_DEVICE      8   /* no CUDA device */

/* node types of the reference bc[] map (the reference's def.h values are not
 * published; these are the values this library and its tools use) */
#define RBC_COMP 0
#define RBC_BUFF 1
#define RBC_WALL 2

/* population storage in HBM */
#define RBC_STORE_F32 0            /* f_i - w_i in FP32: 180 B per lattice update */
#define RBC_STORE_F16 1            /* (f_i - w_i) * scale in FP16: 104 B per lattice update */

/* flow modes.  CHANNEL: z periodic with two BUFF planes at each end, walls from
 * the bc map (the same in every z plane), body-force drive P along z.  SHEAR
 * (init1.cu:133-187, lbm.cu:706-980): a box periodic in x and z (two BUFF
 * layers at each end of both) between two y walls half a node beyond rows 2
 * and ny - 3 that move along z (walls: both at -/+ sr LY / 2 or the top at
 * sr LY, LY = (ny - 4) dx, from iteration FLOWSTART on); no body force
 * (P = 0); with FLOWSTART = 0 rbc_create starts from the walls' linear
 * profile as flu_init does. */
#define RBC_FLOW_CHANNEL 0
#define RBC_FLOW_SHEAR   1
#define RBC_WALLS_BOTH   0
#define RBC_WALLS_TOP    1

/* membrane constitutive law (stress.cu:94-99) */
#define RBC_LAW_SKALAK     0
#define RBC_LAW_NEOHOOKEAN 1

/* device status flags (rbc_get_status) */
#define RBC_FLAG_VC_NOT_CONVERGED  0x1
#define RBC_FLAG_NONFINITE         0x2
#define RBC_FLAG_SPREAD_OVERFLOW   0x4   /* informational: a cell used the direct-atomic spread path */
#define RBC_FLAG_SOLVE_RESIDUAL    0x8   /* membrane load solve: |r| / |b| of the Jacobi-scaled
                                            system above 1e-3 (|r|^2 > 1e-6 |b|^2) */
#define RBC_FLAG_VOF_NOT_CONVERGED 0x10  /* a front-tracking solve hit vof_itrmax (the reference's error(5)) */

typedef struct rbc_params {
    /* lattice (reference frame, nz includes the 4 BUFF planes) */
    int    nx, ny, nz;
    double dx, dt;
    double tau;          /* BGK relaxation time (tau = 3 Df + 1/2) */
    double Cr;           /* Courant number macro Cr */
    double P;            /* body-force macro P (force density 2 rho P along z) */
    double B;            /* IB-force macro B (force density 2 rho B F) */
    int    flowstart;    /* FLOWSTART: drive off for iter <= flowstart */
    double freq;         /* FREQ: drive factor 1 + 0.5 sin(pi dt iter / FREQ); +inf = constant */
    /* periodic lengths and extents (reference macros LX, LZ and cdo->xmin ...) */
    double LX, LZ;
    double xmin, xmax, zmin, zmax;
    /* membrane */
    double C;            /* Skalak area-dilation ratio */
    double rgs;          /* tension normalisation cel->rg (1.0 for red cells) */
    int    law;          /* RBC_LAW_* */
    double br;           /* bending modulus BR of fourpoint_bend (stress.cu:448-578); 0 = none */
    int    M;            /* sub-cycling factor M >= 1 (main.cu:78-106); no VOF, batch or adjoint with M > 1 */
    int    rk_order;     /* RUNGE_KUTTA of the advection: 1, 2 or 4 (1 and 2 need dx = dt = 1) */
    /* implementation choices */
    int    storage;      /* RBC_STORE_* */
    int    membrane_fp64;/* 1: element mechanics in FP64, 0: FP32 */
    int    solver_iters; /* Chebyshev iterations of the load solve; 0 = default (16) */
    int    device;       /* CUDA device ordinal; -1 = device 0 of this library's runtime */
    /* flow mode */
    int    flow;         /* RBC_FLOW_CHANNEL (CapsuleCHANNELFLOW) or RBC_FLOW_SHEAR (CapsuleSHEARFLOW) */
    double sr;           /* cdo->sr, shear rate of the moving walls (shear mode; lattice units) */
    int    walls;        /* RBC_WALLS_BOTH (allwall: walls at -/+ sr LY/2) or RBC_WALLS_TOP (topwall: top at sr LY) */
    /* channel mode: > 0 = the walls are the circular tube x^2 + y^2 = tube_r^2 and its links
     * bounce back by linear interpolation at the circle (lbm_cylinder.cu:61-231); 0 = half-way */
    double tube_r;
    /* bending (BR != 0) about spontaneous angles: 0 = angle 0 for every edge, as
     * the reference runs (init1.cu:849-850 overwrite the computed angles with
     * c0 = 1, s0 = 0); 1 = the initial shape's dihedral angles, the values
     * init1.cu:797-848 (init3.cu:313-364) compute before that override */
    int    bend_spont;
    /* volume fraction of the cells (VOF, fronttrack.cu / thincwlic.cu): vof_k = K > 0
     * (CN != 0) tracks it, by front tracking at rbc_create (vof_init) and every K steps
     * and THINC/WLIC advection every step; the collision then relaxes with omega =
     * 1 / (3 (1 + (LAMBDA1 - 1) vf) Df + 1/2) (lbm.cu:1131).  0 = not tracked (vf = 0). */
    double lambda1;      /* LAMBDA1: viscosity ratio of the cells' interior */
    int    vof_k;        /* K */
    double vof_residual; /* RESIDUAL of the front-tracking solve */
    int    vof_itrmax;   /* ITRMAX of that solve */
} rbc_params;

typedef struct rbc_mesh {
    int ncell;           /* cel->n */
    int vertex;          /* cel->vertex */
    int element;         /* cel->element */
    /* local triangle connectivity shared by every cell, [element*3], 0-based,
     * outward winding: (x_b - x_a) x (x_c - x_a) points out of the cell */
    const int *tri;
    /* positions defining the reference (stress-free) shape and the initial
     * state, AoS [3*ncell*vertex] like fem->xr / fem->x (init2.cu:311-325) */
    const double *xr;
} rbc_mesh;

typedef struct rbc_handle rbc_handle;

/* ---- lifetime -------------------------------------------------------- */

/* Replaces cdo_init/flu_init/fem_init/mem_init/volume_init for the step:
 * validates p and bc[nx*ny*nz], builds the link tables and the reference
 * metric from mesh->xr, sets the lattice to rest equilibrium (rho = 1, u = 0),
 * stores V0 and the centroids.  mesh may be NULL or have ncell = 0 (pure fluid).
 * Synchronous. */
int rbc_create(const rbc_params *p, const rbc_mesh *mesh, const int *bc, rbc_handle **out);
int rbc_destroy(rbc_handle *h);
/* human-readable text of the last error on h (or of the last create failure
 * when h is NULL) */
const char *rbc_last_error(const rbc_handle *h);

/* ---- state in and out, reference layouts (synchronous) ---------------- */

/* fn[nx*ny*nz*19]: pre-collision populations as lbm_d3q19 leaves them in
 * ltc->fnD (lbm.cu:1575).  Only COMP nodes are read.  The lattice crosses to
 * the device in chunks of about 16 MB through a ring of four slots while the
 * chunks already there are converted, so the call takes about the time of the
 * host-to-device copy (fastest from pinned host memory).  The ring (four
 * chunks and two planes) is allocated by rbc_create for lattices of more than
 * four chunks, else by the first import. */
int rbc_import_ref_lattice(rbc_handle *h, const double *fn);
/* Any pointer may be NULL.  fn: populations on COMP nodes, 0 elsewhere.
 * dn/un/vn/wn [nx*ny*nz]: density and velocity of the last lbm step with the
 * reference's half-force shift (lbm.cu:1116-1118) on COMP nodes, their periodic
 * images on BUFF nodes (lbm.cu:1378-1432), and rho = 1, u = 0 on WALL nodes
 * (the values the reference's WALL nodes keep from flu_init).  With M > 1 the
 * density and velocity are those of ltc->dmD / umD: the sums over the steps of
 * the current cycle, the velocity averaged after its last step (lbm.cu:1097-1126,
 * 1435-1460). */
int rbc_export_ref_lattice(rbc_handle *h, double *fn, double *dn, double *un, double *vn, double *wn);
/* Eulerian spread force ltc->fx/fy/fz [nx*ny*nz] after rbc_ibm_st1 and before
 * rbc_lbm_d3q19 (COMP nodes, folded as ibm.cu:214-296 leaves them). */
int rbc_export_ref_force(rbc_handle *h, double *fx, double *fy, double *fz);
/* Any pointer may be NULL.  x,y,z [nv]: cel->x/y/z; xd [3*nv]: fem->xd;
 * nd [4*ne]: fem->nd; volume0 [ncell]; gx [3*ncell]: cel->gx.  The layout
 * conversions (xd and gx to [3][n], nd to the covariant metric) run on the
 * device after plain copies, through a staging buffer rbc_create allocates. */
int rbc_import_ref_cells(rbc_handle *h, const double *x, const double *y, const double *z,
                         const double *xd, const double *nd, const double *volume0, const double *gx);
/* Vertex forces cel->fx/fy/fz [nv] as stress() leaves them, for running
 * rbc_ibm_st1 on forces computed elsewhere. */
int rbc_import_ref_vertex_force(rbc_handle *h, const double *fx, const double *fy, const double *fz);
/* Any pointer may be NULL.  u,v,w: cel->u/v/w; fx,fy,fz: cel->fx/fy/fz. */
int rbc_export_ref_cells(rbc_handle *h, double *x, double *y, double *z, double *xd,
                         double *u, double *v, double *w, double *fx, double *fy, double *fz,
                         double *gx);
/* ---- white cells (N_W > 0: init3.cu, stress.cu:620-655, ibm.cu:334-360 and
 * 670-690, volume_correction.cu:260-340) ----------------------------------- */

/* A second cell population stepped with the first: its own mesh, tension
 * normalisation rgs (cel->rg_w = GSw / GS) and bending modulus br (BRw); the
 * same law and C as the red cells.  It spreads into and advects with the same
 * lattice and has its own volume correction.  Replaces wbc_init (init3.cu) for
 * the step; the mesh's ncell is cel->n_w.  Synchronous; once per handle. */
int rbc_add_wbc(rbc_handle *h, const rbc_mesh *mesh, double rgs, double br);
/* cel->n_w, vertex_w, element_w (all 0 without white cells); any pointer may be NULL */
int rbc_wbc_dims(const rbc_handle *h, int *ncell, int *vertex, int *element);
/* rbc_import_ref_cells / rbc_export_ref_cells / rbc_cell_metrics for the white
 * cells (cel->x_w ..., fem->xd_w, fem->nd_w, cel->volume0_w, cel->gx_w) */
int rbc_import_ref_wbc(rbc_handle *h, const double *x, const double *y, const double *z,
                       const double *xd, const double *nd, const double *volume0, const double *gx);
int rbc_export_ref_wbc(rbc_handle *h, double *x, double *y, double *z, double *xd,
                       double *u, double *v, double *w, double *fx, double *fy, double *fz,
                       double *gx);
int rbc_wbc_metrics(rbc_handle *h, double *volume, double *area, double *centroid);

/* ltc->vf and ltc->vf2 (red and white cells) [nx*ny*nz] in the reference
 * layout: BUFF nodes hold their periodic images, WALL nodes 0; import reads
 * COMP nodes.  Either pointer may be NULL.  RBC_ERR_STATE without vof_k > 0. */
int rbc_export_ref_vof(rbc_handle *h, double *vf, double *vf2);
int rbc_import_ref_vof(rbc_handle *h, const double *vf, const double *vf2);

/* prc->iter as the stage entry points see it (rbc_step increments it first,
 * as main.cu:75 does) */
int rbc_set_iter(rbc_handle *h, int iter);
int rbc_get_iter(const rbc_handle *h, int *iter);

/* ---- the step ---------------------------------------------------------- */

/* calc_tension + calc_load + q2f, then fourpoint_bend when BR != 0 */
int rbc_stress(rbc_handle *h);
int rbc_ibm_st1(rbc_handle *h);
/* With M > 1 the velocity sums and the force reset follow the place of step
 * prc->iter (rbc_set_iter) among its M: the caller runs rbc_stress and
 * rbc_ibm_st1 at the first of every M steps and rbc_ibm_st2 and
 * rbc_volume_correction at the last, as main.cu:78-106 does. */
int rbc_lbm_d3q19(rbc_handle *h);
int rbc_ibm_st2(rbc_handle *h);
/* *iters (may be NULL) receives the reference's return value, iterations - 1.
 * Synchronous when iters != NULL. */
int rbc_volume_correction(rbc_handle *h, int *iters);
/* thinc_wlic (thincwlic.cu:316): THINC/WLIC advection of the volume fraction
 * with the last lbm step's velocity; nothing without vof_k > 0. */
int rbc_thinc_wlic(rbc_handle *h);
/* front_tracking (fronttrack.cu:628): the volume fraction of the current cells
 * by the Poisson solve of the indicator; *iters (may be NULL) receives the red
 * cells' solver sweeps (-1 = not converged, RBC_FLAG_VOF_NOT_CONVERGED).
 * Synchronous when iters != NULL.  rbc_step runs it every vof_k steps. */
int rbc_front_tracking(rbc_handle *h, int *iters);
/* nsteps full steps, each a replay of a CUDA graph of one step.  Asynchronous
 * (rbc_synchronize or any export waits for it).  With M > 1, nsteps lattice
 * steps: each runs the stages of its place among its M (main.cu:78-106), and a
 * call may end inside a cycle. */
int rbc_step(rbc_handle *h, int nsteps);

/* ---- diagnostics ------------------------------------------------------ */

/* Synchronous.  flags: RBC_FLAG_* accumulated since the last call (cleared
 * by the call); vc_iters_max: largest volume-correction return value seen. */
int rbc_get_status(rbc_handle *h, int *flags, int *vc_iters_max);
/* Synchronous.  FP64 per-cell volume, area and vertex centroid ([ncell],
 * [ncell], [3*ncell]); any pointer may be NULL.  Right after rbc_step (or a
 * batch step) these are the values the step's volume correction computed for
 * the final positions (cel->volume, cel->area, cel->gx), read back without a
 * kernel; after any other call that may change the state a kernel measures
 * them. */
int rbc_cell_metrics(rbc_handle *h, double *volume, double *area, double *centroid);
/* Asynchronous form of rbc_cell_metrics for a caller that consumes each
 * step's metrics while the next steps run: enqueues on the handle's stream
 * the device-to-host copies of the same values into out (5 * ncell doubles:
 * volume[ncell], area[ncell], then the centroid as x[ncell], y[ncell],
 * z[ncell]) and returns without waiting.  out must stay valid until the
 * copies complete (rbc_synchronize, or an event recorded on the handle's
 * stream after this call); page-locked memory keeps the call asynchronous. */
int rbc_cell_metrics_async(rbc_handle *h, double *out);
int rbc_synchronize(rbc_handle *h);
/* Number of kernel launches issued by this library since creation. */
int rbc_launch_count(const rbc_handle *h, long long *count);
/* The CUDA stream (cudaStream_t) all work of h runs on. */
int rbc_get_stream(const rbc_handle *h, void **stream);
/* Runs nsteps full steps with direct launches (no graph) and a CUDA event
 * around every kernel; kernel_ms[RBC_NUM_KERNELS] receives the summed device
 * time per kernel in the order of RBC_KERNEL_NAMES (with BR != 0 the bending
 * kernel is timed in the "membrane" slot; "vof" holds the THINC/WLIC sweeps and
 * the front tracking of the steps it runs in).  Synchronous. */
#define RBC_NUM_KERNELS 8
#define RBC_KERNEL_NAMES {"step_begin", "membrane", "spread", "lbm_collide_stream", "force_reset", "advect", "vof", "volume"}
int rbc_profile_steps(rbc_handle *h, int nsteps, double *kernel_ms);

/* ---- batches of independent simulations ----------------------------------- */

/* Several independent simulations (for instance capillaries of different
 * sizes and parameters, each its own handle) stepped together.  The reference
 * runs one simulation per process; its main.cu:73-110 loop is what each
 * simulation of the batch executes.  Two forms:
 *   fused (the default where possible): each batch step is one CUDA graph of
 *     seven launches -- step begin, the occupancy-word clear, membrane,
 *     spread, collide-stream, advection, volume correction -- each running
 *     the blocks of every simulation (a table of per-simulation arguments and
 *     block offsets), with the same device code as a simulation's own step,
 *     so the results are the same bit for bit.  Needs simulations that share
 *     storage, flow mode, membrane precision and vertices per cell, with no
 *     white cells, bending, output averages, volume fraction or tube;
 *   child graphs (otherwise, or rbc_batch_set_form(b, 0)): each batch step is
 *     one graph launch whose nodes are the simulations' whole steps.
 * The handles stay owned by the caller and usable (stage calls, imports,
 * exports, rbc_step) between batch steps; destroy the batch first. */
typedef struct rbc_batch rbc_batch;
/* handles: n distinct handles on one device.  Text of errors: rbc_batch_last_error(NULL). */
int rbc_batch_create(rbc_handle *const *handles, int n, rbc_batch **out);
int rbc_batch_destroy(rbc_batch *b);
const char *rbc_batch_last_error(const rbc_batch *b);
/* nsteps steps of every simulation.  Asynchronous; each handle's later work
 * is ordered after it, and rbc_batch_synchronize waits for it. */
int rbc_batch_step(rbc_batch *b, int nsteps);
int rbc_batch_synchronize(rbc_batch *b);
/* The CUDA stream (cudaStream_t) the batch graph launches run on. */
int rbc_batch_get_stream(const rbc_batch *b, void **stream);
/* Simulations per dependency chain of the batch graph (default 1: all
 * concurrent): simulations i and i + 1 with the same i / chain run one after
 * the other, chains concurrently. */
int rbc_batch_set_chain(rbc_batch *b, int chain);
int rbc_batch_get_chain(const rbc_batch *b, int *chain);
/* Autotuner: times each candidate over 1 + steps_per_trial batch steps and
 * keeps the fastest.  Fused form: the launch shapes (collide-stream threads
 * per block 128 / 256 and z planes per thread 1 / 2 / 4, membrane vertices per
 * thread: the one-simulation choice and the next); child graphs: chain = 1, 2,
 * 4, ... up to 64.  *chain_out (may be NULL) receives the chain.  The timed
 * steps are real steps: every simulation advances by them. */
int rbc_batch_autotune(rbc_batch *b, int steps_per_trial, int *chain_out);
/* fused: 1 (default) for the fused form where the simulations allow it, 0 for
 * child graphs.  rbc_batch_get_form: *fused = the form the next step uses;
 * *obstacle (may be NULL) = why the fused form is not possible ("" if it is). */
int rbc_batch_set_form(rbc_batch *b, int fused);
int rbc_batch_get_form(const rbc_batch *b, int *fused, const char **obstacle);
/* Launch shapes of the fused form: collide-stream threads per block (128 or
 * 256), z planes per thread (0 = 2 with FP32 storage, 4 with FP16; else 1..8)
 * and membrane vertices per thread (0 = as one simulation; else 1..4 within the
 * block's thread limit).  Results do not depend on them. */
int rbc_batch_set_shape(rbc_batch *b, int lbm_threads, int lbm_planes, int membrane_vpt);
int rbc_batch_get_shape(const rbc_batch *b, int *lbm_threads, int *lbm_planes, int *membrane_vpt);
/* Kernels the batch launched (fused: 7 per step; child graphs: every
 * simulation's step kernels). */
int rbc_batch_launch_count(const rbc_batch *b, long long *count);

/* ---- adjoint (gradients through the step) -------------------------------- */

/* No counterpart in the reference.  Exact discrete adjoint of this library's
 * own step (membrane, spread, collide-stream, RK4 advection, volume
 * correction) with checkpointing: gradients of a function L of the final
 * vertex positions (cel->x) with respect to the coefficients P, B, C and to
 * the initial positions.  FP32 population storage and BR = 0 only
 * (RBC_ERR_UNSUPPORTED otherwise).
 *
 * rbc_adjoint_record: runs nsteps steps from the current state (as rbc_step
 * would) and keeps a checkpoint of the state every ckpt_every steps and after
 * the last.  Device memory: (nsteps / ckpt_every + 1) checkpoints of
 * 4 Q B per node + 48 B per vertex, and ckpt_every steps of stored stages
 * (104 B per node + 84 B per vertex) used by the backward sweep.
 * Synchronous. */
int rbc_adjoint_record(rbc_handle *h, int nsteps, int ckpt_every);
/* rbc_adjoint_record_binomial: the same run for a reverse sweep under binomial
 * (revolve) checkpointing, for lattices whose segments of stored stages would
 * not fit: the run is cut into units of `unit` steps, and the backward sweep
 * reverses them under the binomial schedule with `snaps` snapshot slots beside
 * the initial state (A. Griewank, A. Walther, "Algorithm 799: revolve", ACM
 * TOMS 26, 2000): each unit is advanced at most r times before it is
 * recorded, r the least with C(snaps + r + 1, snaps + 1) >= units.  The
 * forward run keeps the snapshots the schedule takes before its first
 * recording.  Device memory: snaps + 2 checkpoints of 4 Q B per node + 48 B
 * per vertex and 2 * unit steps of stored stages (104 B per node + 84 B per
 * vertex), independent of nsteps.  rbc_adjoint_backward then follows the
 * schedule (recordings alternate between the two stores, so a unit's
 * recording overlaps the reversal of the unit after it).  Synchronous. */
int rbc_adjoint_record_binomial(rbc_handle *h, int nsteps, int unit, int snaps);
/* The recorded run's schedule: units (segments between checkpoints for
 * rbc_adjoint_record), steps per unit, checkpoint slots including the initial
 * state's, and the units one backward sweep advances without recording (0 for
 * rbc_adjoint_record).  Any pointer may be NULL.  RBC_ERR_STATE before a
 * record. */
int rbc_adjoint_schedule(const rbc_handle *h, int *units, int *unit_steps, int *snapshots, long long *advances);
/* The binomial schedule of `units` units with `snaps` free slots, from the
 * initial state in slot 0, as actions (needs no device): ops[i] is
 * 0 advance args[i] units, 1 keep the state in slot args[i], 2 restore slot
 * args[i], 3 record unit args[i] (the state advances past it), 4 reverse unit
 * args[i].  *len receives the number of actions; with cap 0 only *len is set,
 * a cap below it is RBC_ERR_ARG. */
#define RBC_ADJ_ADVANCE 0
#define RBC_ADJ_SNAP    1
#define RBC_ADJ_RESTORE 2
#define RBC_ADJ_RECORD  3
#define RBC_ADJ_REVERSE 4
int rbc_adjoint_binomial_plan(int units, int snaps, int *ops, int *args, int cap, int *len);
/* rbc_adjoint_backward: reverse sweep of the recorded run.
 *   xbar, ybar, zbar  host [nv] each: dL/d(final cel->x, y, z); NULL = 0
 *   grad              host [3] out: dL/dP, dL/dB, dL/dC
 *   dx0, dy0, dz0     host [nv] each, may be NULL: dL/d(initial positions),
 *                     the sum of the adjoints of the initial cel->x and
 *                     fem->xd (equal at the start of a run from rbc_create)
 *   adj_flags         may be NULL: bit 0 set when some step's volume
 *                     correction moved the vertices more than 16 times (the
 *                     moves beyond are not differentiated)
 *   ms                may be NULL: device time of the sweep (recomputation
 *                     included), milliseconds
 * Each segment between checkpoints is recomputed once, stage by stage, then
 * reversed.  The handle is left at the state after the recorded run.  May be
 * called again with other seeds.  Synchronous.  With the reference's macros:
 * P = g / 2 and B = Gs / 2 (dx = dt = 1), so dL/dg = dL/dP / 2 and
 * dL/dGs = dL/dB / 2. */
int rbc_adjoint_backward(rbc_handle *h, const double *xbar, const double *ybar, const double *zbar,
                         double *grad, double *dx0, double *dy0, double *dz0, int *adj_flags, float *ms);
/* Replaces the coefficients P (drive), B (IB force) and C (area dilation) of
 * a handle.  The handle's step graphs are rebuilt on the next rbc_step and a
 * recorded adjoint run is dropped; a batch holding the handle must be
 * destroyed and created again.  Synchronous. */
int rbc_set_coefficients(rbc_handle *h, double P, double B, double C);

/* ---- files in the reference's formats (etc.cu) ---------------------------- */

/* The reference's output_data / restart_file files for a red-cell run (no
 * white cells, no cytoadhesion), byte for byte: restart.bin (etc.cu:738-766,
 * read by restart_file etc.cu:164-270), cell%04d.bin (etc.cu:566-590),
 * prof%04d.bin (etc.cu:547-560) and center.dat (OutputCapsuleCenter /
 * InputCapsuleCenter etc.cu:110-160).  The caller names the files (the
 * reference builds the names from prc->fnum).  vf / vf2 (VOF indicator, only
 * used with a viscosity contrast) are written as 0, the reference's unset
 * rx / ry / rz as 0; both are ignored when read.  Synchronous. */

/* FILEOUTPUT: from the next step on, fem->qi (the load of the membrane solve)
 * and fem->tp (the principal tensions of each element) are averaged over
 * output intervals of fileoutput steps as the reference does (reset in the
 * first step of an interval, stress.cu:101-118, 280-300); 0 stops it and the
 * files then hold the last averages, or zeros when none was ever kept. */
int rbc_set_output_interval(rbc_handle *h, int fileoutput);
int rbc_write_restart(rbc_handle *h, const char *path, int fnum);
/* Imports a restart.bin written for this handle's lattice and cells: the
 * populations, positions (cel->x and fem->xd), the averages and the iteration
 * counter (0 with fnum 0 when the file's fnum exceeds 100, etc.cu:205).
 * *fnum (may be NULL) receives the file's output counter.  A file of another
 * size is RBC_ERR_ARG. */
int rbc_read_restart(rbc_handle *h, const char *path, int *fnum);
int rbc_write_cell_file(rbc_handle *h, const char *path);
int rbc_write_prof_file(rbc_handle *h, const char *path);
int rbc_write_center_file(rbc_handle *h, const char *path);
/* cel->gx, the centroids the volume correction unwraps about */
int rbc_read_center_file(rbc_handle *h, const char *path);

/* ---- without allocation -------------------------------------------------- */

/* No counterpart in the reference.  Per-cell FP64 volume, area and vertex
 * centroid (the quantities of rbc_cell_metrics) of cells whose positions the
 * caller already holds on the device, for callers that cannot allocate device
 * memory: this call needs no handle and calls no allocator.  Its scratch is a
 * static device array of RBC_NOALLOC_MAX_CELLS cells (160 KB) that every GPU
 * loading the library keeps until exit.
 *   x        device, [3][ncell*vertex] SoA positions (x block, y block, z block)
 *   tri      device, [element*3] local connectivity shared by all cells; every
 *            entry must lie in 0..vertex-1 (entries outside are skipped with
 *            their triangles and the call returns RBC_ERR_ARG)
 *   LX, xmin, xmax  periodic length and range of x when x is periodic (the
 *            shear mode, RBC_FLOW_SHEAR); LX <= 0 for the channel and the tube,
 *            whose x is bounded by walls
 *   LZ, zmin, zmax  periodic length and range of z
 *            Cells are unwrapped along each periodic axis about their first
 *            vertex and their centroids wrapped into [min, max], as the
 *            handle's volume correction does (cells must span less than half
 *            of each period).
 *   device   CUDA device ordinal, or -1 for the calling thread's current device;
 *            the calling thread's current device is the same after the call
 *   stream   cudaStream_t to run on (NULL = default stream)
 *   volume, area [ncell], centroid [3*ncell] (x, y, z of each cell): host outputs
 * Synchronous.  ncell above RBC_NOALLOC_MAX_CELLS, vertex above
 * RBC_NOALLOC_MAX_VERTEX, LZ <= 0 or NULL pointers return RBC_ERR_ARG (text in
 * rbc_last_error(NULL)).  The first call on a device looks up the scratch
 * array's device address and sets the kernel's shared-memory limit; make that
 * first call before any CUDA graph capture.  All calls share the scratch
 * array: calls that overlap on the GPU (other streams, other host threads)
 * race and must be serialised. */
#define RBC_NOALLOC_MAX_CELLS  4096
#define RBC_NOALLOC_MAX_VERTEX 4096
int rbc_cell_metrics_noalloc(const double *x, int ncell, int vertex, int element, const int *tri,
                             double LX, double xmin, double xmax, double LZ, double zmin, double zmax,
                             int device, void *stream, double *volume, double *area, double *centroid);

/* Launch shapes (no counterpart in the reference, which launches one thread
 * per node): results do not depend on them, only the speed.
 *   RBC_SHAPE_LBM_PLANES  z planes each collide-stream thread updates: 1, 2, 4
 *                         or 8, or 0 to choose from the lattice size (2 with
 *                         FP32 storage, 4 with FP16, fewer on lattices too
 *                         small to fill the GPU).
 * A change takes effect at the next step (the step graphs are rebuilt);
 * batches built before keep their graphs until they are rebuilt. */
#define RBC_SHAPE_LBM_PLANES 1
int rbc_set_launch_shape(rbc_handle *h, int what, int value);
int rbc_get_launch_shape(const rbc_handle *h, int what, int *value);

/* Sizes of the internal lattice and of the cells. */
int rbc_dims(const rbc_handle *h, int *nx, int *ny, int *nz_periodic, int *ncell, int *vertex, int *element);

#ifdef __cplusplus
}
#endif
#endif
