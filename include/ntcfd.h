/*
 * ntcfd.h -- C-ABI of the B200 projection-method time step.
 *
 * This is the drop-in boundary for NTUSTCFD's time-step loop body
 * (main.f90:209-259): Smagorinsky viscosity, QUICK predictor, SOR pressure
 * Poisson solve, projection, direct-forcing immersed boundary, force
 * integral, velocity update and boundary conditions.  The reference calls
 * argument-less Fortran subroutines that work on MODULE variables
 * (variables_module.f90); here the same state lives in device memory owned
 * by an opaque context, and the Fortran driver reaches it through
 * ISO_C_BINDING (see fortran/ntcfd_iface.f90).
 *
 * Conventions shared by every entry point:
 *  - Halo arrays are Fortran order (i fastest), index range -1..n+2 in each
 *    direction, i.e. (nx+4)*(ny+4)*(nz+4) doubles, exactly the layout of
 *    `real*8, dimension(-1:nx+2,-1:ny+2,-1:nz+2)` in variables_module.f90:215-223.
 *  - Interior arrays (pre, uc, vc, wc) are (nx,ny,nz), Fortran order
 *    (variables_module.f90:225).
 *  - 1-D metrics iDx/Dxs/... have n+4 entries, index -1..n+2
 *    (variables_module.f90:306-316); node coordinates X/Y/Z have n+5
 *    entries, index -1..n+3 (variables_module.f90:292-296).
 *  - Every pointer argument is HOST memory; calls are synchronous at return.
 *  - Every call returns 0 on success, a negative NTCFD_E* code on error
 *    (ntcfd_last_error() gives the message), or the positive warning
 *    NTCFD_NOT_CONVERGED when an SOR solve stopped at itmax (the reference
 *    continues silently in that case, GS.f90:11).
 *  - A context is used by one host thread at a time and owns one CUDA stream.
 */
#ifndef NTCFD_H
#define NTCFD_H

#ifdef __cplusplus
extern "C" {
#endif

#define NTCFD_OK              0
#define NTCFD_NOT_CONVERGED   1   /* warning: at least one SOR solve hit itmax */
#define NTCFD_EINVAL        (-1)  /* bad parameter or argument */
#define NTCFD_ECUDA         (-2)  /* CUDA runtime error */
#define NTCFD_ENOMEM        (-3)  /* device allocation failed */
#define NTCFD_ENONFINITE    (-4)  /* NaN/Inf detected in the SOR residual */
#define NTCFD_ESTATE        (-5)  /* call out of order (e.g. no metrics yet) */
#define NTCFD_ETIMEOUT      (-6)  /* a bounded device wait gave up */

/* Boundary-condition kinds: the strings 'no-slip', 'Neumann', 'Dirichlet'
 * of variables_module.f90:110-132, plus PERIODIC (no reference counterpart). */
enum { NTCFD_BC_NOSLIP = 0, NTCFD_BC_NEUMANN = 1, NTCFD_BC_DIRICHLET = 2,
       NTCFD_BC_PERIODIC = 3,
       NTCFD_BC_INTERFACE = 4 /* Back/Front only, all three components: the face is
                                 shared with the neighbouring z-slab (ntcfd_slab_stage) */ };
/* Walls, in the order boundary_conditions.f90 applies them (13-301). */
enum { NTCFD_WEST = 0, NTCFD_EAST = 1, NTCFD_SOUTH = 2, NTCFD_NORTH = 3,
       NTCFD_BACK = 4, NTCFD_FRONT = 5 };
enum { NTCFD_FP64 = 0, NTCFD_MIXED = 1 };
/* K2 predictor: discretisation_QUICK_centre.f90 (the one main.f90:213 calls),
 * or the reference's uncalled alternatives discretisation_QUICK.f90,
 * discretisation_upwind.f90, discretisation_centre.f90, with their flag Q1
 * read as LES and their own inline eddy viscosity.  The alternatives predict
 * u* on i < nx, v* on j < ny, w* on k < nz (the wall faces keep u), and
 * ntcfd_adjoint does not differentiate them. */
enum { NTCFD_QUICK_CENTRE = 0, NTCFD_QUICK = 1, NTCFD_UPWIND = 2, NTCFD_CENTRE = 3 };
enum { NTCFD_SMAG_REF_ALIASED = 0, NTCFD_SMAG_STAGGERED = 1 };
enum { NTCFD_SOR_REDBLACK = 0, NTCFD_SOR_LEX = 1 };    /* LEX: oracle only */
/* How the sweeps of one correction cycle run on the device:
 * STREAMING -- two kernels per sweep (one per colour) reading e from
 *              global memory, the loop driven by CUDA-graph conditional nodes;
 * RESIDENT  -- one persistent cooperative kernel per cycle with e kept in
 *              shared memory (only when the grid's e fits on the chip);
 * AUTO      -- RESIDENT when it fits, else STREAMING.  Both run the same
 *              red-black iteration and stop rule. */
enum { NTCFD_SOR_AUTO = 0, NTCFD_SOR_STREAMING = 1, NTCFD_SOR_RESIDENT = 2 };

typedef struct ntcfd_params {
    int nx, ny, nz;          /* interior cells (variables_module.f90:13-17) */
    double Re;               /* nu = 1/Re (reading_data.f90:38) */
    double dt;               /* time step (variables_module.f90:11) */
    double omega;            /* SOR relaxation (main.f90:44) */
    double zeta;             /* SOR stop: max|pNew-p| <= zeta (main.f90:46, GS.f90:11) */
    int itmax;               /* SOR sweep cap (main.f90:48) */
    int LES;                 /* 1: add Smagorinsky nu_t (main.f90:60) */
    double Cs;               /* Smagorinsky constant (variables_module.f90:277) */
    int scheme;              /* NTCFD_QUICK_CENTRE (default), NTCFD_QUICK, NTCFD_UPWIND, NTCFD_CENTRE */
    int precision;           /* NTCFD_FP64 or NTCFD_MIXED */
    int sor_order;           /* NTCFD_SOR_REDBLACK on the device */
    int smag_mode;           /* NTCFD_SMAG_REF_ALIASED (reference indexing) or _STAGGERED */
    int check_every;         /* test the SOR stop rule every c sweeps (1 = every sweep) */
    int bc[6][3];            /* [wall][u,v,w] kind */
    double bc_value[6][3];   /* Dirichlet value (the reference hard-codes 1.0) */
    double u_solid[3];       /* solid velocity in the forcing (variables_module.f90:331-335) */
    double lx;               /* force-coefficient normalisation (virtualForceIntegrator.f90:80-81) */
    int mixed_cycle;         /* sweeps per defect-correction cycle; 0: 8 for MIXED, itmax for FP64 */
    int diag_divergence;     /* 1: report max|div u^{n+1}| in ntcfd_step_info.div_max */
    int device;              /* CUDA device ordinal that holds the grid */
    int sor_path;            /* NTCFD_SOR_AUTO, NTCFD_SOR_STREAMING or NTCFD_SOR_RESIDENT */
    int eager;               /* 1: launch the step's kernels one by one from the host (no
                                CUDA graph; for kernel profilers and debugging, slower) */
    int reserved[3];         /* must be zero */
} ntcfd_params;

typedef struct ntcfd_step_info {
    int sor_iters;           /* sweeps this step (GS.f90:96-103 prints the same count) */
    int converged;           /* 1 if the stop rule fired before itmax */
    double sor_last_change;  /* max|pNew-p| of the last checked sweep */
    double cDrag, cLift;     /* virtualForceIntegrator.f90:80-81 */
    double div_max;          /* max |div u^{n+1}| * V (FP64) when diag_divergence = 1 */
    int dc_cycles;           /* defect-correction cycles used */
    int launches;            /* device kernels launched for this step */
    int sor_path;            /* NTCFD_SOR_STREAMING or NTCFD_SOR_RESIDENT: the path that ran */
    int pad;
    double aoa;              /* angle of attack of the step's mask under ntcfd_set_dynamic_aoa, else 0 */
} ntcfd_step_info;

/* Average device time of single kernels of the step, for the roofline. */
typedef struct ntcfd_kernel_times {
    float predictor_ms;      /* K2 (with K1 when LES = 1), one launch */
    float rhs_ms;            /* K3a */
    float defect_ms;         /* defect pass of a correction cycle */
    float sweep_ms;          /* one half-sweep (one colour) */
    float project_ms;        /* K4, measured on a copy of the velocity */
    float bc_ms;             /* the three K6 launches together */
    float resident_ms;       /* one resident-SOR launch running resident_sweeps sweeps (0 if unused) */
    float resident_sweeps;
} ntcfd_kernel_times;

typedef struct ntcfd_ctx ntcfd_ctx;

/* Fills p with the reference defaults: 40^3, Re=10, dt=1e-3, omega=1.5,
 * zeta=1e-4, itmax=3000, LES=0, Cs=0.18, cavity walls with the lid on the
 * north wall moving in w (variables_module.f90:9-23,110-132,277; main.f90:44-60). */
void ntcfd_default_params(ntcfd_params* p);

/* Replaces program init: allocation of the MODULE arrays and
 * initial_conditions() (initial_conditions.f90:9-29, all fields zero). */
int  ntcfd_create(const ntcfd_params* p, ntcfd_ctx** out);
void ntcfd_destroy(ntcfd_ctx* ctx);
const char* ntcfd_last_error(const ntcfd_ctx* ctx);

/* Grid metrics made by gridder_equal/gridder_Unequal (gridder.f90:97-157). */
int ntcfd_set_metrics(ntcfd_ctx* ctx,
                      const double* iDx, const double* Dxs,
                      const double* iDy, const double* Dys,
                      const double* iDz, const double* Dzs);
/* Node coordinates X, Y, Z (gridder.f90:34-93); needed by the mask builders. */
int ntcfd_set_coords(ntcfd_ctx* ctx, const double* X, const double* Y, const double* Z);

/* Volume fraction ETA (variables_module.f90:159), a halo array. */
int ntcfd_set_mask(ntcfd_ctx* ctx, const double* eta);
int ntcfd_get_mask(ntcfd_ctx* ctx, double* eta);
/* RayCasting (airfoil.f90:580-915) on the device: polygon (az[m], ay[m]),
 * m < npts, is shifted by -0.25, rotated by -aoa_deg, moved to (zc, yc) and
 * scan-converted into ETA with 50x50 sub-cells on cut cells.  ties_out
 * (may be NULL) receives the number of exact vertex/grid ties met, which
 * the reference resolves by moving the grid (airfoil.f90:700-702). */
int ntcfd_build_mask_polygon(ntcfd_ctx* ctx, const double* az, const double* ay, int npts,
                             double aoa_deg, double zc, double yc, int* ties_out);
/* A smoothed, differentiable mask of the same body, for gradients with
 * respect to its angle of attack (no counterpart in the reference).  The
 * polygon is moved exactly as ntcfd_build_mask_polygon moves it
 * (airfoil.f90:597-611); each cell's ETA is a C1 ramp of the signed distance
 * d (negative inside) from its (y,z) centre to the polygon: with
 * tau = -d / width, ETA = 1 for tau >= 1, 0 for tau <= -1 and
 * 0.5 + 0.75 tau - 0.25 tau^3 between (so the mask is the ray-cast body
 * blurred over +-width).  The context keeps dETA/dAOA, and ntcfd_adjoint then
 * also reports dJ/dAOA through the rotating body (dJ_daoa_body).  Any other
 * mask call replaces it. */
int ntcfd_build_mask_smooth(ntcfd_ctx* ctx, const double* az, const double* ay, int npts,
                            double aoa_deg, double zc, double yc, double width);
/* Same result as ntcfd_build_mask_polygon, for callers that must not
 * allocate device memory after set-up.  No counterpart in the reference.
 *
 * ntcfd_build_mask_polygon allocates and frees device scratch (the moved
 * polygon, the cut-cell list, a tie counter) on every call.  A driver that
 * rebuilds the mask inside its time loop -- a dynamic angle of attack re-runs
 * the ray casting every step -- cannot afford that: cudaFree waits for all
 * work on the device, so each step would stall, and a caller whose device
 * memory is already handed out to its own allocator may find cudaMalloc
 * failing mid-run.  This variant keeps that scratch in one fixed array that
 * the library reserves on every device that loads it (2.5 MiB, held
 * until the process exits) and calls no cudaMalloc, cudaFree or other
 * allocating routine; ETA goes to the context's existing storage.  The
 * polygon is turned, its cut cells found and compacted and their sub-cell
 * fractions summed on the device; the call waits for the stream once, to
 * read the tie count.
 *
 * Limits: npts <= 16384 polygon points and ny*nz <= 262144 cells in the
 * (k,j) plane; larger inputs return NTCFD_EINVAL before any device work.
 * The first call on a device looks up the array's device address (once per
 * device); make that first call before any stream capture.  All calls on a
 * device share the array: its control block, counters and cut-cell flags
 * are cleared by each call, and two calls that overlap on the GPU (from two host threads
 * or two contexts on one device) race on it. */
int ntcfd_build_mask_polygon_noalloc(ntcfd_ctx* ctx, const double* az, const double* ay,
                                     int npts, double aoa_deg, double zc, double yc,
                                     int* ties_out);
/* DFIB_Cylinder (DFIB.f90:74-145): cylinder along x, centre (zc, yc), radius r,
 * 50x50 sub-cells within half a cell diagonal of the surface, real*4 arithmetic. */
int ntcfd_build_mask_cylinder(ntcfd_ctx* ctx, double zc, double yc, double r);

/* Velocity and pressure halo arrays in and out (exact FP64 checkpoints).
 * These calls and ntcfd_set_mask/get_mask copy each array in one piece
 * through a device staging array of one halo array, which the context makes
 * on the first such call and keeps until ntcfd_destroy. */
int ntcfd_set_state(ntcfd_ctx* ctx, const double* u, const double* v,
                    const double* w, const double* p);
int ntcfd_get_state(ntcfd_ctx* ctx, double* u, double* v, double* w, double* p);

/* boundary_conditions() (boundary_conditions.f90:13-374) on the device
 * state; the driver calls it once after ntcfd_set_state, as main.f90:100 does. */
int ntcfd_apply_bc(ntcfd_ctx* ctx);

/* Output fields of the last completed step: pre = p after the SOR solve
 * (GS.f90:86-94) and the centred velocities uc, vc, wc computed from the
 * projected, forced velocity before the end-of-step boundary conditions
 * (calcul_new_velocity.f90:171-181).  Each (nx,ny,nz); any may be NULL. */
int ntcfd_get_output(ntcfd_ctx* ctx, double* pre, double* uc, double* vc, double* wc);

/* nsteps passes of the loop body main.f90:209-259 plus `time += dt`.
 * per_step (nsteps entries) may be NULL. */
int ntcfd_step(ntcfd_ctx* ctx, int nsteps, ntcfd_step_info* per_step);

/* Simulated time (main.f90:271). */
double ntcfd_time(const ntcfd_ctx* ctx);

/* Device time of the last ntcfd_step call: CUDA events recorded on the
 * context's stream before the first and after the last step launch. */
int ntcfd_last_step_ms(const ntcfd_ctx* ctx, float* ms);

/* Times `reps` standalone launches of each step kernel on the context's
 * stream with CUDA events and returns the averages.  The velocity, pressure
 * and ETA of the context are left unchanged. */
int ntcfd_time_kernels(ntcfd_ctx* ctx, int reps, ntcfd_kernel_times* out);

/* dynamic_AOA + RayCasting inside the time loop (airfoil.f90:311-321,
 * main.f90:144-155).  From the context's step start_step on (steps counted
 * from 1 over every ntcfd_step call), each step first sets
 *     AOA = aoa1 + 10 |sin(2 pi f (time - dt (start_step - 1)))|,
 *     f = reduce_frequency / pi,
 * with time the simulated time before the step and pi the reference's
 * default-real literal 3.14159265359, and rebuilds ETA by ray casting the
 * polygon (az, ay) at that angle about (zc, yc) as ntcfd_build_mask_polygon
 * does.  The host evaluates each step's angle and its cosine and sine; the
 * rotation, the ray casting and ETA are computed on the device inside the
 * step's CUDA graph (a second graph: the mask kernels, then the step under a
 * conditional node), so a call of many steps makes no per-step host round
 * trip.  The arrays are the context's own (allocated here; no limit on npts
 * or ny*nz beyond device memory), so contexts on one device do not share
 * them.  The angle used is reported in ntcfd_step_info.aoa.  A step whose
 * polygon meets an exact vertex/grid tie stops the call with NTCFD_EINVAL
 * (the reference moves the grid instead): that step and the rest of the call
 * do nothing, ETA holds the tied step's mask, and per_step, ntcfd_time and
 * the step count account for exactly the steps that ran.  npts = 0 switches
 * the dynamic angle off.  An eager context (or a driver that does not take
 * the conditional graph) launches the same kernels one by one and reads the
 * tie count after each step's mask. */
int ntcfd_set_dynamic_aoa(ntcfd_ctx* ctx, const double* az, const double* ay, int npts,
                          double aoa1, double reduce_frequency, double zc, double yc,
                          int start_step);

/* z-slab decomposition (Mpi_division.f90:6-24): one context (one GPU, one
 * process) per slab of z planes, created with the slab's nz, the slab's
 * slice of the z metrics (ghost entries from the neighbours' cells) and
 * NTCFD_BC_INTERFACE on each face shared with a neighbour.  Such a context
 * does not take ntcfd_step; the caller runs each step as
 *     exchange u, v, w (2 planes)                  main.f90:163-183
 *     NTCFD_STAGE_PREDICT
 *     exchange w* (1 plane)                        main.f90:220-226
 *     exchange p (1 plane); NTCFD_STAGE_RHS
 *     repeat: for the global red then black colour: NTCFD_STAGE_HALFSWEEP
 *             with the slab's own colour (the global one flipped when the
 *             slab's first plane has an even global index), then exchange
 *             that colour's e (1 plane);              GS.f90:20-28
 *             max over the slabs of ntcfd_slab_change; stop as GS.f90:11
 *     NTCFD_STAGE_CORRECT; exchange p (1 plane)     main.f90:236-242
 *     NTCFD_STAGE_PROJECT
 * where "exchange f (n planes)" moves a slab's first n interior planes of f
 * into the lower neighbour's top n ghost planes and its last n interior
 * planes into the upper neighbour's bottom n ghost planes.  The stages run
 * the FP64 streaming kernels of ntcfd_step, so the decomposed step repeats
 * the single-domain FP64 streaming step bit for bit.  The force integral is
 * not formed on slabs.  FP64 contexts only. */
enum { NTCFD_FIELD_U = 0, NTCFD_FIELD_V = 1, NTCFD_FIELD_W = 2, NTCFD_FIELD_P = 3,
       NTCFD_FIELD_WSTAR = 4, NTCFD_FIELD_E_RED = 5, NTCFD_FIELD_E_BLACK = 6 };
enum { NTCFD_STAGE_PREDICT = 0, NTCFD_STAGE_RHS = 1, NTCFD_STAGE_HALFSWEEP = 2,
       NTCFD_STAGE_CORRECT = 3, NTCFD_STAGE_PROJECT = 4 };
/* Launches one stage on the context's stream (colour: the half-sweep's
 * colour in the slab's own indexing, 0 = (i+j+k) even). */
int ntcfd_slab_stage(ntcfd_ctx* ctx, int stage, int colour);
/* max |change| of the half-sweeps since the last call (then cleared). */
int ntcfd_slab_change(ntcfd_ctx* ctx, double* max_change);
/* Elements of one z plane of a field (natural or colour-split layout). */
long long ntcfd_slab_plane_elems(const ntcfd_ctx* ctx, int field);
/* Copies planes k0..k0+count-1 (k in -1..nz+2) of a field out of the
 * context (put = 0) or into it (put = 1); buf holds count * plane_elems
 * doubles in host or device memory.  Waits for the copy. */
int ntcfd_slab_planes(ntcfd_ctx* ctx, int field, int k0, int count, double* buf, int put);

/* The centred output of ntcfd_get_output without waiting for it
 * (filereachtime every isto steps, main.f90:318-324): the fields of the last
 * completed step are formed on the context's stream and copied into pre, uc,
 * vc, wc on a second stream while the following ntcfd_step calls run.  The
 * arrays (any may be NULL) belong to the copy until ntcfd_output_wait
 * returns: the caller neither reads nor frees them before that.  Pinned
 * (page-locked) arrays are written by the copy engine directly; pageable
 * ones through a context-owned pinned buffer and a stream callback, off the
 * caller's thread.  One output is in flight at a time: ntcfd_output_async
 * first waits for the previous one.  The first call allocates its buffers. */
int ntcfd_output_async(ntcfd_ctx* ctx, double* pre, double* uc, double* vc, double* wc);
int ntcfd_output_wait(ntcfd_ctx* ctx);

/* ------------------------------------------------------------------------
 * Body force and discrete adjoint.  No counterpart in the reference: its
 * momentum equation has no source term and it computes no derivatives.
 * ---------------------------------------------------------------------- */

/* Per-cell body force added by the predictor: u* += dt fu, v* += dt fv,
 * w* += dt fw at the staggered points (i,j,k) of each component.  Each array
 * is (nx,ny,nz) in Fortran order; a NULL array counts as zero, and three
 * NULLs remove the force. */
int ntcfd_set_body_force(ntcfd_ctx* ctx, const double* fu, const double* fv, const double* fw);

typedef struct ntcfd_adj_spec {
    int nsteps;              /* K: steps taken from the context's current state */
    int checkpoint_every;    /* M >= 1: (u,v,w,p) kept every M steps, the rest recomputed */
    double w_drag, w_lift;   /* J = (1/K) sum over the K steps of (w_drag cDrag + w_lift cLift) */
    double adj_zeta;         /* adjoint Poisson stop rule: max|change| <= adj_zeta * max|rhs| (0: 1e-7) */
    double adj_omega;        /* SOR relaxation of the adjoint solves, 0 < adj_omega < 2 (0: 1.9; the
                                forward keeps the reference's omega, the adjoint solve is free to
                                relax closer to the optimum) */
    int adj_itmax;           /* sweep cap of one adjoint Poisson solve (0: 20000) */
    int inflow_wall;         /* NTCFD_WEST..NTCFD_FRONT, or -1: the wall whose Dirichlet values are */
    int inflow_normal;       /*   bc_value[inflow_wall][inflow_normal]     = U cos(theta) */
    int inflow_tangential;   /*   bc_value[inflow_wall][inflow_tangential] = U sin(theta) */
    int initial_bc;          /* 1: apply boundary_conditions() to the state first (as main.f90:100
                                does at start-up) and differentiate through it; 0: the state,
                                ghosts included, is held fixed */
    int reserved[3];         /* must be zero */
} ntcfd_adj_spec;

typedef struct ntcfd_adj_result {
    double J;                /* objective of the forward pass */
    double dJ_dbc[6][3];     /* dJ / d bc_value[wall][component] (Dirichlet walls; 0 elsewhere) */
    double dJ_dU;            /* inflow speed and angle (radians) from inflow_wall, else 0 */
    double dJ_dtheta;
    double forward_ms;       /* device time of the forward pass (K steps and their checkpoints) */
    double total_ms;         /* wall time of the whole call */
    double recompute_ms;     /* device time of the steps re-run from checkpoints */
    double solve_ms;         /* device time of the adjoint Poisson solves */
    long long adj_sweeps;    /* sweeps of all adjoint Poisson solves */
    int adj_unconverged;     /* adjoint solves that stopped at adj_itmax */
    int recomputed_steps;    /* forward steps re-run from checkpoints */
    int fwd_status;          /* status of the forward pass (0 or NTCFD_NOT_CONVERGED) */
    int pad;
    double dJ_daoa_body;     /* dJ / d(the body's angle of attack), per radian, through the body's
                                rotation, when ETA is the mask of ntcfd_build_mask_smooth; else 0 */
} ntcfd_adj_result;

/* Discrete adjoint of K steps.  Runs the K steps forward from the current
 * state (checkpointing every M steps), then the reverse pass: each step's
 * boundary conditions, force integral, projection and direct forcing,
 * converged pressure solve (the same SOR kernels on the transposed system),
 * divergence, QUICK predictor and Smagorinsky nu_t transposed about the
 * recomputed forward state.  The initial state is held fixed (after the
 * optional initial boundary conditions, see initial_bc); the pressure
 * solves are differentiated as exact solves (their initial guess does not
 * enter), the QUICK upwind branches and the force-integral guards as fixed.
 * dJ_df* (each (nx,ny,nz), Fortran order, may be NULL) receive dJ/dfu,
 * dJ/dfv, dJ/dfw of the body force.  per_step (K entries, may be NULL)
 * receives the forward steps' records.  On return the context holds the
 * state after the K steps, as ntcfd_step(ctx, K, ...) would leave it. */
int ntcfd_adjoint(ntcfd_ctx* ctx, const ntcfd_adj_spec* spec, ntcfd_adj_result* result,
                  double* dJ_dfu, double* dJ_dfv, double* dJ_dfw, ntcfd_step_info* per_step);

#ifdef __cplusplus
}
#endif

#endif /* NTCFD_H */
