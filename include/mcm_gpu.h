/*
 * mcm_gpu.h -- C ABI of the B200 (sm_100a) SPH explicit step for MCM 2.07.
 *
 * The reference (MarkoTopalovic/MCMtop) has no plugin or FFI layer: its time
 * loop MCM/mcm_solution.f90:37-138 calls argument-less subroutines that act on
 * the module arrays of MCM/mcm_database.f90 (par, gpar, mcm_mat).  This ABI
 * replaces the physics calls of that loop; the Fortran loop, its output,
 * termination test and Ctrl-C handling stay on the host:
 *
 *   reference loop body (mcm_solution.f90)       this ABI
 *   :41  mcm_neighbours  \
 *   :45  mcm_strain       > mcm_gpu_step_a(h, dt, &critts)
 *   :53  mcm_constitutive/
 *   :58-62 dt update     (host, unchanged)
 *   :69  mcm_momentum    \
 *   :73  mcm_boundcond    > mcm_gpu_step_b(h, energies)
 *   :77  mcm_calctotale  /
 *   :81-108 output / termination / ctrl-c (host, unchanged)
 *   :112 mcm_update_velocity \ mcm_gpu_step_c(h, dt, dtold, coord_maxmin)
 *   :116 mcm_move            /
 *
 * mcm_gpu_run() fuses whole loop iterations (dt update on the device) for
 * stretches with no output in between.
 *
 * Conventions: plain pointers and sizes; host arrays use the Fortran layout of
 * the reference (vectors (3,np), tensors (3,3,np), column-major); particle ids
 * are 1-based reference indices.  Host pointers are borrowed for the call only.
 * Every entry point returns an mcm_gpu_status; the library never exits, aborts
 * or traps a device.  One host thread per handle; handles are independent.
 */
#ifndef MCM_GPU_H
#define MCM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define MCM_GPU_ABI_VERSION 3
#define MCM_GPU_MAX_MATERIALS 16

/* Status codes.  The reference's fatal paths call mcm_shutdown(2)
 * (MCM/mcm_shutdown.f90); here they return a code instead. */
typedef enum {
    MCM_OK = 0,
    MCM_ENBR_OVERFLOW = 1,     /* neighbour table too narrow; regrown and retried internally
                                  (MCM/mcm_ll_neighbours.f90:44,301-309) */
    MCM_EGHOST_OVERFLOW = 2,   /* ghost storage too small; regrown and retried internally
                                  (MCM/mcm_ghost_setup.f90:269-282) */
    MCM_ECOMPLEX_C = 3,        /* eos41 c^2 < 0 (MCM/mcm_eos41c.f90:73-79) */
    MCM_ECAP_NOCONV = 4,       /* cap model Newton loop did not converge (MCM/mcm_f3dm25.f90) */
    MCM_ETIMEOUT = 5,          /* a bounded device wait ran out */
    MCM_ECUDA = 6,             /* CUDA runtime error (see mcm_gpu_last_error) */
    MCM_ENOMEM = 7,            /* device allocation failed */
    MCM_EINVAL = 8,            /* bad argument */
    MCM_EUNSUPPORTED = 9,      /* option outside the ported path (e.g. 1-D and 2-D problems) */
    MCM_EGRID_OVERFLOW = 10,   /* cell grid larger than its storage; regrown and retried internally */
    MCM_EGHOST_LAYER = 11,     /* a real particle lies in a ghost-layer cell (undefined in the reference) */
    MCM_EGRID_TOO_LARGE = 12   /* the linked-list grid would exceed 2^31 cells
                                  (MCM/mcm_setuplist.f90:85-92 shuts down when
                                  the grid cannot be allocated) */
} mcm_gpu_status;

/* Arithmetic of the step. */
typedef enum {
    MCM_PREC_FP64_EXACT = 0,   /* FP64, no fused multiply-add, reference accumulation order */
    MCM_PREC_FP64 = 1,         /* FP64 with fused multiply-add */
    MCM_PREC_MIXED = 2         /* FP32 strain-rate and momentum pair sums on cell-relative
                                  positions, lane sums combined by error-free (TwoSum)
                                  reduction; FP64 state, constitutive update, position/velocity
                                  integration, energy and critical-timestep reductions
                                  (disctype 0) */
} mcm_gpu_precision;

/* One material, as the reference holds it after mcm_matin, the mcm_sets routines and mcm_calcg:
 * `type material` of MCM/mcm_database.f90:235-257. */
typedef struct {
    int model;                 /* 1, 3, 4 (cap model: disctype 0), 9, 10 */
    int eos;                   /* 1, 4, 13, 28, 41 (models 9, 10) */
    int visc_type;             /* 1: nodal artificial viscosity */
    double rho;                /* reference density (rho0 of every particle of this material) */
    double g;                  /* shear modulus (mcm_calcg) */
    double av_l, av_q;         /* artificial viscosity coefficients */
    double mass;               /* total material mass (massopt 0) */
    double h;                  /* smoothing length */
    double rho_min, rho_max;   /* density limits */
    double strinput[48];       /* constitutive constants after mcm_sets* */
    double eosinput[24];       /* EOS constants */
    double k_cont, n_cont;     /* repulsive-contact strength K and exponent n (contact cards,
                                  MCM/mcm_contactype.f90:35; read when contacttype > 0) */
} mcm_gpu_material;

/* Run options: control cards (MCM/mcm_control_v2.f90:88-124), boundary planes
 * (MCM/mcm_inp_symmetry_v2.f90:115-137), base accelerations. */
typedef struct {
    int ndim;                  /* 3 (1-D and 2-D return MCM_EUNSUPPORTED) */
    int disctype;              /* 0 basic SPH, 1 Bonet mixed-corrected SPH */
    int tcrit_opt;             /* 0 DYNA formula, 1 h/(c+|v|), 2 mindist/(c+|v|) */
    int contacttype;           /* 0: kernel contact (other materials are neighbours); > 0: they are
                                  contacts instead, and Monaghan's repulsive acceleration over them
                                  (MCM/mcm_rep_contact.f90:37-94, called at mcm_solution.f90:64)
                                  starts each particle's momentum sum (mcm_oldacceleration.f90:49-56) */
    int h_opt;                 /* smoothing length: 0 constant, 1 from the volumetric strain rate,
                                  2 from the density (MCM/mcm_update_h.f90) */
    int veloc_opt;             /* 1: XSPH velocity smoothing (MCM/mcm_update_velocity.f90:61-87) */
    int krtype;                /* 1: cubic B-spline */
    int drelax;                /* dynamic relaxation active */
    double drelax_scale;
    int boundary;              /* mcm_boundary: ghost planes active */
    int boundary_code[6];      /* (side,dim) as mcm_boundary_code(2,3): xmin xmax ymin ymax zmin zmax;
                                  0 none, 1 symmetry, 2 periodic */
    double boundary_x[6];      /* plane coordinates, same order */
    int baseaccel;
    double base_a[3];
    double tssf;               /* timestep scale factor */
    double hmax;               /* mcm_hmax (grid cell = 2 hmax) */
    int precision;             /* mcm_gpu_precision */
    int nbr_stride;            /* initial neighbour-table stride (0: automatic) */
    int reorder_interval;      /* steps between particle re-sorts (0: never) */
    int block_size;            /* threads per block for the pair kernels (0: tuned default) */
    double nbr_skin;           /* 0: neighbour lists rebuilt from the cell list every step (the
                                  reference).  > 0 (FP64 and mixed precision, constant h): a skin
                                  list per particle of the particles within h_i + h_j + nbr_skin*hmax,
                                  rebuilt only when some particle has moved nbr_skin*hmax/2 since the
                                  last build, filtered every step to the reference's neighbour sets
                                  (not its order).  No counterpart in the reference. */
    int compensated_sums;      /* MCM_PREC_MIXED: 1 adds each lane's FP32 pair terms with Kahan
                                  compensation before the TwoSum lane combination; 0 adds them
                                  plainly (the faster default).  Ignored by the FP64 precisions. */
} mcm_gpu_config;

/* Host views of the particle arrays (Fortran layout, np particles).  NULL
 * members are skipped.  Mirrors the fields of `type particle`
 * (MCM/mcm_database.f90:159-216) that the step reads or writes. */
typedef struct {
    double *x, *v, *a;                         /* (3,np) */
    double *mass, *h, *hold, *rho, *rhoold, *e, *p, *c, *vabs;
    double *efps, *pcut, *p_cut, *fail, *mindist, *critts, *tracerod;
    double *etry, *einc, *capa;
    double *sigma, *s, *q, *qold, *alfa, *rod, *spin;   /* (3,3,np) */
    int *mat, *dispbc, *nnbr, *g_nnbr, *ptype;
    double *h0;                                /* initial h (h_opt 2); upload: NULL takes h */
    double *repulsion;                         /* (3,np) contact acceleration par%repulsion
                                                  (contacttype > 0); download only */
} mcm_gpu_fields;

typedef struct mcm_gpu_handle mcm_gpu_handle;

/* Time scalars of mcm_database (mcm_dt, mcm_dtold, mcm_ptime, mcm_endtime). */
typedef struct {
    double dt, dtold, ptime, endtime;
} mcm_gpu_time;

/* ---------------------------------------------------------------- set-up */

/* Selects the CUDA device that handles created by this host thread use
 * (the library links its own CUDA runtime). */
int mcm_gpu_set_device(int device);

/* Applies the deck defaults and rearrangements of MCM/mcm_matin.f90:46-56,
 * MCM/mcm_sets1.f90, mcm_sets3.f90, mcm_sets4.f90 (with its initial-cap and
 * tension cut-off iterations), mcm_sets10.f90 and mcm_calcg.f90 to a
 * material given as read from its cards.  Replaces those routines for callers
 * that do not run the Fortran input phase. */
int mcm_gpu_material_from_deck(mcm_gpu_material *m);

/* Allocates device storage for np particles.  Replaces the allocation part of
 * MCM/mcm_database.f90:mcm_allocate_memory and MCM/mcm_init_neighb.f90:25-46. */
int mcm_gpu_create(const mcm_gpu_config *cfg, const mcm_gpu_material *mats, int nmat,
                   int np, mcm_gpu_handle **out);
int mcm_gpu_destroy(mcm_gpu_handle *h);

/* Copies an already initialised particle state (what mcm_initial leaves in
 * par) to the device.  coord_maxmin (mcm_coord_maxmin(2,3), may be NULL: then
 * it is recomputed from x as MCM/mcm_initvbls.f90:81-91 does). */
int mcm_gpu_upload(mcm_gpu_handle *h, const mcm_gpu_fields *f, const double *coord_maxmin);

/* Runs mcm_initial (MCM/mcm_initial.f90:33-101) on the device from deck-level
 * particle data: f->x, f->v, f->mat, f->dispbc, and, when the deck gives them,
 * f->mass (massopt 1), f->h (init_h_opt 1), f->rho and f->e (init_rhoe 1).
 * massopt/init_h_opt/init_rhoe select which of those are read.  On return *t
 * holds the first dt (MCM/mcm_initial.f90:85-93) with ptime = 0. */
int mcm_gpu_initialise(mcm_gpu_handle *h, const mcm_gpu_fields *f, int massopt, int init_h_opt,
                       int init_rhoe, double itss, mcm_gpu_time *t);

/* Copies the non-NULL members of f back in the reference's particle order
 * (whatever order the device keeps its storage in).  Upload, initialise and
 * download move each host array in one copy through a device staging buffer
 * of 72 bytes per particle, allocated by the first of them, and convert the
 * layout on the device: page-locked host buffers move at the link's speed. */
int mcm_gpu_download(mcm_gpu_handle *h, mcm_gpu_fields *f);

/* ------------------------------------------------------------------ step */

/* Returns critts as soon as the neighbour search, strain rate and
 * constitutive update of the step are done.  The momentum sum and the energy
 * sums of step_b do not depend on the new dt (step_c moves the particles), so
 * step_a also enqueues them behind that work: they run on the device while
 * the caller updates dt, and the step_b that follows enqueues nothing (the
 * acceleration of a download between step_a and step_b is already the
 * step's).  An upload or mcm_gpu_run between step_a and step_b discards it. */
int mcm_gpu_step_a(mcm_gpu_handle *h, double dt, double *critts);
/* energies: per material ke, ie, mom(3) -> 5*nmat doubles (mcm_mat%ke, %ie, %mom),
 * then kinetice, internale, totale.  May be NULL.
 * step_b with energies NULL and step_c with coord_maxmin NULL (the next grid
 * reads the box on the device) only enqueue their work and return without
 * waiting; a device error they meet is returned by the next call that waits
 * (step_a, or step_b/step_c with an output, download). */
int mcm_gpu_step_b(mcm_gpu_handle *h, double *energies);
int mcm_gpu_step_c(mcm_gpu_handle *h, double dt, double dtold, double *coord_maxmin);

/* Up to nsteps whole loop iterations with the dt update of
 * MCM/mcm_solution.f90:58-62 and the termination test of :101 on the device.
 * *done receives the iterations completed (the last one may end at the
 * termination test, before the velocity and position update). */
int mcm_gpu_run(mcm_gpu_handle *h, int nsteps, mcm_gpu_time *t, int *done);

/* ----------------------------------------------------------- inspection */

/* Neighbour lists of the last search in reference order, 1-based ids.
 * nbr: (stride, np) like mcm_nbrlist(maxnbr,np); g_nbr: ghost indices like
 * mcm_g_nbrlist.  Either array may be NULL.  Returns MCM_EINVAL if a stride
 * is too small (the required strides are written to *stride / *g_stride). */
int mcm_gpu_neighbours(mcm_gpu_handle *h, int *nnbr, int *nbr, int *stride,
                       int *g_nnbr, int *g_nbr, int *g_stride);
/* Contact lists of the last search (contacttype > 0): particles of other
 * materials within reach, in the order mcm_ll_neighbours.f90:150-174 fills
 * mcm_contlist (1-based ids), and ghost contacts like mcm_g_contlist.  Same
 * conventions as mcm_gpu_neighbours; with contacttype 0 every count is 0. */
int mcm_gpu_contacts(mcm_gpu_handle *h, int *ncont, int *cont, int *stride,
                     int *g_ncont, int *g_cont, int *g_stride);
/* Per-material contact forces of the last step_b (mcm_mat%xcf, %ycf, %zcf:
 * the sums of mass x repulsion of MCM/mcm_oldacceleration.f90:52-55, written
 * to the time-history file by MCM/mcm_timehist.f90:46): 3*nmat doubles,
 * x y z per material.  Zero with contacttype 0 and with disctype 1, whose
 * momentum routine (MCM/mcm_corr_acceleration.f90) does not sum them. */
int mcm_gpu_contact_forces(mcm_gpu_handle *h, double *xyz);
/* Ghosts of the last mcm_ghost_setup: *ngp, source particle (1-based), x (3,ngp), v (3,ngp). */
int mcm_gpu_ghosts(mcm_gpu_handle *h, int *ngp, int *par, double *x, double *v, int cap);
/* Linked-list grid of the last search: gridlim(3), gridmin(3), gridsize(3). */
int mcm_gpu_grid(mcm_gpu_handle *h, int *gridlim, double *gridmin, double *gridsize);
int mcm_gpu_energies(mcm_gpu_handle *h, double *energies);

/* Skin-list builds since mcm_gpu_create (nbr_skin > 0; 0 otherwise). */
int mcm_gpu_skin_builds(mcm_gpu_handle *h, long long *builds);
/* Mean neighbour count of the last search (for the roofline accounting). */
int mcm_gpu_stats(mcm_gpu_handle *h, double *mean_nbr, int *max_nbr, int *stride, int *ngp);

/* -------------------------------------------------- allocation-free call */

/* No counterpart in the reference.  The per-material energy sums that
 * mcm_gpu_step_b returns (ke = sum 0.5 m vabs^2, ie = sum e, mom(3) = sum m |v_d|
 * per material, then kinetice, internale, totale: 5*nmat+3 doubles into
 * `energies`), summed over all np particles with no active-particle filter,
 * as step_b sums them, from DEVICE arrays the caller owns -- mass, vabs, e,
 * mat of length np and v in the (3,np) layout -- without allocating device
 * memory: for callers that cannot call cudaMalloc (a host code that gives all
 * device memory to its own pool, or must keep cudaMalloc/cudaFree and their
 * synchronisation out of the time step).  Particles whose mat lies outside
 * 1..nmat are skipped.  Its scratch is a fixed __device__ array of
 * 296 x 5 x 16 doubles (189 440 bytes per GPU, held until exit); nmat above
 * MCM_GPU_MAX_MATERIALS returns MCM_EINVAL.  The first call on each device
 * looks up the array's device address (make that first call before any
 * stream capture) and keeps it for the process: do not call it after a
 * cudaDeviceReset of that device.  Calls share the array,
 * so calls whose kernels overlap on the GPU race.  Runs on `stream` (NULL:
 * the default stream) and waits for it; an error already pending from the
 * caller's earlier CUDA work returns MCM_ECUDA before anything is launched. */
int mcm_gpu_calctotale_noalloc(const double *mass, const double *vabs, const double *v, const double *e,
                               const int *mat, int np, int nmat, double *energies, void *stream);

/* ------------------------------------------------------------- adjoint */

/* No counterpart in the reference (it has no differentiation).  Reverse-mode
 * gradients of a function of the final state with respect to the initial
 * state and to the material parameters, through the whole step: disctype 0,
 * every material model 10, or model 9 without viscosity (materials 1 and 2),
 * with EOS 1, 4, 13, 28 or 41, reorder_interval 0, constant h, no repulsive
 * contact, no skin lists.  The forward runs
 * in the handle's precision; the reverse kernels are FP64 and differentiate
 * the FP64 step along that forward trajectory (with MCM_PREC_MIXED: the
 * gradient of the step along the FP32-pair-sum trajectory).  The dt schedule is an input (the critical-timestep
 * minimum is not differentiated) and each step's neighbour lists are frozen
 * at their forward values.
 *
 * mcm_gpu_adjoint_forward runs nsteps loop iterations from the current state
 * with step_a(dts[n]), dt update to dts[n+1], step_b, step_c (dts has
 * nsteps+1 entries; dts[0] is the dt of the first step_a, normally the one
 * mcm_gpu_initialise returned) and keeps a full-state checkpoint every
 * checkpoint_every steps.  mcm_gpu_adjoint_backward takes the adjoints of the
 * final x and v (Fortran (3,np) layout; NULL = zero), recomputes each
 * checkpoint segment forward and runs the reverse steps backwards, and
 * returns dL/dx and dL/dv of the initial state (xbar0, vbar0, (3,np)) and, in
 * param_bar[nmat][4], dL/d(strinput[0], strinput[1], strinput[2],
 * eosinput[1]) of each material, in the card's units: for model 10 G, yield
 * stress and hardening modulus; eosinput[1] is the slope s of EOS 41 and 4,
 * the linear coefficient c1 of EOS 1 and gamma of EOS 28.  The device state is left as the
 * forward run left it. */
int mcm_gpu_adjoint_forward(mcm_gpu_handle *h, int nsteps, const double *dts, int checkpoint_every);
int mcm_gpu_adjoint_backward(mcm_gpu_handle *h, const double *xbar, const double *vbar, double *param_bar,
                             double *xbar0, double *vbar0);

/* ------------------------------------------------ launch shape, batches */

/* No counterpart in the reference (a serial code).  Launch shape of a handle's
 * neighbour search and cooperative gathers (the FP64-fast and mixed strain and
 * momentum kernels; the FP64-exact step keeps one thread per particle).  The
 * results do not depend on it, except that per-material energy sums are
 * combined over a different number of block partials.  Zero fields keep the
 * current value. */
typedef struct {
    int search_threads;      /* threads per block of the search: 64, 128 or 256 */
    int pair_threads;        /* threads per block of the gathers: 64, 128 or 256 */
    int pair_blocks_per_sm;  /* blocks per SM the gathers' persistent grid is sized for: 1..16 (reported as
                                0 while it is the blocks resident per SM, the default) */
    int nbr_stride;          /* neighbour-table row width in entries (rounded up to 4; still regrown
                                when a list outgrows it) */
    int search_kind;         /* 1: one thread per particle (the default), 2: one warp per particle,
                                3: one warp per cell (candidates staged in shared memory) */
    int pair_kind;           /* mixed-precision strain and momentum gathers: 1 neighbour records
                                through L1 (the default), 2 each block's rows of neighbour cells
                                staged in shared memory (the same sums) */
    int adj_kind;            /* reverse of the per-particle update in mcm_gpu_adjoint_backward: 1 one
                                hand-written reverse pass when every material is model 10 with EOS 41
                                (the default), 2 forward-mode dual numbers (any supported material) */
    double ms_per_step;      /* mcm_gpu_autotune: device time per loop iteration of the chosen shape */
} mcm_gpu_tuning;

int mcm_gpu_set_tuning(mcm_gpu_handle *h, const mcm_gpu_tuning *t);
int mcm_gpu_get_tuning(mcm_gpu_handle *h, mcm_gpu_tuning *t);
/* Times nsteps fused loop iterations (mcm_gpu_run) from the current state for
 * each candidate shape (search and gather block sizes, persistent-grid size,
 * and the neighbour-table stride rounded to 16 entries or not), keeps the
 * fastest, restores the state and time scalars, and returns the choice with
 * its time in *best (may be NULL).  Needs a copy of the particle state in
 * device memory for the duration of the call. */
int mcm_gpu_autotune(mcm_gpu_handle *h, int nsteps, mcm_gpu_tuning *best);

/* No counterpart in the reference.  Many independent bodies (one handle each,
 * initialised, on the device that is current at create, reorder_interval 0)
 * advanced together: one loop iteration of every body is one CUDA-graph
 * launch.  The bodies are spread over `lanes` streams (1..64), largest first
 * onto the least loaded lane, so bodies of uneven size run concurrently and
 * fill the GPU; each keeps its own dt, time scalars and termination.  The
 * handles must not be used through other entry points while a batch run is
 * in progress; they stay valid after mcm_gpu_batch_destroy. */
typedef struct mcm_gpu_batch mcm_gpu_batch;
int mcm_gpu_batch_create(mcm_gpu_handle *const *bodies, int nbodies, int lanes, mcm_gpu_batch **out);
/* Up to nsteps loop iterations of every body (mcm_gpu_run semantics per
 * body): times[b] in/out, done[b] = iterations body b completed (may be
 * NULL).  A body whose neighbour or ghost storage must grow is regrown and
 * brought level on its own stream; the graph is re-captured after a regrow. */
int mcm_gpu_batch_run(mcm_gpu_batch *b, int nsteps, mcm_gpu_time *times, int *done);
/* Times nsteps batched iterations for several lane counts from the current
 * states, restores every body's state and time scalars, and keeps the fastest
 * lane count (*lanes, *ms_per_step may be NULL). */
int mcm_gpu_batch_autotune(mcm_gpu_batch *b, int nsteps, int *lanes, double *ms_per_step);
/* No counterpart in the reference.  Gradients of every body of a batch:
 * mcm_gpu_adjoint_forward and mcm_gpu_adjoint_backward of each body (same
 * arguments, per body: dts[b] with nsteps+1 entries, xbar[b], vbar[b],
 * param_bar[b] (nmat x 4), xbar0[b], vbar0[b]; a NULL array of pointers is
 * NULL for every body), run by host worker threads -- at most the batch's
 * lane count and 16 -- that take the bodies largest first, each body's work
 * on its own stream, so that the bodies' kernels overlap on the GPU.  Each
 * body's results are those of its single-body calls.  Returns the first
 * failing body's status (the workers then stop taking bodies). */
int mcm_gpu_batch_adjoint_forward(mcm_gpu_batch *b, int nsteps, const double *const *dts, int checkpoint_every);
int mcm_gpu_batch_adjoint_backward(mcm_gpu_batch *b, const double *const *xbar, const double *const *vbar,
                                   double *const *param_bar, double *const *xbar0, double *const *vbar0);
int mcm_gpu_batch_destroy(mcm_gpu_batch *b);

/* ----------------------------------------------------------- measurement */

/* Diagnostic fields (rod, spin, tracerod, etry, einc, rhoold, critts, s, a)
 * are refreshed every step when enabled (the default).  The physics state is
 * computed identically either way; disabling only skips writing outputs that
 * no later part of the step reads. */
int mcm_gpu_set_diagnostics(mcm_gpu_handle *h, int enable);
/* Brackets every kernel group enqueued on the handle's stream with CUDA events
 * (enable = 1) and resets the launch counter.  The reference has no profiler;
 * its only timing is the commented-out MCM/mcm_write_timings.f90. */
int mcm_gpu_profile(mcm_gpu_handle *h, int enable);
/* Device time and launches of kernel group `region` (0..14) since
 * mcm_gpu_profile; returns MCM_EINVAL past the last group. */
int mcm_gpu_profile_report(mcm_gpu_handle *h, int region, char *name, int name_len, double *total_ms,
                           int *launches);
/* Kernels launched by this handle since the last mcm_gpu_profile call. */
long long mcm_gpu_kernel_launches(mcm_gpu_handle *h);
/* op 0: record a start event on the handle's stream; op 1: record a stop
 * event, wait for it and return the elapsed device time in *ms. */
int mcm_gpu_timer(mcm_gpu_handle *h, int op, double *ms);

const char *mcm_gpu_strerror(int status);
/* Text of the last CUDA error or failed check on this handle. */
const char *mcm_gpu_last_error(mcm_gpu_handle *h);
int mcm_gpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
