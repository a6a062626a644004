/*
 * mcm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C interface of the CPU restatement of MCM 2.07's explicit SPH time step
 * (MarkoTopalovic/MCMtop, Fortran 90).  The oracle is the checker for the
 * CUDA path: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it.  The product library never links or calls it.
 *
 * Parity status: UNPINNED.  The reference ships no tests, golden vectors or
 * example decks, and no Fortran compiler exists on either machine, so the
 * restatement is checked only by line-by-line review against the cited
 * Fortran, by self-built known-answer tests and by physical invariants.
 */
#ifndef MCM_ORACLE_H
#define MCM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One material as it comes off the deck (MCM/mcm_matin.f90:41-54 and the
 * property cards :124-148), i.e. BEFORE the mcm_sets* rearrangement.  Zero
 * fields take the same defaults as mcm_matin.f90:46-56. */
typedef struct {
    int model;          /* 1, 3, 4 (cap), 9, 10 */
    int eos;            /* 0, 1, 4, 13, 28, 41 */
    int visc_type;      /* 0 -> 1 (nodal AV) */
    double rho;         /* reference density */
    double av_l, av_q;  /* artificial viscosity (0 -> 0.06 / 1.5) */
    double mass;        /* total material mass (massopt 0) */
    double h;           /* smoothing length (init_h_opt 0) */
    double rho_min, rho_max;
    double strinput[48];
    double eosinput[24];
    double k_cont, n_cont;  /* contact cards (MCM/mcm_contactype.f90:35), contacttype > 0 */
} mcmo_material;

/* Control cards (MCM/mcm_control_v2.f90:88-124), the symmetry cards
 * (MCM/mcm_inp_symmetry_v2.f90:29-53) and the base acceleration card
 * (MCM/mcm_baseaccel_in.f90:23-33). */
typedef struct {
    int ndim;           /* axopt 1..3 */
    int disctype;       /* 0 basic SPH, 1 mixed-corrected SPH */
    int nummat;
    int np;
    double endtime, tssf, itss, drelax_scale;
    int init_v_opt, massopt, init_h_opt, init_rhoe;
    int contacttype, tcrit_opt, veloc_opt, mirr_opt;
    int nthp[3];
    int h_opt, krtype, maxnbr;
    int sym_flag[6];    /* xmin xmax ymin ymax zmin zmax: 0 none, 1 symmetry, 2 periodic */
    double sym_x[6];
    double base_a[3];
} mcmo_deck;

/* Status codes (shared meaning with include/mcm_gpu.h). */
#define MCMO_OK 0
#define MCMO_EUNSUPPORTED 9
#define MCMO_ECOMPLEX_C 3
#define MCMO_EINVAL 8
#define MCMO_ECAP_NOCONV 4

/* x, v: Fortran layout (3,np); mat, dispbc: (np); pardata: (4,np) holding
 * mass, h, rho, e (MCM/mcm_nodein.f90:86-131) or NULL. */
void *mcmo_create(const mcmo_deck *deck, const mcmo_material *mats,
                  const double *x, const double *v, const int *mat,
                  const int *dispbc, const double *pardata, int *status);
void mcmo_destroy(void *sim);

/* One pass of the mcm_solution loop body (MCM/mcm_solution.f90:37-138),
 * split at the same points as the GPU C ABI. */
int mcmo_step_a(void *sim, double *critts);     /* neighbours, strain, constitutive */
int mcmo_dt_update(void *sim);                  /* mcm_solution.f90:58-62 */
int mcmo_step_b(void *sim);                     /* momentum, boundcond, calctotale */
int mcmo_ended(void *sim);                      /* mcm_solution.f90:101 */
int mcmo_step_c(void *sim);                     /* update_velocity, move */
/* Whole loop iterations; stops early at termination.  *done = steps run. */
int mcmo_run(void *sim, int nsteps, int *done);

/* Per-particle field copies (Fortran layout: vectors (3,np), tensors (3,3,np)). */
int mcmo_get(void *sim, const char *field, double *out);
int mcmo_get_int(void *sim, const char *field, int *out);
int mcmo_set(void *sim, const char *field, const double *in);
double mcmo_scalar(void *sim, const char *name);
int mcmo_set_scalar(void *sim, const char *name, double value);
/* Neighbour lists: returns count; 1-based ids as in mcm_nbrlist. */
int mcmo_nbrlist(void *sim, int i, int *out, int cap);
int mcmo_g_nbrlist(void *sim, int i, int *out, int cap);
/* Contact lists (other materials' particles, contacttype > 0) and the
 * per-material contact forces xcf, ycf, zcf of the last mcm_oldacceleration. */
int mcmo_contlist(void *sim, int i, int *out, int cap);
int mcmo_g_contlist(void *sim, int i, int *out, int cap);
int mcmo_contact_forces(void *sim, double *xyz);
/* Ghosts created by the last mcm_ghost_setup: source particle id and x. */
int mcmo_ghosts(void *sim, int *par_out, double *x_out, double *v_out, int cap);
int mcmo_grid(void *sim, int *gridlim, double *gridmin, double *gridsize);
int mcmo_material_energy(void *sim, double *ke, double *ie, double *mom);
int mcmo_material_table(void *sim, int m, double *strinput, double *eosinput,
                        double *g);

/* Kernel known-answer hooks (MCM/mcm_kernel.f90, MCM/mcm_gradw.f90). */
double mcmo_kernel_w(int ndim, const double *xi, const double *xj, double havg);
void mcmo_gradw(int ndim, const double *xi, const double *xj, double havg,
                double *dwdx);

#ifdef __cplusplus
}
#endif
#endif
