// mcm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// A C++17 FP64 restatement of the explicit SPH time step of MCM 2.07
// (MarkoTopalovic/MCMtop).  Every routine follows the Fortran file cited in
// its comment, in the reference's loop order, neighbour order (linked-list
// head insertion, z/y/x cell loops) and accumulation order, so that the CUDA
// path can be compared against it field by field.  Single-precision Fortran
// literals are reproduced as (double)float; Intel's mixed-kind sign/dim/max
// are promoted to FP64.  Build with -ffp-contract=off: the reference does not
// fuse multiply-adds.
//
// Parity status: UNPINNED (no reference tests, golden vectors or Fortran
// compiler exist to pin it); see the header.
//
// Documented deviations from the reference (all outside the configurations'
// reachable states):
//  * neighbour and ghost storage is unbounded, so the overflow/regrow paths of
//    MCM/mcm_ll_neighbours.f90:44,301-309 and MCM/mcm_ghost_setup.f90:269-282
//    are not needed; the final lists equal the reference's after its retry.
//  * MCM/mcm_f3dm10.f90:82-89 reads an uninitialised `defps` when fail /= 1;
//    here it is 0.
//  * only 3-D Cartesian problems (axopt 3) are restated for disctype 1; the
//    2-D branch of MCM/mcm_math_func.f90:inverse leaves entries undefined.

#include "mcm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

typedef double real;

inline real sq(real a) { return a * a; }
// Fortran `dim(x,y)` (MCM/mcm_f3dm10.f90:84)
inline real fdim_(real x, real y) { return x > y ? x - y : 0.0; }
// Fortran `sign(a,b)` with a>=0
inline real fsign(real a, real b) { return (b >= 0.0) ? std::fabs(a) : -std::fabs(a); }
inline real F32(float f) { return (real)f; }

struct Material {
    int model = 0, eos = 0, visc_type = 0;
    real rho = 0, g = 0, av_l = 0, av_q = 0, mass = 0, h = 0, rho_min = 0, rho_max = 0;
    real ke = 0, ie = 0, xcf = 0, ycf = 0, zcf = 0;
    real mom[3] = {0, 0, 0};
    real k_cont = 0, n_cont = 0;   // contact cards (MCM/mcm_contactype.f90:35)
    real strinput[48];
    real strinput2[48];
    real eosinput[24];
    // cm(i,j) view of strinput as cm(5,*)
    real &cm(int i, int j) { return strinput[(i - 1) + 5 * (j - 1)]; }
};

struct Particle {
    bool active = false;
    int mat = 0, dispbc = 0, llpointer = 0, nnbr = 0, ncont = 0, g_nnbr = 0, g_ncont = 0;
    real mass = 0, h = 0, hold = 0, h0 = 0, rho = 0, rho0 = 0, rhoold = 0, p = 0, e = 0,
         etry = 0, einc = 0, c = 0, vabs = 0, tracerod = 0, pcut = 0, p_cut = 0, efps = 0,
         fail = 0, temper = 0, mindist = 0, critts = 0, capa = 0;
    int ptype = 0;
    real epx[6] = {0, 0, 0, 0, 0, 0};
    real alfa[3][3] = {};
    real x[3] = {0, 0, 0}, xzero[3] = {0, 0, 0}, v[3] = {0, 0, 0}, a[3] = {0, 0, 0};
    real repulsion[3] = {0, 0, 0};   // contact acceleration (MCM/mcm_database.f90:206)
    real rod[3][3] = {}, spin[3][3] = {}, sigma[3][3] = {}, s[3][3] = {}, q[3][3] = {},
         qold[3][3] = {}, qq[3][3] = {};
    std::vector<int> nbr, cont, gnbr, gcont;
};

struct Ghost {
    int par = 0, mat = 0, llpointer = 0;
    real mass = 0, h = 0, hold = 0, rho = 0;
    real x[3] = {0, 0, 0}, xzero[3] = {0, 0, 0}, v[3] = {0, 0, 0};
    real sigma[3][3] = {}, q[3][3] = {};
};

struct Sim {
    // deck / control
    int ndim = 3, disctype = 0, nummat = 1, np = 0;
    int ssp = 1, esp = 0, svp = 1, evp = 0;
    real endtime = 0, tssf = 0, itss = 0, drelax_scale = 0;
    bool drelax = false, boundary = false, baseaccel = false;
    int init_v_opt = 0, massopt = 0, init_h_opt = 0, init_rhoe = 0;
    int contacttype = 0, tcrit_opt = 0, veloc_opt = 0, h_opt = 0, krtype = 1;
    int nthp[3] = {0, 0, 0};
    int maxnbr = 40, maxcont = 40, g_maxnbr = 20, g_maxcont = 20;
    real base_a[3] = {0, 0, 0};
    int boundary_code[2][3] = {};
    real boundary_x[2][3] = {};
    int boundary_type[3] = {1, 1, 1};
    real mult[6][3] = {}, add[6][3] = {};
    real pi = 0;
    // state
    std::vector<Particle> par;   // 1-based
    std::vector<Ghost> gpar;     // 1-based
    std::vector<Material> mat;   // 1-based
    int ngp = 0;
    real hmax = 0;
    real gridsize[3] = {0, 0, 0}, gridmin[3] = {0, 0, 0};
    int gridlim[3] = {1, 1, 1};
    std::vector<int> llgrid;
    real coord_maxmin[2][3] = {};
    real dt = 0, dtold = 0, ptime = 0, critts = 0, init_ts = 0;
    real kinetice = 0, internale = 0, totale = 0, thermale = 0;
    int timestep = 0;

    int &ll(int i, int j, int k) {
        return llgrid[(size_t)(i - 1) + (size_t)gridlim[0] * ((size_t)(j - 1) + (size_t)gridlim[1] * (size_t)(k - 1))];
    }

    // ------------------------------------------------------------------ input
    int setup(const mcmo_deck *d, const mcmo_material *m, const double *x, const double *v,
              const int *matid, const int *dispbc, const double *pardata);
    void sets1(Material &M);
    void sets3(Material &M);
    void sets10(Material &M);
    int sets4(Material &M);
    // ------------------------------------------------------------- init path
    void initial();
    void init_boundcond();
    void calcmass();
    void initvbls();
    void calcg();
    void calcrhopc();
    void eoscalc(int i);
    void eos1p(int i); void eos4p(int i); void eos13p(int i); void eos28p(int i); void eos41p(int i);
    void initsigma();
    void initrod();
    void init_h();
    void init_neighb();
    void initold();
    // --------------------------------------------------------------- step
    int step_a(real *critts_out);
    void dt_update();
    void step_b();
    bool ended() const { return ptime - dt >= endtime; }
    void step_c();
    // neighbours
    void neighbours();
    void setuplist();
    void init_boundary();
    void ghost_setup();
    void create_ghost_from_real(int id, int i, int j, int k, const real *mlt, const real *ad);
    void create_ghost_from_ghost(int id, int i, int j, int k, const real *mlt, const real *ad);
    void ll_neighbours(int ip_flag);
    // kernels
    real kernel1(const real *xi, const real *xj, real havg) const;
    void grad1(real *dwdx, real &dwdr, const real *xi, const real *xj, real havg) const;
    // strain
    void strain();
    void update_h();
    void xsph();
    void oldstrain();
    void corr_strain();
    void get_j_strain_info(int i, int k, real *x, real *v, real &mass, real &rho, real &h, real &hold);
    void inverse(const real B[3][3], real inv[3][3]) const;
    // constitutive
    int constitutive();
    void rhoupd();
    void stress_rot1(int i);
    void f3dm1(Material &M, int i);
    void f3dm3(Material &M, int i);
    void f3dm9(Material &M, int i);
    void f3dm10(Material &M, int i);
    int f3dm25(Material &M, int i);
    int sueos(int i);
    int eos1c(int i); int eos4c(int i); int eos13c(int i); int eos28c(int i); int eos41c(int i);
    void aviscosity(int i);
    void nodalav(int i);
    void hieupd(int i);
    void eqos(int i);
    void eqos1(int i); void eqos4(int i); void eqos13(int i); void eqos28(int i); void eqos41(int i);
    void stress_up(int i);
    void lieupd(int i);
    void calccritts();
    // repulsive contact (contacttype > 0)
    void rep_cont();
    real calc_fij(const real *xi, const real *xj, real havg, real inv_w_deltap) const;
    void get_j_cont_info(int i, int k, real *x, real &mass, real &rho, real &h, real &kj) const;
    // momentum
    void momentum();
    void update_ghost_stress();
    void oldacceleration();
    void corr_acceleration();
    void get_j_moment_info(int i, int k, real *x, real &mass, real &rho, real &h, real &hold,
                           real sig[3][3], real qq[3][3]);
    void boundcond();
    void calctotale();
    void update_velocity();
    void move();
    void check_sym_pen();

    int status = 0;
};

// =========================================================================
// Input processing: defaults of MCM/mcm_control_v2.f90:193-200, material
// defaults MCM/mcm_matin.f90:46-56 and the mcm_sets* routines.
// =========================================================================

// MCM/mcm_sets1.f90:23-51
void Sim::sets1(Material &M) {
    real prop[48];
    prop[0] = M.cm(1, 1); prop[1] = M.cm(1, 2); prop[2] = M.cm(1, 3); prop[3] = M.cm(1, 4);
    prop[4] = M.cm(1, 5); prop[5] = M.cm(2, 1); prop[6] = M.cm(3, 1);
    for (int i = 2; i <= 5; ++i)
        for (int j = 1; j <= 5; ++j) M.cm(i, j) = 0.0;
    real q1 = M.cm(1, 1) * M.cm(1, 2) / ((1.0 + M.cm(1, 2)) * (1.0 - 2.0 * M.cm(1, 2)));
    real q2 = M.cm(1, 1) * 0.5 / (1.0 + M.cm(1, 2));
    real q3 = q1 + 2.0 * q2;
    M.cm(2, 1) = q3; M.cm(3, 2) = q3; M.cm(4, 3) = q3; M.cm(5, 4) = q2;
    M.cm(2, 2) = q1; M.cm(2, 3) = q1; M.cm(3, 1) = q1; M.cm(3, 3) = q1; M.cm(4, 1) = q1; M.cm(4, 2) = q1;
    M.cm(2, 6) = M.cm(1, 6);
    M.cm(1, 6) = M.cm(1, 1) * M.cm(1, 4) / (M.cm(1, 1) - M.cm(1, 4));
    M.cm(1, 7) = prop[5];
    M.cm(2, 7) = prop[6];
}

// MCM/mcm_sets3.f90:23-43
void Sim::sets3(Material &M) {
    real prop7 = M.cm(2, 6);
    for (int i = 2; i <= 5; ++i)
        for (int j = 1; j <= 6; ++j) M.cm(i, j) = 0.0;
    real q1 = M.cm(1, 1) * M.cm(1, 2) / ((1.0 + M.cm(1, 2)) * (1.0 - 2.0 * M.cm(1, 2)));
    real q2 = M.cm(1, 1) * 0.5 / (1.0 + M.cm(1, 2));
    real q3 = q1 + 2.0 * q2;
    M.cm(2, 1) = q3;
    M.cm(5, 4) = q2;
    M.cm(2, 4) = M.cm(1, 1) * M.cm(1, 4) / (M.cm(1, 1) - M.cm(1, 4));
    M.cm(2, 6) = prop7;
}

// MCM/mcm_sets4.f90:21-41 and its initel (:43-98).  Both routines are
// `implicit double precision (a-h,o-z)`: everything is FP64 except the
// integer ltype and the single-precision literals (tol = 1.0e-3, 1.e10,
// 1.e-15 assigned to doubles keep their float values).  initel's Newton loops
// only print a message past maxit = 200 iterations and keep going; here they
// stop after 100000 and the material is rejected.
int Sim::sets4(Material &M) {
    real alpha = M.cm(1, 3), theta = M.cm(1, 4), gama = M.cm(1, 5), beta = M.cm(1, 6), r = M.cm(2, 1);
    real xint = M.cm(2, 5);
    real tempE = (9.0 * M.cm(1, 1) * M.cm(1, 2)) / (3.0 * M.cm(1, 1) + M.cm(1, 2));
    real tempNi = (3.0 * M.cm(1, 1) - tempE) / (6.0 * M.cm(1, 1));
    real q1 = tempE * tempNi / ((1.0 + tempNi) * (1.0 - 2.0 * tempNi));
    real q2 = tempE * 0.5 / (1.0 + tempNi);
    real q3 = q1 + 2.0 * q2;
    M.cm(5, 2) = q3;
    // initel: initial cap kappa0 from X0 = kappa + R Fe(kappa), then the
    // tension cut-off Fe(fcut) = 0
    const real tol = F32(1.0e-3f);
    real capint = 0.0, delcap = F32(1.e10f), delf = F32(1.e10f), fcut = 0.0;
    for (int it = 0;; ++it) {
        real fe = alpha - gama * std::exp(-beta * capint) + theta * capint;
        real psik = xint - capint - r * fe;
        real err1 = std::fabs(psik);
        real err2 = std::fabs(delcap) / (std::fabs(capint) + F32(1.e-15f));
        if (!((err1 > tol) && (err2 > tol))) break;
        if (it > 100000) return MCMO_EINVAL;
        real fep = beta * gama * std::exp(-beta * capint) + theta;
        real dpsik = -1.0 - r * fep;
        delcap = psik / dpsik;
        capint = capint - delcap;
    }
    for (int it = 0;; ++it) {
        real fe = alpha - gama * std::exp(-beta * fcut) + theta * fcut;
        real err1 = std::fabs(fe);
        real err2 = std::fabs(delf) / (std::fabs(fcut) + F32(1.e-15f));
        if (!((err1 > tol) && (err2 > tol))) break;
        if (it > 100000) return MCMO_EINVAL;
        real fep = gama * beta * std::exp(-beta * fcut) + theta;
        delf = fe / fep;
        fcut = fcut - delf;
    }
    M.cm(3, 3) = capint;
    M.cm(3, 4) = fcut;
    return MCMO_OK;
}

// MCM/mcm_sets10.f90:21-35
void Sim::sets10(Material &M) {
    real prop[48];
    for (int i = 0; i < 48; ++i) prop[i] = M.strinput[i];
    if (prop[3] == 0.0) prop[3] = F32(-1.e30f);
    if (prop[6] == 0.0) prop[6] = F32(1.000000001f);
    for (int i = 0; i < 48; ++i) M.strinput[i] = prop[i];
    for (int i = 2; i <= 16; ++i)
        if (prop[i + 15 - 1] < prop[i + 16 - 1]) M.strinput[15] = (real)i;
}

int Sim::setup(const mcmo_deck *d, const mcmo_material *m, const double *x, const double *v,
               const int *matid, const int *dispbc, const double *pardata) {
    pi = std::acos(-1.0);  // MCM/mcm_startup.f90:33
    ndim = d->ndim;
    if (ndim != 3 && d->disctype == 1) return MCMO_EUNSUPPORTED;
    if (ndim < 1 || ndim > 3) return MCMO_EINVAL;
    disctype = d->disctype;
    nummat = d->nummat;
    np = d->np;
    endtime = d->endtime; tssf = d->tssf; itss = d->itss; drelax_scale = d->drelax_scale;
    init_v_opt = d->init_v_opt; massopt = d->massopt; init_h_opt = d->init_h_opt; init_rhoe = d->init_rhoe;
    contacttype = d->contacttype; tcrit_opt = d->tcrit_opt; veloc_opt = d->veloc_opt;
    h_opt = d->h_opt; krtype = d->krtype; maxnbr = d->maxnbr;
    for (int k = 0; k < 3; ++k) nthp[k] = d->nthp[k];
    if (contacttype < 0 || h_opt < 0 || h_opt > 2 || veloc_opt < 0 || veloc_opt > 1) return MCMO_EUNSUPPORTED;
    // MCM/mcm_control_v2.f90:193-243
    if (tssf == 0.0) tssf = 0.8;
    if (krtype == 0) krtype = 1;
    if (krtype != 1) return MCMO_EUNSUPPORTED;
    if (maxnbr == 0) maxnbr = 40;
    boundary = (d->mirr_opt == 1);
    maxcont = maxnbr;
    g_maxnbr = maxnbr / 2;
    g_maxcont = g_maxnbr;
    drelax = (drelax_scale > 0.1 && drelax_scale < 1.0);
    ssp = 1; svp = 1; esp = np; evp = np;
    baseaccel = (nthp[0] == 1 || nthp[1] == 1 || nthp[2] == 1);
    // materials: MCM/mcm_matin.f90:41-161
    mat.assign(nummat + 1, Material());
    for (int n = 1; n <= nummat; ++n) {
        Material &M = mat[n];
        const mcmo_material &s = m[n - 1];
        M.model = s.model; M.eos = s.eos; M.visc_type = s.visc_type;
        M.rho = s.rho; M.av_l = s.av_l; M.av_q = s.av_q; M.mass = s.mass; M.h = s.h;
        M.rho_min = s.rho_min; M.rho_max = s.rho_max;
        M.k_cont = s.k_cont; M.n_cont = s.n_cont;
        for (int k = 0; k < 48; ++k) { M.strinput[k] = s.strinput[k]; M.strinput2[k] = 0; }
        for (int k = 0; k < 24; ++k) M.eosinput[k] = s.eosinput[k];
        if (M.visc_type == 0) M.visc_type = 1;
        if (M.av_l == 0.0) M.av_l = 0.06;
        if (M.av_q == 0.0) M.av_q = 1.5;
        if (M.rho_min == 0.0) M.rho_min = 1.0E-10;
        if (M.rho_max == 0.0) M.rho_max = 1.0E+10;
        switch (M.model) {
            case 1: case 3:
                if (M.eos != 0) return MCMO_EINVAL;
                break;
            case 4:
                if (M.eos != 0) return MCMO_EINVAL;
                break;
            case 9: case 10:
                if (!(M.eos == 1 || M.eos == 4 || M.eos == 13 || M.eos == 28 || M.eos == 41)) return MCMO_EINVAL;
                break;
            default: return MCMO_EINVAL;
        }
        if (M.model == 1) sets1(M);
        else if (M.model == 3) sets3(M);
        else if (M.model == 4) { if (sets4(M) != MCMO_OK) return MCMO_EINVAL; }
        else if (M.model == 10) sets10(M);
    }
    // symmetry planes: MCM/mcm_inp_symmetry_v2.f90:83-137
    if (boundary) {
        bool found = false;
        for (int i = 0; i < 6; ++i) if (d->sym_flag[i] == 1) found = true;
        for (int i = 0; i < 6; ++i) if (d->sym_flag[i] == 2) found = true;
        for (int i = 0; i < 6; i += 2)
            if ((d->sym_flag[i] == 2) != (d->sym_flag[i + 1] == 2)) return MCMO_EINVAL;
        if (!found) boundary = false;
        for (int i = 0; i < 3; ++i) {
            boundary_code[0][i] = d->sym_flag[2 * i];
            boundary_code[1][i] = d->sym_flag[2 * i + 1];
            boundary_x[0][i] = d->sym_x[2 * i];
            boundary_x[1][i] = d->sym_x[2 * i + 1];
        }
        for (int i = 0; i < 3; ++i) {
            boundary_type[i] = 1;
            if (boundary_code[0][i] > 0) boundary_type[i] += 1;
            if (boundary_code[1][i] > 0) boundary_type[i] += 2;
        }
    }
    // MCM/mcm_baseaccel_in.f90:23-33
    for (int k = 0; k < 3; ++k) base_a[k] = (nthp[k] == 1) ? d->base_a[k] : 0.0;
    // particles: MCM/mcm_initialise_database.f90, MCM/mcm_nodein.f90, MCM/mcm_Inputvel.f90
    par.assign(np + 1, Particle());
    for (int i = 1; i <= np; ++i) {
        Particle &P = par[i];
        for (int j = 0; j < ndim; ++j) P.x[j] = x[3 * (i - 1) + j];
        if (init_v_opt == 1)
            for (int j = 0; j < ndim; ++j) P.v[j] = v[3 * (i - 1) + j];
        P.mat = matid[i - 1];
        if (P.mat < 1 || P.mat > nummat) return MCMO_EINVAL;
        P.dispbc = dispbc ? dispbc[i - 1] : 0;
        if (pardata) {
            if (massopt == 1) P.mass = pardata[4 * (i - 1) + 0];
            if (init_h_opt == 1) P.h = pardata[4 * (i - 1) + 1];
            if (init_rhoe == 1) { P.rho = pardata[4 * (i - 1) + 2]; P.e = pardata[4 * (i - 1) + 3]; }
        }
    }
    gpar.assign(1, Ghost());
    return MCMO_OK;
}

// =========================================================================
// mcm_initial (MCM/mcm_initial.f90:28-122)
// =========================================================================

void Sim::initial() {
    init_boundcond();
    calcmass();
    initvbls();
    calcg();
    calcrhopc();
    initsigma();
    initrod();
    init_h();
    timestep = 1;
    for (int i = ssp; i <= esp; ++i) {
        par[i].tracerod = 0.0;
        for (int l = 0; l < ndim; ++l) par[i].tracerod = par[i].tracerod + par[i].rod[l][l];
        aviscosity(i);
    }
    init_neighb();
    calccritts();
    if (itss != 0.0) dt = std::min(itss, critts * tssf);
    else dt = critts * tssf;
    calctotale();
    initold();
    init_ts = dt;  // MCM/mcm_solution.f90:33
}

// MCM/mcm_init_boundcond.f90:25-54
void Sim::init_boundcond() {
    for (int i = svp; i <= evp; ++i) {
        real *v = par[i].v;
        switch (par[i].dispbc) {
            case 1: v[0] = 0.0; break;
            case 2: v[1] = 0.0; break;
            case 3: v[2] = 0.0; break;
            case 4: v[0] = 0.0; v[1] = 0.0; break;
            case 5: v[1] = 0.0; v[2] = 0.0; break;
            case 6: v[0] = 0.0; v[2] = 0.0; break;
            case 7: v[0] = 0.0; v[1] = 0.0; v[2] = 0.0; break;
            default: break;
        }
    }
}

// MCM/mcm_calcmass.f90:20-34, calcmzero :122-152 (Cartesian only)
void Sim::calcmass() {
    if (massopt != 0) return;
    std::vector<int> nppermat(nummat + 1, 0);
    for (int i = svp; i <= evp; ++i) nppermat[par[i].mat] += 1;
    for (int i = svp; i <= evp; ++i) par[i].mass = mat[par[i].mat].mass / (real)nppermat[par[i].mat];
}

// MCM/mcm_initvbls.f90:23-91
void Sim::initvbls() {
    for (int i = 1; i <= np; ++i) par[i].active = true;
    for (int i = 1; i <= np; ++i)
        for (int j = 0; j < ndim; ++j) par[i].xzero[j] = par[i].x[j];
    for (int i = 1; i <= np; ++i) par[i].a[0] = par[i].a[1] = par[i].a[2] = 0.0;
    thermale = 0.0;
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        P.efps = 0.0; P.fail = 1.0; P.temper = 0.0;
        switch (mat[P.mat].model) {
            case 1: case 3: case 4: P.pcut = -9.90E+20; break;
            case 9: P.pcut = mat[P.mat].strinput[0]; break;
            case 10: P.pcut = mat[P.mat].strinput[3]; break;
        }
    }
    for (int i = svp; i <= evp; ++i) {
        Particle &P = par[i];
        P.vabs = 0.0;
        for (int j = 0; j < ndim; ++j) P.vabs = P.vabs + P.v[j] * P.v[j];
        P.vabs = std::sqrt(P.vabs);
    }
    for (int i = 0; i < 3; ++i) { coord_maxmin[0][i] = 1.0e+20; coord_maxmin[1][i] = -1.0e+20; }
    for (int i = 1; i <= np; ++i)
        for (int j = 0; j < ndim; ++j) {
            if (par[i].x[j] < coord_maxmin[0][j]) coord_maxmin[0][j] = par[i].x[j];
            if (par[i].x[j] > coord_maxmin[1][j]) coord_maxmin[1][j] = par[i].x[j];
        }
}

// MCM/mcm_calcg.f90:31-59
void Sim::calcg() {
    for (int i = 1; i <= nummat; ++i) {
        Material &M = mat[i];
        switch (M.model) {
            case 1: case 3: M.g = M.strinput[0] / (2.0 * (1.0 + M.strinput[5])); break;
            case 4: M.g = M.strinput[5]; break;
            case 9: M.g = 0.0; break;
            case 10: M.g = M.strinput[0]; break;
        }
    }
}

// MCM/mcm_calcrhopc.f90:31-95
void Sim::calcrhopc() {
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        P.rho0 = mat[P.mat].rho;
        switch (mat[P.mat].model) {
            case 1: case 3:
                if (init_rhoe != 1) { P.rho = P.rho0; P.e = 0.0; }
                P.p = 0.0;
                P.c = std::sqrt(mat[P.mat].strinput[1] / P.rho);
                break;
            case 4:   // MCM/mcm_calcrhopc.f90:57-67: strinput(10) = cm(5,2), set by mcm_sets4
                if (init_rhoe != 1) { P.rho = P.rho0; P.e = 0.0; }
                P.p = 0.0;
                P.c = std::sqrt(mat[P.mat].strinput[9] / P.rho);
                break;
            case 9: {
                eoscalc(i);
                real pmax = mat[P.mat].strinput[0];
                if (P.p < pmax) P.p = pmax;
                break;
            }
            case 10: eoscalc(i); break;
        }
    }
}

// MCM/mcm_eoscalc.f90:27-113
void Sim::eoscalc(int i) {
    Particle &P = par[i];
    Material &M = mat[P.mat];
    switch (M.eos) {
        case 1:
            if (init_rhoe != 1) { P.rho = P.rho0 / M.eosinput[8]; P.e = M.eosinput[7] * P.mass / P.rho; }
            eos1p(i); eos1c(i); break;
        case 4:
            if (init_rhoe != 1) { P.rho = P.rho0 / M.eosinput[7]; P.e = M.eosinput[6] * P.mass / P.rho; }
            eos4p(i); eos4c(i); break;
        case 13:
            if (init_rhoe != 1) { P.rho = P.rho0 / M.eosinput[3]; P.e = M.eosinput[2] * P.mass / P.rho; }
            eos13p(i); eos13c(i); break;
        case 28:
            if (init_rhoe != 1) { P.rho = P.rho0 / M.eosinput[3]; P.e = M.eosinput[2] * P.mass; }
            eos28p(i); eos28c(i); break;
        case 41:
            if (init_rhoe != 1) { P.rho = P.rho0 / M.eosinput[5]; P.e = M.eosinput[2] * M.eosinput[3] * P.mass / P.rho; }
            eos41p(i); eos41c(i); break;
    }
}

// MCM/mcm_eos1p.f90:30-47
void Sim::eos1p(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real c0 = ei[0], c1 = ei[1], c2 = ei[2], c3 = ei[3], c4 = ei[4], c5 = ei[5], c6 = ei[6];
    real mu = P.rho / P.rho0 - 1.0;
    real mu_t = std::max(mu, 0.0);
    real e1 = P.e * P.rho0 / P.mass;
    e1 = 0.0;
    P.p = c0 + (c1 + c3 * (mu * mu)) * mu + c2 * (mu_t * mu_t) + (c4 + c5 * mu + c6 * (mu_t * mu_t)) * e1;
}

// MCM/mcm_eos4p.f90:32-61
void Sim::eos4p(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real c1 = ei[0], s1 = ei[1], s2 = ei[2], s3 = ei[3], gamma = ei[4], a1 = ei[5];
    real e1 = P.e * P.rho0 / P.mass;
    real mu = P.rho / P.rho0 - 1.0;
    if (mu > 0.0) {
        real termone = mu * (1.0 - (gamma / 2.0));
        real termtwo = (a1 / 2.0) * mu * mu;
        real eosnum = mu * P.rho0 * (c1 * c1) * (1.0 + termone - termtwo);
        real mu21 = (mu * mu) / (mu + 1.0);
        real mu32 = (mu * mu * mu) / ((mu + 1.0) * (mu + 1.0));
        real eosden = 1.0 - (s1 - 1.0) * mu - s2 * mu21 - s3 * mu32;
        P.p = eosnum / (eosden * eosden) + (gamma + a1 * mu) * e1;
    } else {
        P.p = P.rho0 * (c1 * c1) * mu + (gamma + a1 * mu) * e1;
    }
}

// MCM/mcm_eos13p.f90:29-35
void Sim::eos13p(int i) {
    Particle &P = par[i];
    real gamma = mat[P.mat].eosinput[0];
    real e1 = P.e / P.mass;
    P.p = P.rho * (gamma - 1.0) * e1;
}

// MCM/mcm_eos28p.f90:28-33
void Sim::eos28p(int i) {
    Particle &P = par[i];
    real B = mat[P.mat].eosinput[0], gamma = mat[P.mat].eosinput[1];
    P.p = B * (std::pow(P.rho / P.rho0, gamma) - 1.0);
}

// MCM/mcm_eos41p.f90:31-76
void Sim::eos41p(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real cc = ei[0], sl = ei[1], gamma = ei[4];
    real e1 = P.e / P.mass;
    real ao = P.rho0 * (cc * cc);
    real mu = P.rho / P.rho0 - 1.0;
    real bo = ao * (1.0 + 2.0 * (sl - 1.0));
    real co = ao * (2.0 * (sl - 1.0) + 3.0 * ((sl - 1.0) * (sl - 1.0)));
    gamma = gamma * P.rho0 / P.rho;
    real f = gamma * mu;
    real ph;
    if (mu > 0.0) ph = ao * mu + bo * (mu * mu) + co * (mu * mu * mu);
    else ph = ao * mu;
    real pn = ph * (1.0 - 0.5 * f) + P.rho * gamma * e1;
    if (pn < P.pcut) {
        pn = P.pcut;
        P.rho = P.rho / (1.0 - P.tracerod * dt);
    }
    P.p = pn;
}

// MCM/mcm_initsigma.f90:26-49
void Sim::initsigma() {
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        for (int k = 0; k < 6; ++k) P.epx[k] = 0.0;
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) P.sigma[k][j] = (j == k) ? -P.p : 0.0;
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) { P.s[k][j] = 0.0; P.alfa[k][j] = 0.0; }
    }
}

// MCM/mcm_initrod.f90:26-33
void Sim::initrod() {
    for (int i = ssp; i <= esp; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) { par[i].rod[k][j] = 0.0; par[i].spin[k][j] = 0.0; }
}

// MCM/mcm_init_h.f90:22-48 (the hmax loop indexes particles 1..nummat, as written)
void Sim::init_h() {
    hmax = 0.0;
    if (init_h_opt == 0) {
        for (int i = 1; i <= np; ++i) par[i].h = mat[par[i].mat].h;
        for (int i = 1; i <= nummat; ++i) hmax = std::max(hmax, mat[par[i].mat].h);
    } else {
        for (int i = 1; i <= np; ++i) hmax = std::max(hmax, par[i].h);
    }
    for (int i = 1; i <= np; ++i) { par[i].h0 = par[i].h; par[i].hold = par[i].h; }
}

// MCM/mcm_init_neighb.f90:25-84
void Sim::init_neighb() {
    for (int i = 1; i <= np; ++i) { par[i].nnbr = 0; par[i].g_nnbr = 0; }
    setuplist();
    if (boundary) {
        init_boundary();
        ghost_setup();
    }
    ll_neighbours(disctype);
}

// MCM/mcm_initold.f90:22-26
void Sim::initold() {
    for (int i = ssp; i <= esp; ++i) {
        par[i].rhoold = par[i].rho;
        std::memcpy(par[i].qold, par[i].q, sizeof(par[i].q));
    }
}

// =========================================================================
// Neighbour search
// =========================================================================

// MCM/mcm_neighbours.f90:19-41 (the per-particle format loop is vestigial)
void Sim::neighbours() {
    setuplist();
    if (boundary) ghost_setup();
    ll_neighbours(disctype == 1 ? 1 : 0);
}

// MCM/mcm_setuplist.f90:30-141
void Sim::setuplist() {
    const real factor = 2.0;
    for (int i = 0; i < 3; ++i) {
        gridmin[i] = 0.0;
        gridlim[i] = 1;
        gridsize[i] = 1.0 / (factor * hmax);
    }
    for (int i = 0; i < ndim; ++i) {
        switch (boundary_type[i]) {
            case 1:
                gridmin[i] = coord_maxmin[0][i] - 0.01 * hmax;
                gridlim[i] = (int)(gridsize[i] * (coord_maxmin[1][i] - gridmin[i])) + 1;
                break;
            case 2:
                gridmin[i] = boundary_x[0][i];
                gridlim[i] = (int)(gridsize[i] * (coord_maxmin[1][i] - gridmin[i])) + 1;
                break;
            case 3:
                gridlim[i] = (int)(gridsize[i] * (boundary_x[1][i] - coord_maxmin[0][i])) + 1;
                gridmin[i] = boundary_x[1][i] - gridlim[i] * factor * hmax;
                break;
            case 4:
                gridmin[i] = boundary_x[0][i];
                gridlim[i] = (int)(gridsize[i] * (boundary_x[1][i] - boundary_x[0][i]));
                gridlim[i] = std::max(gridlim[i], 1);
                gridsize[i] = (real)(float)gridlim[i] / (boundary_x[1][i] - boundary_x[0][i]);
                break;
        }
    }
    for (int i = 0; i < ndim; ++i) {
        int c0 = boundary_code[0][i];
        if (c0 == 1 || c0 == 2) {
            gridlim[i] = gridlim[i] + 1;
            gridmin[i] = gridmin[i] - (1.0 / gridsize[i]);
        }
        int c1 = boundary_code[1][i];
        if (c1 == 1 || c1 == 2) gridlim[i] = gridlim[i] + 1;
    }
    llgrid.assign((size_t)gridlim[0] * gridlim[1] * gridlim[2], 0);
    int boxcrd[3] = {1, 1, 1};
    for (int i = 1; i <= np; ++i) {
        if (!par[i].active) continue;
        bool in = true;
        for (int j = 0; j < ndim; ++j) {
            boxcrd[j] = (int)(gridsize[j] * (par[i].x[j] - gridmin[j])) + 1;
            if (boxcrd[j] < 1) in = false;
            if (boxcrd[j] > gridlim[j]) in = false;
        }
        if (in) {
            par[i].llpointer = ll(boxcrd[0], boxcrd[1], boxcrd[2]);
            ll(boxcrd[0], boxcrd[1], boxcrd[2]) = i;
        } else {
            par[i].llpointer = -1;
        }
    }
}

// MCM/mcm_init_boundary.f90:28-116 (the multipliers; storage is unbounded here)
void Sim::init_boundary() {
    // plane order: 0 xmin, 1 xmax, 2 ymin, 3 ymax, 4 zmin, 5 zmax
    for (int d = 0; d < 3; ++d) {
        for (int side = 0; side < 2; ++side) {
            int pl = 2 * d + side;
            int code = boundary_code[side][d];
            for (int k = 0; k < 3; ++k) { mult[pl][k] = 1.0; add[pl][k] = 0.0; }
            if (code == 1) {
                mult[pl][d] = -1.0;
                add[pl][d] = 2.0 * boundary_x[side][d];
            } else if (code == 2) {
                if (side == 0) add[pl][d] = -(boundary_x[1][d] - boundary_x[0][d]);
                else add[pl][d] = boundary_x[1][d] - boundary_x[0][d];
            }
        }
    }
}

// MCM/mcm_ghost_setup.f90:293-357
void Sim::create_ghost_from_real(int id, int i, int j, int k, const real *mlt, const real *ad) {
    ngp = ngp + 1;
    if ((int)gpar.size() <= ngp) gpar.resize(ngp + 1);
    Ghost &G = gpar[ngp];
    const Particle &P = par[id];
    G.par = id; G.mat = P.mat; G.mass = P.mass; G.h = P.h; G.hold = P.hold; G.rho = P.rho;
    for (int m = 0; m < 3; ++m) {
        G.x[m] = P.x[m] * mlt[m] + ad[m];
        G.xzero[m] = P.xzero[m] * mlt[m] + ad[m];
        G.v[m] = P.v[m] * mlt[m];
    }
    G.llpointer = ll(i, j, k);
    ll(i, j, k) = -ngp;
}

// MCM/mcm_ghost_setup.f90:361-425
void Sim::create_ghost_from_ghost(int id, int i, int j, int k, const real *mlt, const real *ad) {
    ngp = ngp + 1;
    if ((int)gpar.size() <= ngp) gpar.resize(ngp + 1);
    Ghost S = gpar[id];  // copy: resize above may move storage
    Ghost &G = gpar[ngp];
    G.par = S.par; G.mat = S.mat; G.mass = S.mass; G.h = S.h; G.hold = S.hold; G.rho = S.rho;
    for (int m = 0; m < 3; ++m) {
        G.x[m] = S.x[m] * mlt[m] + ad[m];
        G.xzero[m] = S.xzero[m] * mlt[m] + ad[m];
        G.v[m] = S.v[m] * mlt[m];
    }
    G.llpointer = ll(i, j, k);
    ll(i, j, k) = -ngp;
}

// MCM/mcm_ghost_setup.f90:29-284 (planes in the order xmin xmax ymin ymax zmin zmax)
void Sim::ghost_setup() {
    ngp = 0;
    gpar.assign(1, Ghost());
    for (int d = 0; d < 3; ++d) {
        for (int side = 0; side < 2; ++side) {
            int code = boundary_code[side][d];
            if (code != 1 && code != 2) continue;
            int pl = 2 * d + side;
            int src;
            if (side == 0) src = (code == 1) ? 2 : gridlim[d] - 1;
            else src = (code == 1) ? gridlim[d] - 1 : 2;
            int dst = (side == 0) ? 1 : gridlim[d];
            // loop over the 2-D layer in the reference's order
            int a_dim, b_dim;  // outer, inner
            if (d == 0) { a_dim = 2; b_dim = 1; }
            else if (d == 1) { a_dim = 2; b_dim = 0; }
            else { a_dim = 1; b_dim = 0; }
            for (int a = 1; a <= gridlim[a_dim]; ++a) {
                for (int b = 1; b <= gridlim[b_dim]; ++b) {
                    int cs[3], cd[3];
                    cs[d] = src; cd[d] = dst;
                    cs[a_dim] = a; cd[a_dim] = a;
                    cs[b_dim] = b; cd[b_dim] = b;
                    int id = ll(cs[0], cs[1], cs[2]);
                    if (id > 0) {
                        while (id != 0) {
                            create_ghost_from_real(id, cd[0], cd[1], cd[2], mult[pl], add[pl]);
                            id = par[id].llpointer;
                        }
                    } else {
                        while (id != 0) {
                            create_ghost_from_ghost(std::abs(id), cd[0], cd[1], cd[2], mult[pl], add[pl]);
                            id = gpar[std::abs(id)].llpointer;
                        }
                    }
                }
            }
        }
    }
}

// MCM/mcm_ll_neighbours.f90:1-311 (storage unbounded; see header)
void Sim::ll_neighbours(int ip_flag) {
    const real factor = 2.0;
    maxnbr = maxnbr + 5 + ip_flag;
    maxcont = maxcont + 5;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 1; i <= np; ++i) {
        int boxcrd[3] = {1, 1, 1};                   // per particle: private to the thread
        int looplim[2][3] = {{1, 1, 1}, {1, 1, 1}};
        Particle &P = par[i];
        P.nnbr = 0; P.ncont = 0; P.g_nnbr = 0; P.g_ncont = 0;
        P.nbr.clear(); P.cont.clear(); P.gnbr.clear(); P.gcont.clear();
        P.mindist = 1.0e20;
        real mindist_cp = 1.0e20;
        if (P.llpointer > -1) {
            for (int j = 0; j < ndim; ++j) {
                boxcrd[j] = (int)(gridsize[j] * (P.x[j] - gridmin[j])) + 1;
                looplim[0][j] = std::max(boxcrd[j] - 1, 1);
                looplim[1][j] = std::min(boxcrd[j] + 1, gridlim[j]);
            }
            for (int n = looplim[0][2]; n <= looplim[1][2]; ++n)
                for (int m = looplim[0][1]; m <= looplim[1][1]; ++m)
                    for (int l = looplim[0][0]; l <= looplim[1][0]; ++l) {
                        int id = ll(l, m, n);
                        if (id > -1) {
                            while (true) {
                                if (id < 1) break;
                                if (id != i) {
                                    real dist_sq = 0.0;
                                    for (int j = 0; j < ndim; ++j) dist_sq = dist_sq + sq(par[id].x[j] - P.x[j]);
                                    real h_avg = factor * 0.5 * (par[id].h + P.h);
                                    real h_sq = h_avg * h_avg;
                                    if (dist_sq < h_sq) {
                                        if (par[id].mat == P.mat) {
                                            P.mindist = std::min(P.mindist, dist_sq);
                                            P.nnbr += 1;
                                            P.nbr.push_back(id);
                                        } else {
                                            mindist_cp = std::min(mindist_cp, dist_sq);
                                            P.ncont += 1;
                                            P.cont.push_back(id);
                                        }
                                    }
                                }
                                id = par[id].llpointer;
                            }
                        } else {
                            while (true) {
                                if (id > -1) break;
                                id = std::abs(id);
                                real dist_sq = 0.0;
                                for (int j = 0; j < ndim; ++j) dist_sq = dist_sq + sq(gpar[id].x[j] - P.x[j]);
                                real h_avg = factor * 0.5 * (gpar[id].h + P.h);
                                real h_sq = h_avg * h_avg;
                                if (dist_sq < h_sq) {
                                    if (gpar[id].mat == P.mat) {
                                        P.mindist = std::min(P.mindist, dist_sq);
                                        P.g_nnbr += 1;
                                        P.gnbr.push_back(id);
                                    } else {
                                        mindist_cp = std::min(mindist_cp, dist_sq);
                                        P.g_ncont += 1;
                                        P.gcont.push_back(id);
                                    }
                                }
                                id = gpar[id].llpointer;
                            }
                        }
                    }
            if (contacttype == 0) {
                for (int c : P.cont) P.nbr.push_back(c);
                P.nnbr = P.nnbr + P.ncont;
                P.mindist = std::min(P.mindist, mindist_cp);
                if (boundary) {
                    for (int c : P.gcont) P.gnbr.push_back(c);
                    P.g_nnbr = P.g_nnbr + P.g_ncont;
                }
            }
            P.mindist = std::sqrt(P.mindist);
        }
    }
    maxnbr = 0; maxcont = 0;
    for (int i = 1; i <= np; ++i) { maxnbr = std::max(maxnbr, par[i].nnbr); maxcont = std::max(maxcont, par[i].ncont); }
    if (boundary) {
        g_maxnbr = 0; g_maxcont = 0;
        for (int i = 1; i <= np; ++i) { g_maxnbr = std::max(g_maxnbr, par[i].g_nnbr); g_maxcont = std::max(g_maxcont, par[i].g_ncont); }
    }
    if (ip_flag == 1) {
        for (int i = 1; i <= np; ++i) {
            par[i].nnbr = par[i].nnbr + 1;
            maxnbr = std::max(maxnbr, par[i].nnbr);
            par[i].nbr.push_back(i);
        }
    }
}

// =========================================================================
// Kernel (MCM/mcm_kernel.f90:42-95) and gradient (MCM/mcm_gradw.f90:41-103)
// =========================================================================

real Sim::kernel1(const real *xi, const real *xj, real havg) const {
    real const1 = 0;
    switch (ndim) {
        case 3: const1 = 1.0 / (pi * havg * havg * havg); break;
        case 2: const1 = 10.0 / (7.0 * pi * havg * havg); break;
        case 1: const1 = 2.0 / (3.0 * havg); break;
    }
    real const2 = const1 / 4.0;
    real rad = 0.0;
    for (int n = 0; n < ndim; ++n) {
        real xij = xi[n] - xj[n];
        rad = rad + xij * xij;
    }
    rad = std::sqrt(rad);
    real z = rad / havg;
    if (z < 1.0) return const1 * (((0.75 * z - 1.5) * z) * z + 1.0);
    if (z < 2.0) { real t = 2.0 - z; return const2 * (t * t * t); }
    return 0.0;
}

void Sim::grad1(real *dwdx, real &dwdr, const real *xi, const real *xj, real havg) const {
    real const1 = 0;
    switch (ndim) {
        case 3: const1 = 1.0 / (pi * havg * havg * havg); break;
        case 2: const1 = 10.0 / (7.0 * pi * havg * havg); break;
        case 1: const1 = 2.0 / (3.0 * havg); break;
    }
    real const2 = const1 * 0.25;
    real xij[3] = {0, 0, 0};
    real rad = 0.0;
    for (int n = 0; n < ndim; ++n) {
        xij[n] = xi[n] - xj[n];
        rad = rad + xij[n] * xij[n];
    }
    rad = std::sqrt(rad);
    real z = rad / havg;
    real dw;
    if (z < 1.0) dw = const1 * ((9.0 / 4.0 * z - 3.0) * z);
    else if (z < 2.0) { real t = 2.0 - z; dw = -3.0 * const2 * (t * t); }
    else dw = 0.0;
    for (int n = 0; n < ndim; ++n) {
        if (rad == 0.0) { dwdx[n] = 0.0; dwdr = 0.0; }
        else { dwdx[n] = dw * xij[n] / (rad * havg); dwdr = dw / havg; }
    }
}

// =========================================================================
// Strain rate (MCM/mcm_strain.f90, mcm_oldstrain.f90, mcm_corr_strain.f90)
// =========================================================================

// MCM/mcm_get_j_strain_info.f90:27-54
void Sim::get_j_strain_info(int i, int k, real *x, real *v, real &mass, real &rho, real &h, real &hold) {
    const Particle &P = par[i];
    if (k <= P.nnbr) {
        const Particle &J = par[P.nbr[k - 1]];
        for (int m = 0; m < 3; ++m) { x[m] = J.x[m]; v[m] = J.v[m]; }
        mass = J.mass; h = J.h; hold = J.hold; rho = J.rho;
    } else {
        const Ghost &J = gpar[P.gnbr[k - P.nnbr - 1]];
        for (int m = 0; m < 3; ++m) { x[m] = J.x[m]; v[m] = J.v[m]; }
        mass = J.mass; h = J.h; hold = J.hold; rho = J.rho;
    }
}

// MCM/mcm_strain.f90:20-61
void Sim::strain() {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 1; i <= np; ++i)
        for (int j = 0; j < ndim; ++j) par[i].x[j] = par[i].x[j] - 0.5 * par[i].v[j] * dt;
    if (disctype == 0) oldstrain();
    else corr_strain();
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 1; i <= np; ++i)
        for (int j = 0; j < ndim; ++j) par[i].x[j] = par[i].x[j] + 0.5 * par[i].v[j] * dt;
}

// MCM/mcm_oldstrain.f90:34-64
void Sim::oldstrain() {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        real grad_v[3][3] = {};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) { P.rod[a][b] = 0.0; P.spin[a][b] = 0.0; }
        real vi[3] = {P.v[0], P.v[1], P.v[2]};
        int nk = P.nnbr + P.g_nnbr;
        for (int k = 1; k <= nk; ++k) {
            real xj[3], vj[3], massj, rhoj, hj, holdj;
            get_j_strain_info(i, k, xj, vj, massj, rhoj, hj, holdj);
            real Volj = massj / rhoj;
            real havg = 0.5 * (P.h + hj);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, P.x, xj, havg);
            for (int n = 0; n < ndim; ++n)
                for (int m = 0; m < ndim; ++m)
                    grad_v[n][m] = grad_v[n][m] + Volj * (vj[n] - vi[n]) * dwdx[m];
        }
        for (int n = 0; n < ndim; ++n)
            for (int m = 0; m < ndim; ++m) {
                P.rod[n][m] = 0.5 * (grad_v[n][m] + grad_v[m][n]);
                P.spin[n][m] = 0.5 * (grad_v[n][m] - grad_v[m][n]);
            }
        P.tracerod = P.rod[0][0] + P.rod[1][1] + P.rod[2][2];
    }
}

// MCM/mcm_math_func.f90:16-82 (3-D branch, :50-79)
void Sim::inverse(const real M[3][3], real inv[3][3]) const {
    real sd[3][3];
    sd[0][0] = M[1][1] * M[2][2] - M[1][2] * M[2][1];
    sd[0][1] = M[1][0] * M[2][2] - M[1][2] * M[2][0];
    sd[0][2] = M[1][0] * M[2][1] - M[1][1] * M[2][0];
    sd[1][0] = M[0][1] * M[2][2] - M[0][2] * M[2][1];
    sd[1][1] = M[0][0] * M[2][2] - M[0][2] * M[2][0];
    sd[1][2] = M[0][0] * M[2][1] - M[0][1] * M[2][0];
    sd[2][0] = M[0][1] * M[1][2] - M[0][2] * M[1][1];
    sd[2][1] = M[0][0] * M[1][2] - M[0][2] * M[1][0];
    sd[2][2] = M[0][0] * M[1][1] - M[0][1] * M[1][0];
    real det = M[0][0] * sd[0][0] - M[0][1] * sd[0][1] + M[0][2] * sd[0][2];
    if (std::fabs(det) < 1.0e-08) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) inv[a][b] = (a == b) ? 1.0 : 0.0;
    } else {
        real invdet = 1.0 / det;
        inv[0][0] = sd[0][0] * invdet;
        inv[0][1] = -sd[1][0] * invdet;
        inv[0][2] = sd[2][0] * invdet;
        inv[1][0] = -sd[0][1] * invdet;
        inv[1][1] = sd[1][1] * invdet;
        inv[1][2] = -sd[2][1] * invdet;
        inv[2][0] = sd[0][2] * invdet;
        inv[2][1] = -sd[1][2] * invdet;
        inv[2][2] = sd[2][2] * invdet;
    }
}

// MCM/mcm_corr_strain.f90:37-146
void Sim::corr_strain() {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) { P.rod[a][b] = 0.0; P.spin[a][b] = 0.0; }
        int nk = P.nnbr + P.g_nnbr;
        real sum_w = 0.0, sum_gradw[3] = {0, 0, 0};
        for (int k = 1; k <= nk; ++k) {
            real xj[3], vj[3], massj, rhoj, hj, holdj;
            get_j_strain_info(i, k, xj, vj, massj, rhoj, hj, holdj);
            real Volj = massj / rhoj;
            real havg = 0.5 * (P.h + hj);
            real w = kernel1(P.x, xj, havg);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, P.x, xj, havg);
            sum_w = sum_w + Volj * w;
            for (int l = 0; l < ndim; ++l) sum_gradw[l] = sum_gradw[l] + Volj * dwdx[l];
        }
        real B[3][3] = {};
        for (int k = 1; k <= nk; ++k) {
            real xj[3], vj[3], massj, rhoj, hj, holdj;
            get_j_strain_info(i, k, xj, vj, massj, rhoj, hj, holdj);
            real Volj = massj / rhoj;
            real havg = 0.5 * (P.h + hj);
            real w = kernel1(P.x, xj, havg);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, P.x, xj, havg);
            real cg[3];
            for (int m = 0; m < ndim; ++m) cg[m] = (dwdx[m] * sum_w - w * sum_gradw[m]) / (sum_w * sum_w);
            for (int m = 0; m < ndim; ++m)
                for (int n = 0; n < ndim; ++n) B[n][m] = B[n][m] + Volj * (xj[n] - P.x[n]) * cg[m];
        }
        real invB[3][3];
        inverse(B, invB);
        real f[3][3] = {};
        for (int k = 1; k <= nk; ++k) {
            real xj[3], vj[3], massj, rhoj, hj, holdj;
            get_j_strain_info(i, k, xj, vj, massj, rhoj, hj, holdj);
            real Volj = massj / rhoj;
            real havg = 0.5 * (P.h + hj);
            real w = kernel1(P.x, xj, havg);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, P.x, xj, havg);
            real cg[3];
            for (int m = 0; m < ndim; ++m) cg[m] = (dwdx[m] * sum_w - w * sum_gradw[m]) / (sum_w * sum_w);
            real c2[3];
            for (int n = 0; n < 3; ++n) c2[n] = invB[n][0] * cg[0] + invB[n][1] * cg[1] + invB[n][2] * cg[2];
            for (int n = 0; n < ndim; ++n)
                for (int m = 0; m < ndim; ++m) f[n][m] = f[n][m] + Volj * vj[n] * c2[m];
        }
        for (int n = 0; n < ndim; ++n)
            for (int m = 0; m < ndim; ++m) {
                P.rod[n][m] = 0.5 * (f[n][m] + f[m][n]);
                P.spin[n][m] = 0.5 * (f[n][m] - f[m][n]);
            }
        P.tracerod = P.rod[0][0] + P.rod[1][1] + P.rod[2][2];
    }
}

// =========================================================================
// Constitutive update (MCM/mcm_constitutive.f90:26-87)
// =========================================================================

int Sim::constitutive() {
    rhoupd();
    for (int m = 1; m <= nummat; ++m) {
        int md = mat[m].model;
        if (md != 1 && md != 3 && md != 4 && md != 9 && md != 10) return MCMO_EUNSUPPORTED;
    }
    int bad = 0, cap_bad = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) reduction(max : bad, cap_bad)
#endif
    for (int nn = ssp; nn <= esp; ++nn) {
        Material &M = mat[par[nn].mat];
        switch (M.model) {
            case 1: stress_rot1(nn); f3dm1(M, nn); aviscosity(nn); lieupd(nn); break;
            case 3: stress_rot1(nn); f3dm3(M, nn); aviscosity(nn); lieupd(nn); break;
            case 4:
                stress_rot1(nn);
                if (f3dm25(M, nn) != MCMO_OK) cap_bad = 1;
                aviscosity(nn); lieupd(nn);
                break;
            case 9: {
                stress_rot1(nn); f3dm9(M, nn);
                if (sueos(nn) != MCMO_OK) bad = 1;
                aviscosity(nn); hieupd(nn); eqos(nn); stress_up(nn);
                break;
            }
            case 10: {
                stress_rot1(nn); f3dm10(M, nn);
                if (sueos(nn) != MCMO_OK) bad = 1;
                aviscosity(nn); hieupd(nn); eqos(nn); stress_up(nn);
                break;
            }
            default: break;
        }
    }
    calccritts();
    if (cap_bad) return MCMO_ECAP_NOCONV;
    return bad ? MCMO_ECOMPLEX_C : MCMO_OK;
}

// MCM/mcm_rhoupd.f90:19-66 (the bound warnings only print)
void Sim::rhoupd() {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        P.rhoold = P.rho;
        real othird = 1.0 / 3.0;
        P.rho = P.rho * (1.0 - P.tracerod * dt);
        const Material &M = mat[P.mat];
        for (int rep = 0; rep < 2; ++rep) {
            if (P.rho > M.rho_max) {
                P.rho = P.rho / (1.0 - P.tracerod * dt);
                P.rod[0][0] = P.rod[0][0] - othird * P.tracerod;
                P.rod[1][1] = P.rod[1][1] - othird * P.tracerod;
                P.rod[2][2] = P.rod[2][2] - othird * P.tracerod;
                P.tracerod = 0.0;
                if (rep == 1) P.h = P.hold;
                P.h = M.h * std::pow(M.rho / P.rho, 1.0 / (real)(float)ndim);
            }
        }
    }
}

// MCM/mcm_stress_rot1.f90:1-203 (iorder = 3: exponential map)
void Sim::stress_rot1(int i) {
    Particle &P = par[i];
    const real etol = F32(1.0e-3f);
    const real z1 = 1.0 / 3.0, z2 = 2.0 / 15.0, z3 = 17.0 / 315.0, z4 = 62.0 / 2835.0;
    real st[3][3];
    std::memcpy(st, P.sigma, sizeof(st));
    real dt2 = 0.5 * dt;
    real wzz = -dt2 * P.spin[0][1];
    real wyy = dt2 * P.spin[0][2];
    real wxx = -dt2 * P.spin[1][2];
    real wxx2 = wxx * wxx, wyy2 = wyy * wyy, wzz2 = wzz * wzz;
    real qm2 = wxx2 + wyy2 + wzz2;
    real qm = std::sqrt(qm2);
    real dd = std::tan(qm * 0.5);
    real cc;
    if (qm < etol) {
        real aa = qm2 * 0.25;
        cc = 0.5 * (1.0 + aa * (z1 + aa * (z2 + aa * (z3 + aa * z4))));
    } else {
        cc = dd / qm;
    }
    real bb = 2.0 * cc / (1.0 + dd * dd);
    real aa = bb * cc;
    real Q[3][3];
    Q[0][0] = 1.0 - aa * (wyy2 + wzz2);
    Q[1][1] = 1.0 - aa * (wxx2 + wzz2);
    Q[2][2] = 1.0 - aa * (wxx2 + wyy2);
    Q[0][1] = aa * wxx * wyy;
    Q[0][2] = aa * wxx * wzz;
    Q[1][2] = aa * wyy * wzz;
    Q[1][0] = Q[0][1];
    Q[2][0] = Q[0][2];
    Q[2][1] = Q[1][2];
    real bwxx = bb * wxx, bwyy = bb * wyy, bwzz = bb * wzz;
    Q[0][1] = Q[0][1] - bwzz;
    Q[1][0] = Q[1][0] + bwzz;
    Q[0][2] = Q[0][2] + bwyy;
    Q[2][0] = Q[2][0] - bwyy;
    Q[1][2] = Q[1][2] - bwxx;
    Q[2][1] = Q[2][1] + bwxx;
    real qs[3][3];
    qs[0][0] = Q[0][0] * st[0][0] + Q[0][1] * st[0][1] + Q[0][2] * st[2][0];
    qs[0][1] = Q[0][0] * st[0][1] + Q[0][1] * st[1][1] + Q[0][2] * st[1][2];
    qs[0][2] = Q[0][0] * st[2][0] + Q[0][1] * st[1][2] + Q[0][2] * st[2][2];
    qs[1][0] = Q[1][0] * st[0][0] + Q[1][1] * st[0][1] + Q[1][2] * st[2][0];
    qs[1][1] = Q[1][0] * st[0][1] + Q[1][1] * st[1][1] + Q[1][2] * st[1][2];
    qs[1][2] = Q[1][0] * st[2][0] + Q[1][1] * st[1][2] + Q[1][2] * st[2][2];
    qs[2][0] = Q[2][0] * st[0][0] + Q[2][1] * st[0][1] + Q[2][2] * st[2][0];
    qs[2][1] = Q[2][0] * st[0][1] + Q[2][1] * st[1][1] + Q[2][2] * st[1][2];
    qs[2][2] = Q[2][0] * st[2][0] + Q[2][1] * st[1][2] + Q[2][2] * st[2][2];
    P.sigma[0][0] = qs[0][0] * Q[0][0] + qs[0][1] * Q[0][1] + qs[0][2] * Q[0][2];
    P.sigma[1][1] = qs[1][0] * Q[1][0] + qs[1][1] * Q[1][1] + qs[1][2] * Q[1][2];
    P.sigma[2][2] = qs[2][0] * Q[2][0] + qs[2][1] * Q[2][1] + qs[2][2] * Q[2][2];
    P.sigma[0][1] = qs[0][0] * Q[1][0] + qs[0][1] * Q[1][1] + qs[0][2] * Q[1][2];
    P.sigma[1][2] = qs[1][0] * Q[2][0] + qs[1][1] * Q[2][1] + qs[1][2] * Q[2][2];
    P.sigma[2][0] = qs[0][0] * Q[2][0] + qs[0][1] * Q[2][1] + qs[0][2] * Q[2][2];
    P.sigma[1][0] = P.sigma[0][1];
    P.sigma[2][1] = P.sigma[1][2];
    P.sigma[0][2] = P.sigma[2][0];
    // qq <- qq * Q (MCM/mcm_stress_rot1.f90:189-199): a write-only field
    real qa[3][3];
    std::memcpy(qa, P.qq, sizeof(qa));
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) P.qq[r][c] = qa[r][0] * Q[0][c] + qa[r][1] * Q[1][c] + qa[r][2] * Q[2][c];
}

// MCM/mcm_f3dm1.f90:27-71
void Sim::f3dm1(Material &M, int i) {
    Particle &P = par[i];
    real othird = 1.0 / 3.0;
    real ym = M.cm(1, 1), pr = M.cm(1, 2), gg = M.cm(5, 4);
    real gdt = dt * gg;
    real gd2 = 2.0 * gdt;
    real blk = dt * ym / ((1.0 - 2.0 * pr));
    real davg = othird * P.tracerod;
    real p_incr = blk * davg;
    real (&r)[3][3] = P.rod;
    real (&s)[3][3] = P.sigma;
    real (&q)[3][3] = P.q;
    P.einc = (r[0][0] * (s[0][0] + q[0][0]) + r[1][1] * (s[1][1] + q[1][1]) + r[2][2] * (s[2][2] + q[2][2]) +
              2.0 * (r[0][1] * (s[0][1] + q[0][1]) + r[0][2] * (s[0][2] + q[0][2]) + r[1][2] * (s[1][2] + q[1][2]))) * dt;
    s[0][0] = s[0][0] + p_incr + gd2 * (r[0][0] - davg);
    s[1][1] = s[1][1] + p_incr + gd2 * (r[1][1] - davg);
    s[2][2] = s[2][2] + p_incr + gd2 * (r[2][2] - davg);
    s[0][1] = s[0][1] + gd2 * r[0][1];
    s[0][2] = s[0][2] + gd2 * r[0][2];
    s[1][2] = s[1][2] + gd2 * r[1][2];
    s[1][0] = s[0][1]; s[2][0] = s[0][2]; s[2][1] = s[1][2];
    P.einc = 0.5 * ((r[0][0] * s[0][0] + r[1][1] * s[1][1] + r[2][2] * s[2][2] +
                     2.0 * (r[0][1] * s[0][1] + r[0][2] * s[0][2] + r[1][2] * s[1][2])) * dt + P.einc);
    P.p = -othird * (s[0][0] + s[1][1] + s[2][2]);
}

// MCM/mcm_f3dm3.f90:31-156
void Sim::f3dm3(Material &M, int i) {
    Particle &P = par[i];
    real othird = 1.0 / 3.0;
    real qh = M.cm(2, 4), qb = M.cm(1, 5), qs = M.cm(1, 3), ym = M.cm(1, 1), pr = M.cm(1, 2);
    real efps_f = M.cm(2, 6);
    real gg = 2.0 * M.cm(5, 4);
    real gdt = dt * gg;
    real qbqh = qb * qh;
    int efps_flag = (int)std::lround(M.cm(1, 6));
    real blk = dt * ym / ((1.0 - 2.0 * pr));
    real davg = othird * P.tracerod;
    real p_incr = blk * davg;
    P.p = P.p - p_incr;
    real (&r)[3][3] = P.rod;
    real (&sg)[3][3] = P.sigma;
    real (&q)[3][3] = P.q;
    real (&s)[3][3] = P.s;
    real (&al)[3][3] = P.alfa;
    P.einc = (r[0][0] * (sg[0][0] + q[0][0]) + r[1][1] * (sg[1][1] + q[1][1]) + r[2][2] * (sg[2][2] + q[2][2]) +
              2.0 * (r[0][1] * (sg[0][1] + q[0][1]) + r[0][2] * (sg[0][2] + q[0][2]) + r[1][2] * (sg[1][2] + q[1][2]))) * dt;
    sg[0][0] = sg[0][0] + p_incr + gdt * (r[0][0] - davg);
    sg[1][1] = sg[1][1] + p_incr + gdt * (r[1][1] - davg);
    sg[2][2] = sg[2][2] + p_incr + gdt * (r[2][2] - davg);
    sg[0][1] = sg[0][1] + gdt * r[0][1];
    sg[0][2] = sg[0][2] + gdt * r[0][2];
    sg[1][2] = sg[1][2] + gdt * r[1][2];
    sg[1][0] = sg[0][1]; sg[2][0] = sg[0][2]; sg[2][1] = sg[1][2];
    real k = qs + qbqh * P.efps;
    s[0][0] = P.p + sg[0][0] - al[0][0];
    s[1][1] = P.p + sg[1][1] - al[1][1];
    s[2][2] = P.p + sg[2][2] - al[2][2];
    s[0][1] = sg[0][1] - al[0][1];
    s[0][2] = sg[0][2] - al[0][2];
    s[1][2] = sg[1][2] - al[1][2];
    s[1][0] = s[0][1]; s[2][0] = s[0][2]; s[2][1] = s[1][2];
    real j2 = s[1][2] * s[1][2] + s[0][2] * s[0][2] + s[0][1] * s[0][1] - s[0][0] * s[1][1] - s[1][1] * s[2][2] -
              s[0][0] * s[2][2];
    real k2 = 3.0 * j2 - k * k;
    real scle = 0.5 * (1.0 + fsign(1.0, k2));
    real fac1 = 1.0 / (1.5 * gg + qh);
    real fac2 = 1.5 * gg;
    real fac3 = (1.0 - qb) * qh;
    real j1 = std::sqrt(3.0 * std::fabs(j2)) + 1.0 - scle;
    real defps = scle * fac1 * (j1 - k);
    P.efps = P.efps + defps;
    real des = scle * fac2 * defps / j1;
    real depn = scle * fac3 * defps / j1;
    sg[0][0] = sg[0][0] - des * s[0][0];
    sg[1][1] = sg[1][1] - des * s[1][1];
    sg[2][2] = sg[2][2] - des * s[2][2];
    sg[0][1] = sg[0][1] - des * s[0][1];
    sg[0][2] = sg[0][2] - des * s[0][2];
    sg[1][2] = sg[1][2] - des * s[1][2];
    sg[1][0] = sg[0][1]; sg[2][0] = sg[0][2]; sg[2][1] = sg[1][2];
    al[0][0] = al[0][0] + depn * s[0][0];
    al[1][1] = al[1][1] + depn * s[1][1];
    al[2][2] = al[2][2] + depn * s[2][2];
    al[0][1] = al[0][1] + depn * s[0][1];
    al[0][2] = al[0][2] + depn * s[0][2];
    al[1][2] = al[1][2] + depn * s[1][2];
    al[1][0] = al[0][1]; al[2][0] = al[0][2]; al[2][1] = al[1][2];
    if (efps_flag == 1) {
        if (P.efps > efps_f) {
            real press = othird * (sg[0][0] + sg[1][1] + sg[2][2]);
            sg[0][0] = press; sg[0][1] = 0.0; sg[0][2] = 0.0;
            sg[1][1] = press; sg[1][0] = 0.0; sg[1][2] = 0.0;
            sg[2][2] = press; sg[2][0] = 0.0; sg[2][1] = 0.0;
        }
    }
    P.einc = 0.5 * ((r[0][0] * sg[0][0] + r[1][1] * sg[1][1] + r[2][2] * sg[2][2] +
                     2.0 * (r[0][1] * sg[0][1] + r[0][2] * sg[0][2] + r[1][2] * sg[1][2])) * dt + P.einc);
}

// MCM/mcm_f3dm9.f90:27-49 (s(1,2) is never assigned; xmu indexed by material id)
void Sim::f3dm9(Material &M, int i) {
    Particle &P = par[i];
    real othird = 1.0 / 3.0;
    real xmu = M.cm(2, P.mat);
    if (xmu == 0.0) {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) P.s[a][b] = 0.0;
    } else {
        real davg = -othird * P.tracerod;
        P.s[0][0] = xmu * (P.rod[0][0] + davg);
        P.s[1][1] = xmu * (P.rod[1][1] + davg);
        P.s[2][2] = xmu * (P.rod[2][2] + davg);
        P.s[0][2] = xmu * P.rod[0][1];
        P.s[0][2] = xmu * P.rod[0][2];
        P.s[1][2] = xmu * P.rod[1][2];
        P.s[1][0] = P.s[0][1];
        P.s[2][0] = P.s[0][2];
        P.s[2][1] = P.s[1][2];
    }
}

// MCM/mcm_f3dm10.f90:28-157
void Sim::f3dm10(Material &M, int i) {
    Particle &P = par[i];
    const real *cm = M.strinput;
    real othird = 1.0 / 3.0;
    real gg = cm[0], qs = cm[1], qh = cm[2], a1 = cm[4], a2 = cm[5];
    int ispall = (int)cm[6];
    real epf = cm[7];
    real g2 = 2.0 * dt * gg;
    real davg = othird * P.tracerod;
    real (&sg)[3][3] = P.sigma;
    real (&s)[3][3] = P.s;
    real (&r)[3][3] = P.rod;
    P.p = -othird * (sg[0][0] + sg[1][1] + sg[2][2]);
    P.p_cut = P.pcut;
    real ak = qs + qh * P.efps + (a1 + a2 * P.p) * std::max(0.0, P.p);
    s[0][0] = sg[0][0] + P.p + g2 * (r[0][0] + davg);
    s[1][1] = sg[1][1] + P.p + g2 * (r[1][1] + davg);
    s[2][2] = sg[2][2] + P.p + g2 * (r[2][2] + davg);
    s[0][1] = sg[0][1] + 0.5 * g2 * r[0][1];
    s[0][2] = sg[0][2] + 0.5 * g2 * r[0][2];
    s[1][2] = sg[1][2] + 0.5 * g2 * r[1][2];
    if (ispall == 3) {
        real deltap = P.p - P.p_cut;
        real scle = 0.50 * (1.0 + fsign(1.0, deltap));
        P.pcut = scle * P.p_cut;
        s[0][0] = scle * s[0][0]; s[1][1] = scle * s[1][1]; s[2][2] = scle * s[2][2];
        s[0][1] = scle * s[0][1]; s[0][2] = scle * s[0][2]; s[1][2] = scle * s[1][2];
        s[1][0] = s[0][1]; s[2][0] = s[0][2]; s[2][1] = s[1][2];
        P.p_cut = P.pcut;
    }
    real aj2 = 0.5 * (s[0][0] * s[0][0] + s[1][1] * s[1][1] + s[2][2] * s[2][2]) + s[0][1] * s[0][1] +
               s[0][2] * s[0][2] + s[1][2] * s[1][2];
    real sj2 = std::sqrt(3.0 * aj2);
    real defps = 0.0;
    if (P.fail == 1.0) {
        real thrg = othird / gg;
        defps = fdim_(sj2, ak) / (F32(1.e-30f) + fdim_(1.0, -thrg * qh));
        defps = thrg * std::min(sj2, defps);
        P.efps = P.efps + defps;
    }
    ak = std::max(ak + qh * defps, 0.0);
    real seps = F32(1.e-30f) * gg;
    real scle = (ak + seps) / (std::max(ak, sj2) + seps);
    s[0][0] = scle * s[0][0]; s[1][1] = scle * s[1][1]; s[2][2] = scle * s[2][2];
    s[0][1] = scle * s[0][1]; s[0][2] = scle * s[0][2]; s[1][2] = scle * s[1][2];
    s[1][0] = s[0][1]; s[2][0] = s[0][2]; s[2][1] = s[1][2];
    if (epf != 0.0) {
        if (P.efps > epf) {
            P.fail = 0.0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) s[a][b] = 0.0;
        }
    }
    if (ispall == 2) {
        aj2 = 0.5 * (s[0][0] * s[0][0] + s[1][1] * s[1][1] + s[2][2] * s[2][2]) + s[0][1] * s[0][1] +
              s[0][2] * s[0][2] + s[1][2] * s[1][2] + F32(1.e-12f);
        sj2 = s[0][0] * s[1][2] * s[1][2] + s[1][1] * s[0][2] * s[0][2] + s[2][2] * s[0][1] * s[0][1] -
              s[0][0] * s[1][1] * s[2][2] - 2.0 * s[0][1] * s[0][2] * s[1][2];
        real akt = -std::sqrt(27.0 / aj2) * sj2 * 0.5 / aj2;
        akt = fsign(std::min(std::fabs(akt), 1.0), akt);
        real ywh = std::acos(akt) * othird;
        sj2 = 2.0 * std::sqrt(aj2 * othird) * std::cos(ywh);
        real davg1 = P.p - sj2 - P.p_cut;
        real scle2 = 0.50 * (1.0 + fsign(1.0, davg1));
        P.pcut = scle2 * P.p_cut;
        s[0][0] = scle2 * s[0][0]; s[1][1] = scle2 * s[1][1]; s[2][2] = scle2 * s[2][2];
        s[0][1] = scle2 * s[0][1]; s[0][2] = scle2 * s[0][2]; s[1][2] = scle2 * s[1][2];
        s[1][0] = s[0][1]; s[2][0] = s[0][2]; s[2][1] = s[1][2];
        P.p_cut = P.pcut;
    }
}

// MCM/mcm_sueos.f90:22-46
int Sim::sueos(int i) {
    switch (mat[par[i].mat].eos) {
        case 1: return eos1c(i);
        case 4: return eos4c(i);
        case 13: return eos13c(i);
        case 28: return eos28c(i);
        case 41: return eos41c(i);
    }
    return MCMO_OK;
}

// MCM/mcm_eos1c.f90:32-67 (complex c forced to continue)
int Sim::eos1c(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real c1 = ei[1], c2 = ei[2], c3 = ei[3], c4 = ei[4], c5 = ei[5], c6 = ei[6];
    real mu = P.rho / P.rho0 - 1.0;
    real mu_t = std::max(mu, 0.0);
    real e1 = P.e * P.rho0 / P.mass;
    e1 = 0.0;
    real dmudrho = 1 / P.rho0;
    real termone = c1 * dmudrho + (c2 * (dmudrho * dmudrho)) + (3.0 * c3 * dmudrho) * mu * mu;
    real termtwo = (c5 * dmudrho + c6 * dmudrho * dmudrho) * e1;
    real dpdrho = termone + termtwo;
    real dpde = c4 + c5 * mu + c6 * (mu_t * mu_t);
    real mr = P.mass / P.rho;
    real c_sq = ((4.0 / 3.0) * mat[P.mat].g / P.rho0 + dpdrho + P.p / P.rho0 * (mr * mr) * dpde);
    if (c_sq > 0.0) P.c = std::sqrt(c_sq);
    else P.c = std::sqrt(std::fabs(c_sq));
    return MCMO_OK;
}

// MCM/mcm_eos4c.f90:33-90 (complex c forced to continue)
int Sim::eos4c(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real c1 = ei[0], s1 = ei[1], s2 = ei[2], s3 = ei[3], gamma = ei[4], a1 = ei[5];
    real e1 = P.e * P.rho0 / P.mass;
    real mu = P.rho / P.rho0 - 1.0;
    real dpdrho;
    if (mu > 0.0) {
        real termone = mu * (1.0 - (gamma / 2.0));
        real termtwo = (a1 / 2.0) * mu * mu;
        real eosnum = mu * P.rho0 * (c1 * c1) * (1.0 + termone - termtwo);
        real mu11 = mu / (mu + 1.0);
        real mu21 = (mu * mu) / (mu + 1.0);
        real mu22 = (mu * mu) / ((mu + 1.0) * (mu + 1.0));
        real mu32 = (mu * mu * mu) / ((mu + 1.0) * (mu + 1.0));
        real mu33 = (mu * mu * mu) / ((mu + 1.0) * (mu + 1.0) * (mu + 1.0));
        real eosden = 1.0 - (s1 - 1.0) * mu - s2 * mu21 - s3 * mu32;
        real termthree = P.rho0 * (c1 * c1) * (1.0 + 2.0 * termone - 3.0 * termtwo);
        real termfour = 1.0 - s1 - 2.0 * s2 * mu11 + s2 * mu22 - 3.0 * s3 * mu22 + 2.0 * s3 * mu33;
        dpdrho = (termthree / (eosden * eosden) - 2.0 * eosnum * termfour / (eosden * eosden * eosden)) / P.rho0 +
                 a1 * e1 / P.rho0;
    } else {
        dpdrho = (c1 * c1) + a1 * e1 / P.rho0;
    }
    real dpde = gamma + a1 * mu;
    real mr = P.mass / P.rho;
    real c_sq = ((4.0 / 3.0) * mat[P.mat].g / P.rho0 + dpdrho + P.p / P.rho0 * (mr * mr) * dpde);
    if (c_sq > 0.0) P.c = std::sqrt(c_sq);
    else P.c = std::sqrt(std::fabs(c_sq));
    return MCMO_OK;
}

// MCM/mcm_eos13c.f90:29-37
int Sim::eos13c(int i) {
    Particle &P = par[i];
    real gamma = mat[P.mat].eosinput[0];
    real e1 = P.e / P.mass;
    P.c = std::sqrt((gamma - 1.0) * gamma * e1);
    return MCMO_OK;
}

// MCM/mcm_eos28c.f90:28-33
int Sim::eos28c(int i) {
    Particle &P = par[i];
    real b = mat[P.mat].eosinput[0], gamma = mat[P.mat].eosinput[1];
    P.c = std::sqrt(b * gamma / P.rho0);
    return MCMO_OK;
}

// MCM/mcm_eos41c.f90:31-85 (c2 < 0 stops the reference; a status here)
int Sim::eos41c(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real cc = ei[0], sl = ei[1], gamma0 = ei[4];
    real e1 = P.e / P.mass;
    real ao = P.rho0 * (cc * cc);
    real mu = P.rho / P.rho0 - 1.0;
    real gamma = gamma0 * P.rho0 / P.rho;
    real bo = ao * (1.0 + 2.0 * (sl - 1.0));
    real co = ao * (2.0 * (sl - 1.0) + 3.0 * ((sl - 1.0) * (sl - 1.0)));
    real f = gamma * mu;
    real a1 = ao * (1.0 - f);
    real b1 = bo * (2.0 - 1.5 * f);
    real c1 = co * (3.0 - 2.0 * f);
    real dpdrho;
    if (mu > 0.0) dpdrho = (a1 + b1 * mu + c1 * (mu * mu)) / P.rho0 + gamma * e1;
    else dpdrho = ao * (1.0 - f) / P.rho0 + gamma * e1;
    real c2;
    if (P.p == P.pcut) {
        c2 = cc * cc;
    } else {
        real dpdi = gamma * P.rho;
        real didrho = P.p / (P.rho * P.rho);
        dpdrho = dpdrho + dpdi * didrho;
        c2 = dpdrho;
    }
    int st = MCMO_OK;
    if (c2 < 0.0) st = MCMO_ECOMPLEX_C;
    P.c = std::sqrt(c2);
    return st;
}

// MCM/mcm_aviscosity.f90:28-39
void Sim::aviscosity(int i) {
    if (mat[par[i].mat].visc_type == 1) nodalav(i);
}

// MCM/mcm_nodalav.f90:32-47
void Sim::nodalav(int i) {
    Particle &P = par[i];
    const Material &M = mat[P.mat];
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) P.q[j][k] = 0.0;
    if (P.tracerod < 0.0) {
        real ht = P.h * P.tracerod;
        real q = M.av_l * P.rho * P.c * P.h * std::fabs(P.tracerod) + M.av_q * P.rho * (ht * ht);
        for (int j = 0; j < 3; ++j) P.q[j][j] = q;
    }
}

// MCM/mcm_hieupd.f90:27-64
void Sim::hieupd(int i) {
    Particle &P = par[i];
    real othird = 1.0 / 3.0;
    real pold = -othird * (P.sigma[0][0] + P.sigma[1][1] + P.sigma[2][2]);
    real trace_q = othird * (P.q[0][0] + P.q[1][1] + P.q[2][2]);
    real volold = P.mass / P.rhoold;
    real volnew = P.mass / P.rho;
    real de[3][3];
    for (int l = 0; l < 3; ++l)
        for (int k = 0; k < 3; ++k) {
            if (k == l) de[k][l] = P.rod[k][l] * (0.5 * (P.sigma[k][l] + pold + P.s[k][l]) - P.q[k][l] + trace_q);
            else de[k][l] = P.rod[k][l] * (0.5 * (P.sigma[k][l] + P.s[k][l]) - P.q[k][l]);
        }
    real vavg = 0.5 * (volnew + volold);
    real eincr = 0.0;
    for (int l = 0; l < 3; ++l)
        for (int k = 0; k < 3; ++k) eincr = eincr + de[k][l];
    eincr = vavg * eincr;
    real dvol = volnew - volold;
    real mean_incr = dvol * (0.5 * pold + trace_q);
    P.etry = P.e + dt * eincr - mean_incr;
    std::memcpy(P.qold, P.q, sizeof(P.q));
}

// MCM/mcm_eqos.f90:24-55
void Sim::eqos(int i) {
    switch (mat[par[i].mat].eos) {
        case 1: eqos1(i); break;
        case 4: eqos4(i); break;
        case 13: eqos13(i); break;
        case 28: eqos28(i); break;
        case 41: eqos41(i); break;
    }
}

// MCM/mcm_eqos1.f90:32-75
void Sim::eqos1(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real c0 = ei[0], c1 = ei[1], c2 = ei[2], c3 = ei[3], c4 = ei[4], c5 = ei[5], c6 = ei[6];
    real mu = P.rho / P.rho0 - 1.0;
    real mu_t = std::max(mu, 0.0);
    real dvol = P.mass / P.rho - P.mass / P.rhoold;
    real vol0 = P.mass / P.rho0;
    real e1try = P.etry / vol0;
    real termone = c0 + (c1 + c3 * (mu * mu)) * mu + c2 * (mu_t * mu_t);
    real termtwo = c4 + c5 * mu + c6 * (mu_t * mu_t);
    P.p = (termone + termtwo * e1try) / (1 + termtwo * (dvol / vol0));
    if (P.p < P.pcut) {
        P.p = P.pcut;
        P.rho = P.rho / (1.0 - P.tracerod * dt);
    } else {
        P.e = P.etry - 0.5 * dvol * P.p;
    }
}

// MCM/mcm_eqos4.f90:30-82
void Sim::eqos4(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real c1 = ei[0], s1 = ei[1], s2 = ei[2], s3 = ei[3], gamma = ei[4], a1 = ei[5];
    real mu = P.rho / P.rho0 - 1.0;
    real dvol = P.mass / P.rho - P.mass / P.rhoold;
    real vol0 = P.mass / P.rho0;
    real e1try = P.etry / vol0;
    if (mu > 0.0) {
        real termone = mu * (1.0 - (gamma / 2.0));
        real termtwo = (a1 / 2.0) * mu * mu;
        real eosnum = mu * P.rho0 * (c1 * c1) * (1.0 + termone - termtwo);
        real mu21 = (mu * mu) / (mu + 1.0);
        real mu32 = (mu * mu * mu) / ((mu + 1.0) * (mu + 1.0));
        real eosden = 1.0 - (s1 - 1.0) * mu - s2 * mu21 - s3 * mu32;
        P.p = (eosnum / (eosden * eosden) + (gamma + a1 * mu) * e1try) / (1.0 + 0.5 * (gamma + a1 * mu) * dvol / vol0);
    } else {
        P.p = (P.rho0 * (c1 * c1) * mu + (gamma + a1 * mu) * e1try) / (1.0 + 0.5 * (gamma + a1 * mu) * dvol / vol0);
    }
    if (P.p < P.pcut) {
        P.p = P.pcut;
        P.rho = P.rho / (1.0 - P.tracerod * dt);
    } else {
        P.e = P.etry - 0.5 * dvol * P.p;
    }
}

// MCM/mcm_eqos13.f90:30-46
void Sim::eqos13(int i) {
    Particle &P = par[i];
    real gamma_m1 = mat[P.mat].eosinput[0] - 1.0;
    real e1try = P.etry / P.mass;
    real dvol = P.mass / P.rho - P.mass / P.rhoold;
    P.p = (P.rho * gamma_m1 * e1try) / (1.0 + 0.5 * P.rho * gamma_m1 * dvol / P.mass);
    P.e = P.etry - 0.5 * dvol * P.p;
}

// MCM/mcm_eqos28.f90:30-45
void Sim::eqos28(int i) {
    Particle &P = par[i];
    real b = mat[P.mat].eosinput[0], gamma = mat[P.mat].eosinput[1];
    real dvol = P.mass / P.rho - P.mass / P.rhoold;
    P.p = b * (std::pow(P.rho / P.rho0, gamma) - 1.0);
    P.e = P.etry - 0.5 * dvol * P.p;
}

// MCM/mcm_eqos41.f90:32-102
void Sim::eqos41(int i) {
    Particle &P = par[i];
    const real *ei = mat[P.mat].eosinput;
    real cc = ei[0], sl = ei[1], gama0 = ei[4];
    real etry1 = P.etry / P.mass;
    real ao = P.rho0 * (cc * cc);
    real mu = P.rho / P.rho0 - 1.0;
    real dvol = P.mass / P.rho - P.mass / P.rhoold;
    real vol0 = P.mass / P.rho0;
    real gama = gama0 * P.rho0 / P.rho;
    real bo = ao * (1.0 + 2.0 * (sl - 1.0));
    real co = ao * (2.0 * (sl - 1.0) + 3.0 * ((sl - 1.0) * (sl - 1.0)));
    real f = gama * mu;
    real ph;
    if (mu > 0.0) ph = ao * mu + bo * (mu * mu) + co * (mu * mu * mu);
    else ph = ao * mu;
    real pn = (ph * (1.0 - 0.5 * f) + P.rho * gama * etry1) / (1.0 + 0.5 * P.rho * gama * dvol / vol0);
    if (pn < P.pcut) {
        pn = P.pcut;
        P.rho = P.rho / (1.0 - P.tracerod * dt);
    } else {
        P.e = etry1 * P.mass - 0.5 * dvol * pn;
    }
    P.p = pn;
}

// MCM/mcm_stress_up.f90:28-36
void Sim::stress_up(int i) {
    Particle &P = par[i];
    P.sigma[0][0] = P.s[0][0] - P.p;
    P.sigma[1][1] = P.s[1][1] - P.p;
    P.sigma[2][2] = P.s[2][2] - P.p;
    P.sigma[0][1] = P.s[0][1];
    P.sigma[0][2] = P.s[0][2];
    P.sigma[1][2] = P.s[1][2];
    P.sigma[1][0] = P.sigma[0][1];
    P.sigma[2][0] = P.sigma[0][2];
    P.sigma[2][1] = P.sigma[1][2];
}

// MCM/mcm_lieupd.f90:26-33
void Sim::lieupd(int nn) {
    Particle &P = par[nn];
    real qpm = 0.0;
    for (int l = 0; l < 3; ++l)
        for (int k = 0; k < 3; ++k) qpm = qpm + P.q[k][l] * P.rod[k][l];
    P.e = P.e + (P.einc - dt * qpm) * P.mass / P.rho;
}

// ------------------------------------------------------------ cap model
// Model 4: the generalised cap model of MCM/mcm_f3dm25.f90 (f3dm25a :37-827,
// feit :906-966, fcit :968-1038).  f3dm25a has no `implicit none`: every local
// it does not declare is default REAL (single precision; names i-n INTEGER).
// Those locals are float here, the declared ones (sig*, dd*, p, bulk, capan,
// davgm, gdt, gd2, ...) double, and mixed expressions are evaluated in the
// wider kind, left to right.  Single-precision exp is taken as the correctly
// rounded float of a double exp (fexp); sqrt and the four operations are IEEE
// in both kinds.  Quirks kept:
//  * the local `capa` (not par%capa) is never assigned: static and zero under
//    /Qsave, so the first Fe of :197 is Fe(0);
//  * only the upper triangle of sigma is written back (:813-815): the lower
//    triangle keeps the rotated stress of mcm_stress_rot1, which the next
//    rotation (sigma(3,1)) and the momentum sum read;
//  * `nplot = cm(2,5)` and `xint = cm(2,5)` (mcm_sets4.f90:28) share a slot,
//    while f3dm25 reads X0 for the hardening law from cm(2,4) (`z`).
// A return-map iteration that does not converge (feit/fcit, 100 iterations)
// stops the reference; here it returns MCMO_ECAP_NOCONV.

inline float fexp(float x) { return (float)std::exp((double)x); }

struct CapConst {
    float shear, alpha, theta, gama, beta, r, dDyna, w, z, tcut, fcut;
    double bulk;
    int ltype, ivec;
};

// One iteration of the failure-surface return (feit :923-960 and the
// unrolled copies of f3dm25a :491-596).  capa is par%capa (double).
static void cap_fail_iter(const CapConst &C, double &capa, double sig[6], float s[6], float &x1, float &x2d) {
    float xk = (float)(capa + C.r * (C.alpha - C.gama * std::exp(-C.beta * capa) + C.theta * capa));
    float dhdk = (float)((C.w * C.dDyna * fexp(-C.dDyna * xk)) *
                         (1.0 + C.r * (C.theta + C.gama * C.beta * std::exp(-C.beta * capa))));
    float omega = C.theta + C.gama * C.beta * fexp(-C.beta * x1);
    float dcd = (float)(C.shear + 9.0 * C.bulk * (double)(omega * omega));
    float f = x2d - (C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1);
    float delcap = -(3.0f * omega * f / (dcd * dhdk));
    float delam = -(dhdk * delcap / (3.0f * omega));
    capa = capa + delcap;
    (void)xk;
    float fac1 = C.shear / x2d;
    float fac2 = (float)(3.0 * C.bulk * omega);
    sig[0] = sig[0] - delam * (fac1 * s[0] - fac2);
    sig[1] = sig[1] - delam * (fac1 * s[1] - fac2);
    sig[2] = sig[2] - delam * (fac1 * s[2] - fac2);
    sig[3] = sig[3] - delam * fac1 * s[3];
    sig[4] = sig[4] - delam * fac1 * s[4];
    sig[5] = sig[5] - delam * fac1 * s[5];
    x1 = (float)(sig[0] + sig[1] + sig[2]);
    s[0] = (float)(sig[0] - x1 / 3.0f);
    s[1] = (float)(sig[1] - x1 / 3.0f);
    s[2] = (float)(sig[2] - x1 / 3.0f);
    s[3] = (float)sig[3];
    s[4] = (float)sig[4];
    s[5] = (float)sig[5];
    x2d = std::sqrt(0.5f * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
}

// One iteration of the cap return (fcit :986-1022 and f3dm25a :652-800).
// Returns the cap function value of the convergence test of fcit (:1023) and
// the elcap of the iteration (before the capa update).
static float cap_cap_iter(const CapConst &C, double &capa, double sig[6], float s[6], float &x1, float &x2d,
                          float &elcap_out) {
    const float unit = 1.0f;
    float xk = (float)(capa + C.r * (C.alpha - C.gama * std::exp(-C.beta * capa) + C.theta * capa));
    float dhdk = (float)((C.w * C.dDyna * fexp(-C.dDyna * xk)) *
                         (1.0 + C.r * (C.theta + C.gama * C.beta * std::exp(-C.beta * capa))));
    float dfdk;
    if (capa >= 0.0) {
        dfdk = (float)(-(2.0f * (std::fabs((double)x1 - capa) / (double)(C.r * C.r) +
                                 (C.alpha - C.gama * std::exp(-C.beta * capa) + C.theta * capa) *
                                     (C.theta + C.gama * C.beta * std::exp(-C.beta * capa)))));
    } else {
        dfdk = (float)(-(((2.0f * xk) * (1.0 + C.r * (C.theta + C.gama * C.beta * std::exp(-C.beta * capa)))) /
                         (double)(C.r * C.r)));
    }
    float elcap = (float)std::max(capa, (double)(0.0f * unit));
    float omega = std::min(-(2.0f * std::fabs(x1 - elcap) / (C.r * C.r)), -1.e-15f * unit);
    float dcd = (float)((4.0f * C.shear * (x2d * x2d)) +
                        9.0 * C.bulk * (double)((2.0f * (x1 - elcap) / (C.r * C.r)) * (2.0f * (x1 - elcap) / (C.r * C.r))));
    float f = x2d * x2d + (x1 - elcap) * (x1 - elcap) / (C.r * C.r) - (xk - elcap) * (xk - elcap) / (C.r * C.r);
    float delcap = -(f / (dfdk + (dcd * dhdk) / (3.0f * omega)));
    float delam = -(dhdk * delcap / (3.0f * omega));
    capa = capa + delcap;
    xk = (float)(capa + C.r * (C.alpha - C.gama * std::exp(-C.beta * capa) + C.theta * capa));
    float fac1 = 2.0f * C.shear;
    float fac2 = (float)(6.0 * C.bulk * (double)std::fabs(x1 - elcap) / (double)(C.r * C.r));
    sig[0] = sig[0] - delam * (fac1 * s[0] + fac2);
    sig[1] = sig[1] - delam * (fac1 * s[1] + fac2);
    sig[2] = sig[2] - delam * (fac1 * s[2] + fac2);
    sig[3] = sig[3] - delam * fac1 * s[3];
    sig[4] = sig[4] - delam * fac1 * s[4];
    sig[5] = sig[5] - delam * fac1 * s[5];
    x1 = (float)(sig[0] + sig[1] + sig[2]);
    s[0] = (float)(sig[0] - x1 / 3.0f);
    s[1] = (float)(sig[1] - x1 / 3.0f);
    s[2] = (float)(sig[2] - x1 / 3.0f);
    s[3] = (float)sig[3];
    s[4] = (float)sig[4];
    s[5] = (float)sig[5];
    x2d = std::sqrt(0.5f * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    elcap_out = elcap;
    return x2d * x2d + (x1 - elcap) * (x1 - elcap) / (C.r * C.r) - (xk - elcap) * (xk - elcap) / (C.r * C.r);
}

int Sim::f3dm25(Material &M, int i) {
    Particle &P = par[i];
    const float unit = 1.0f, third = 1.0f / 3.0f, geop = 0.0f, tol = 1.0e-7f;
    CapConst C;
    C.bulk = M.cm(1, 1);
    C.shear = (float)M.cm(1, 2);
    C.alpha = (float)M.cm(1, 3);
    C.theta = (float)M.cm(1, 4);
    C.gama = (float)M.cm(1, 5);
    C.beta = (float)M.cm(1, 6);
    C.r = (float)M.cm(2, 1);
    C.dDyna = (float)M.cm(2, 2);
    C.w = (float)M.cm(2, 3);
    const float falfac = (float)M.cm(4, 1);
    C.alpha = C.alpha - falfac;
    C.z = (float)M.cm(2, 4);
    C.ivec = (M.cm(3, 5) != 0.0) ? 0 : 1;
    C.ltype = (int)M.cm(2, 6);
    C.tcut = (float)M.cm(3, 1);
    C.fcut = (float)M.cm(3, 4);
    const float t = std::max(C.fcut, C.tcut + 3.0f * geop);
    const float fet = C.alpha - C.gama * fexp(-C.beta * t) + C.theta * t;
    const float fept = C.gama * C.beta * fexp(-C.beta * t) + C.theta;
    P.capa = std::max(P.capa, M.cm(3, 3));
    double sig[6] = {-P.sigma[0][0], -P.sigma[1][1], -P.sigma[2][2], -P.sigma[0][1], -P.sigma[0][2], -P.sigma[1][2]};
    const double dd1 = -P.rod[0][0], dd2 = -P.rod[1][1], dd3 = -P.rod[2][2];
    const double dd4 = -P.rod[0][1] / 2.0, dd5 = -P.rod[0][2] / 2.0, dd6 = -P.rod[1][2] / 2.0;
    const double dd = (dd1 + dd2 + dd3);
    const double davgm = (double)(1.0f / 3.0f) * dd;
    const float dt1 = (float)dt;
    double p = 3.0 * C.bulk * (double)dt1 * davgm;
    const double gdt = dt * (double)C.shear;
    const double gd2 = 2.0 * gdt;
    const float gtr11 = (float)(sig[0] + p + gd2 * (dd1 - davgm));
    const float gtr22 = (float)(sig[1] + p + gd2 * (dd2 - davgm));
    const float gtr33 = (float)(sig[2] + p + gd2 * (dd3 - davgm));
    const float gtr12 = (float)(sig[3] + gd2 * dd4);
    const float gtr23 = (float)(sig[4] + gd2 * dd5);
    const float gtr31 = (float)(sig[5] + gd2 * dd6);
    const float x1tr = gtr11 + gtr22 + gtr33;
    float s[6];
    s[0] = gtr11 - (1.0f / 3.0f) * x1tr;
    s[1] = gtr22 - (1.0f / 3.0f) * x1tr;
    s[2] = gtr33 - (1.0f / 3.0f) * x1tr;
    const float sdtr11 = s[0], sdtr22 = s[1], sdtr33 = s[2];
    float x2dtr = 0.5f * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0f * (gtr12 * gtr12 + gtr23 * gtr23 + gtr31 * gtr31));
    x2dtr = std::sqrt(x2dtr);
    const float capa_local = 0.0f;   // never assigned in f3dm25a (see above)
    float fe = C.alpha - C.gama * fexp(-C.beta * capa_local) + C.theta * capa_local;
    const float xkn = capa_local + C.r * fe;
    const float elcapn = (float)std::max(P.capa, (double)(0.0f * unit));
    const float tmises = std::fabs(xkn - elcapn) / C.r;
    fe = C.alpha - C.gama * fexp(-C.beta * x1tr) + C.theta * x1tr;
    const float f1tr = x2dtr - std::min(fe, tmises);
    const float tcrit = (float)((double)t - 9.0 * C.bulk / (double)C.shear * (double)(x2dtr - fet) * (double)fept);
    fe = C.alpha - C.gama * fexp(-C.beta * elcapn) + C.theta * elcapn;
    const float fep = C.beta * C.gama * fexp(-C.beta * elcapn) + C.theta;
    const float fc2tr = ((xkn - elcapn) * (xkn - elcapn) - (x1tr - elcapn) * (x1tr - elcapn)) / (C.r * C.r);
    const float f2tr = x2dtr * x2dtr - fc2tr;
    const float x1crt = (float)((double)elcapn - ((double)((x2dtr - fe) * 9.0f) * C.bulk) * (double)fep / (double)C.shear);
    fe = (float)(C.alpha - C.gama * std::exp(-C.beta * P.capa) + C.theta * P.capa);
    const float capal = (float)std::min((double)(0.0f * unit), P.capa - (double)(tol * fe));
    fe = C.alpha - C.gama * fexp(-C.beta * capal) + C.theta * capal;
    const float xk0 = capal + C.r * fe;
    const float evpn = C.w * (1.0f - fexp(C.dDyna * (C.z - xkn)));
    const float devpb = C.w * (1.0f - fexp(C.dDyna * (C.z - xk0))) - evpn;
    const double capan = P.capa;
    const int ltype = C.ltype;
    // mode selection (:219-253)
    int imode = 0;
    if ((x1tr <= t) && (x2dtr <= fet) && (ltype == 1) && (capan > 0.0) && (devpb >= 0.0f)) imode = 2;
    else if ((x1tr <= t) && (x2dtr <= fet) && (ltype == 1) && (capan > 0.0) && (devpb < 0.0f)) imode = 7;
    else if ((x1tr <= t) && (x2dtr <= fet) && ((ltype == 2) || (capan <= 0.0))) imode = 3;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr <= tcrit) && (ltype == 1) && (capan > 0.0) && (devpb >= 0.0f)) imode = 4;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr <= tcrit) && (ltype == 1) && (capan > 0.0) && (devpb < 0.0f)) imode = 6;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr <= tcrit) && ((ltype == 2) || (capan <= 0.0))) imode = 5;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr > tcrit) && (capan >= 0.0)) imode = 10;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr > tcrit) && (capan < 0.0)) imode = 8;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr <= tol)) imode = 1;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr > tol) && (x1tr >= x1crt)) imode = 9;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr > tol) && (x1tr < x1crt) && (capan >= 0.0)) imode = 10;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr > tol) && (x1tr < x1crt) && (capan < 0.0)) imode = 8;
    else if ((x1tr > t) && (x1tr > elcapn) && (f2tr < tol)) imode = 1;
    else if ((x1tr > t) && (x1tr > elcapn) && (f2tr >= tol)) imode = 11;
    P.ptype = imode;
    float x1 = 0.0f, x2d = 0.0f, ratio = 0.0f;
    auto set_scaled = [&](const float *sd, float rat) {   // sig = s*ratio + p, off-diagonals gtr*ratio
        sig[0] = (double)(sd[0] * rat) + p;
        sig[1] = (double)(sd[1] * rat) + p;
        sig[2] = (double)(sd[2] * rat) + p;
        sig[3] = (double)(gtr12 * rat);
        sig[4] = (double)(gtr23 * rat);
        sig[5] = (double)(gtr31 * rat);
    };
    auto set_plain = [&]() {   // sig = s + p, off-diagonals gtr
        sig[0] = (double)s[0] + p;
        sig[1] = (double)s[1] + p;
        sig[2] = (double)s[2] + p;
        sig[3] = (double)gtr12;
        sig[4] = (double)gtr23;
        sig[5] = (double)gtr31;
    };
    auto move_cap = [&]() {   // modes 6 and 7 (:359-364, :381-386)
        const float x1old = (float)(sig[0] + sig[1] + sig[2]);
        const float devp = (float)(dd - (double)(x1 - x1old) / (3.0 * C.bulk));
        const float xhat = std::min(devpb, devp);
        P.capa = P.capa + (double)devp * ((double)capal - capan) / (double)xhat;
        P.capa = std::max(P.capa, (double)(0.0f * unit));
    };
    switch (imode) {
        case 1:
            x1 = x1tr; x2d = x2dtr; P.capa = capan;
            p = (double)(third * x1 + geop);
            set_plain();
            break;
        case 2:
            x1 = t; x2d = x2dtr; P.capa = 0.0;
            p = (double)(third * x1 + geop);
            set_plain();
            break;
        case 3:
            x1 = t; x2d = x2dtr; P.capa = capan;
            p = (double)(third * x1 + geop);
            set_plain();
            break;
        case 4:
            x1 = t; x2d = fet; P.capa = 0.0;
            p = (double)(third * x1 + geop);
            ratio = x2d / x2dtr;
            set_scaled(s, ratio);
            break;
        case 5:
            x1 = t; x2d = fet; P.capa = capan;
            p = (double)(third * x1 + geop);
            ratio = x2d / x2dtr;
            set_scaled(s, ratio);
            break;
        case 6:
            x1 = t; x2d = fet;
            move_cap();
            p = (double)(third * x1 + geop);
            ratio = x2d / x2dtr;
            set_scaled(s, ratio);
            break;
        case 7:
            x1 = t; x2d = x2dtr;
            move_cap();
            p = (double)(third * x1 + geop);
            set_plain();
            break;
        case 8:
            x1 = x1tr;
            fe = C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1;
            x2d = std::min(fe, tmises);
            P.capa = capan;
            ratio = x2d / x2dtr;
            p = (double)(third * x1 + geop);
            set_scaled(s, ratio);
            break;
        case 9:
            x1 = elcapn;
            x2d = C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1;
            P.capa = capan;
            ratio = x2d / x2dtr;
            p = (double)(third * x1 + geop);
            set_scaled(s, ratio);
            break;
        case 10: {
            double sg[6] = {gtr11, gtr22, gtr33, gtr12, gtr23, gtr31};
            P.capa = capan;
            x1 = x1tr;
            x2d = x2dtr;
            float si[6];
            for (int k = 0; k < 3; ++k) si[k] = (float)(sg[k] - x1tr / 3.0f);
            for (int k = 3; k < 6; ++k) si[k] = (float)sg[k];
            if (C.ivec == 0) {
                // feit: iterate to |f| <= 1e-8 (at most 100 iterations)
                bool conv = false;
                for (int it = 1; it <= 100; ++it) {
                    cap_fail_iter(C, P.capa, sg, si, x1, x2d);
                    const float f = x2d - (C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1);
                    if (std::fabs(f) <= 1.0e-8f) { conv = true; break; }
                }
                if (!conv) return MCMO_ECAP_NOCONV;
            } else {
                for (int it = 0; it < 4; ++it) cap_fail_iter(C, P.capa, sg, si, x1, x2d);
            }
            if (x1 > elcapn) x1 = elcapn;
            if ((ltype == 2) || (capan == 0.0)) P.capa = capan;
            if ((double)x1 > P.capa) P.capa = x1;
            if ((ltype == 1) && (capan >= 0.0)) P.capa = std::max(P.capa, (double)(0.0f * unit));
            fe = C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1;
            x2d = std::min(fe, tmises);
            ratio = x2d / x2dtr;
            p = (double)(third * x1 + geop);
            if (C.ivec == 0) {
                set_scaled(s, ratio);
            } else {
                const float sd[3] = {sdtr11, sdtr22, sdtr33};
                set_scaled(sd, ratio);
            }
            break;
        }
        case 11: {
            double sg[6] = {gtr11, gtr22, gtr33, gtr12, gtr23, gtr31};
            P.capa = capan;
            x1 = x1tr;
            x2d = x2dtr;
            float si[6];
            for (int k = 0; k < 3; ++k) si[k] = (float)(sg[k] - x1tr / 3.0f);
            for (int k = 3; k < 6; ++k) si[k] = (float)sg[k];
            float elcap = 0.0f;
            bool done = false;
            const int nit = (C.ivec == 0) ? 100 : 4;
            for (int it = 1; it <= nit; ++it) {
                const float f = cap_cap_iter(C, P.capa, sg, si, x1, x2d, elcap);
                if (C.ivec == 0 && std::fabs(f) <= 1.0e-8f) { done = true; break; }
            }
            if (C.ivec == 0 && !done) return MCMO_ECAP_NOCONV;
            if (x1 < elcap) {
                x1 = elcap + std::fabs(x1 - elcap);
                sg[0] = (double)(si[0] + x1 / 3.0f);
                sg[1] = (double)(si[1] + x1 / 3.0f);
                sg[2] = (double)(si[2] + x1 / 3.0f);
            }
            for (int k = 0; k < 6; ++k) sig[k] = sg[k];
            break;
        }
        default: break;
    }
    // write-back (:813-827): the upper triangle only
    P.sigma[0][0] = -sig[0];
    P.sigma[1][1] = -sig[1];
    P.sigma[2][2] = -sig[2];
    P.sigma[0][1] = -sig[3];
    P.sigma[0][2] = -sig[4];
    P.sigma[1][2] = -sig[5];
    P.p = -(1.0 / 3.0) * (P.sigma[0][0] + P.sigma[1][1] + P.sigma[2][2]);
    return MCMO_OK;
}

// MCM/mcm_calccritts.f90:32-87
void Sim::calccritts() {
    critts = 1.0e20;
    for (int i = ssp; i <= esp; ++i) {
        Particle &P = par[i];
        const Material &M = mat[P.mat];
        if (tcrit_opt == 0) {
            real veae = 0, ae = 0;
            real vol = P.mass / P.rho;
            switch (ndim) {
                case 1: veae = vol; ae = 1; break;
                case 2: veae = std::sqrt(vol); ae = std::sqrt(vol); break;
                case 3: veae = std::pow(vol, 1.0 / 3.0); ae = std::pow(vol, 2.0 / 3.0); break;
            }
            real qu = (M.av_l * P.c + M.av_q * P.mass / P.rho * P.tracerod) / ae;
            P.critts = veae / (qu + std::sqrt(qu * qu + P.c * P.c));
        } else if (tcrit_opt == 1) {
            P.critts = P.h / (P.c + P.vabs);
        } else if (tcrit_opt == 2) {
            P.critts = P.mindist / (P.c + P.vabs);
        }
        if (P.active)
            if (P.critts < critts) critts = P.critts;
    }
}

// =========================================================================
// Momentum (MCM/mcm_momentum.f90, mcm_oldacceleration.f90, mcm_corr_acceleration.f90)
// =========================================================================

void Sim::momentum() {
    if (boundary) update_ghost_stress();
    if (disctype == 0) oldacceleration();
    else corr_acceleration();
}

// MCM/mcm_update_ghost_stress.f90:28-41 (all off-diagonals flipped)
void Sim::update_ghost_stress() {
    for (int g = 1; g <= ngp; ++g) {
        int id = gpar[g].par;
        for (int k = 0; k < 3; ++k)
            for (int j = 0; j < 3; ++j) {
                real f = (j == k) ? 1.0 : -1.0;
                gpar[g].sigma[j][k] = f * par[id].sigma[j][k];
                gpar[g].q[j][k] = f * par[id].q[j][k];
            }
    }
}

// MCM/mcm_get_j_moment_info.f90:31-58
void Sim::get_j_moment_info(int i, int k, real *x, real &mass, real &rho, real &h, real &hold,
                            real sig[3][3], real qq[3][3]) {
    const Particle &P = par[i];
    if (k <= P.nnbr) {
        const Particle &J = par[P.nbr[k - 1]];
        for (int m = 0; m < 3; ++m) x[m] = J.x[m];
        mass = J.mass; h = J.h; hold = J.hold; rho = J.rho;
        std::memcpy(sig, J.sigma, sizeof(J.sigma));
        std::memcpy(qq, J.q, sizeof(J.q));
    } else {
        const Ghost &J = gpar[P.gnbr[k - P.nnbr - 1]];
        for (int m = 0; m < 3; ++m) x[m] = J.x[m];
        mass = J.mass; h = J.h; hold = J.hold; rho = J.rho;
        std::memcpy(sig, J.sigma, sizeof(J.sigma));
        std::memcpy(qq, J.q, sizeof(J.q));
    }
}

// =========================================================================
// Repulsive contact (MCM/mcm_rep_contact.f90, mcm_get_j_cont_info.f90),
// called by MCM/mcm_solution.f90:64 when contacttype > 0, after the dt update
// and before mcm_momentum.  It reads the contact lists that
// mcm_ll_neighbours builds from particles of other materials (:150-174).
// =========================================================================

// MCM/mcm_get_j_cont_info.f90:31-58.  For k > ncont the reference reads the
// ghost index from the REAL contact list (mcm_contlist(k,i), :48), whose
// entries past ncont are left over from earlier searches or never written;
// the ghost contact list the search builds for that purpose (mcm_g_contlist)
// is read here instead.
void Sim::get_j_cont_info(int i, int k, real *x, real &mass, real &rho, real &h, real &kj) const {
    const Particle &P = par[i];
    if (k <= P.ncont) {
        const Particle &J = par[P.cont[k - 1]];
        kj = mat[J.mat].k_cont;
        for (int m = 0; m < 3; ++m) x[m] = J.x[m];
        mass = J.mass; rho = J.rho; h = J.h;
    } else {
        const Ghost &J = gpar[P.gcont[k - P.ncont - 1]];
        kj = mat[J.mat].k_cont;
        for (int m = 0; m < 3; ++m) x[m] = J.x[m];
        mass = J.mass; rho = J.rho; h = J.h;
    }
}

// MCM/mcm_rep_contact.f90:102-161 (mcm_calc_fij).  The velocity difference of
// :133-134 reads the uninitialised locals vi, vj and feeds only xijdotvij,
// which nothing uses (:156-157 are commented out), so it is not restated.
real Sim::calc_fij(const real *xi, const real *xj, real havg, real inv_w_deltap) const {
    real rad = 0.0;
    for (int n = 0; n < ndim; ++n) {
        real xij = xi[n] - xj[n];
        rad = rad + xij * xij;
    }
    rad = std::sqrt(rad);
    real z = rad / havg;
    if (z < 1.0) return inv_w_deltap * (((0.75 * z - 1.5) * z) * z + 1.0);
    if (z < 2.0) {
        real t = 2.0 - z;
        return 0.25 * inv_w_deltap * (t * t * t);
    }
    return 0.0;
}

// MCM/mcm_rep_contact.f90:37-94: Monaghan's repulsive acceleration
// -sum_j m_j (K_i + K_j) f_ij^n grad W_ij over the real and ghost contacts,
// only for particles with at least one real contact (:41).
void Sim::rep_cont() {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = svp; i <= evp; ++i) {
        Particle &P = par[i];
        for (int l = 0; l < ndim; ++l) P.repulsion[l] = 0.0;
        if (P.ncont > 0) {
            const real ki = mat[P.mat].k_cont;
            const real n = mat[P.mat].n_cont;
            for (int j = 1; j <= P.ncont + P.g_ncont; ++j) {
                real xj[3] = {0, 0, 0}, massj, rhoj, hj, kj;
                get_j_cont_info(i, j, xj, massj, rhoj, hj, kj);
                real havg = 0.5 * (P.h + hj);
                // inverse of W(delta p) for the cubic B-spline (:55-68)
                real ratio = hj / havg;
                real inv_w_deltap;
                if (ratio < 1.0) inv_w_deltap = 1.0 / (((0.75 * ratio - 1.5) * ratio) * ratio + 1.0);
                else { real t = 2.0 - ratio; inv_w_deltap = 1.0 / (t * t * t); }
                real dwdx[3] = {0, 0, 0}, dwdr = 0;
                grad1(dwdx, dwdr, P.x, xj, havg);
                real fij = calc_fij(P.x, xj, havg, inv_w_deltap);
                real kij = ki + kj;
                for (int l = 0; l < ndim; ++l)
                    P.repulsion[l] = P.repulsion[l] - (massj * (kij * std::pow(fij, n)) * dwdx[l]);
            }
        }
    }
}

// MCM/mcm_oldacceleration.f90:36-90.  With contacttype > 0 the acceleration
// starts from par%repulsion and the per-material contact forces xcf, ycf, zcf
// (written to the time-history file) sum mass x repulsion (:44-56).
void Sim::oldacceleration() {
    for (int i = 1; i <= nummat; ++i) { mat[i].xcf = 0.0; mat[i].ycf = 0.0; mat[i].zcf = 0.0; }
    if (contacttype > 0)
        for (int i = svp; i <= evp; ++i) {
            const Particle &P = par[i];
            mat[P.mat].xcf = mat[P.mat].xcf + P.mass * P.repulsion[0];
            mat[P.mat].ycf = mat[P.mat].ycf + P.mass * P.repulsion[1];
            mat[P.mat].zcf = mat[P.mat].zcf + P.mass * P.repulsion[2];
        }
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = svp; i <= evp; ++i) {
        Particle &P = par[i];
        P.a[0] = P.a[1] = P.a[2] = 0.0;
        if (contacttype > 0)
            for (int l = 0; l < ndim; ++l) P.a[l] = P.a[l] + P.repulsion[l];
        real rhoi = P.rho;
        real sigmai[3][3], qi[3][3];
        std::memcpy(sigmai, P.sigma, sizeof(sigmai));
        std::memcpy(qi, P.q, sizeof(qi));
        int nk = P.nnbr + P.g_nnbr;
        for (int k = 1; k <= nk; ++k) {
            real xj[3], massj, rhoj, hj, holdj, sigmaj[3][3], qj[3][3];
            get_j_moment_info(i, k, xj, massj, rhoj, hj, holdj, sigmaj, qj);
            real havg = 0.5 * (P.h + hj);
            real deltasig[3] = {0, 0, 0};
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, P.x, xj, havg);
            for (int n = 0; n < ndim; ++n)
                for (int m = 0; m < ndim; ++m)
                    deltasig[n] = deltasig[n] + ((sigmaj[m][n] - qj[m][n]) / (rhoj * rhoj) +
                                                 (sigmai[m][n] - qi[m][n]) / (rhoi * rhoi)) * dwdx[m];
            for (int l = 0; l < ndim; ++l) P.a[l] = P.a[l] + massj * deltasig[l];
        }
    }
}

// MCM/mcm_corr_acceleration.f90:37-163 (kernel centred at j; self slot zeroed;
// the final sum uses the mass of the last neighbour visited).  With
// contacttype > 0 the acceleration starts from par%repulsion (:45-49); this
// routine does not touch the per-material contact forces.
void Sim::corr_acceleration() {
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = svp; i <= evp; ++i) {
        Particle &P = par[i];
        P.a[0] = P.a[1] = P.a[2] = 0.0;
        if (contacttype > 0)
            for (int l = 0; l < ndim; ++l) P.a[l] = P.a[l] + P.repulsion[l];
        real rhoi = P.rho;
        real sigmai[3][3], qi[3][3];
        std::memcpy(sigmai, P.sigma, sizeof(sigmai));
        std::memcpy(qi, P.q, sizeof(qi));
        int nk = P.nnbr + P.g_nnbr;
        real sum_w = 0, sum_gradw[3] = {0, 0, 0};
        real massj = 0;
        for (int k = 1; k <= nk; ++k) {
            real xj[3], rhoj, hj, holdj, sigmaj[3][3], qj[3][3];
            get_j_moment_info(i, k, xj, massj, rhoj, hj, holdj, sigmaj, qj);
            real Volj = massj / rhoj;
            real havg = 0.5 * (P.h + hj);
            real w = kernel1(xj, P.x, havg);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, xj, P.x, havg);
            sum_w = sum_w + Volj * w;
            for (int l = 0; l < ndim; ++l) sum_gradw[l] = sum_gradw[l] + Volj * dwdx[l];
        }
        real B[3][3] = {};
        for (int k = 1; k <= nk; ++k) {
            real xj[3], rhoj, hj, holdj, sigmaj[3][3], qj[3][3];
            get_j_moment_info(i, k, xj, massj, rhoj, hj, holdj, sigmaj, qj);
            real Volj = massj / rhoj;
            real havg = 0.5 * (P.h + hj);
            real w = kernel1(xj, P.x, havg);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, xj, P.x, havg);
            real cg[3];
            for (int m = 0; m < ndim; ++m) cg[m] = (dwdx[m] * sum_w - w * sum_gradw[m]) / (sum_w * sum_w);
            for (int m = 0; m < ndim; ++m)
                for (int n = 0; n < ndim; ++n) B[n][m] = B[n][m] + Volj * (xj[n] - P.x[n]) * cg[m];
        }
        real invB[3][3];
        inverse(B, invB);
        real deltasig[3][3][3] = {};
        for (int k = 1; k <= nk; ++k) {
            real xj[3], rhoj, hj, holdj, sigmaj[3][3], qj[3][3];
            get_j_moment_info(i, k, xj, massj, rhoj, hj, holdj, sigmaj, qj);
            real havg = 0.5 * (P.h + hj);
            real w = kernel1(xj, P.x, havg);
            real dwdx[3] = {0, 0, 0}, dwdr = 0;
            grad1(dwdx, dwdr, xj, P.x, havg);
            real cg[3];
            for (int m = 0; m < ndim; ++m) cg[m] = (dwdx[m] * sum_w - w * sum_gradw[m]) / (sum_w * sum_w);
            for (int n = 0; n < ndim; ++n)
                for (int m = 0; m < ndim; ++m) {
                    real dsig = (sigmaj[m][n] - qj[m][n]) / (rhoj * rhoj) + (sigmai[m][n] - qi[m][n]) / (rhoi * rhoi);
                    if (k == P.nnbr) dsig = 0.0;
                    for (int l = 0; l < ndim; ++l) deltasig[m][n][l] = deltasig[m][n][l] + dsig * cg[l];
                }
        }
        for (int n = 0; n < ndim; ++n)
            for (int m = 0; m < ndim; ++m)
                for (int l = 0; l < ndim; ++l) P.a[n] = P.a[n] + massj * deltasig[n][m][l] * invB[l][m];
    }
}

// MCM/mcm_boundcond.f90:23-62
void Sim::boundcond() {
    if (baseaccel)
        for (int i = svp; i <= evp; ++i)
            for (int j = 0; j < ndim; ++j) par[i].a[j] = par[i].a[j] + base_a[j];
    for (int i = svp; i <= evp; ++i) {
        real *a = par[i].a;
        switch (par[i].dispbc) {
            case 1: a[0] = 0.0; break;
            case 2: a[1] = 0.0; break;
            case 3: a[2] = 0.0; break;
            case 4: a[0] = 0.0; a[1] = 0.0; break;
            case 5: a[1] = 0.0; a[2] = 0.0; break;
            case 6: a[0] = 0.0; a[2] = 0.0; break;
            case 7: a[0] = 0.0; a[1] = 0.0; a[2] = 0.0; break;
            default: break;
        }
    }
}

// MCM/mcm_calctotale.f90:27-60
void Sim::calctotale() {
    for (int i = 1; i <= nummat; ++i) { mat[i].ie = 0.0; mat[i].ke = 0.0; mat[i].mom[0] = mat[i].mom[1] = mat[i].mom[2] = 0.0; }
    for (int i = svp; i <= evp; ++i) {
        if (!par[i].active) continue;
        Material &M = mat[par[i].mat];
        M.ke = M.ke + 0.5 * par[i].mass * (par[i].vabs * par[i].vabs);
        for (int j = 0; j < 3; ++j) M.mom[j] = M.mom[j] + par[i].mass * std::fabs(par[i].v[j]);
    }
    for (int i = ssp; i <= esp; ++i) {
        if (!par[i].active) continue;
        Material &M = mat[par[i].mat];
        M.ie = M.ie + par[i].e;
    }
    kinetice = 0.0; internale = 0.0;
    for (int i = 1; i <= nummat; ++i) { kinetice = kinetice + mat[i].ke; internale = internale + mat[i].ie; }
    totale = kinetice + internale;
}

// MCM/mcm_update_h.f90:25-55: h follows the volumetric strain rate (h_opt 1)
// or the density (h_opt 2) for particles at or above their cut-off pressure,
// and hmax, the next grid's cell size, is their largest h.  With no such
// particle the reference would set hmax to 0 (a zero division in the grid);
// the previous hmax is kept instead.
void Sim::update_h() {
    real hm = 0.0;
    if (h_opt == 1) {
        for (int i = ssp; i <= esp; ++i) {
            Particle &P = par[i];
            if (P.p >= P.pcut) {
                P.hold = P.h;
                P.h = P.hold * (1.0 + P.tracerod * dt / (real)(float)ndim);
                hm = std::max(hm, P.h);
            }
        }
    } else if (h_opt == 2) {
        const real power = 1.0 / (real)(float)ndim;
        for (int i = ssp; i <= esp; ++i) {
            Particle &P = par[i];
            if (P.p >= P.pcut) {
                P.hold = P.h;
                P.h = P.h0 * std::pow(P.rho0 / P.rho, power);
                hm = std::max(hm, P.h);
            }
        }
    }
    if (hm > 0.0) hmax = hm;
}

// MCM/mcm_update_velocity.f90:61-87: XSPH.  The neighbours' velocities are
// the updated ones for real particles and the ghosts' copies from the start of
// the step; W uses the neighbour's h; the sums are applied after all are done.
void Sim::xsph() {
    const real epsilon = 0.100;
    std::vector<real> sv(3 * (size_t)(np + 1), 0.0);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = 1; i <= np; ++i) {
        Particle &P = par[i];
        real s[3] = {0.0, 0.0, 0.0};
        for (int j = 1; j <= P.nnbr + P.g_nnbr; ++j) {
            real xj[3], vj[3], massj, rhoj, hj, holdj;
            get_j_strain_info(i, j, xj, vj, massj, rhoj, hj, holdj);
            real w = kernel1(P.x, xj, hj);
            real volj = massj / (0.5 * (rhoj + P.rho));
            for (int k = 0; k < ndim; ++k) s[k] = s[k] + volj * (vj[k] - P.v[k]) * w;
        }
        for (int k = 0; k < 3; ++k) sv[3 * (size_t)i + k] = s[k];
    }
    for (int i = 1; i <= np; ++i)
        for (int j = 0; j < ndim; ++j) par[i].v[j] = par[i].v[j] + epsilon * sv[3 * (size_t)i + j];
}

// MCM/mcm_update_velocity.f90:29-56, then XSPH (veloc_opt 1)
void Sim::update_velocity() {
    real dtn = 0.5 * (dt + dtold);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int i = svp; i <= evp; ++i) {
        Particle &P = par[i];
        P.vabs = 0.0;
        for (int j = 0; j < ndim; ++j) {
            if (drelax) P.v[j] = drelax_scale * P.v[j] + P.a[j] * dtn;
            else P.v[j] = P.v[j] + P.a[j] * dtn;
            P.vabs = P.vabs + P.v[j] * P.v[j];
        }
        P.vabs = std::sqrt(P.vabs);
    }
    if (veloc_opt == 1) xsph();
}

// MCM/mcm_move.f90:25-55
void Sim::move() {
    for (int i = 0; i < ndim; ++i) { coord_maxmin[0][i] = 1.0e+20; coord_maxmin[1][i] = -1.0e+20; }
    for (int i = 1; i <= np; ++i)
        for (int j = 0; j < ndim; ++j) {
            par[i].x[j] = par[i].x[j] + par[i].v[j] * dt;
            if (par[i].x[j] < coord_maxmin[0][j]) coord_maxmin[0][j] = par[i].x[j];
            if (par[i].x[j] > coord_maxmin[1][j]) coord_maxmin[1][j] = par[i].x[j];
        }
    if (boundary) check_sym_pen();
}

// MCM/mcm_check_sym_pen.f90:27-179
void Sim::check_sym_pen() {
    for (int d = 0; d < 3; ++d) {
        if (boundary_code[0][d] == 1 && coord_maxmin[0][d] < boundary_x[0][d])
            for (int i = svp; i <= evp; ++i)
                if (par[i].x[d] < boundary_x[0][d]) { par[i].x[d] = 2.0 * boundary_x[0][d] - par[i].x[d]; par[i].v[d] = -par[i].v[d]; }
        if (boundary_code[1][d] == 1 && coord_maxmin[1][d] > boundary_x[1][d])
            for (int i = svp; i <= evp; ++i)
                if (par[i].x[d] > boundary_x[1][d]) { par[i].x[d] = 2.0 * boundary_x[1][d] - par[i].x[d]; par[i].v[d] = -par[i].v[d]; }
        if (boundary_code[0][d] == 2) {
            real dx = boundary_x[1][d] - boundary_x[0][d];
            if (coord_maxmin[0][d] < boundary_x[0][d])
                for (int i = svp; i <= evp; ++i)
                    if (par[i].x[d] < boundary_x[0][d]) par[i].x[d] = par[i].x[d] + dx;
            if (coord_maxmin[1][d] > boundary_x[1][d])
                for (int i = svp; i <= evp; ++i)
                    if (par[i].x[d] > boundary_x[1][d]) par[i].x[d] = par[i].x[d] - dx;
        }
    }
}

// =========================================================================
// The loop body (MCM/mcm_solution.f90:37-138)
// =========================================================================

int Sim::step_a(real *critts_out) {
    neighbours();
    strain();
    if (h_opt > 0) update_h();
    int st = constitutive();
    if (critts_out) *critts_out = critts;
    return st;
}

void Sim::dt_update() {
    dtold = dt;
    dt = tssf * critts;
    dt = std::min(dt, 1.1 * dtold);
    ptime = ptime + dt;
}

void Sim::step_b() {
    if (contacttype > 0) rep_cont();   // MCM/mcm_solution.f90:64
    momentum();
    boundcond();
    calctotale();
}

void Sim::step_c() {
    update_velocity();
    move();
    timestep = timestep + 1;
}

bool field_ptr(Particle &P, const std::string &f, real *&ptr, int &n) {
    n = 1;
    if (f == "x") { ptr = P.x; n = 3; }
    else if (f == "xzero") { ptr = P.xzero; n = 3; }
    else if (f == "v") { ptr = P.v; n = 3; }
    else if (f == "a") { ptr = P.a; n = 3; }
    else if (f == "repulsion") { ptr = P.repulsion; n = 3; }
    else if (f == "rod") { ptr = &P.rod[0][0]; n = 9; }
    else if (f == "spin") { ptr = &P.spin[0][0]; n = 9; }
    else if (f == "sigma") { ptr = &P.sigma[0][0]; n = 9; }
    else if (f == "s") { ptr = &P.s[0][0]; n = 9; }
    else if (f == "q") { ptr = &P.q[0][0]; n = 9; }
    else if (f == "qold") { ptr = &P.qold[0][0]; n = 9; }
    else if (f == "alfa") { ptr = &P.alfa[0][0]; n = 9; }
    else if (f == "mass") ptr = &P.mass;
    else if (f == "h") ptr = &P.h;
    else if (f == "hold") ptr = &P.hold;
    else if (f == "h0") ptr = &P.h0;
    else if (f == "rho") ptr = &P.rho;
    else if (f == "rho0") ptr = &P.rho0;
    else if (f == "rhoold") ptr = &P.rhoold;
    else if (f == "p") ptr = &P.p;
    else if (f == "e") ptr = &P.e;
    else if (f == "etry") ptr = &P.etry;
    else if (f == "einc") ptr = &P.einc;
    else if (f == "c") ptr = &P.c;
    else if (f == "vabs") ptr = &P.vabs;
    else if (f == "tracerod") ptr = &P.tracerod;
    else if (f == "pcut") ptr = &P.pcut;
    else if (f == "p_cut") ptr = &P.p_cut;
    else if (f == "efps") ptr = &P.efps;
    else if (f == "fail") ptr = &P.fail;
    else if (f == "mindist") ptr = &P.mindist;
    else if (f == "critts") ptr = &P.critts;
    else if (f == "capa") ptr = &P.capa;
    else return false;
    return true;
}

}  // namespace

// ===================================================================== C API

extern "C" {

void *mcmo_create(const mcmo_deck *deck, const mcmo_material *mats, const double *x, const double *v,
                  const int *mat, const int *dispbc, const double *pardata, int *status) {
    Sim *s = new Sim();
    int st = s->setup(deck, mats, x, v, mat, dispbc, pardata);
    if (st != MCMO_OK) {
        if (status) *status = st;
        delete s;
        return nullptr;
    }
    s->initial();
    if (status) *status = MCMO_OK;
    return s;
}

void mcmo_destroy(void *sim) { delete static_cast<Sim *>(sim); }

int mcmo_step_a(void *sim, double *critts) { return static_cast<Sim *>(sim)->step_a(critts); }
int mcmo_dt_update(void *sim) { static_cast<Sim *>(sim)->dt_update(); return MCMO_OK; }
int mcmo_step_b(void *sim) { static_cast<Sim *>(sim)->step_b(); return MCMO_OK; }
int mcmo_ended(void *sim) { return static_cast<Sim *>(sim)->ended() ? 1 : 0; }
int mcmo_step_c(void *sim) { static_cast<Sim *>(sim)->step_c(); return MCMO_OK; }

int mcmo_run(void *sim, int nsteps, int *done) {
    Sim *s = static_cast<Sim *>(sim);
    int st = MCMO_OK;
    int k = 0;
    for (; k < nsteps; ++k) {
        st = s->step_a(nullptr);
        if (st != MCMO_OK) break;
        s->dt_update();
        s->step_b();
        if (s->ended()) { ++k; break; }
        s->step_c();
    }
    if (done) *done = k;
    return st;
}

int mcmo_get(void *sim, const char *field, double *out) {
    Sim *s = static_cast<Sim *>(sim);
    std::string f(field);
    for (int i = 1; i <= s->np; ++i) {
        real *p; int n;
        if (!field_ptr(s->par[i], f, p, n)) return MCMO_EINVAL;
        if (n == 9) {
            // Fortran (3,3) column-major: element (r,c) at r + 3c
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) out[(size_t)9 * (i - 1) + r + 3 * c] = p[3 * r + c];
        } else {
            for (int k = 0; k < n; ++k) out[(size_t)n * (i - 1) + k] = p[k];
        }
    }
    return MCMO_OK;
}

int mcmo_set(void *sim, const char *field, const double *in) {
    Sim *s = static_cast<Sim *>(sim);
    std::string f(field);
    for (int i = 1; i <= s->np; ++i) {
        real *p; int n;
        if (!field_ptr(s->par[i], f, p, n)) return MCMO_EINVAL;
        if (n == 9) {
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) p[3 * r + c] = in[(size_t)9 * (i - 1) + r + 3 * c];
        } else {
            for (int k = 0; k < n; ++k) p[k] = in[(size_t)n * (i - 1) + k];
        }
    }
    return MCMO_OK;
}

int mcmo_get_int(void *sim, const char *field, int *out) {
    Sim *s = static_cast<Sim *>(sim);
    std::string f(field);
    for (int i = 1; i <= s->np; ++i) {
        const Particle &P = s->par[i];
        int v;
        if (f == "nnbr") v = P.nnbr;
        else if (f == "g_nnbr") v = P.g_nnbr;
        else if (f == "ncont") v = P.ncont;
        else if (f == "g_ncont") v = P.g_ncont;
        else if (f == "mat") v = P.mat;
        else if (f == "dispbc") v = P.dispbc;
        else if (f == "llpointer") v = P.llpointer;
        else if (f == "ptype") v = P.ptype;
        else return MCMO_EINVAL;
        out[i - 1] = v;
    }
    return MCMO_OK;
}

double mcmo_scalar(void *sim, const char *name) {
    Sim *s = static_cast<Sim *>(sim);
    std::string n(name);
    if (n == "dt") return s->dt;
    if (n == "dtold") return s->dtold;
    if (n == "ptime") return s->ptime;
    if (n == "critts") return s->critts;
    if (n == "hmax") return s->hmax;
    if (n == "kinetice") return s->kinetice;
    if (n == "internale") return s->internale;
    if (n == "totale") return s->totale;
    if (n == "ngp") return s->ngp;
    if (n == "maxnbr") return s->maxnbr;
    if (n == "g_maxnbr") return s->g_maxnbr;
    if (n == "timestep") return s->timestep;
    if (n == "tssf") return s->tssf;
    if (n == "pi") return s->pi;
    if (n == "boundary") return s->boundary ? 1 : 0;
    for (int k = 0; k < 6; ++k) {
        static const char *names[6] = {"xmin", "xmax", "ymin", "ymax", "zmin", "zmax"};
        if (n == std::string("bbox_") + names[k]) return s->coord_maxmin[k % 2][k / 2];
    }
    return std::nan("");
}

int mcmo_set_scalar(void *sim, const char *name, double value) {
    Sim *s = static_cast<Sim *>(sim);
    std::string n(name);
    if (n == "dt") s->dt = value;
    else if (n == "dtold") s->dtold = value;
    else if (n == "ptime") s->ptime = value;
    else if (n == "endtime") s->endtime = value;
    else return MCMO_EINVAL;
    return MCMO_OK;
}

int mcmo_nbrlist(void *sim, int i, int *out, int cap) {
    Sim *s = static_cast<Sim *>(sim);
    const Particle &P = s->par[i];
    int n = (int)P.nbr.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = P.nbr[k];
    return n;
}

int mcmo_g_nbrlist(void *sim, int i, int *out, int cap) {
    Sim *s = static_cast<Sim *>(sim);
    const Particle &P = s->par[i];
    int n = (int)P.gnbr.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = P.gnbr[k];
    return n;
}

int mcmo_contlist(void *sim, int i, int *out, int cap) {
    Sim *s = static_cast<Sim *>(sim);
    const Particle &P = s->par[i];
    int n = (int)P.cont.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = P.cont[k];
    return n;
}

int mcmo_g_contlist(void *sim, int i, int *out, int cap) {
    Sim *s = static_cast<Sim *>(sim);
    const Particle &P = s->par[i];
    int n = (int)P.gcont.size();
    for (int k = 0; k < n && k < cap; ++k) out[k] = P.gcont[k];
    return n;
}

int mcmo_contact_forces(void *sim, double *xyz) {
    Sim *s = static_cast<Sim *>(sim);
    for (int m = 1; m <= s->nummat; ++m) {
        xyz[3 * (m - 1) + 0] = s->mat[m].xcf;
        xyz[3 * (m - 1) + 1] = s->mat[m].ycf;
        xyz[3 * (m - 1) + 2] = s->mat[m].zcf;
    }
    return MCMO_OK;
}

int mcmo_ghosts(void *sim, int *par_out, double *x_out, double *v_out, int cap) {
    Sim *s = static_cast<Sim *>(sim);
    for (int g = 1; g <= s->ngp && g <= cap; ++g) {
        if (par_out) par_out[g - 1] = s->gpar[g].par;
        for (int m = 0; m < 3; ++m) {
            if (x_out) x_out[3 * (g - 1) + m] = s->gpar[g].x[m];
            if (v_out) v_out[3 * (g - 1) + m] = s->gpar[g].v[m];
        }
    }
    return s->ngp;
}

int mcmo_grid(void *sim, int *gridlim, double *gridmin, double *gridsize) {
    Sim *s = static_cast<Sim *>(sim);
    for (int k = 0; k < 3; ++k) {
        gridlim[k] = s->gridlim[k];
        gridmin[k] = s->gridmin[k];
        gridsize[k] = s->gridsize[k];
    }
    return MCMO_OK;
}

int mcmo_material_energy(void *sim, double *ke, double *ie, double *mom) {
    Sim *s = static_cast<Sim *>(sim);
    for (int m = 1; m <= s->nummat; ++m) {
        ke[m - 1] = s->mat[m].ke;
        ie[m - 1] = s->mat[m].ie;
        for (int j = 0; j < 3; ++j) mom[3 * (m - 1) + j] = s->mat[m].mom[j];
    }
    return MCMO_OK;
}

int mcmo_material_table(void *sim, int m, double *strinput, double *eosinput, double *g) {
    Sim *s = static_cast<Sim *>(sim);
    if (m < 1 || m > s->nummat) return MCMO_EINVAL;
    for (int k = 0; k < 48; ++k) strinput[k] = s->mat[m].strinput[k];
    for (int k = 0; k < 24; ++k) eosinput[k] = s->mat[m].eosinput[k];
    *g = s->mat[m].g;
    return MCMO_OK;
}

double mcmo_kernel_w(int ndim, const double *xi, const double *xj, double havg) {
    Sim s;
    s.ndim = ndim;
    s.pi = std::acos(-1.0);
    return s.kernel1(xi, xj, havg);
}

void mcmo_gradw(int ndim, const double *xi, const double *xj, double havg, double *dwdx) {
    Sim s;
    s.ndim = ndim;
    s.pi = std::acos(-1.0);
    real dwdr = 0;
    s.grad1(dwdx, dwdr, xi, xj, havg);
}

}  // extern "C"
