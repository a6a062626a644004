// common.cuh -- device data layout shared by the kernels of the MCM step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mcm_gpu.h"

namespace mcm {

constexpr int kMaxMat = MCM_GPU_MAX_MATERIALS;
constexpr int kWarp = 32;
constexpr int kNoCell = -1;

// Material constants on the device (mirrors mcm_gpu_material).
struct DevMaterial {
    int model, eos, visc_type, pad;
    double rho, g, av_l, av_q, mass, h, rho_min, rho_max;
    double strinput[48];
    double eosinput[24];
    double k_cont, n_cont;   // repulsive contact (contacttype > 0)
};

// Scalars of the time loop kept on the device so that whole steps can be
// enqueued (and captured) without host round trips.
struct DevTime {
    double dt, dtold, ptime, endtime;
    double critts;
    int ended;        // MCM/mcm_solution.f90:101 fired
    int steps_done;   // completed loop iterations in the current mcm_gpu_run
};

// First error raised on the device; later kernels of the step return early.
struct DevStatus {
    int code;
    int req_stride;   // neighbour-list entries needed (real part); -1: a row is too long
    int req_gstride;  // neighbour-table width needed (ghost part)
    int req_ngp;      // ghost storage needed
    int req_sstride;  // skin-list entries needed
    int req_cstride;  // contact-list entries needed (real contacts)
    int req_gcstride; // contact-list entries needed (ghost contacts)
    long long req_cells;
    int bad_index;
    int max_nbr, max_gnbr;
    unsigned long long sum_nbr;  // for the mean neighbour count
};

// Linked-list grid of MCM/mcm_setuplist.f90, recomputed every step.
struct DevGrid {
    double gridmin[3];
    double gridsize[3];
    int gridlim[3];
    int pad;
    long long ncells;
    double hcut;      // largest h of the particles in cells (bounds the search reach)
};

// Boundary planes (MCM/mcm_init_boundary.f90:28-116).
struct DevPlanes {
    int code[2][3];
    double bx[2][3];
    int type[3];
    double mult[6][3];
    double add[6][3];
};

// Run options used inside kernels.
struct DevParams {
    int ndim, disctype, tcrit_opt, boundary, baseaccel, drelax, nmat, diag;
    int asym;         // a material of the cap model is present: the momentum sum reads both triangles of sigma
    int h_opt;        // variable smoothing length (MCM/mcm_update_h.f90): 0 fixed, 1 strain rate, 2 density
    int veloc_opt;    // 1: XSPH velocity smoothing (MCM/mcm_update_velocity.f90:61-87)
    int contacttype;  // 0: particles of other materials are neighbours (kernel contact); > 0: contacts
    int contact;      // contacttype > 0 with more than one material: contact lists and repulsion are built
    int kahan;        // mixed precision: pair sums compensated per lane (Kahan) before the lane combination
    int xsort;        // each cell's particles in ascending x (FP64-fast, mixed); else descending reference index
    double drelax_scale, tssf, hmax;
    double skin;      // > 0: neighbour lists filtered from skin lists kept within h_i + h_j + skin * hmax
    double base_a[3];
    DevPlanes planes;
};

// Per-particle field identifiers of the FP64 state (one array of npad
// doubles each).  Symmetric tensors keep 6 components: 11 22 33 12 13 23.
enum Field {
    FX = 0, FY, FZ, FVX, FVY, FVZ, FH, FMASS, FRHO, FE, FP, FC, FEFPS, FPCUT, FPCUT2, FFAIL, FVABS, FHOLD,
    FS11, FS22, FS33, FS12, FS13, FS23,      // sigma
    FQ,                                      // isotropic artificial viscosity
    FD11, FD22, FD33, FD12, FD13, FD23,      // deviator s
    FA11, FA22, FA33, FA12, FA13, FA23,      // back stress alfa (model 3)
    FCAPA,
    // diagnostics refreshed by the split path (and on request)
    FR11, FR22, FR33, FR12, FR13, FR23,      // rod
    FW12, FW13, FW23,                        // spin
    FTR, FETRY, FEINC, FRHOOLD, FMINDIST, FCRITTS, FAX, FAY, FAZ,
    // lower triangle of sigma (21, 31, 32): equal to the upper one except for
    // the cap model, whose return map writes the upper triangle only
    FL21, FL31, FL32,
    FH0,                                     // initial smoothing length (h_opt 2)
    FXS0, FXS1, FXS2,                        // XSPH velocity sums of the step
    FRPX, FRPY, FRPZ,                        // repulsive contact acceleration (contacttype > 0)
    NFIELD
};

struct Fields {
    double *f[NFIELD];
    int *mat, *dispbc, *orig, *ptype;
};

__host__ __device__ inline long long cell_key(int bx, int by, int bz, const int *gl) {
    return (long long)(bx - 1) + (long long)gl[0] * ((long long)(by - 1) + (long long)gl[1] * (long long)(bz - 1));
}

// Lower corner of cell b (1-based) along axis d of the grid.
__host__ __device__ inline double cell_origin(const DevGrid &g, int d, int b) {
    return g.gridmin[d] + (double)(b - 1) * (1.0 / g.gridsize[d]);
}

__device__ __forceinline__ void raise_status(DevStatus *st, int code, int idx = -1) {
    if (atomicCAS(&st->code, 0, code) == 0) st->bad_index = idx;
}

}  // namespace mcm
