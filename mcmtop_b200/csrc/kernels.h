// kernels.h -- launch interface between the C-ABI host code and the kernel
// translation units.  StepArgs carries every device pointer and size a step
// needs; it is passed by value to the kernels.
#pragma once
#include "common.cuh"

namespace mcm {

struct StepArgs {
    int n;            // particles
    int npad;         // column pitch of per-particle arrays (multiple of 32)
    int nmat;
    int nstride;      // neighbour-list capacity per position (entries, multiple of 4)
    int gstride;      // ghost-neighbour table width (int32 entries)
    int ghost_cap;    // ghost storage
    long long cell_cap;   // cell-array storage
    int layer_cap;    // scratch for one boundary layer
    int split_mode;   // 1: step_a/b/c entry points (dt supplied by the host); 0: fused run
    DevParams prm;
    const DevMaterial *mats;
    Fields F;
    DevTime *time;
    DevStatus *status;
    DevGrid *grid;
    double *bbox;     // [2][3]: min, max (mcm_coord_maxmin)
    double *hmax;     // [0]: mcm_hmax, the grid's cell half-size; [1]: bits of the step's new maximum (h_opt > 0)
    // cell list.  "Position" p is a particle's rank in cell order (cells in
    // key order, each cell in descending reference index, particles outside
    // the grid last); cell_list[p] is its state index.
    int *key;         // per state index: cell key or -1
    int *cell_count;  // cell_cap
    int *cell_start;  // cell_cap + 1
    int *cell_list;   // npad: position -> state index
    int *n_inside;    // particles inside the grid (device counter)
    double4 *cpos;    // per position: x, y, z, h at neighbour time
    float4 *cposf;    // per position: x, y, z relative to the cell origin (FP32), h
    float4 *cposg;    // x-ordered steps, per position: x relative to the grid origin, y, z relative to the cell origin (FP32), h
    int *cmat;        // per position: material
    int *ckey;        // per position: cell key or -1
    int *scan_sums;   // block sums of the scan
    int2 *gcell;      // per cell: first ghost index, ghost count
    // ghosts (SoA, ghost_cap each)
    double *gx, *gy, *gz, *gvx, *gvy, *gvz, *gmass, *gh, *ghold, *grho;
    int *gpar, *gmat;
    int *gflip;       // per ghost: bit d set if its position is the parent's mirrored along axis d
    int *ngp;         // device ghost counter
    int *plane_base;  // ghost index base of the plane being built
    int *layer_count, *layer_off;
    // neighbour lists, per position p, in the reference order (same-material
    // neighbours, then contacts; rows in z, y order, cells in x order, each
    // cell in descending reference index): entry k of p at
    // nidx[p*nstride + k] = q | code << 26, q the neighbour's position and
    // code = (dx+1) + 3(dy+1) + 9(dz+1) the offset of its cell from p's.
    // The self entry of disctype 1 is not stored.  Ghost neighbours: int32
    // ghost indices, entry k of p at gnbr[k*npad + p].
    unsigned int *nidx;
    int *gnbr, *nnbr, *gnnbr;
    // contact lists (prm.contact): particles of other materials, entry k of
    // position p at cidx[p*cstride + k] (same encoding as nidx), ghost
    // contacts at gcont[k*npad + p]; counts per position
    unsigned int *cidx;
    int *gcont, *ncont, *gncont;
    int cstride, gcstride;
    // skin lists (prm.skin > 0): per STATE index i, the state indices of the
    // particles within h_i + h_j + skin at the last build, sup[i*sstride + k],
    // supn[i] of them; the positions x at that build (xref, 3 x npad); pos_of[i]
    // the cell-order position of state index i in the current cell list
    int *sup, *supn, *pos_of;
    int sstride;
    double *xref;
    int *skin_flags;                 // [0] force a build, [1] this step builds, [2] builds so far
    unsigned long long *skin_d2;     // bits of the largest squared displacement since the build
    double *reorder_tmp;   // npad doubles of scratch for the state permutation
    double *reorder_grp;   // kReorderGroup x npad doubles: a group of fields permuted at once (reorder_interval > 0)
    // gather records
    double4 *rec0, *rec1, *rec2;   // per particle
    double4 *grec0, *grec1, *grec2;  // per ghost
    double4 *rec3, *grec3;           // prm.asym: the lower triangle of (sigma - q)/rho^2 (21 31 32)
    float4 *frec0;                   // mixed path: 4 npad float4 (strain or momentum records)
    float4 *gfrec1, *gfrec2;         // mixed path, per ghost
    // reductions
    double *red;      // block partials
    int red_blocks;   // capacity of red in blocks (partial vectors)
    // launch shape, chosen by mcm_gpu_set_tuning or mcm_gpu_autotune (0: default)
    int search_threads;   // threads per block of the neighbour search
    int search_kind;      // 0 or 1: one thread per particle (k_search); 2: one warp per particle (k_search_warp);
                          // 3: one warp per cell (k_search_cell)
    int pair_threads;     // threads per block of the cooperative strain and momentum gathers
    int pair_bps;         // blocks per SM the cooperative gathers' persistent grid is sized for (0: resident)
    int pair_kind;        // mixed gathers: 0 or 1 neighbour records through L1; 2 rows staged in shared memory
    double *energy;   // 5*nmat + 3
};

// cells.cu
void launch_grid_setup(const StepArgs &a, cudaStream_t s);
void launch_cell_build(const StepArgs &a, cudaStream_t s);
void launch_ghosts(const StepArgs &a, cudaStream_t s);
void launch_search(const StepArgs &a, cudaStream_t s);
// skin lists: displacement check, conditional skin-list build, per-step filter
void launch_skin_search(const StepArgs &a, cudaStream_t s);
void launch_skin_force(const StepArgs &a, cudaStream_t s);   // the next step rebuilds the skin lists
constexpr int kReorderGroup = 8;   // fields permuted by one kernel
constexpr int kReorderLaunches = (NFIELD + kReorderGroup - 1) / kReorderGroup + 8;
void launch_reorder(const StepArgs &a, cudaStream_t s);

// reduce.cu
void launch_critts_reduce(const StepArgs &a, cudaStream_t s, int nblocks);
void launch_init_critts_reduce(const StepArgs &a, cudaStream_t s, int nblocks);
void launch_energy_bbox_reduce(const StepArgs &a, cudaStream_t s, int nblocks, int energy, int bbox);
void launch_set_time(const StepArgs &a, cudaStream_t s, double dt, double dtold, int set_dtold);
// energy partials of several materials in the rows of the momentum kernel's nblocks blocks
void launch_energy_step_partials(const StepArgs &a, cudaStream_t s, int nblocks);
// per-material sums of mass x repulsion into out[3*nmat] (device memory)
void launch_contact_forces(const StepArgs &a, cudaStream_t s, double *out);
void launch_finish_step(const StepArgs &a, cudaStream_t s);

// step_mixed.cu: FP32 pair sums over FP32 gather records (the constitutive
// update of the mixed path is the FP64 fast one)
namespace mixed {
void launch_strain_prep(const StepArgs &a, cudaStream_t s);
void launch_strain(const StepArgs &a, cudaStream_t s);
void launch_mom_prep(const StepArgs &a, cudaStream_t s);
int launch_momentum(const StepArgs &a, cudaStream_t s, int integrate);
}  // namespace mixed

// adjoint.cu: reverse step of the FP64 step (model 10 + EOS 41, disctype 0)
namespace adj {
constexpr int kParams = 4;   // per material: G, yield stress, hardening modulus, EOS-41 slope s
struct AdjArgs {
    // adjoint of the state (by state index): in = after the step, out = before it
    double *xb[3], *vb[3], *rhob, *eb, *pb, *efpsb, *sigb[6];
    double *ab[3];                                   // acceleration
    double *yrho, *ye, *yp, *yefps, *ysig[6], *yq;   // post-constitutive state
    double *rho0b;       // the step's initial density, through the ghost copies
    double *gb[9];       // velocity gradient G (row n = velocity component, column m = derivative)
    const double *pre[NFIELD];   // the step's initial state (snapshot)
    double *theta_b;     // [nmat][kParams], accumulated
    double4 *rec;        // per cell-order position, kRecSlots double4: what the reverse gathers read of a neighbour
    double dt_prev, dt, dtold;   // dt of the strain/constitutive part, of the update, the one before
    int rev;             // 1: every material is model 10 with EOS 41 (one reverse pass), 0: dual-number passes
};
constexpr int kRecSlots = 5;   // double4 slots per position in AdjArgs::rec
// one reverse step = these three, in this order
void launch_reverse_momentum(const StepArgs &a, const AdjArgs &b, cudaStream_t s);       // move, velocity, momentum
void launch_reverse_constitutive(const StepArgs &a, const AdjArgs &b, cudaStream_t s);   // per-particle update
void launch_reverse_strain(const StepArgs &a, const AdjArgs &b, cudaStream_t s);         // strain rate
}  // namespace adj

// step kernels (one namespace per arithmetic flavour)
#define MCM_DECLARE_STEP(NS)                                                        \
    namespace NS {                                                                  \
    void launch_strain_prep(const StepArgs &a, cudaStream_t s);                     \
    void launch_strain(const StepArgs &a, cudaStream_t s);                          \
    int launch_constitutive(const StepArgs &a, cudaStream_t s);                     \
    void launch_mom_prep(const StepArgs &a, cudaStream_t s);                        \
    void launch_rep_cont(const StepArgs &a, cudaStream_t s);                        \
    int launch_momentum(const StepArgs &a, cudaStream_t s, int integrate);          \
    int launch_update_move(const StepArgs &a, cudaStream_t s);                      \
    int launch_xsph_move(const StepArgs &a, cudaStream_t s);                        \
    int launch_initial(const StepArgs &a, cudaStream_t s, int massopt, int init_h_opt, int init_rhoe, const int *nppermat); \
    int launch_init_critts(const StepArgs &a, cudaStream_t s);                      \
    }
MCM_DECLARE_STEP(exact)
MCM_DECLARE_STEP(fast)
#undef MCM_DECLARE_STEP

// Layout of one particle's record in a host array of the C ABI: entry k of
// the record comes from (goes to) field[k], times sign[k] on download; a
// negative field is zero on download and skipped on upload.
struct PackSpec {
    int width;
    int field[9];
    double sign[9];
};
void launch_unpack(const StepArgs &a, const PackSpec &s, const double *stage, cudaStream_t st);
void launch_pack(const StepArgs &a, const PackSpec &s, double *stage, cudaStream_t st);

constexpr int kRedThreads = 256;

// Blocks of `kernel` resident on one SM at `threads` per block (the
// occupancy calculator's answer, kept per kernel and block size).
int resident_per_sm(const void *kernel, int threads);

// Launch shape of the cooperative gathers: per block, pair_threads / lanes
// particles; the persistent grid covers every particle group once or one
// wave of 148 * pair_bps blocks (pair_bps 0: the blocks of `kernel` resident
// per SM), whichever is fewer, and never more blocks than the partials
// buffer holds.
inline int pair_threads_of(const StepArgs &a) { return a.pair_threads > 0 ? a.pair_threads : 256; }
inline int pair_blocks_of(const StepArgs &a, int lanes, const void *kernel) {
    const int per = pair_threads_of(a) / lanes;
    int b = (a.n + per - 1) / per;
    const int cap = 148 * (a.pair_bps > 0 ? a.pair_bps : resident_per_sm(kernel, pair_threads_of(a)));
    if (b > cap) b = cap;
    if (a.red_blocks > 0 && b > a.red_blocks) b = a.red_blocks;
    return b < 1 ? 1 : b;
}
inline int search_threads_of(const StepArgs &a) { return a.search_threads > 0 ? a.search_threads : 256; }

}  // namespace mcm
