// abi.cu -- host side of the C ABI declared in include/mcm_gpu.h.
//
// A handle owns one CUDA stream and the device state of one body.  Each entry
// point enqueues the kernels of its part of the loop body of
// MCM/mcm_solution.f90 and reads back the device status.  The neighbour table,
// ghost storage and cell arrays are sized on demand: when a kernel reports that
// one is too small, the step is re-run after the storage has been regrown,
// which mirrors the regrow-and-retry of MCM/mcm_ll_neighbours.f90:44,301-309.
// The particle state is untouched by a step that stops at such a check,
// because the search and ghost set-up precede every state update.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handle.h"

#include <map>
#include <mutex>
#include <utility>

using namespace mcm;
using namespace mcm_host;

namespace mcm {
int resident_per_sm(const void *kernel, int threads) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> known;
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(kernel, threads);
    auto it = known.find(key);
    if (it != known.end()) return it->second;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        nb = 1;
    }
    known[key] = nb;
    return nb;
}
}  // namespace mcm

namespace mcm_host {

const char *kRegionName[R_NREG] = {"cell_list", "ghosts", "search", "strain_prep", "strain", "constitutive",
                                   "critts_dt", "momentum_prep", "momentum_integrate", "energy_bbox_reduce",
                                   "update_move", "misc", "adjoint_momentum", "adjoint_constitutive",
                                   "adjoint_strain"};

DevParams make_params(const mcm_gpu_config &c, int nmat) {
    DevParams p;
    std::memset(&p, 0, sizeof(p));
    p.ndim = c.ndim;
    p.disctype = c.disctype;
    p.tcrit_opt = c.tcrit_opt;
    p.boundary = c.boundary;
    p.baseaccel = c.baseaccel;
    p.drelax = c.drelax;
    p.nmat = nmat;
    p.diag = 1;
    p.drelax_scale = c.drelax_scale;
    p.tssf = c.tssf;
    p.hmax = c.hmax;
    p.h_opt = c.h_opt;
    p.contacttype = c.contacttype;
    p.contact = (c.contacttype > 0 && nmat > 1) ? 1 : 0;
    p.skin = c.nbr_skin > 0.0 ? c.nbr_skin : 0.0;
    p.kahan = (c.precision == MCM_PREC_MIXED && c.compensated_sums) ? 1 : 0;
    // the sums of the FP64-fast and mixed steps do not follow the reference's
    // neighbour order: their cells are kept in x order, which lets the search
    // window each row of cells in x
    p.xsort = c.precision != MCM_PREC_FP64_EXACT ? 1 : 0;
    p.veloc_opt = c.veloc_opt;
    for (int k = 0; k < 3; ++k) p.base_a[k] = c.baseaccel ? c.base_a[k] : 0.0;
    DevPlanes &pl = p.planes;
    for (int d = 0; d < 3; ++d) {
        for (int side = 0; side < 2; ++side) {
            int code = c.boundary ? c.boundary_code[2 * d + side] : 0;
            pl.code[side][d] = code;
            pl.bx[side][d] = c.boundary_x[2 * d + side];
        }
        pl.type[d] = 1;
        if (pl.code[0][d] > 0) pl.type[d] += 1;
        if (pl.code[1][d] > 0) pl.type[d] += 2;
    }
    // MCM/mcm_init_boundary.f90:28-116
    for (int d = 0; d < 3; ++d) {
        for (int side = 0; side < 2; ++side) {
            int plane = 2 * d + side;
            for (int k = 0; k < 3; ++k) { pl.mult[plane][k] = 1.0; pl.add[plane][k] = 0.0; }
            int code = pl.code[side][d];
            if (code == 1) {
                pl.mult[plane][d] = -1.0;
                pl.add[plane][d] = 2.0 * pl.bx[side][d];
            } else if (code == 2) {
                double span = pl.bx[1][d] - pl.bx[0][d];
                pl.add[plane][d] = (side == 0) ? -span : span;
            }
        }
    }
    return p;
}

// ------------------------------------------------------------ allocation
int alloc_particles(mcm_gpu_handle *h) {
    const size_t np = h->npad;
    int st;
    if ((st = dalloc(h, &h->d_fields, (size_t)NFIELD * np))) return st;
    CK(cudaMemsetAsync(h->d_fields, 0, sizeof(double) * NFIELD * np, h->stream));
    for (int f = 0; f < NFIELD; ++f) h->A.F.f[f] = h->d_fields + (size_t)f * np;
    if ((st = dalloc(h, &h->d_ints, 4 * np))) return st;
    CK(cudaMemsetAsync(h->d_ints, 0, sizeof(int) * 4 * np, h->stream));
    h->A.F.mat = h->d_ints;
    h->A.F.dispbc = h->d_ints + np;
    h->A.F.orig = h->d_ints + 2 * np;
    h->A.F.ptype = h->d_ints + 3 * np;
    if ((st = dalloc(h, &h->A.key, np))) return st;
    if ((st = dalloc(h, &h->A.cell_list, np))) return st;
    if ((st = dalloc(h, &h->A.cpos, np))) return st;
    if ((st = dalloc(h, &h->A.cposf, np))) return st;
    if (h->A.prm.xsort && (st = dalloc(h, &h->A.cposg, np))) return st;
    if ((st = dalloc(h, &h->A.cmat, np))) return st;
    if ((st = dalloc(h, &h->A.ckey, np))) return st;
    if ((st = dalloc(h, &h->A.reorder_tmp, np))) return st;
    if (h->cfg.reorder_interval > 0 && (st = dalloc(h, &h->A.reorder_grp, (size_t)kReorderGroup * np))) return st;
    if ((st = dalloc(h, &h->A.nnbr, np))) return st;
    if ((st = dalloc(h, &h->A.gnnbr, np))) return st;
    CK(cudaMemsetAsync(h->A.nnbr, 0, sizeof(int) * np, h->stream));
    CK(cudaMemsetAsync(h->A.gnnbr, 0, sizeof(int) * np, h->stream));
    if (h->A.prm.skin > 0.0) {
        if ((st = dalloc(h, &h->A.pos_of, np))) return st;
        if ((st = dalloc(h, &h->A.supn, np))) return st;
        if ((st = dalloc(h, &h->A.xref, 3 * np))) return st;
    }
    if (h->A.prm.contact) {
        if ((st = dalloc(h, &h->A.ncont, np))) return st;
        if ((st = dalloc(h, &h->A.gncont, np))) return st;
        CK(cudaMemsetAsync(h->A.ncont, 0, sizeof(int) * np, h->stream));
        CK(cudaMemsetAsync(h->A.gncont, 0, sizeof(int) * np, h->stream));
    }
    if ((st = dalloc(h, &h->A.rec0, np))) return st;
    if ((st = dalloc(h, &h->A.rec1, np))) return st;
    if ((st = dalloc(h, &h->A.rec2, np))) return st;
    if (h->A.prm.asym && (st = dalloc(h, &h->A.rec3, np))) return st;
    // partial vectors: one per block of the cooperative momentum kernel (at
    // least 16 particles per block of 256 threads, at most 148 x 16 blocks
    // for narrower blocks) or of the per-particle kernels (256 threads)
    h->red_cap = (int)std::max<size_t>((np + 15) / 16, 148 * 16) + 8;
    h->A.red_blocks = h->red_cap;
    if ((st = dalloc(h, &h->A.red, (size_t)h->red_cap * (5 * h->nmat + 6)))) return st;
    if (h->cfg.precision == MCM_PREC_MIXED) {
        // 64 bytes per particle: strain records are 32 bytes at a 2-float4
        // stride; momentum records 32 bytes there plus 16 in the third
        // quarter of the buffer (and the cap model's 16 in the fourth)
        if ((st = dalloc(h, &h->A.frec0, 4 * np))) return st;
    }
    return MCM_OK;
}

int alloc_cells(mcm_gpu_handle *h, long long cap) {
    int st;
    h->A.cell_cap = cap;
    if ((st = dalloc(h, &h->A.cell_count, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.cell_start, (size_t)cap + 1))) return st;
    long long nsum = (cap + 4095) / 4096 + 2;
    if ((st = dalloc(h, &h->A.scan_sums, (size_t)nsum))) return st;
    if ((st = dalloc(h, &h->A.gcell, (size_t)cap))) return st;
    h->A.layer_cap = (int)std::min<long long>(cap, 1LL << 30);
    if ((st = dalloc(h, &h->A.layer_count, (size_t)h->A.layer_cap))) return st;
    if ((st = dalloc(h, &h->A.layer_off, (size_t)h->A.layer_cap))) return st;
    return MCM_OK;
}

int alloc_ghosts(mcm_gpu_handle *h, int cap) {
    int st;
    h->A.ghost_cap = cap;
    double **dd[] = {&h->A.gx, &h->A.gy, &h->A.gz, &h->A.gvx, &h->A.gvy, &h->A.gvz,
                     &h->A.gmass, &h->A.gh, &h->A.ghold, &h->A.grho};
    for (double **p : dd)
        if ((st = dalloc(h, p, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.gpar, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.gmat, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.gflip, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.grec0, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.grec1, (size_t)cap))) return st;
    if ((st = dalloc(h, &h->A.grec2, (size_t)cap))) return st;
    if (h->A.prm.asym && (st = dalloc(h, &h->A.grec3, (size_t)cap))) return st;
    if (h->cfg.precision == MCM_PREC_MIXED) {
        if ((st = dalloc(h, &h->A.gfrec1, (size_t)cap))) return st;
        if ((st = dalloc(h, &h->A.gfrec2, (size_t)cap))) return st;
    }
    return MCM_OK;
}

int alloc_table(mcm_gpu_handle *h, int nstride, int gstride) {
    int st;
    h->A.nstride = round_up(nstride, 4);
    h->A.gstride = gstride;
    if ((st = dalloc(h, &h->A.nidx, (size_t)h->A.nstride * h->npad))) return st;
    if ((st = dalloc(h, &h->A.gnbr, (size_t)gstride * h->npad))) return st;
    return MCM_OK;
}

// Contact lists (contacttype > 0 with several materials): particles of other
// materials within reach, the lists mcm_rep_cont reads.
int alloc_contacts(mcm_gpu_handle *h, int cstride, int gcstride) {
    int st;
    h->A.cstride = round_up(cstride, 4);
    h->A.gcstride = gcstride;
    if ((st = dalloc(h, &h->A.cidx, (size_t)h->A.cstride * h->npad))) return st;
    if ((st = dalloc(h, &h->A.gcont, (size_t)gcstride * h->npad))) return st;
    return MCM_OK;
}

// Skin lists (nbr_skin > 0): sstride entries per particle; a new table holds
// no lists, so the next step builds them.
int alloc_skin(mcm_gpu_handle *h, int sstride) {
    int st;
    h->A.sstride = round_up(sstride, 4);
    if ((st = dalloc(h, &h->A.sup, (size_t)h->A.sstride * h->npad))) return st;
    launch_skin_force(h->A, h->stream);
    CK(cudaGetLastError());
    return MCM_OK;
}

// A copy ordered on the handle's stream and complete on return.  A plain
// cudaMemcpy runs on the legacy default stream, which does not order against
// the handle's non-blocking stream: kernels enqueued after it could read the
// destination before a host-to-device copy of pageable memory has landed,
// and a device-to-host copy could read results not yet written.
cudaError_t scopy(mcm_gpu_handle *h, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    return e;
}

int reset_status(mcm_gpu_handle *h) {
    CK(cudaMemsetAsync(h->A.status, 0, sizeof(DevStatus), h->stream));
    return MCM_OK;
}

int sync_status(mcm_gpu_handle *h) {
    CK(cudaMemcpyAsync(h->h_status, h->A.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->h_time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaGetLastError());
    return MCM_OK;
}

// Regrows whatever the last status asked for.  Returns 1 if something grew.
int regrow(mcm_gpu_handle *h, int *grew) {
    *grew = 0;
    const DevStatus &s = *h->h_status;
    int st;
    switch (s.code) {
        case MCM_ENBR_OVERFLOW: {
            int ns = h->A.nstride, ng = h->A.gstride;
            if (s.req_stride > ns || s.req_gstride > ng) {
                if (s.req_stride > ns) ns = s.req_stride + s.req_stride / 8 + 8;
                if (s.req_gstride > ng) ng = round_up(s.req_gstride + s.req_gstride / 8 + 8, 8);
                if ((st = alloc_table(h, ns, ng))) return st;
                *grew = 1;
            }
            if (h->A.prm.skin > 0.0 && s.req_sstride > h->A.sstride) {
                if ((st = alloc_skin(h, s.req_sstride + s.req_sstride / 8 + 8))) return st;
                *grew = 1;
            }
            int cs = h->A.cstride, gcs = h->A.gcstride;
            if (h->A.prm.contact && (s.req_cstride > cs || s.req_gcstride > gcs)) {
                if (s.req_cstride > cs) cs = s.req_cstride + s.req_cstride / 8 + 8;
                if (s.req_gcstride > gcs) gcs = round_up(s.req_gcstride + s.req_gcstride / 8 + 8, 8);
                if ((st = alloc_contacts(h, cs, gcs))) return st;
                *grew = 1;
            }
            break;
        }
        case MCM_EGHOST_OVERFLOW: {
            int cap = std::max(s.req_ngp + s.req_ngp / 4 + 1024, h->A.ghost_cap * 2);
            if ((st = alloc_ghosts(h, cap))) return st;
            *grew = 1;
            break;
        }
        case MCM_EGRID_OVERFLOW: {
            long long need = std::max<long long>(s.req_cells, h->A.cell_cap * 2);
            long long cap = need + need / 2 + 1024;
            if ((st = alloc_cells(h, cap))) return st;
            *grew = 1;
            break;
        }
        default: break;
    }
    return MCM_OK;
}

// ---------------------------------------------------------------- dispatch
int launch_strain(mcm_gpu_handle *h) {
    const int prec = h->cfg.precision;
    {
        Scope sc(h, R_STRAIN_PREP, 1);
        if (prec == MCM_PREC_FP64_EXACT) exact::launch_strain_prep(h->A, h->stream);
        else if (prec == MCM_PREC_MIXED) mixed::launch_strain_prep(h->A, h->stream);
        else fast::launch_strain_prep(h->A, h->stream);
    }
    {
        Scope sc(h, R_STRAIN, 1);
        if (prec == MCM_PREC_FP64_EXACT) exact::launch_strain(h->A, h->stream);
        else if (prec == MCM_PREC_MIXED) mixed::launch_strain(h->A, h->stream);
        else fast::launch_strain(h->A, h->stream);
    }
    Scope sc(h, R_CONST, 1);
    switch (prec) {
        case MCM_PREC_FP64_EXACT: return exact::launch_constitutive(h->A, h->stream);
        default: return fast::launch_constitutive(h->A, h->stream);
    }
}
int launch_mom(mcm_gpu_handle *h, int integrate) {
    const int prec = h->cfg.precision;
    if (h->A.prm.contact) {
        // MCM/mcm_solution.f90:64: repulsive contact before the momentum sum
        Scope sc(h, R_MOM_PREP, 1);
        if (prec == MCM_PREC_FP64_EXACT) exact::launch_rep_cont(h->A, h->stream);
        else fast::launch_rep_cont(h->A, h->stream);
    }
    {
        Scope sc(h, R_MOM_PREP, 1);
        if (prec == MCM_PREC_FP64_EXACT) exact::launch_mom_prep(h->A, h->stream);
        else if (prec == MCM_PREC_MIXED) mixed::launch_mom_prep(h->A, h->stream);
        else fast::launch_mom_prep(h->A, h->stream);
    }
    // the cooperative gathers of several materials add a fixed-order energy-partials kernel
    Scope sc(h, R_MOMENTUM, (prec != MCM_PREC_FP64_EXACT && h->nmat > 1) ? 2 : 1);
    switch (prec) {
        case MCM_PREC_FP64_EXACT: return exact::launch_momentum(h->A, h->stream, integrate);
        case MCM_PREC_MIXED: return mixed::launch_momentum(h->A, h->stream, integrate);
        default: return fast::launch_momentum(h->A, h->stream, integrate);
    }
}
int launch_move(mcm_gpu_handle *h) {
    if (h->A.prm.veloc_opt) {
        Scope sc(h, R_MOVE, 3);
        if (h->cfg.precision == MCM_PREC_FP64_EXACT) return exact::launch_xsph_move(h->A, h->stream);
        return fast::launch_xsph_move(h->A, h->stream);
    }
    Scope sc(h, R_MOVE, 1);
    switch (h->cfg.precision) {
        case MCM_PREC_FP64_EXACT: return exact::launch_update_move(h->A, h->stream);
        default: return fast::launch_update_move(h->A, h->stream);
    }
}

int active_planes(const mcm_gpu_handle *h) {
    int n = 0;
    for (int p = 0; p < 6; ++p) {
        int c = h->A.prm.planes.code[p & 1][p >> 1];
        if ((c == 1 || c == 2) && (p >> 1) < h->A.prm.ndim) ++n;
    }
    return n;
}

// neighbours -> strain -> constitutive -> critts (MCM/mcm_solution.f90:41-53)
void enqueue_part_a(mcm_gpu_handle *h) {
    StepArgs &a = h->A;
    const int every = h->cfg.reorder_interval;
    if (every > 0 && h->have_cells && (h->steps_enqueued % every) == 0) {
        Scope sc(h, R_MISC, kReorderLaunches + (a.prm.skin > 0.0 ? 1 : 0));
        launch_reorder(a, h->stream);
        // the skin lists hold state indices, which the re-sort permutes
        if (a.prm.skin > 0.0) launch_skin_force(a, h->stream);
    }
    ++h->steps_enqueued;
    h->have_cells = true;
    {
        Scope sc(h, R_CELLS, 8);
        launch_grid_setup(a, h->stream);
        launch_cell_build(a, h->stream);
    }
    if (a.prm.boundary) {
        Scope sc(h, R_GHOSTS, 3 * active_planes(h));
        launch_ghosts(a, h->stream);
    }
    if (a.prm.skin > 0.0) {
        Scope sc(h, R_SEARCH, 4);
        launch_skin_search(a, h->stream);
    } else {
        Scope sc(h, R_SEARCH, 1);
        launch_search(a, h->stream);
    }
    int nb = launch_strain(h);
    Scope sc(h, R_CRITTS, 1);
    launch_critts_reduce(a, h->stream, nb);
}

// momentum -> boundcond -> calctotale (-> update_velocity -> move)
void enqueue_part_b(mcm_gpu_handle *h, int integrate) {
    if (h->A.prm.veloc_opt && integrate) {
        // XSPH needs every updated velocity before any particle moves
        int nb = launch_mom(h, 0);
        {
            Scope sc(h, R_REDUCE, 2);
            launch_energy_bbox_reduce(h->A, h->stream, nb, 1, 0);
        }
        nb = launch_move(h);
        Scope sc(h, R_REDUCE, 1);
        launch_energy_bbox_reduce(h->A, h->stream, nb, 0, 1);
        return;
    }
    int nb = launch_mom(h, integrate);
    Scope sc(h, R_REDUCE, 2);
    launch_energy_bbox_reduce(h->A, h->stream, nb, 1, integrate);
}

int check_handle(mcm_gpu_handle *h) {
    if (!h) return MCM_EINVAL;
    if (!h->initialised) return set_error(h, MCM_EINVAL, "state not uploaded");
    CK(cudaSetDevice(h->device));
    return MCM_OK;
}

// ------------------------------------------------------------- transfers
// Fortran (3,np) vector -> three device arrays
// Host arrays cross PCIe as one contiguous copy each, into a device staging
// buffer (9 doubles per particle, allocated on first use), and kernels
// convert between the Fortran record layout and the per-field arrays.
PackSpec spec_none(int width) {
    PackSpec s;
    s.width = width;
    for (int k = 0; k < 9; ++k) { s.field[k] = -1; s.sign[k] = 1.0; }
    return s;
}
// Fortran (3,np) vector
PackSpec spec_vec3(int f0) {
    PackSpec s = spec_none(3);
    for (int k = 0; k < 3; ++k) s.field[k] = f0 + k;
    return s;
}
// entry (r, c) of a Fortran (3,3) record is r + 3c; a symmetric tensor keeps
// 11 22 33 12 13 23 in fields f0..f0+5
constexpr int kSymIdx[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
PackSpec spec_sym(int f0, bool both) {
    PackSpec s = spec_none(9);
    for (int t = 0; t < 6; ++t) {
        s.field[kSymIdx[t][0] + 3 * kSymIdx[t][1]] = f0 + t;
        if (both) s.field[kSymIdx[t][1] + 3 * kSymIdx[t][0]] = f0 + t;
    }
    return s;
}
// sigma: upper triangle from 11..23, lower triangle (21, 31, 32) from its own fields
PackSpec spec_sigma() {
    PackSpec s = spec_sym(FS11, false);
    s.field[1] = FL21; s.field[2] = FL31; s.field[5] = FL32;
    return s;
}
PackSpec spec_spin() {
    PackSpec s = spec_none(9);
    const int fl[3] = {FW12, FW13, FW23};
    const int rc[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int t = 0; t < 3; ++t) {
        s.field[rc[t][0] + 3 * rc[t][1]] = fl[t];
        s.field[rc[t][1] + 3 * rc[t][0]] = fl[t];
        s.sign[rc[t][1] + 3 * rc[t][0]] = -1.0;
    }
    return s;
}
PackSpec spec_iso(int f, bool full) {   // q: the isotropic value on the diagonal
    PackSpec s = spec_none(9);
    s.field[0] = f;
    if (full) { s.field[4] = f; s.field[8] = f; }
    return s;
}

int stage_ready(mcm_gpu_handle *h) {
    if (h->d_stage) return MCM_OK;
    return dalloc(h, &h->d_stage, 9 * (size_t)h->npad);
}

int put_rec(mcm_gpu_handle *h, const double *src, const PackSpec &s) {
    int st;
    if ((st = stage_ready(h))) return st;
    CK(cudaMemcpyAsync(h->d_stage, src, sizeof(double) * s.width * (size_t)h->np, cudaMemcpyHostToDevice,
                       h->stream));
    launch_unpack(h->A, s, h->d_stage, h->stream);
    CK(cudaGetLastError());
    return MCM_OK;
}

int get_rec(mcm_gpu_handle *h, double *dst, const PackSpec &s) {
    int st;
    if ((st = stage_ready(h))) return st;
    launch_pack(h->A, s, h->d_stage, h->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, h->d_stage, sizeof(double) * s.width * (size_t)h->np, cudaMemcpyDeviceToHost,
                       h->stream));
    return MCM_OK;
}

int put_vec3(mcm_gpu_handle *h, const double *src, int f0) { return put_rec(h, src, spec_vec3(f0)); }

int put_scalar(mcm_gpu_handle *h, const double *src, int f) {
    CK(cudaMemcpyAsync(h->A.F.f[f], src, sizeof(double) * h->np, cudaMemcpyHostToDevice, h->stream));
    return MCM_OK;
}


}  // namespace

// ====================================================================== ABI
extern "C" {

int mcm_gpu_abi_version(void) { return MCM_GPU_ABI_VERSION; }

int mcm_gpu_set_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return MCM_ECUDA;
    if (device < 0 || device >= n) return MCM_EINVAL;
    return cudaSetDevice(device) == cudaSuccess ? MCM_OK : MCM_ECUDA;
}

const char *mcm_gpu_strerror(int status) {
    switch (status) {
        case MCM_OK: return "ok";
        case MCM_ENBR_OVERFLOW: return "neighbour table overflow";
        case MCM_EGHOST_OVERFLOW: return "ghost storage overflow";
        case MCM_ECOMPLEX_C: return "complex speed of sound (eos41 c^2 < 0)";
        case MCM_ECAP_NOCONV: return "cap model iteration did not converge";
        case MCM_ETIMEOUT: return "bounded device wait timed out";
        case MCM_ECUDA: return "CUDA runtime error";
        case MCM_ENOMEM: return "device allocation failed";
        case MCM_EINVAL: return "invalid argument";
        case MCM_EUNSUPPORTED: return "option not supported by the GPU step";
        case MCM_EGRID_OVERFLOW: return "cell grid storage overflow";
        case MCM_EGHOST_LAYER: return "real particle in a ghost-layer cell";
        case MCM_EGRID_TOO_LARGE: return "linked-list grid too large";
    }
    return "unknown status";
}

const char *mcm_gpu_last_error(mcm_gpu_handle *h) { return h ? h->last_error.c_str() : "no handle"; }

// MCM/mcm_matin.f90:46-56, MCM/mcm_sets1.f90:23-51, mcm_sets3.f90:25-43,
// mcm_sets10.f90:23-36, MCM/mcm_calcg.f90:31-59.
int mcm_gpu_material_from_deck(mcm_gpu_material *m) {
    if (!m) return MCM_EINVAL;
    if (m->visc_type == 0) m->visc_type = 1;
    if (m->av_l == 0.0) m->av_l = 0.06;
    if (m->av_q == 0.0) m->av_q = 1.5;
    if (m->rho_min == 0.0) m->rho_min = 1.0E-10;
    if (m->rho_max == 0.0) m->rho_max = 1.0E+10;
    double *cm = m->strinput;
    auto C = [cm](int i, int j) -> double & { return cm[(i - 1) + 5 * (j - 1)]; };
    switch (m->model) {
        case 1: {
            double p6 = C(2, 1), p7 = C(3, 1);
            for (int i = 2; i <= 5; ++i)
                for (int j = 1; j <= 5; ++j) C(i, j) = 0.0;
            double q1 = C(1, 1) * C(1, 2) / ((1.0 + C(1, 2)) * (1.0 - 2.0 * C(1, 2)));
            double q2 = C(1, 1) * 0.5 / (1.0 + C(1, 2));
            double q3 = q1 + 2.0 * q2;
            C(2, 1) = q3; C(3, 2) = q3; C(4, 3) = q3; C(5, 4) = q2;
            C(2, 2) = q1; C(2, 3) = q1; C(3, 1) = q1; C(3, 3) = q1; C(4, 1) = q1; C(4, 2) = q1;
            C(2, 6) = C(1, 6);
            C(1, 6) = C(1, 1) * C(1, 4) / (C(1, 1) - C(1, 4));
            C(1, 7) = p6;
            C(2, 7) = p7;
            if (m->eos != 0) return MCM_EINVAL;
            m->g = cm[0] / (2.0 * (1.0 + cm[5]));
            break;
        }
        case 3: {
            double p7 = C(2, 6);
            for (int i = 2; i <= 5; ++i)
                for (int j = 1; j <= 6; ++j) C(i, j) = 0.0;
            double q1 = C(1, 1) * C(1, 2) / ((1.0 + C(1, 2)) * (1.0 - 2.0 * C(1, 2)));
            double q2 = C(1, 1) * 0.5 / (1.0 + C(1, 2));
            double q3 = q1 + 2.0 * q2;
            C(2, 1) = q3;
            C(5, 4) = q2;
            C(2, 4) = C(1, 1) * C(1, 4) / (C(1, 1) - C(1, 4));
            C(2, 6) = p7;
            if (m->eos != 0) return MCM_EINVAL;
            m->g = cm[0] / (2.0 * (1.0 + cm[5]));
            break;
        }
        case 9:
            m->g = 0.0;
            if (!(m->eos == 1 || m->eos == 4 || m->eos == 13 || m->eos == 28 || m->eos == 41)) return MCM_EINVAL;
            break;
        case 10: {
            double prop[48];
            for (int i = 0; i < 48; ++i) prop[i] = cm[i];
            if (prop[3] == 0.0) prop[3] = (double)-1.e30f;
            if (prop[6] == 0.0) prop[6] = (double)1.000000001f;
            for (int i = 0; i < 48; ++i) cm[i] = prop[i];
            for (int i = 2; i <= 16; ++i)
                if (prop[i + 14] < prop[i + 15]) cm[15] = (double)i;
            m->g = cm[0];
            if (!(m->eos == 1 || m->eos == 4 || m->eos == 13 || m->eos == 28 || m->eos == 41)) return MCM_EINVAL;
            break;
        }
        case 4: {
            // MCM/mcm_sets4.f90:21-41: the elastic modulus cm(5,2) = lambda + 2 mu
            // from K and G, then initel (:43-98, implicit double precision,
            // single-precision literals kept): the initial cap kappa0 with
            // X0 = kappa0 + R Fe(kappa0), X0 = cm(2,5), and the tension cut-off
            // Fe(fcut) = 0, by Newton iterations to an absolute/relative
            // tolerance of 1e-3.  The reference only prints a warning past 200
            // iterations and keeps going; here a material that needs more
            // than 100000 is rejected.
            if (m->eos != 0) return MCM_EINVAL;
            const double alpha = C(1, 3), theta = C(1, 4), gama = C(1, 5), beta = C(1, 6), r = C(2, 1);
            const double xint = C(2, 5);
            const double tempE = (9.0 * C(1, 1) * C(1, 2)) / (3.0 * C(1, 1) + C(1, 2));
            const double tempNi = (3.0 * C(1, 1) - tempE) / (6.0 * C(1, 1));
            const double q1 = tempE * tempNi / ((1.0 + tempNi) * (1.0 - 2.0 * tempNi));
            const double q2 = tempE * 0.5 / (1.0 + tempNi);
            C(5, 2) = q1 + 2.0 * q2;
            const double tol = (double)1.0e-3f, tiny = (double)1.e-15f;
            double capint = 0.0, delcap = (double)1.e10f, delf = (double)1.e10f, fcut = 0.0;
            for (int it = 0;; ++it) {
                const double fe = alpha - gama * std::exp(-beta * capint) + theta * capint;
                const double psik = xint - capint - r * fe;
                if (!((std::fabs(psik) > tol) && (std::fabs(delcap) / (std::fabs(capint) + tiny) > tol))) break;
                if (it > 100000) return MCM_EINVAL;
                const double fep = beta * gama * std::exp(-beta * capint) + theta;
                delcap = psik / (-1.0 - r * fep);
                capint = capint - delcap;
            }
            for (int it = 0;; ++it) {
                const double fe = alpha - gama * std::exp(-beta * fcut) + theta * fcut;
                if (!((std::fabs(fe) > tol) && (std::fabs(delf) / (std::fabs(fcut) + tiny) > tol))) break;
                if (it > 100000) return MCM_EINVAL;
                const double fep = gama * beta * std::exp(-beta * fcut) + theta;
                delf = fe / fep;
                fcut = fcut - delf;
            }
            C(3, 3) = capint;
            C(3, 4) = fcut;
            const int ltype = (int)C(2, 6);
            if (ltype != 1 && ltype != 2) return MCM_EINVAL;   // the mode table of f3dm25 covers soil and rock
            m->g = cm[5];   // MCM/mcm_calcg.f90:43-45: cm(1,2), the shear modulus
            break;
        }
        default:
            return MCM_EINVAL;
    }
    return MCM_OK;
}

int mcm_gpu_create(const mcm_gpu_config *cfg, const mcm_gpu_material *mats, int nmat, int np,
                   mcm_gpu_handle **out) {
    if (!cfg || !mats || !out || np <= 0 || nmat <= 0 || nmat > MCM_GPU_MAX_MATERIALS) return MCM_EINVAL;
    *out = nullptr;
    if (cfg->ndim != 3) return MCM_EUNSUPPORTED;
    if (cfg->contacttype < 0) return MCM_EINVAL;
    if (!(cfg->nbr_skin >= 0.0)) return MCM_EINVAL;
    // skin lists: the reference's neighbour order is not kept, and the skin
    // bound assumes smoothing lengths that do not change between builds
    if (cfg->nbr_skin > 0.0 && (cfg->precision == MCM_PREC_FP64_EXACT || cfg->h_opt != 0)) return MCM_EUNSUPPORTED;
    if (cfg->h_opt < 0 || cfg->h_opt > 2 || cfg->veloc_opt < 0 || cfg->veloc_opt > 1) return MCM_EINVAL;
    if (cfg->krtype != 0 && cfg->krtype != 1) return MCM_EUNSUPPORTED;
    if (cfg->disctype != 0 && cfg->disctype != 1) return MCM_EINVAL;
    if (cfg->tcrit_opt < 0 || cfg->tcrit_opt > 2) return MCM_EINVAL;
    if (cfg->precision < 0 || cfg->precision > 2) return MCM_EINVAL;
    bool cap_model = false;
    for (int m = 0; m < nmat; ++m) {
        int md = mats[m].model;
        if (md != 1 && md != 3 && md != 4 && md != 9 && md != 10) return MCM_EINVAL;
        cap_model = cap_model || md == 4;
    }
    // the cap model leaves sigma asymmetric: the simple-SPH momentum sums of
    // every precision read both triangles; the corrected-SPH sum carries 6 components
    if (cap_model && cfg->disctype != 0) return MCM_EUNSUPPORTED;
    if (cfg->boundary) {
        for (int d = 0; d < 3; ++d) {
            bool p0 = cfg->boundary_code[2 * d] == 2, p1 = cfg->boundary_code[2 * d + 1] == 2;
            if (p0 != p1) return MCM_EINVAL;   // MCM/mcm_inp_symmetry_v2.f90:89-109
        }
    }
    // mixed path: simple SPH sums only; gather entries carry 26-bit positions
    // neighbour-list entries carry 26-bit positions; the mixed path has simple SPH sums only
    if (np >= (1 << 26)) return MCM_EUNSUPPORTED;
    if (cfg->precision == MCM_PREC_MIXED && cfg->disctype != 0) return MCM_EUNSUPPORTED;
    mcm_gpu_handle *h = new mcm_gpu_handle();
    h->cfg = *cfg;
    if (h->cfg.tssf == 0.0) h->cfg.tssf = 0.8;   // MCM/mcm_control_v2.f90:193
    h->np = np;
    h->npad = round_up(np, 32);
    h->nmat = nmat;
    h->mats.assign(mats, mats + nmat);
    cudaError_t e = cudaGetDevice(&h->device);
    if (e != cudaSuccess) { delete h; return MCM_ECUDA; }
    int st = MCM_OK;
#define TRY(x) do { st = (x); if (st) { mcm_gpu_destroy(h); return st; } } while (0)
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return MCM_ECUDA; }
    std::memset(&h->A, 0, sizeof(h->A));
    h->A.n = np;
    h->A.npad = h->npad;
    h->A.nmat = nmat;
    h->A.split_mode = 1;
    h->A.prm = make_params(h->cfg, nmat);
    h->A.prm.asym = cap_model ? 1 : 0;
    // materials
    std::vector<DevMaterial> dm(nmat);
    for (int m = 0; m < nmat; ++m) {
        DevMaterial &d = dm[m];
        std::memset(&d, 0, sizeof(d));
        d.model = mats[m].model; d.eos = mats[m].eos; d.visc_type = mats[m].visc_type;
        d.rho = mats[m].rho; d.g = mats[m].g; d.av_l = mats[m].av_l; d.av_q = mats[m].av_q;
        d.mass = mats[m].mass; d.h = mats[m].h; d.rho_min = mats[m].rho_min; d.rho_max = mats[m].rho_max;
        d.k_cont = mats[m].k_cont; d.n_cont = mats[m].n_cont;
        std::memcpy(d.strinput, mats[m].strinput, sizeof(d.strinput));
        std::memcpy(d.eosinput, mats[m].eosinput, sizeof(d.eosinput));
    }
    TRY(dalloc(h, &h->d_mats, (size_t)nmat));
    if (scopy(h, h->d_mats, dm.data(), sizeof(DevMaterial) * nmat, cudaMemcpyHostToDevice) != cudaSuccess) {
        mcm_gpu_destroy(h);
        return MCM_ECUDA;
    }
    h->A.mats = h->d_mats;
    // scalars
    size_t scal = sizeof(DevTime) + sizeof(DevStatus) + sizeof(DevGrid) + 64 + sizeof(double) * (5 * nmat + 8) + 64;
    if (cudaMalloc(&h->d_scalars, 4096 + scal) != cudaSuccess) { mcm_gpu_destroy(h); return MCM_ENOMEM; }
    if (cudaMemsetAsync(h->d_scalars, 0, 4096 + scal, h->stream) != cudaSuccess) { mcm_gpu_destroy(h); return MCM_ECUDA; }
    char *p = (char *)h->d_scalars;
    h->A.time = (DevTime *)p; p += 256;
    h->A.status = (DevStatus *)p; p += 256;
    h->A.grid = (DevGrid *)p; p += 256;
    h->A.bbox = (double *)p; p += 256;
    h->A.ngp = (int *)p; p += 64;
    h->A.plane_base = (int *)p; p += 32;
    h->A.n_inside = (int *)p; p += 32;
    h->A.hmax = (double *)p; p += 32;
    h->A.skin_d2 = (unsigned long long *)p; p += 32;
    h->A.skin_flags = (int *)p; p += 32;
    h->A.energy = (double *)p;
    cudaMallocHost((void **)&h->h_time, 4096);
    char *q = (char *)h->h_time;
    h->h_status = (DevStatus *)(q + 256);
    h->h_grid = (DevGrid *)(q + 512);
    h->h_bbox = (double *)(q + 768);
    h->h_ngp = (int *)(q + 1024);
    h->h_energy = (double *)(q + 1088);
    TRY(alloc_particles(h));
    int entries = cfg->nbr_stride > 0 ? cfg->nbr_stride : 100;
    TRY(alloc_table(h, entries, cfg->boundary ? 48 : 8));
    if (h->A.prm.contact) TRY(alloc_contacts(h, 16, 8));
    if (h->A.prm.skin > 0.0) TRY(alloc_skin(h, entries + entries / 2));
    TRY(alloc_cells(h, 1 << 16));
    TRY(alloc_ghosts(h, cfg->boundary ? std::max(4096, np / 8) : 32));
    TRY(dalloc(h, &h->d_nppermat, (size_t)nmat));
#undef TRY
    *out = h;
    return MCM_OK;
}

int mcm_gpu_destroy(mcm_gpu_handle *h) {
    if (!h) return MCM_EINVAL;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void *ptrs[] = {h->d_fields, h->d_stage, h->A.frec0, h->A.gfrec1, h->A.gfrec2,
                    h->d_ints, h->d_mats, h->d_scalars, h->d_nppermat,
                    h->A.key, h->A.cell_list, h->A.nnbr, h->A.gnnbr, h->A.rec0, h->A.rec1, h->A.rec2,
                    h->A.cpos, h->A.cposf, h->A.cposg, h->A.cmat, h->A.ckey, h->A.reorder_tmp, h->A.reorder_grp, h->A.nidx,
                    h->A.red, h->A.cell_count, h->A.cell_start, h->A.scan_sums, h->A.gcell,
                    h->A.layer_count, h->A.layer_off, h->A.gx, h->A.gy, h->A.gz, h->A.gvx, h->A.gvy,
                    h->A.gvz, h->A.gmass, h->A.gh, h->A.ghold, h->A.grho, h->A.gpar, h->A.gmat, h->A.gflip,
                    h->A.grec0, h->A.grec1, h->A.grec2, h->A.gnbr, h->A.rec3, h->A.grec3,
                    h->A.cidx, h->A.gcont, h->A.ncont, h->A.gncont,
                    h->A.sup, h->A.supn, h->A.pos_of, h->A.xref};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (double *p : h->adj_ckpt)
        if (p) cudaFree(p);
    if (h->adj_seg) cudaFree(h->adj_seg);
    for (auto &r : h->adj_rec)
        if (r.buf) cudaFree(r.buf);
    if (h->adj_final) cudaFree(h->adj_final);
    if (h->d_adj) cudaFree(h->d_adj);
    if (h->d_theta) cudaFree(h->d_theta);
    if (h->h_time) cudaFreeHost(h->h_time);
    for (auto &v : h->prof_pairs)
        for (auto &pr : v) { h->ev_pool.push_back(pr.first); h->ev_pool.push_back(pr.second); }
    for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : h->timer)
        if (e) cudaEventDestroy(e);
    if (h->part_a_done) cudaEventDestroy(h->part_a_done);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MCM_OK;
}

}  // extern "C"

namespace mcm_host {

// bbox from x (MCM/mcm_initvbls.f90:81-91) when none is supplied
__global__ void k_bbox_partials(StepArgs a) {
    __shared__ double sm[2][32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nv = 5 * a.nmat + 6;
    double *out = a.red + (size_t)blockIdx.x * nv;
    for (int d = 0; d < 3; ++d) {
        double lo = 1.0e20, hi = -1.0e20;
        if (i < a.n) { lo = a.F.f[FX + d][i]; hi = lo; }
        for (int o = 16; o > 0; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        __syncthreads();
        if (lane == 0) { sm[0][w] = lo; sm[1][w] = hi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { lo = fmin(lo, sm[0][k]); hi = fmax(hi, sm[1][k]); }
            out[5 * a.nmat + d] = lo;
            out[5 * a.nmat + 3 + d] = hi;
        }
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 5 * a.nmat; ++v) out[v] = 0.0;
}

__global__ void k_energy_partials(StepArgs a) {
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nv = 5 * a.nmat + 6;
    double *out = a.red + (size_t)blockIdx.x * nv;
    int mati = 0;
    double vals[5] = {0, 0, 0, 0, 0};
    if (i < a.n) {
        mati = a.F.mat[i];
        double mass = a.F.f[FMASS][i], vabs = a.F.f[FVABS][i];
        vals[0] = 0.5 * mass * (vabs * vabs);
        vals[1] = a.F.f[FE][i];
        vals[2] = mass * fabs(a.F.f[FVX][i]);
        vals[3] = mass * fabs(a.F.f[FVY][i]);
        vals[4] = mass * fabs(a.F.f[FVZ][i]);
    }
    for (int m = 1; m <= a.nmat; ++m) {
        for (int v = 0; v < 5; ++v) {
            double x = (mati == m) ? vals[v] : 0.0;
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
            __syncthreads();
            if (lane == 0) sm[w] = x;
            __syncthreads();
            if (threadIdx.x == 0) {
                double r = 0.0;
                for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sm[k];
                out[5 * (m - 1) + v] = r;
            }
        }
    }
}

__global__ void k_iota(int *p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = i;
}

int compute_bbox(mcm_gpu_handle *h) {
    int nb = (h->np + kRedThreads - 1) / kRedThreads;
    k_bbox_partials<<<nb, kRedThreads, 0, h->stream>>>(h->A);
    launch_energy_bbox_reduce(h->A, h->stream, nb, 0, 1);
    CK(cudaGetLastError());
    return MCM_OK;
}

int compute_energy(mcm_gpu_handle *h) {
    int nb = (h->np + kRedThreads - 1) / kRedThreads;
    k_energy_partials<<<nb, kRedThreads, 0, h->stream>>>(h->A);
    launch_energy_bbox_reduce(h->A, h->stream, nb, 1, 0);
    CK(cudaGetLastError());
    return MCM_OK;
}

// Runs the neighbour search alone (mcm_init_neighb), regrowing storage.
int run_search_only(mcm_gpu_handle *h) {
    for (int attempt = 0; attempt < 8; ++attempt) {
        int st;
        if ((st = reset_status(h))) return st;
        StepArgs &a = h->A;
        launch_grid_setup(a, h->stream);
        launch_cell_build(a, h->stream);
        if (a.prm.boundary) launch_ghosts(a, h->stream);
        launch_search(a, h->stream);
        if ((st = sync_status(h))) return st;
        int code = h->h_status->code;
        if (code == MCM_OK) {
            h->have_cells = true;
            return MCM_OK;
        }
        int grew = 0;
        if ((st = regrow(h, &grew))) return st;
        if (!grew) return set_error(h, code, mcm_gpu_strerror(code));
    }
    return set_error(h, MCM_ENBR_OVERFLOW, "storage did not converge");
}

// Enqueues part a with retries; returns the final status.
int finish_upload(mcm_gpu_handle *h, const double *coord_maxmin) {
    int st;
    k_iota<<<256, 256, 0, h->stream>>>(h->A.F.orig, h->np);
    const double hm[2] = {h->A.prm.hmax, 0.0};
    CK(cudaMemcpyAsync(h->A.hmax, hm, sizeof(hm), cudaMemcpyHostToDevice, h->stream));
    if (coord_maxmin) {
        double b[6];
        for (int d = 0; d < 3; ++d) { b[d] = coord_maxmin[2 * d]; b[3 + d] = coord_maxmin[2 * d + 1]; }
        CK(cudaMemcpyAsync(h->A.bbox, b, sizeof(b), cudaMemcpyHostToDevice, h->stream));
    } else {
        if ((st = compute_bbox(h))) return st;
    }
    // new positions and smoothing lengths: the next step builds the skin lists
    if (h->A.prm.skin > 0.0) launch_skin_force(h->A, h->stream);
    CK(cudaStreamSynchronize(h->stream));
    h->initialised = true;
    return MCM_OK;
}

}  // namespace

extern "C" {

int mcm_gpu_upload(mcm_gpu_handle *h, const mcm_gpu_fields *f, const double *coord_maxmin) {
    if (!h || !f || !f->x || !f->mat) return MCM_EINVAL;
    h->part_b_enqueued = false;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    const int n = h->np;
    int st;
    CK(cudaStreamSynchronize(h->stream));
    // checked before any copy starts, so that no copy is left reading the caller's buffers
    for (int i = 0; i < n; ++i)
        if (f->mat[i] < 1 || f->mat[i] > h->nmat) return set_error(h, MCM_EINVAL, "material id out of range");
    if ((st = put_vec3(h, f->x, FX))) return st;
    if (f->v && (st = put_vec3(h, f->v, FVX))) return st;
    if (f->a && (st = put_vec3(h, f->a, FAX))) return st;
    struct { const double *p; int f; } sc[] = {
        {f->mass, FMASS}, {f->h, FH}, {f->hold, FHOLD}, {f->rho, FRHO}, {f->rhoold, FRHOOLD}, {f->e, FE},
        {f->p, FP}, {f->c, FC}, {f->vabs, FVABS}, {f->efps, FEFPS}, {f->pcut, FPCUT}, {f->p_cut, FPCUT2},
        {f->fail, FFAIL}, {f->mindist, FMINDIST}, {f->critts, FCRITTS}, {f->tracerod, FTR},
        {f->etry, FETRY}, {f->einc, FEINC}, {f->capa, FCAPA}};
    for (auto &s : sc)
        if (s.p && (st = put_scalar(h, s.p, s.f))) return st;
    if (f->h0 || f->h) {
        if ((st = put_scalar(h, f->h0 ? f->h0 : f->h, FH0))) return st;
    }
    if (f->sigma && (st = put_rec(h, f->sigma, spec_sigma()))) return st;
    if (f->s && (st = put_rec(h, f->s, spec_sym(FD11, false)))) return st;
    if (f->alfa && (st = put_rec(h, f->alfa, spec_sym(FA11, false)))) return st;
    if (f->rod && (st = put_rec(h, f->rod, spec_sym(FR11, false)))) return st;
    if (f->q && (st = put_rec(h, f->q, spec_iso(FQ, false)))) return st;
    CK(scopy(h, h->A.F.mat, f->mat, sizeof(int) * n, cudaMemcpyHostToDevice));
    if (f->dispbc) CK(scopy(h, h->A.F.dispbc, f->dispbc, sizeof(int) * n, cudaMemcpyHostToDevice));
    else CK(cudaMemsetAsync(h->A.F.dispbc, 0, sizeof(int) * n, h->stream));
    if (f->ptype) CK(scopy(h, h->A.F.ptype, f->ptype, sizeof(int) * n, cudaMemcpyHostToDevice));
    return finish_upload(h, coord_maxmin);
}

int mcm_gpu_initialise(mcm_gpu_handle *h, const mcm_gpu_fields *f, int massopt, int init_h_opt, int init_rhoe,
                       double itss, mcm_gpu_time *t) {
    if (!h || !f || !f->x || !f->mat || !t) return MCM_EINVAL;
    CK(cudaSetDevice(h->device));
    const int n = h->np;
    int st;
    // every check before the first copy, so that no copy is left reading the caller's buffers
    if ((massopt == 1 && !f->mass) || (init_h_opt == 1 && !f->h) || (init_rhoe == 1 && (!f->rho || !f->e)))
        return MCM_EINVAL;
    std::vector<int> cnt(h->nmat, 0);
    for (int i = 0; i < n; ++i) {
        if (f->mat[i] < 1 || f->mat[i] > h->nmat) return set_error(h, MCM_EINVAL, "material id out of range");
        cnt[f->mat[i] - 1] += 1;
    }
    CK(cudaStreamSynchronize(h->stream));
    if ((st = put_vec3(h, f->x, FX))) return st;
    if (f->v) { if ((st = put_vec3(h, f->v, FVX))) return st; }
    else {
        for (int k = 0; k < 3; ++k) CK(cudaMemsetAsync(h->A.F.f[FVX + k], 0, sizeof(double) * n, h->stream));
    }
    if (massopt == 1 && (st = put_scalar(h, f->mass, FMASS))) return st;
    if (init_h_opt == 1 && (st = put_scalar(h, f->h, FH))) return st;
    if (init_rhoe == 1) {
        if ((st = put_scalar(h, f->rho, FRHO))) return st;
        if ((st = put_scalar(h, f->e, FE))) return st;
    }
    CK(scopy(h, h->A.F.mat, f->mat, sizeof(int) * n, cudaMemcpyHostToDevice));
    if (f->dispbc) CK(scopy(h, h->A.F.dispbc, f->dispbc, sizeof(int) * n, cudaMemcpyHostToDevice));
    else CK(cudaMemsetAsync(h->A.F.dispbc, 0, sizeof(int) * n, h->stream));
    CK(scopy(h, h->d_nppermat, cnt.data(), sizeof(int) * h->nmat, cudaMemcpyHostToDevice));
    // hmax (MCM/mcm_init_h.f90:22-37; the material loop indexes particles 1..nummat)
    double hmax = 0.0;
    if (init_h_opt == 0) {
        for (int i = 0; i < h->nmat && i < n; ++i) hmax = std::max(hmax, h->mats[f->mat[i] - 1].h);
    } else {
        for (int i = 0; i < n; ++i) hmax = std::max(hmax, f->h[i]);
    }
    h->cfg.hmax = hmax;
    h->A.prm.hmax = hmax;
    if ((st = reset_status(h))) return st;
    switch (h->cfg.precision) {
        case MCM_PREC_FP64_EXACT: exact::launch_initial(h->A, h->stream, massopt, init_h_opt, init_rhoe, h->d_nppermat); break;
        default: fast::launch_initial(h->A, h->stream, massopt, init_h_opt, init_rhoe, h->d_nppermat); break;
    }
    CK(cudaGetLastError());
    if ((st = finish_upload(h, nullptr))) return st;
    if ((st = sync_status(h))) return st;
    if (h->h_status->code) return set_error(h, h->h_status->code, "initialisation");
    // init_neighb (MCM/mcm_initial.f90:74) and calccritts (:81)
    if ((st = run_search_only(h))) return st;
    int nb = (h->cfg.precision == MCM_PREC_FP64_EXACT) ? exact::launch_init_critts(h->A, h->stream)
                                                        : fast::launch_init_critts(h->A, h->stream);
    launch_init_critts_reduce(h->A, h->stream, nb);
    if ((st = compute_energy(h))) return st;
    if ((st = sync_status(h))) return st;
    double critts = h->h_time->critts;
    double dt = (itss != 0.0) ? std::min(itss, critts * h->cfg.tssf) : critts * h->cfg.tssf;
    t->dt = dt;
    t->dtold = 0.0;
    t->ptime = 0.0;
    DevTime dtm;
    std::memset(&dtm, 0, sizeof(dtm));
    dtm.dt = dt; dtm.dtold = 0.0; dtm.ptime = 0.0; dtm.endtime = t->endtime; dtm.critts = critts;
    CK(scopy(h, h->A.time, &dtm, sizeof(dtm), cudaMemcpyHostToDevice));
    return MCM_OK;
}

int mcm_gpu_step_a(mcm_gpu_handle *h, double dt, double *critts) {
    int st;
    if ((st = check_handle(h))) return st;
    h->A.split_mode = 1;
    h->part_b_enqueued = false;
    {
        Scope sc(h, R_MISC, 1);
        launch_set_time(h->A, h->stream, dt, 0.0, 0);
    }
    if (!h->part_a_done) CK(cudaEventCreateWithFlags(&h->part_a_done, cudaEventDisableTiming));
    for (int attempt = 0; attempt < 8; ++attempt) {
        if ((st = reset_status(h))) return st;
        enqueue_part_a(h);
        CK(cudaMemcpyAsync(h->h_status, h->A.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(h->h_time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaEventRecord(h->part_a_done, h->stream));
        // the momentum sum of the split loop does not read dt (step_c moves):
        // it runs while the caller computes the next dt from critts; after a
        // failed part A its kernels see the raised status and do nothing
        enqueue_part_b(h, 0);
        CK(cudaEventSynchronize(h->part_a_done));
        CK(cudaGetLastError());
        const int code = h->h_status->code;
        if (code == MCM_OK) {
            h->part_b_enqueued = true;
            h->last_max_gnbr = h->h_status->max_gnbr;
            if (critts) *critts = h->h_time->critts;
            return MCM_OK;
        }
        CK(cudaStreamSynchronize(h->stream));
        int grew = 0;
        if ((st = regrow(h, &grew))) return st;
        if (!grew) return set_error(h, code, mcm_gpu_strerror(code));
    }
    return set_error(h, MCM_ENBR_OVERFLOW, "storage did not converge");
}

int mcm_gpu_step_b(mcm_gpu_handle *h, double *energies) {
    int st;
    if ((st = check_handle(h))) return st;
    h->A.split_mode = 1;
    if (!h->part_b_enqueued) {   // step_a has not enqueued it (a call out of the usual order)
        if ((st = reset_status(h))) return st;
        enqueue_part_b(h, 0);
    }
    h->part_b_enqueued = false;
    if (!energies) return MCM_OK;   // nothing to wait for: errors surface at the next waiting call
    CK(cudaMemcpyAsync(h->h_energy, h->A.energy, sizeof(double) * (5 * h->nmat + 3), cudaMemcpyDeviceToHost,
                       h->stream));
    if ((st = sync_status(h))) return st;
    if (h->h_status->code) return set_error(h, h->h_status->code, "step_b");
    std::memcpy(energies, h->h_energy, sizeof(double) * (5 * h->nmat + 3));
    return MCM_OK;
}

int mcm_gpu_step_c(mcm_gpu_handle *h, double dt, double dtold, double *coord_maxmin) {
    int st;
    if ((st = check_handle(h))) return st;
    h->A.split_mode = 1;
    if ((st = reset_status(h))) return st;
    {
        Scope sc(h, R_MISC, 1);
        launch_set_time(h->A, h->stream, dt, dtold, 1);
    }
    int nb = launch_move(h);
    {
        Scope sc(h, R_REDUCE, 1);
        launch_energy_bbox_reduce(h->A, h->stream, nb, 0, 1);
    }
    if (!coord_maxmin) return MCM_OK;   // the next grid reads the box on the device
    CK(cudaMemcpyAsync(h->h_bbox, h->A.bbox, sizeof(double) * 6, cudaMemcpyDeviceToHost, h->stream));
    if ((st = sync_status(h))) return st;
    if (h->h_status->code) return set_error(h, h->h_status->code, "step_c");
    for (int d = 0; d < 3; ++d) { coord_maxmin[2 * d] = h->h_bbox[d]; coord_maxmin[2 * d + 1] = h->h_bbox[3 + d]; }
    return MCM_OK;
}

int mcm_gpu_run(mcm_gpu_handle *h, int nsteps, mcm_gpu_time *t, int *done) {
    int st;
    if ((st = check_handle(h))) return st;
    if (!t || nsteps < 0) return MCM_EINVAL;
    if (done) *done = 0;
    h->A.split_mode = 0;
    h->part_b_enqueued = false;
    DevTime dtm;
    std::memset(&dtm, 0, sizeof(dtm));
    dtm.dt = t->dt; dtm.dtold = t->dtold; dtm.ptime = t->ptime; dtm.endtime = t->endtime;
    CK(cudaMemcpyAsync(h->A.time, &dtm, sizeof(dtm), cudaMemcpyHostToDevice, h->stream));
    int total = 0;
    int attempts = 0;
    int finished = 0;
    while (total < nsteps && !finished) {
        int batch = std::min(nsteps - total, 64);
        if ((st = reset_status(h))) return st;
        for (int k = 0; k < batch; ++k) {
            enqueue_part_a(h);
            enqueue_part_b(h, 1);
            Scope sc(h, R_MISC, 1);
            launch_finish_step(h->A, h->stream);
        }
        if ((st = sync_status(h))) return st;
        int ran = h->h_time->steps_done;
        total += ran;
        // clear the per-batch counter
        CK(cudaMemsetAsync(&h->A.time->steps_done, 0, sizeof(int), h->stream));
        if (h->h_time->ended >= 2) finished = 1;
        int code = h->h_status->code;
        if (code != MCM_OK) {
            int grew = 0;
            if ((st = regrow(h, &grew))) return st;
            if (!grew || ++attempts > 16) {
                if (done) *done = total;
                CK(scopy(h, h->h_time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost));
                t->dt = h->h_time->dt; t->dtold = h->h_time->dtold; t->ptime = h->h_time->ptime;
                return set_error(h, code, mcm_gpu_strerror(code));
            }
        }
    }
    CK(scopy(h, h->h_time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost));
    t->dt = h->h_time->dt; t->dtold = h->h_time->dtold; t->ptime = h->h_time->ptime;
    if (done) *done = total;
    h->A.split_mode = 1;
    return MCM_OK;
}

int mcm_gpu_download(mcm_gpu_handle *h, mcm_gpu_fields *f) {
    int st;
    if ((st = check_handle(h))) return st;
    if (!f) return MCM_EINVAL;
    CK(cudaStreamSynchronize(h->stream));
    const int n = h->np;
    std::vector<int> orig(n);
    CK(scopy(h, orig.data(), h->A.F.orig, sizeof(int) * n, cudaMemcpyDeviceToHost));
    if (f->x && (st = get_rec(h, f->x, spec_vec3(FX)))) return st;
    if (f->v && (st = get_rec(h, f->v, spec_vec3(FVX)))) return st;
    if (f->a && (st = get_rec(h, f->a, spec_vec3(FAX)))) return st;
    if (f->repulsion && (st = get_rec(h, f->repulsion, spec_vec3(FRPX)))) return st;
    struct { double *p; int f; } sc[] = {
        {f->mass, FMASS}, {f->h, FH}, {f->hold, FHOLD}, {f->rho, FRHO}, {f->rhoold, FRHOOLD}, {f->e, FE},
        {f->p, FP}, {f->c, FC}, {f->vabs, FVABS}, {f->efps, FEFPS}, {f->pcut, FPCUT}, {f->p_cut, FPCUT2},
        {f->fail, FFAIL}, {f->mindist, FMINDIST}, {f->critts, FCRITTS}, {f->tracerod, FTR},
        {f->etry, FETRY}, {f->einc, FEINC}, {f->capa, FCAPA}, {f->h0, FH0}};
    for (auto &s : sc) {
        if (!s.p) continue;
        PackSpec one = spec_none(1);
        one.field[0] = s.f;
        if ((st = get_rec(h, s.p, one))) return st;
    }
    if (f->sigma && (st = get_rec(h, f->sigma, spec_sigma()))) return st;
    if (f->s && (st = get_rec(h, f->s, spec_sym(FD11, true)))) return st;
    if (f->alfa && (st = get_rec(h, f->alfa, spec_sym(FA11, true)))) return st;
    if (f->rod && (st = get_rec(h, f->rod, spec_sym(FR11, true)))) return st;
    if (f->spin && (st = get_rec(h, f->spin, spec_spin()))) return st;
    if (f->q && (st = get_rec(h, f->q, spec_iso(FQ, true)))) return st;
    if (f->qold && (st = get_rec(h, f->qold, spec_iso(FQ, true)))) return st;
    CK(cudaStreamSynchronize(h->stream));
    std::vector<int> itmp(n);
    auto geti = [&](int *dst, const int *src) -> int {
        CK(scopy(h, itmp.data(), src, sizeof(int) * n, cudaMemcpyDeviceToHost));
        for (int p = 0; p < n; ++p) dst[orig[p]] = itmp[p];
        return MCM_OK;
    };
    if (f->mat && (st = geti(f->mat, h->A.F.mat))) return st;
    if (f->dispbc && (st = geti(f->dispbc, h->A.F.dispbc))) return st;
    if (f->nnbr || f->g_nnbr) {
        // the counts are per cell-order position: position t holds state index cell_list[t]
        std::vector<int> clist(n);
        CK(scopy(h, clist.data(), h->A.cell_list, sizeof(int) * n, cudaMemcpyDeviceToHost));
        auto getc = [&](int *dst, const int *src) -> int {
            CK(scopy(h, itmp.data(), src, sizeof(int) * n, cudaMemcpyDeviceToHost));
            for (int t = 0; t < n; ++t) dst[orig[clist[t]]] = itmp[t];
            return MCM_OK;
        };
        if (f->nnbr && (st = getc(f->nnbr, h->A.nnbr))) return st;
        if (f->g_nnbr && (st = getc(f->g_nnbr, h->A.gnnbr))) return st;
    }
    if (f->ptype && (st = geti(f->ptype, h->A.F.ptype))) return st;
    return MCM_OK;
}

int mcm_gpu_neighbours(mcm_gpu_handle *h, int *nnbr, int *nbr, int *stride, int *g_nnbr, int *g_nbr, int *g_stride) {
    int st;
    if ((st = check_handle(h))) return st;
    CK(cudaStreamSynchronize(h->stream));
    const int n = h->np, np = h->npad;
    std::vector<int> orig(n), cnt(n), gcnt(n), clist(n), ckey(n);
    CK(scopy(h, orig.data(), h->A.F.orig, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(scopy(h, cnt.data(), h->A.nnbr, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(scopy(h, gcnt.data(), h->A.gnnbr, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(scopy(h, clist.data(), h->A.cell_list, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(scopy(h, ckey.data(), h->A.ckey, sizeof(int) * n, cudaMemcpyDeviceToHost));
    int need = 0, gneed = 0;
    for (int t = 0; t < n; ++t) { need = std::max(need, cnt[t]); gneed = std::max(gneed, gcnt[t]); }
    if (nnbr) for (int t = 0; t < n; ++t) nnbr[orig[clist[t]]] = cnt[t];
    if (g_nnbr) for (int t = 0; t < n; ++t) g_nnbr[orig[clist[t]]] = gcnt[t];
    bool small = (nbr && stride && *stride < need) || (g_nbr && g_stride && *g_stride < gneed);
    if (stride) { if (small || !nbr) *stride = std::max(*stride, need); }
    if (g_stride) { if (small || !g_nbr) *g_stride = std::max(*g_stride, gneed); }
    if (small) return MCM_EINVAL;
    if (nbr && stride) {
        const int ns = h->A.nstride;
        std::vector<unsigned int> tab((size_t)ns * np);
        CK(scopy(h, tab.data(), h->A.nidx, sizeof(unsigned int) * tab.size(), cudaMemcpyDeviceToHost));
        const int self = h->cfg.disctype == 1 ? 1 : 0;
        for (int t = 0; t < n; ++t) {
            int *row = nbr + (size_t)orig[clist[t]] * *stride;
            const int stored = cnt[t] - self;
            for (int k = 0; k < stored; ++k) row[k] = orig[clist[tab[(size_t)t * ns + k] & 0x3ffffffu]] + 1;
            if (self) row[stored] = orig[clist[t]] + 1;
        }
    }
    if (g_nbr && g_stride) {
        std::vector<int> tab((size_t)h->A.gstride * np);
        CK(scopy(h, tab.data(), h->A.gnbr, sizeof(int) * tab.size(), cudaMemcpyDeviceToHost));
        for (int t = 0; t < n; ++t)
            for (int k = 0; k < gcnt[t]; ++k) g_nbr[(size_t)orig[clist[t]] * *g_stride + k] = tab[(size_t)k * np + t] + 1;
    }
    return MCM_OK;
}

int mcm_gpu_contacts(mcm_gpu_handle *h, int *ncont, int *cont, int *stride, int *g_ncont, int *g_cont,
                     int *g_stride) {
    int st;
    if ((st = check_handle(h))) return st;
    CK(cudaStreamSynchronize(h->stream));
    const int n = h->np, np = h->npad;
    std::vector<int> orig(n), cnt(n, 0), gcnt(n, 0), clist(n);
    CK(scopy(h, orig.data(), h->A.F.orig, sizeof(int) * n, cudaMemcpyDeviceToHost));
    CK(scopy(h, clist.data(), h->A.cell_list, sizeof(int) * n, cudaMemcpyDeviceToHost));
    const bool on = h->A.prm.contact != 0;
    if (on) {
        CK(scopy(h, cnt.data(), h->A.ncont, sizeof(int) * n, cudaMemcpyDeviceToHost));
        CK(scopy(h, gcnt.data(), h->A.gncont, sizeof(int) * n, cudaMemcpyDeviceToHost));
    }
    int need = 0, gneed = 0;
    for (int t = 0; t < n; ++t) { need = std::max(need, cnt[t]); gneed = std::max(gneed, gcnt[t]); }
    if (ncont) for (int t = 0; t < n; ++t) ncont[orig[clist[t]]] = cnt[t];
    if (g_ncont) for (int t = 0; t < n; ++t) g_ncont[orig[clist[t]]] = gcnt[t];
    bool small = (cont && stride && *stride < need) || (g_cont && g_stride && *g_stride < gneed);
    if (stride) { if (small || !cont) *stride = std::max(*stride, need); }
    if (g_stride) { if (small || !g_cont) *g_stride = std::max(*g_stride, gneed); }
    if (small) return MCM_EINVAL;
    if (!on) return MCM_OK;
    if (cont && stride) {
        const int cs = h->A.cstride;
        std::vector<unsigned int> tab((size_t)cs * np);
        CK(scopy(h, tab.data(), h->A.cidx, sizeof(unsigned int) * tab.size(), cudaMemcpyDeviceToHost));
        for (int t = 0; t < n; ++t) {
            int *row = cont + (size_t)orig[clist[t]] * *stride;
            for (int k = 0; k < cnt[t]; ++k) row[k] = orig[clist[tab[(size_t)t * cs + k] & 0x3ffffffu]] + 1;
        }
    }
    if (g_cont && g_stride) {
        std::vector<int> tab((size_t)h->A.gcstride * np);
        CK(scopy(h, tab.data(), h->A.gcont, sizeof(int) * tab.size(), cudaMemcpyDeviceToHost));
        for (int t = 0; t < n; ++t)
            for (int k = 0; k < gcnt[t]; ++k)
                g_cont[(size_t)orig[clist[t]] * *g_stride + k] = tab[(size_t)k * np + t] + 1;
    }
    return MCM_OK;
}

int mcm_gpu_contact_forces(mcm_gpu_handle *h, double *xyz) {
    int st;
    if ((st = check_handle(h))) return st;
    if (!xyz) return MCM_EINVAL;
    const int nv = 3 * h->nmat;
    if (!h->A.prm.contact || h->cfg.disctype != 0) {
        for (int k = 0; k < nv; ++k) xyz[k] = 0.0;
        return MCM_OK;
    }
    // the rows of the block partials are free between steps
    launch_contact_forces(h->A, h->stream, h->A.red);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(xyz, h->A.red, sizeof(double) * nv, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MCM_OK;
}

int mcm_gpu_ghosts(mcm_gpu_handle *h, int *ngp, int *par, double *x, double *v, int cap) {
    int st;
    if ((st = check_handle(h))) return st;
    CK(cudaStreamSynchronize(h->stream));
    int n = 0;
    CK(scopy(h, &n, h->A.ngp, sizeof(int), cudaMemcpyDeviceToHost));
    if (ngp) *ngp = n;
    int m = std::min(n, cap);
    if (m <= 0) return MCM_OK;
    std::vector<int> orig(h->np);
    CK(scopy(h, orig.data(), h->A.F.orig, sizeof(int) * h->np, cudaMemcpyDeviceToHost));
    if (par) {
        std::vector<int> gp(m);
        CK(scopy(h, gp.data(), h->A.gpar, sizeof(int) * m, cudaMemcpyDeviceToHost));
        for (int g = 0; g < m; ++g) par[g] = orig[gp[g]] + 1;
    }
    std::vector<double> tmp(m);
    double *const xs[3] = {h->A.gx, h->A.gy, h->A.gz};
    double *const vs[3] = {h->A.gvx, h->A.gvy, h->A.gvz};
    for (int k = 0; k < 3; ++k) {
        if (x) {
            CK(scopy(h, tmp.data(), xs[k], sizeof(double) * m, cudaMemcpyDeviceToHost));
            for (int g = 0; g < m; ++g) x[3 * (size_t)g + k] = tmp[g];
        }
        if (v) {
            CK(scopy(h, tmp.data(), vs[k], sizeof(double) * m, cudaMemcpyDeviceToHost));
            for (int g = 0; g < m; ++g) v[3 * (size_t)g + k] = tmp[g];
        }
    }
    return MCM_OK;
}

int mcm_gpu_grid(mcm_gpu_handle *h, int *gridlim, double *gridmin, double *gridsize) {
    int st;
    if ((st = check_handle(h))) return st;
    CK(cudaStreamSynchronize(h->stream));
    DevGrid g;
    CK(scopy(h, &g, h->A.grid, sizeof(g), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; ++k) {
        if (gridlim) gridlim[k] = g.gridlim[k];
        if (gridmin) gridmin[k] = g.gridmin[k];
        if (gridsize) gridsize[k] = g.gridsize[k];
    }
    return MCM_OK;
}

int mcm_gpu_energies(mcm_gpu_handle *h, double *energies) {
    int st;
    if ((st = check_handle(h))) return st;
    if (!energies) return MCM_EINVAL;
    CK(cudaStreamSynchronize(h->stream));
    CK(scopy(h, energies, h->A.energy, sizeof(double) * (5 * h->nmat + 3), cudaMemcpyDeviceToHost));
    return MCM_OK;
}

int mcm_gpu_skin_builds(mcm_gpu_handle *h, long long *builds) {
    int st;
    if ((st = check_handle(h))) return st;
    if (!builds) return MCM_EINVAL;
    *builds = 0;
    if (h->A.prm.skin <= 0.0) return MCM_OK;
    CK(cudaStreamSynchronize(h->stream));
    int flags[3] = {0, 0, 0};
    CK(scopy(h, flags, h->A.skin_flags, sizeof(flags), cudaMemcpyDeviceToHost));
    *builds = flags[2];
    return MCM_OK;
}

int mcm_gpu_stats(mcm_gpu_handle *h, double *mean_nbr, int *max_nbr, int *stride, int *ngp) {
    int st;
    if ((st = check_handle(h))) return st;
    CK(cudaStreamSynchronize(h->stream));
    if (mean_nbr) {
        std::vector<int> cnt(h->np), gcnt(h->np);
        CK(scopy(h, cnt.data(), h->A.nnbr, sizeof(int) * h->np, cudaMemcpyDeviceToHost));
        CK(scopy(h, gcnt.data(), h->A.gnnbr, sizeof(int) * h->np, cudaMemcpyDeviceToHost));
        double s = 0.0;
        for (int p = 0; p < h->np; ++p) s += cnt[p] + gcnt[p];
        *mean_nbr = s / h->np;
    }
    if (max_nbr) {
        DevStatus s;
        CK(scopy(h, &s, h->A.status, sizeof(s), cudaMemcpyDeviceToHost));
        *max_nbr = s.max_nbr;
    }
    if (stride) *stride = h->A.nstride;
    if (ngp) CK(scopy(h, ngp, h->A.ngp, sizeof(int), cudaMemcpyDeviceToHost));
    return MCM_OK;
}

int mcm_gpu_profile(mcm_gpu_handle *h, int enable) {
    if (!h) return MCM_EINVAL;
    CK(cudaStreamSynchronize(h->stream));
    for (auto &v : h->prof_pairs) {
        for (auto &pr : v) { h->ev_pool.push_back(pr.first); h->ev_pool.push_back(pr.second); }
        v.clear();
    }
    h->prof_on = enable != 0;
    h->kernel_launches = 0;
    return MCM_OK;
}

int mcm_gpu_profile_report(mcm_gpu_handle *h, int region, char *name, int name_len, double *total_ms, int *launches) {
    if (!h) return MCM_EINVAL;
    if (region < 0 || region >= R_NREG) return MCM_EINVAL;
    CK(cudaStreamSynchronize(h->stream));
    double ms = 0.0;
    for (auto &pr : h->prof_pairs[region]) {
        float t = 0.f;
        CK(cudaEventElapsedTime(&t, pr.first, pr.second));
        ms += t;
    }
    if (name && name_len > 0) {
        std::strncpy(name, kRegionName[region], (size_t)name_len - 1);
        name[name_len - 1] = 0;
    }
    if (total_ms) *total_ms = ms;
    if (launches) *launches = (int)h->prof_pairs[region].size();
    return MCM_OK;
}

long long mcm_gpu_kernel_launches(mcm_gpu_handle *h) { return h ? h->kernel_launches : -1; }

int mcm_gpu_timer(mcm_gpu_handle *h, int op, double *ms) {
    if (!h) return MCM_EINVAL;
    for (int k = 0; k < 2; ++k)
        if (!h->timer[k]) CK(cudaEventCreate(&h->timer[k]));
    if (op == 0) {
        CK(cudaEventRecord(h->timer[0], h->stream));
        return MCM_OK;
    }
    CK(cudaEventRecord(h->timer[1], h->stream));
    CK(cudaEventSynchronize(h->timer[1]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, h->timer[0], h->timer[1]));
    if (ms) *ms = t;
    return MCM_OK;
}

int mcm_gpu_set_diagnostics(mcm_gpu_handle *h, int enable) {
    if (!h) return MCM_EINVAL;
    h->A.prm.diag = enable ? 1 : 0;
    return MCM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- adjoint
namespace mcm_host {

constexpr int kAdjArrays = 40 + 4 * adj::kRecSlots;   // 40 adjoint arrays, then the gather records

size_t snap_doubles(const mcm_gpu_handle *h) { return (size_t)NFIELD * h->npad + 8; }

int snap_save(mcm_gpu_handle *h, double *buf) {
    CK(cudaMemcpyAsync(buf, h->d_fields, sizeof(double) * NFIELD * h->npad, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(buf + (size_t)NFIELD * h->npad, h->A.bbox, sizeof(double) * 6, cudaMemcpyDeviceToDevice,
                       h->stream));
    CK(cudaMemcpyAsync(buf + (size_t)NFIELD * h->npad + 6, h->A.hmax, sizeof(double) * 2, cudaMemcpyDeviceToDevice,
                       h->stream));
    return MCM_OK;
}
int snap_load(mcm_gpu_handle *h, const double *buf) {
    CK(cudaMemcpyAsync(h->d_fields, buf, sizeof(double) * NFIELD * h->npad, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->A.bbox, buf + (size_t)NFIELD * h->npad, sizeof(double) * 6, cudaMemcpyDeviceToDevice,
                       h->stream));
    CK(cudaMemcpyAsync(h->A.hmax, buf + (size_t)NFIELD * h->npad + 6, sizeof(double) * 2, cudaMemcpyDeviceToDevice,
                       h->stream));
    return MCM_OK;
}

// One loop iteration with the prescribed dt schedule: step_a with dts[n],
// dt update to dts[n+1], step_b, step_c.
int adj_step(mcm_gpu_handle *h, int n, bool move) {
    int st;
    if ((st = mcm_gpu_step_a(h, h->adj_dts[n], nullptr))) return st;
    if ((st = mcm_gpu_step_b(h, nullptr))) return st;
    if (move && (st = mcm_gpu_step_c(h, h->adj_dts[n + 1], h->adj_dts[n], nullptr))) return st;
    return MCM_OK;
}

int adj_check(mcm_gpu_handle *h) {
    if (h->cfg.disctype != 0) return set_error(h, MCM_EUNSUPPORTED, "adjoint: disctype 0 only");
    if (h->cfg.reorder_interval != 0) return set_error(h, MCM_EUNSUPPORTED, "adjoint: reorder_interval must be 0");
    if (h->cfg.h_opt != 0 || h->cfg.veloc_opt != 0)
        return set_error(h, MCM_EUNSUPPORTED, "adjoint: constant smoothing length without XSPH only");
    if (h->A.prm.contact) return set_error(h, MCM_EUNSUPPORTED, "adjoint: no repulsive contact (contacttype > 0)");
    if (h->A.prm.skin > 0.0) return set_error(h, MCM_EUNSUPPORTED, "adjoint: neighbour lists rebuilt every step (nbr_skin 0)");
    // models whose whole state is what the reverse constitutive step carries:
    // model 10, and model 9 without viscosity (its deviator is zero every step;
    // MCM/mcm_f3dm9.f90:30-32); the dual pass keeps 8 constitutive constants,
    // which hold model 9's cm(1..2, mat) for materials 1 and 2
    for (size_t k = 0; k < h->mats.size(); ++k) {
        const mcm_gpu_material &m = h->mats[k];
        const bool eos_ok = m.eos == 1 || m.eos == 4 || m.eos == 13 || m.eos == 28 || m.eos == 41;
        const bool fluid = m.model == 9 && k < 2 && m.strinput[1 + 5 * k] == 0.0;
        if (!eos_ok || !(m.model == 10 || fluid))
            return set_error(h, MCM_EUNSUPPORTED,
                             "adjoint: model 10, or model 9 with zero viscosity (materials 1-2), with EOS 1, 4, 13, 28 "
                             "or 41");
    }
    return MCM_OK;
}

struct DiagOff {
    mcm_gpu_handle *h;
    int saved;
    explicit DiagOff(mcm_gpu_handle *hh) : h(hh), saved(hh->A.prm.diag) { h->A.prm.diag = 0; }
    ~DiagOff() { h->A.prm.diag = saved; }
};

// Step records: what the reverse kernels read of a step's forward pass (the
// state after momentum, the neighbour table, the ghosts), copied once while
// the segment is recomputed, so that the reverse sweep does not run the
// forward part of each step a second time.
constexpr int kGhostD = 9;   // ghost doubles kept: x y z vx vy vz mass h rho (and the int parent and mirror mask)
// Post-step fields the reverse kernels read, as contiguous runs of the field
// enumeration: x | h mass rho | sigma q | rod spin tr | a.  (Material ids and
// displacement conditions do not change: the adjoint runs without re-sorting.)
constexpr int kRecRuns = 5;
constexpr int kRecRun[kRecRuns][2] = {{FX, 3}, {FH, 3}, {FS11, 7}, {FR11, 10}, {FAX, 3}};
constexpr int rec_fields() {
    int n = 0;
    for (int r = 0; r < kRecRuns; ++r) n += kRecRun[r][1];
    return n;
}
static_assert(FMASS == FH + 1 && FRHO == FH + 2 && FQ == FS11 + 6 && FW12 == FR11 + 6 && FTR == FR11 + 9 &&
                  FAZ == FAX + 2,
              "recorded field runs");

// Carves a record buffer into its arrays (256-byte aligned pieces).  With a
// null base it only measures: the returned size is the buffer a record of
// these widths needs.
struct RecordView {
    double *fields, *g[kGhostD];
    unsigned *nidx;
    int *gnbr, *nnbr, *gnnbr, *cell_list, *gpar, *gflip;
};
size_t record_layout(const mcm_gpu_handle *h, char *base, int nstride, int gstride, int ghost_cap, RecordView *v) {
    size_t off = 0;
    auto take = [&](size_t bytes) { char *q = base ? base + off : nullptr; off += (bytes + 255) / 256 * 256; return q; };
    const size_t np = h->npad, gc = (size_t)ghost_cap;
    RecordView t;
    t.fields = (double *)take(sizeof(double) * rec_fields() * np);
    t.nidx = (unsigned *)take(sizeof(unsigned) * (size_t)nstride * np);
    t.gnbr = (int *)take(sizeof(int) * (size_t)gstride * np);
    t.nnbr = (int *)take(sizeof(int) * np);
    t.gnnbr = (int *)take(sizeof(int) * np);
    t.cell_list = (int *)take(sizeof(int) * np);
    for (int k = 0; k < kGhostD; ++k) t.g[k] = (double *)take(sizeof(double) * gc);
    t.gpar = (int *)take(sizeof(int) * gc);
    t.gflip = (int *)take(sizeof(int) * gc);
    if (v) *v = t;
    return off;
}
size_t record_bytes(const mcm_gpu_handle *h) {
    return record_layout(h, nullptr, h->A.nstride, h->A.gstride, h->A.ghost_cap, nullptr);
}
RecordView record_view(const mcm_gpu_handle *h, const mcm_gpu_handle::StepRecord &r) {
    RecordView v;
    record_layout(h, r.buf, r.nstride, r.gstride, r.ghost_cap, &v);
    return v;
}

double *ghost_arrays(StepArgs &a, int k) {
    double *const g[kGhostD] = {a.gx, a.gy, a.gz, a.gvx, a.gvy, a.gvz, a.gmass, a.gh, a.grho};
    return g[k];
}

int record_save(mcm_gpu_handle *h, mcm_gpu_handle::StepRecord &r) {
    const size_t need = record_bytes(h);
    if (r.bytes < need) {
        if (r.buf) cudaFree(r.buf);
        r.buf = nullptr;
        r.bytes = 0;
        CK(cudaMalloc((void **)&r.buf, need));
        r.bytes = need;
    }
    r.nstride = h->A.nstride;
    r.gstride = h->A.gstride;
    r.ghost_cap = h->A.ghost_cap;
    const RecordView v = record_view(h, r);
    const size_t np = h->npad, gc = (size_t)r.ghost_cap;
    StepArgs &a = h->A;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream);
    };
    for (int r = 0, o = 0; r < kRecRuns; o += kRecRun[r][1], ++r)
        CK(cp(v.fields + (size_t)o * np, h->A.F.f[kRecRun[r][0]], sizeof(double) * kRecRun[r][1] * np));
    CK(cp(v.nidx, a.nidx, sizeof(unsigned) * (size_t)r.nstride * np));
    // ghost lists are column-major (entry k of every position in row k): only
    // the rows that hold entries are copied
    const int grows = std::min(h->last_max_gnbr, r.gstride);
    if (grows > 0) CK(cp(v.gnbr, a.gnbr, sizeof(int) * (size_t)grows * np));
    CK(cp(v.nnbr, a.nnbr, sizeof(int) * np));
    CK(cp(v.gnnbr, a.gnnbr, sizeof(int) * np));
    CK(cp(v.cell_list, a.cell_list, sizeof(int) * np));
    for (int k = 0; k < kGhostD; ++k) CK(cp(v.g[k], ghost_arrays(a, k), sizeof(double) * gc));
    CK(cp(v.gpar, a.gpar, sizeof(int) * gc));
    CK(cp(v.gflip, a.gflip, sizeof(int) * gc));
    return MCM_OK;
}

// The step arguments of a recorded step: the live arguments with every array
// the reverse kernels read pointed into the record.
StepArgs record_args(const mcm_gpu_handle *h, const mcm_gpu_handle::StepRecord &r) {
    StepArgs a = h->A;
    const RecordView v = record_view(h, r);
    // fields outside the runs keep pointing at the live state, which the
    // reverse kernels do not read
    for (int r = 0, o = 0; r < kRecRuns; o += kRecRun[r][1], ++r)
        for (int k = 0; k < kRecRun[r][1]; ++k) a.F.f[kRecRun[r][0] + k] = v.fields + (size_t)(o + k) * h->npad;
    a.nstride = r.nstride;
    a.gstride = r.gstride;
    a.ghost_cap = r.ghost_cap;
    a.nidx = v.nidx;
    a.gnbr = v.gnbr;
    a.nnbr = v.nnbr;
    a.gnnbr = v.gnnbr;
    a.cell_list = v.cell_list;
    a.gx = v.g[0]; a.gy = v.g[1]; a.gz = v.g[2];
    a.gvx = v.g[3]; a.gvy = v.g[4]; a.gvz = v.g[5];
    a.gmass = v.g[6]; a.gh = v.g[7]; a.grho = v.g[8];
    a.gpar = v.gpar;
    a.gflip = v.gflip;
    return a;
}

// Records are kept when a segment's worth fits in half of the free memory.
bool records_fit(mcm_gpu_handle *h, int every) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
    size_t held = 0;
    for (auto &r : h->adj_rec) held += r.bytes;
    const size_t need = (size_t)every * (record_bytes(h) + record_bytes(h) / 8);
    return need <= (fr + held) / 2;
}

// The same iteration, enqueued without waiting: storage overflows are found
// from the status after a whole segment (adj_segment).  `record` (may be
// null) receives the step's record between momentum and the move.
int adj_enqueue_step(mcm_gpu_handle *h, int n, bool move, mcm_gpu_handle::StepRecord *record) {
    StepArgs &a = h->A;
    a.split_mode = 1;
    launch_set_time(a, h->stream, h->adj_dts[n], 0.0, 0);
    enqueue_part_a(h);
    enqueue_part_b(h, 0);
    int st;
    if (record && (st = record_save(h, *record))) return st;
    if (move) {
        launch_set_time(a, h->stream, h->adj_dts[n + 1], h->adj_dts[n], 1);
        const int nb = launch_move(h);
        launch_energy_bbox_reduce(a, h->stream, nb, 0, 1);
    }
    CK(cudaGetLastError());
    return MCM_OK;
}

// Steps n0 .. n0+K-1 from the handle's state, which equals the snapshot
// `start`: seg (may be null) receives the state before each step; with
// records, each step's record is kept and the last step stops before its move;
// without them the last step is not run (only its snapshot is taken) unless
// `move_last`.  One status check per segment: after a storage overflow the
// storage is regrown, the state reloaded from `start` and the segment re-run.
int adj_segment(mcm_gpu_handle *h, int n0, int K, const double *start, double *seg, bool records, bool move_last) {
    const size_t sd = snap_doubles(h);
    // records copy every ghost-list row: the longest list is not known before the status is read
    h->last_max_gnbr = 1 << 30;
    for (int attempt = 0; attempt < 8; ++attempt) {
        int st;
        if ((st = reset_status(h))) return st;
        for (int s = 0; s < K; ++s) {
            if (seg && (st = snap_save(h, seg + sd * s))) return st;
            const bool last = (s == K - 1);
            if (records) {
                if ((st = adj_enqueue_step(h, n0 + s, !last || move_last, &h->adj_rec[s]))) return st;
            } else if (!last || move_last) {
                if ((st = adj_enqueue_step(h, n0 + s, true, nullptr))) return st;
            }
        }
        if ((st = sync_status(h))) return st;
        const int code = h->h_status->code;
        if (code == MCM_OK) return MCM_OK;
        int grew = 0;
        if ((st = regrow(h, &grew))) return st;
        if (!grew) return set_error(h, code, mcm_gpu_strerror(code));
        if ((st = snap_load(h, start))) return st;
    }
    return set_error(h, MCM_ENBR_OVERFLOW, "adjoint: storage did not converge");
}

}  // namespace

extern "C" {

int mcm_gpu_adjoint_forward(mcm_gpu_handle *h, int nsteps, const double *dts, int checkpoint_every) {
    int st;
    if ((st = check_handle(h))) return st;
    if (nsteps <= 0 || !dts || checkpoint_every <= 0) return MCM_EINVAL;
    if ((st = adj_check(h))) return st;
    DiagOff diag(h);   // the reverse step reads the strain output, which diagnostics overwrite
    h->adj_dts.assign(dts, dts + nsteps + 1);
    h->adj_steps = nsteps;
    h->adj_every = checkpoint_every;
    const int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
    // checkpoints are kept between calls (a snapshot's size is fixed per
    // handle): only missing ones are allocated, surplus ones freed
    const size_t sd = snap_doubles(h);
    for (size_t c = nck; c < h->adj_ckpt.size(); ++c)
        if (h->adj_ckpt[c]) cudaFree(h->adj_ckpt[c]);
    h->adj_ckpt.resize(nck, nullptr);
    for (int c = 0; c < nck; ++c)
        if (!h->adj_ckpt[c] && (st = dalloc(h, &h->adj_ckpt[c], sd))) return st;
    if (!h->adj_final && (st = dalloc(h, &h->adj_final, sd))) return st;
    for (int c = 0; c < nck; ++c) {
        const int n0 = c * checkpoint_every;
        if ((st = snap_save(h, h->adj_ckpt[c]))) return st;
        if ((st = adj_segment(h, n0, std::min(checkpoint_every, nsteps - n0), h->adj_ckpt[c], nullptr, false, true)))
            return st;
    }
    if ((st = snap_save(h, h->adj_final))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return MCM_OK;
}

int mcm_gpu_adjoint_backward(mcm_gpu_handle *h, const double *xbar, const double *vbar, double *param_bar,
                             double *xbar0, double *vbar0) {
    int st;
    if ((st = check_handle(h))) return st;
    if (h->adj_steps <= 0) return set_error(h, MCM_EINVAL, "adjoint: no forward run recorded");
    if ((st = adj_check(h))) return st;
    DiagOff diag(h);
    const int n = h->np;
    const size_t np = h->npad;
    if (!h->d_adj && (st = dalloc(h, &h->d_adj, (size_t)kAdjArrays * np))) return st;
    CK(cudaMemsetAsync(h->d_adj, 0, sizeof(double) * kAdjArrays * np, h->stream));
    if (!h->d_theta && (st = dalloc(h, &h->d_theta, (size_t)h->nmat * adj::kParams))) return st;
    CK(cudaMemsetAsync(h->d_theta, 0, sizeof(double) * h->nmat * adj::kParams, h->stream));
    std::vector<int> orig(n);
    CK(scopy(h, orig.data(), h->A.F.orig, sizeof(int) * n, cudaMemcpyDeviceToHost));
    adj::AdjArgs b;
    std::memset(&b, 0, sizeof(b));
    double *base = h->d_adj;
    auto arr = [&](int k) { return base + (size_t)k * np; };
    for (int d = 0; d < 3; ++d) { b.xb[d] = arr(d); b.vb[d] = arr(3 + d); b.ab[d] = arr(16 + d); }
    b.rhob = arr(6); b.eb = arr(7); b.pb = arr(8); b.efpsb = arr(9);
    for (int u = 0; u < 6; ++u) { b.sigb[u] = arr(10 + u); b.ysig[u] = arr(23 + u); }
    b.yrho = arr(19); b.ye = arr(20); b.yp = arr(21); b.yefps = arr(22); b.yq = arr(29); b.rho0b = arr(30);
    for (int u = 0; u < 9; ++u) b.gb[u] = arr(31 + u);
    b.rec = reinterpret_cast<double4 *>(arr(40));   // 4 * kRecSlots doubles per position
    b.theta_b = h->d_theta;
    b.rev = h->adj_kind == 1 ? 1 : 0;
    for (const mcm_gpu_material &m : h->mats)
        if (m.model != 10 || m.eos != 41) b.rev = 0;
    // final adjoints, Fortran (3,np) by particle -> state order
    std::vector<double> tmp(n);
    for (int d = 0; d < 3; ++d) {
        if (xbar) {
            for (int i = 0; i < n; ++i) tmp[i] = xbar[3 * (size_t)orig[i] + d];
            CK(scopy(h, b.xb[d], tmp.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        }
        if (vbar) {
            for (int i = 0; i < n; ++i) tmp[i] = vbar[3 * (size_t)orig[i] + d];
            CK(scopy(h, b.vb[d], tmp.data(), sizeof(double) * n, cudaMemcpyHostToDevice));
        }
    }
    const int every = h->adj_every, nck = (int)h->adj_ckpt.size();
    const size_t sd = snap_doubles(h);
    if (h->adj_seg_cap < every) {
        if ((st = dalloc(h, &h->adj_seg, sd * every))) return st;
        h->adj_seg_cap = every;
    }
    // With step records, each step of a segment runs forward once (its record
    // is taken after momentum, before the move); without them the reverse
    // sweep re-runs the forward part of each step from its snapshot.
    const bool keep = records_fit(h, every);
    if (keep && (int)h->adj_rec.size() < every) h->adj_rec.resize(every);
    for (int c = nck - 1; c >= 0; --c) {
        const int n0 = c * every;
        const int K = std::min(every, h->adj_steps - n0);
        if ((st = snap_load(h, h->adj_ckpt[c]))) return st;
        if ((st = adj_segment(h, n0, K, h->adj_ckpt[c], h->adj_seg, keep, false))) return st;
        for (int s = K - 1; s >= 0; --s) {
            const int m = n0 + s;
            const double *pre = h->adj_seg + sd * s;
            StepArgs as;
            if (keep) {
                as = record_args(h, h->adj_rec[s]);
            } else {
                if ((st = snap_load(h, pre))) return st;
                if ((st = adj_step(h, m, false))) return st;   // lists, ghosts, strain, constitutive, momentum
                as = h->A;
            }
            for (int f = 0; f < NFIELD; ++f) b.pre[f] = pre + (size_t)f * np;
            b.dt_prev = h->adj_dts[m];
            b.dtold = h->adj_dts[m];
            b.dt = h->adj_dts[m + 1];
            {
                Scope sc(h, R_ADJ_MOM, 3);
                adj::launch_reverse_momentum(as, b, h->stream);
            }
            {
                Scope sc(h, R_ADJ_CONST, 1);
                adj::launch_reverse_constitutive(as, b, h->stream);
            }
            {
                Scope sc(h, R_ADJ_STRAIN, 1);
                adj::launch_reverse_strain(as, b, h->stream);
            }
            CK(cudaGetLastError());
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    for (int d = 0; d < 3; ++d) {
        if (xbar0) {
            CK(scopy(h, tmp.data(), b.xb[d], sizeof(double) * n, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i) xbar0[3 * (size_t)orig[i] + d] = tmp[i];
        }
        if (vbar0) {
            CK(scopy(h, tmp.data(), b.vb[d], sizeof(double) * n, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; ++i) vbar0[3 * (size_t)orig[i] + d] = tmp[i];
        }
    }
    if (param_bar) CK(scopy(h, param_bar, h->d_theta, sizeof(double) * h->nmat * adj::kParams, cudaMemcpyDeviceToHost));
    // leave the device state as the forward run left it
    if ((st = snap_load(h, h->adj_final))) return st;
    CK(cudaStreamSynchronize(h->stream));
    return MCM_OK;
}

}  // extern "C"
