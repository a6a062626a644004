// handle.h -- the handle behind the C ABI and the host helpers shared by the
// translation units of the C ABI (abi.cu: one body; batch.cu: many bodies and
// the tuner).  Private to the library.
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "kernels.h"

// One body: its stream, device state and host mirrors.
struct mcm_gpu_handle {
    mcm_gpu_config cfg;
    int np = 0, npad = 0, nmat = 0;
    std::vector<mcm_gpu_material> mats;
    cudaStream_t stream = nullptr;
    int device = 0;
    mcm::StepArgs A;
    // owned allocations
    double *d_fields = nullptr;
    double *d_stage = nullptr;   // host-array staging for upload/download (9 x npad), on first use
    int *d_ints = nullptr;
    mcm::DevMaterial *d_mats = nullptr;
    void *d_scalars = nullptr;     // DevTime, DevStatus, DevGrid, bbox, energy, counters
    int *d_nppermat = nullptr;
    // host mirrors (pinned)
    mcm::DevTime *h_time = nullptr;
    mcm::DevStatus *h_status = nullptr;
    mcm::DevGrid *h_grid = nullptr;
    double *h_bbox = nullptr;
    double *h_energy = nullptr;
    int *h_ngp = nullptr;
    std::string last_error;
    bool initialised = false;
    int red_cap = 0;
    double mean_nbr = 0.0;
    // profiling: CUDA events around each kernel group on the handle's stream
    bool prof_on = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_pairs[16];
    long long kernel_launches = 0;
    cudaEvent_t timer[2] = {nullptr, nullptr};
    long long steps_enqueued = 0;
    bool have_cells = false;   // cell_list holds a valid permutation
    // adjoint: prescribed dt schedule, checkpoints (fields + bbox), segment snapshots
    std::vector<double> adj_dts;
    int adj_steps = 0, adj_every = 0;
    int adj_kind = 1;   // reverse constitutive step: 1 hand-written reverse where the materials allow, 2 dual numbers
    std::vector<double *> adj_ckpt;
    double *adj_seg = nullptr;
    int adj_seg_cap = 0;
    double *adj_final = nullptr;
    double *d_adj = nullptr;     // adjoint arrays (40 x npad)
    // per-step record of a segment's forward pass for the reverse sweep (lists,
    // ghosts, post-step fields), kept when the device has room for a segment
    struct StepRecord { char *buf = nullptr; size_t bytes = 0; int nstride = 0, gstride = 0, ghost_cap = 0; };
    std::vector<StepRecord> adj_rec;
    int last_max_gnbr = 0;       // longest ghost-neighbour list of the last step_a
    // split loop: step_a enqueues the momentum sum (independent of the new dt)
    // behind part A and waits only for part A (an event), so the GPU computes
    // the forces while the caller updates dt; step_b then enqueues nothing
    cudaEvent_t part_a_done = nullptr;
    bool part_b_enqueued = false;
    double tuned_ms = 0.0;       // mcm_gpu_autotune: time per iteration of the chosen launch shape
    double *d_theta = nullptr;   // parameter adjoints (nmat x 4)
};


namespace mcm_host {

using namespace mcm;

inline int set_error(mcm_gpu_handle *h, int code, const std::string &msg) {
    if (h) h->last_error = msg;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return set_error(h, e_ == cudaErrorMemoryAllocation ? MCM_ENOMEM : MCM_ECUDA,          \
                             std::string(#call) + " (" + __FILE__ + ":" + std::to_string(__LINE__) +   \
                                 "): " + cudaGetErrorString(e_));                                  \
    } while (0)

template <typename T>
inline int dalloc(mcm_gpu_handle *h, T **p, size_t count) {
    if (*p) { cudaFree(*p); *p = nullptr; }
    if (count == 0) count = 1;
    CK(cudaMalloc((void **)p, sizeof(T) * count));
    return MCM_OK;
}

inline int round_up(int x, int m) { return ((x + m - 1) / m) * m; }

// Kernel groups that the profiler times separately.
enum Region {
    R_CELLS = 0, R_GHOSTS, R_SEARCH, R_STRAIN_PREP, R_STRAIN, R_CONST, R_CRITTS, R_MOM_PREP, R_MOMENTUM,
    R_REDUCE, R_MOVE, R_MISC, R_ADJ_MOM, R_ADJ_CONST, R_ADJ_STRAIN, R_NREG
};
extern const char *kRegionName[R_NREG];

inline cudaEvent_t take_event(mcm_gpu_handle *h) {
    if (h->ev_pool.empty()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    cudaEvent_t e = h->ev_pool.back();
    h->ev_pool.pop_back();
    return e;
}

// Counts the kernels of a group and, when profiling, brackets them with events.
struct Scope {
    mcm_gpu_handle *h;
    int r;
    cudaEvent_t b = nullptr;
    Scope(mcm_gpu_handle *h_, int r_, int nkernels) : h(h_), r(r_) {
        h->kernel_launches += nkernels;
        if (h->prof_on) {
            b = take_event(h);
            cudaEventRecord(b, h->stream);
        }
    }
    ~Scope() {
        if (b) {
            cudaEvent_t e = take_event(h);
            cudaEventRecord(e, h->stream);
            h->prof_pairs[r].push_back({b, e});
        }
    }
};

// abi.cu
int reset_status(mcm_gpu_handle *h);
int sync_status(mcm_gpu_handle *h);
int regrow(mcm_gpu_handle *h, int *grew);
int alloc_table(mcm_gpu_handle *h, int nstride, int gstride);
void enqueue_part_a(mcm_gpu_handle *h);
void enqueue_part_b(mcm_gpu_handle *h, int integrate);
int check_handle(mcm_gpu_handle *h);
size_t snap_doubles(const mcm_gpu_handle *h);
int snap_save(mcm_gpu_handle *h, double *buf);
int snap_load(mcm_gpu_handle *h, const double *buf);

}  // namespace mcm_host
