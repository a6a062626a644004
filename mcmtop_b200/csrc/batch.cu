// batch.cu -- launch-shape tuning of one body and batched runs of many bodies.
//
// Neither has a counterpart in the reference, a serial code that advances one
// body.  The tuner times candidate launch shapes of the gather kernels on a
// saved copy of the state.  A batch advances many independent bodies (one
// handle each) together: one loop iteration of every body -- the kernels of
// mcm_gpu_run's iteration for each handle -- is captured once as a CUDA graph
// over a few streams ("lanes") and replayed, so a step of the whole ensemble
// costs one graph launch, and bodies of uneven size share the GPU instead of
// each under-filling it in turn.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "handle.h"

using namespace mcm;
using namespace mcm_host;

struct mcm_gpu_batch {
    std::vector<mcm_gpu_handle *> bodies;
    int lanes = 1;
    int device = 0;
    cudaStream_t origin = nullptr;
    std::vector<cudaStream_t> lane_streams;
    std::vector<int> lane_of;               // per body
    std::vector<cudaEvent_t> events;        // fork, then one join per lane
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;                      // re-capture before the next launch
    double tuned_ms = 0.0;
};

namespace mcm_host {
namespace {

// The fused loop iterations of mcm_gpu_run, enqueued on the handle's stream
// without host synchronisation.
void enqueue_iteration(mcm_gpu_handle *h) {
    enqueue_part_a(h);
    enqueue_part_b(h, 1);
    Scope sc(h, R_MISC, 1);
    launch_finish_step(h->A, h->stream);
}

// ------------------------------------------------------------------ tuning
struct Shape {
    int search, pair, bps, stride, kind;
};

int search_kind_of(const mcm_gpu_handle *h) { return (h->A.search_kind == 2 || h->A.search_kind == 3) ? h->A.search_kind : 1; }

void apply_shape(mcm_gpu_handle *h, const Shape &s) {
    h->A.search_kind = s.kind;
    h->A.search_threads = s.search;
    h->A.pair_threads = s.pair;
    h->A.pair_bps = s.bps;
}

int valid_block(int t) { return t == 0 || t == 64 || t == 128 || t == 256; }

// State of a body that a tuning run changes: particle fields, bbox and the
// device time scalars (the lists, ghosts and grid are rebuilt every step).
struct Saved {
    double *snap = nullptr;
    DevTime time;
    long long steps_enqueued = 0;
};

int save_body(mcm_gpu_handle *h, Saved &s) {
    if (!s.snap) CK(cudaMalloc((void **)&s.snap, sizeof(double) * snap_doubles(h)));
    int st;
    if ((st = snap_save(h, s.snap))) return st;
    CK(cudaMemcpyAsync(&s.time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    s.steps_enqueued = h->steps_enqueued;
    return MCM_OK;
}

int restore_body(mcm_gpu_handle *h, const Saved &s) {
    int st;
    if ((st = snap_load(h, s.snap))) return st;
    CK(cudaMemcpyAsync(h->A.time, &s.time, sizeof(DevTime), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->steps_enqueued = s.steps_enqueued;
    return MCM_OK;
}

mcm_gpu_time time_of(const DevTime &t) {
    mcm_gpu_time r;
    r.dt = t.dt;
    r.dtold = t.dtold;
    r.ptime = t.ptime;
    r.endtime = t.endtime;
    return r;
}

// ---------------------------------------------------------------- batches
int batch_error(mcm_gpu_batch *b, int body, int code, const std::string &msg) {
    if (body >= 0 && body < (int)b->bodies.size()) b->bodies[body]->last_error = msg;
    return code;
}

// CK for calls that belong to the batch rather than to one body: the message
// goes to the first body's handle.
#define BCK(call)                                                                                   \
    do {                                                                                            \
        const cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                      \
            return batch_error(b, 0, e_ == cudaErrorMemoryAllocation ? MCM_ENOMEM : MCM_ECUDA,      \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

// Largest body first onto the least loaded lane.
void assign_lanes(mcm_gpu_batch *b) {
    const int nb = (int)b->bodies.size();
    std::vector<int> order(nb);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->bodies[x]->np > b->bodies[y]->np; });
    std::vector<long long> load(b->lanes, 0);
    b->lane_of.assign(nb, 0);
    for (int k : order) {
        const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        b->lane_of[k] = l;
        load[l] += b->bodies[k]->np;
    }
    b->dirty = true;
}

int ensure_streams(mcm_gpu_batch *b) {
    while ((int)b->lane_streams.size() < b->lanes) {
        cudaStream_t s;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return MCM_ECUDA;
        b->lane_streams.push_back(s);
    }
    while ((int)b->events.size() < b->lanes + 1) {
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return MCM_ECUDA;
        b->events.push_back(e);
    }
    return MCM_OK;
}

void release_graph(mcm_gpu_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->dirty = true;
}

// Captures one loop iteration of every body: a fork from the origin stream
// to the lanes, each lane's bodies in turn, a join back to the origin.
int capture(mcm_gpu_batch *b) {
    release_graph(b);
    int st;
    if ((st = ensure_streams(b))) return st;
    const int nb = (int)b->bodies.size();
    std::vector<cudaStream_t> own(nb);
    std::vector<bool> prof(nb);
    for (int k = 0; k < nb; ++k) {
        mcm_gpu_handle *h = b->bodies[k];
        own[k] = h->stream;
        prof[k] = h->prof_on;
        h->prof_on = false;   // no event records inside the graph
        h->A.split_mode = 0;
    }
    cudaError_t e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaEventRecord(b->events[0], b->origin);
        for (int l = 0; l < b->lanes; ++l) cudaStreamWaitEvent(b->lane_streams[l], b->events[0], 0);
        for (int l = 0; l < b->lanes; ++l)
            for (int k = 0; k < nb; ++k) {
                if (b->lane_of[k] != l) continue;
                mcm_gpu_handle *h = b->bodies[k];
                h->stream = b->lane_streams[l];
                enqueue_iteration(h);
                h->stream = own[k];
            }
        for (int l = 0; l < b->lanes; ++l) {
            cudaEventRecord(b->events[1 + l], b->lane_streams[l]);
            cudaStreamWaitEvent(b->origin, b->events[1 + l], 0);
        }
        e = cudaStreamEndCapture(b->origin, &b->graph);
    }
    for (int k = 0; k < nb; ++k) {
        b->bodies[k]->stream = own[k];
        b->bodies[k]->prof_on = prof[k];
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) {
        release_graph(b);
        cudaGetLastError();
        return batch_error(b, 0, MCM_ECUDA, std::string("batch graph capture: ") + cudaGetErrorString(e));
    }
    b->dirty = false;
    return MCM_OK;
}

// Runs fn(body index) for every body of the batch on host worker threads
// (at most the batch's lane count, 16 and the bodies), largest bodies first,
// each body's calls on its own stream, so that the bodies' GPU work overlaps.
// Returns the first non-zero status (the other workers stop taking bodies).
template <typename F>
int for_each_body(mcm_gpu_batch *b, F &&fn) {
    const int nb = (int)b->bodies.size();
    std::vector<int> order(nb);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->bodies[x]->np > b->bodies[y]->np; });
    std::atomic<int> next{0}, err{0};
    const int nthreads = std::max(1, std::min({b->lanes, 16, nb}));
    auto work = [&]() {
        if (cudaSetDevice(b->device) != cudaSuccess) {
            int z = 0;
            err.compare_exchange_strong(z, (int)MCM_ECUDA);
            return;
        }
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= nb || err.load() != 0) return;
            const int st = fn(order[k]);
            if (st != MCM_OK) {
                int z = 0;
                err.compare_exchange_strong(z, st);
                return;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return err.load();
}

}  // namespace
}  // namespace mcm_host

extern "C" {

int mcm_gpu_set_tuning(mcm_gpu_handle *h, const mcm_gpu_tuning *t) {
    if (!h || !t) return MCM_EINVAL;
    if (!valid_block(t->search_threads) || !valid_block(t->pair_threads)) return MCM_EINVAL;
    if (t->pair_blocks_per_sm < 0 || t->pair_blocks_per_sm > 16 || t->nbr_stride < 0) return MCM_EINVAL;
    if (t->search_kind < 0 || t->search_kind > 3) return MCM_EINVAL;
    if (t->pair_kind < 0 || t->pair_kind > 2) return MCM_EINVAL;
    if (t->adj_kind < 0 || t->adj_kind > 2) return MCM_EINVAL;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (t->search_threads) h->A.search_threads = t->search_threads;
    if (t->search_kind) h->A.search_kind = t->search_kind;
    if (t->pair_kind) h->A.pair_kind = t->pair_kind;
    if (t->adj_kind) h->adj_kind = t->adj_kind;
    if (t->pair_threads) h->A.pair_threads = t->pair_threads;
    if (t->pair_blocks_per_sm) h->A.pair_bps = t->pair_blocks_per_sm;
    if (t->nbr_stride && t->nbr_stride != h->A.nstride) {
        int st;
        if ((st = alloc_table(h, t->nbr_stride, h->A.gstride))) return st;
    }
    return MCM_OK;
}

int mcm_gpu_get_tuning(mcm_gpu_handle *h, mcm_gpu_tuning *t) {
    if (!h || !t) return MCM_EINVAL;
    t->search_threads = search_threads_of(h->A);
    t->pair_threads = pair_threads_of(h->A);
    t->pair_blocks_per_sm = h->A.pair_bps > 0 ? h->A.pair_bps : 0;
    t->nbr_stride = h->A.nstride;
    t->search_kind = search_kind_of(h);
    t->pair_kind = h->A.pair_kind == 2 ? 2 : 1;
    t->adj_kind = h->adj_kind;
    t->ms_per_step = h->tuned_ms;
    return MCM_OK;
}

int mcm_gpu_autotune(mcm_gpu_handle *h, int nsteps, mcm_gpu_tuning *best) {
    int st;
    if ((st = check_handle(h))) return st;
    if (nsteps < 1) return MCM_EINVAL;
    // re-sorting permutes the integer arrays the snapshot does not hold: off while tuning
    const int every = h->cfg.reorder_interval;
    h->cfg.reorder_interval = 0;
    Saved saved;
    if ((st = save_body(h, saved))) { h->cfg.reorder_interval = every; return st; }
    cudaEvent_t e0 = take_event(h), e1 = take_event(h);
    const Shape cur = {search_threads_of(h->A), pair_threads_of(h->A), h->A.pair_bps > 0 ? h->A.pair_bps : 0,
                       h->A.nstride, search_kind_of(h)};
    auto timed = [&](const Shape &s, double *ms) -> int {
        int r;
        apply_shape(h, s);
        if (s.stride != h->A.nstride && (r = alloc_table(h, s.stride, h->A.gstride))) return r;
        if ((r = restore_body(h, saved))) return r;
        mcm_gpu_time t = time_of(saved.time);
        int done = 0;
        if ((r = mcm_gpu_run(h, 1, &t, &done))) return r;   // warm-up (and any regrow)
        t = time_of(saved.time);
        if ((r = restore_body(h, saved))) return r;
        cudaEventRecord(e0, h->stream);
        if ((r = mcm_gpu_run(h, nsteps, &t, &done))) return r;
        cudaEventRecord(e1, h->stream);
        CK(cudaEventSynchronize(e1));
        float f = 0.f;
        CK(cudaEventElapsedTime(&f, e0, e1));
        *ms = done > 0 ? (double)f / done : 1e30;
        return MCM_OK;
    };
    Shape bestS = cur;
    double bestMs = 1e30;
    // stage 1: block sizes and grid of the search and the gathers
    const int blocks[3] = {64, 128, 256};
    const int bpss[2] = {0, 8};   // 0: one wave of the resident blocks
    for (int sb : blocks)
        for (int pb : blocks)
            for (int g : bpss) {
                if (sb == 64 && pb != 64) continue;   // narrow searches only with narrow gathers
                const Shape s = {sb, pb, g, cur.stride, cur.kind};
                double ms = 0.0;
                if ((st = timed(s, &ms))) goto out;
                if (ms < bestMs) { bestMs = ms; bestS = s; }
            }
    // the other search kinds with the best block sizes
    for (int kind = 1; kind <= 3; ++kind) {
        if (kind == cur.kind) continue;
        Shape s = bestS;
        s.kind = kind;
        double ms = 0.0;
        if ((st = timed(s, &ms))) goto out;
        if (ms < bestMs) { bestMs = ms; bestS = s; }
    }
    // stage 2: neighbour-table stride, tight or rounded to 64-byte rows
    {
        const int need = std::max(h->h_status->max_nbr, 1);
        const int strides[2] = {((need + need / 16 + 4 + 3) / 4) * 4, ((need + need / 16 + 4 + 15) / 16) * 16};
        for (int sw : strides) {
            Shape s = bestS;
            s.stride = sw;
            double ms = 0.0;
            if ((st = timed(s, &ms))) goto out;
            if (ms < bestMs) { bestMs = ms; bestS = s; }
        }
    }
    apply_shape(h, bestS);
    if (bestS.stride != h->A.nstride) st = alloc_table(h, bestS.stride, h->A.gstride);
    h->tuned_ms = bestMs;
out:
    {
        const int r = restore_body(h, saved);
        if (!st) st = r;
    }
    h->ev_pool.push_back(e0);
    h->ev_pool.push_back(e1);
    cudaFree(saved.snap);
    h->cfg.reorder_interval = every;
    if (st) return st;
    if (best) mcm_gpu_get_tuning(h, best);
    return MCM_OK;
}

int mcm_gpu_batch_create(mcm_gpu_handle *const *bodies, int nbodies, int lanes, mcm_gpu_batch **out) {
    if (!bodies || nbodies < 1 || !out || lanes < 1 || lanes > 64) return MCM_EINVAL;
    *out = nullptr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MCM_ECUDA;
    for (int k = 0; k < nbodies; ++k) {
        mcm_gpu_handle *h = bodies[k];
        if (!h || !h->initialised) return MCM_EINVAL;
        if (h->device != dev) return set_error(h, MCM_EINVAL, "batch: bodies on different devices");
        if (h->cfg.reorder_interval != 0) return set_error(h, MCM_EUNSUPPORTED, "batch: reorder_interval must be 0");
        for (int j = 0; j < k; ++j)
            if (bodies[j] == h) return set_error(h, MCM_EINVAL, "batch: a body appears twice");
    }
    mcm_gpu_batch *b = new mcm_gpu_batch();
    b->bodies.assign(bodies, bodies + nbodies);
    b->lanes = std::min(lanes, nbodies);
    b->device = dev;
    if (cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) != cudaSuccess ||
        ensure_streams(b) != MCM_OK) {
        mcm_gpu_batch_destroy(b);
        return MCM_ECUDA;
    }
    assign_lanes(b);
    *out = b;
    return MCM_OK;
}

int mcm_gpu_batch_adjoint_forward(mcm_gpu_batch *b, int nsteps, const double *const *dts, int checkpoint_every) {
    if (!b || !dts || nsteps <= 0 || checkpoint_every <= 0) return MCM_EINVAL;
    for (size_t k = 0; k < b->bodies.size(); ++k)
        if (!dts[k]) return MCM_EINVAL;
    return for_each_body(b, [&](int k) { return mcm_gpu_adjoint_forward(b->bodies[k], nsteps, dts[k], checkpoint_every); });
}

int mcm_gpu_batch_adjoint_backward(mcm_gpu_batch *b, const double *const *xbar, const double *const *vbar,
                                   double *const *param_bar, double *const *xbar0, double *const *vbar0) {
    if (!b) return MCM_EINVAL;
    return for_each_body(b, [&](int k) {
        return mcm_gpu_adjoint_backward(b->bodies[k], xbar ? xbar[k] : nullptr, vbar ? vbar[k] : nullptr,
                                        param_bar ? param_bar[k] : nullptr, xbar0 ? xbar0[k] : nullptr,
                                        vbar0 ? vbar0[k] : nullptr);
    });
}

int mcm_gpu_batch_destroy(mcm_gpu_batch *b) {
    if (!b) return MCM_EINVAL;
    cudaSetDevice(b->device);
    if (b->origin) cudaStreamSynchronize(b->origin);
    release_graph(b);
    for (cudaStream_t s : b->lane_streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    if (b->origin) cudaStreamDestroy(b->origin);
    delete b;
    return MCM_OK;
}

int mcm_gpu_batch_run(mcm_gpu_batch *b, int nsteps, mcm_gpu_time *times, int *done) {
    if (!b || !times || nsteps < 0) return MCM_EINVAL;
    if (cudaSetDevice(b->device) != cudaSuccess) return MCM_ECUDA;
    const int nb = (int)b->bodies.size();
    std::vector<DevTime> t0(nb);
    for (int k = 0; k < nb; ++k) {
        mcm_gpu_handle *h = b->bodies[k];
        if (!h->initialised) return MCM_EINVAL;
        CK(cudaStreamSynchronize(h->stream));   // earlier work of the body is done
        std::memset(&t0[k], 0, sizeof(DevTime));
        t0[k].dt = times[k].dt;
        t0[k].dtold = times[k].dtold;
        t0[k].ptime = times[k].ptime;
        t0[k].endtime = times[k].endtime;
        CK(cudaMemcpyAsync(h->A.time, &t0[k], sizeof(DevTime), cudaMemcpyHostToDevice, b->origin));
        CK(cudaMemsetAsync(h->A.status, 0, sizeof(DevStatus), b->origin));
        if (done) done[k] = 0;
    }
    int st = MCM_OK;
    int total = 0;
    std::vector<int> count(nb, 0);
    while (total < nsteps) {
        const int k = std::min(nsteps - total, 64);
        if (b->dirty && (st = capture(b))) break;
        for (int i = 0; i < k; ++i) {
            const cudaError_t e = cudaGraphLaunch(b->exec, b->origin);
            if (e != cudaSuccess) return batch_error(b, 0, MCM_ECUDA, std::string("batch launch: ") + cudaGetErrorString(e));
        }
        for (int j = 0; j < nb; ++j) {
            mcm_gpu_handle *h = b->bodies[j];
            CK(cudaMemcpyAsync(h->h_status, h->A.status, sizeof(DevStatus), cudaMemcpyDeviceToHost, b->origin));
            CK(cudaMemcpyAsync(h->h_time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost, b->origin));
        }
        BCK(cudaStreamSynchronize(b->origin));
        for (int j = 0; j < nb; ++j) {
            mcm_gpu_handle *h = b->bodies[j];
            const int ran = h->h_time->steps_done;
            const int code = h->h_status->code;
            const bool ended = h->h_time->ended >= 2;
            count[j] += ran;
            CK(cudaMemsetAsync(&h->A.time->steps_done, 0, sizeof(int), b->origin));
            CK(cudaMemsetAsync(h->A.status, 0, sizeof(DevStatus), b->origin));
            if (code == MCM_OK || ended) continue;
            // storage too small: regrow, then bring the body level on its own stream
            int grew = 0;
            if ((st = regrow(h, &grew))) return st;
            if (!grew) return set_error(h, code, mcm_gpu_strerror(code));
            b->dirty = true;
            CK(cudaStreamSynchronize(b->origin));
            mcm_gpu_time t = time_of(*h->h_time);
            int d = 0;
            if ((st = mcm_gpu_run(h, k - ran, &t, &d))) return st;
            count[j] += d;
            CK(cudaMemsetAsync(&h->A.time->steps_done, 0, sizeof(int), b->origin));
            CK(cudaMemsetAsync(h->A.status, 0, sizeof(DevStatus), b->origin));
        }
        total += k;
    }
    BCK(cudaStreamSynchronize(b->origin));
    for (int j = 0; j < nb; ++j) {
        mcm_gpu_handle *h = b->bodies[j];
        CK(cudaMemcpy(h->h_time, h->A.time, sizeof(DevTime), cudaMemcpyDeviceToHost));
        times[j] = time_of(*h->h_time);
        h->A.split_mode = 1;
        if (done) done[j] = count[j];
    }
    return st;
}

int mcm_gpu_batch_autotune(mcm_gpu_batch *b, int nsteps, int *lanes, double *ms_per_step) {
    if (!b || nsteps < 1) return MCM_EINVAL;
    if (cudaSetDevice(b->device) != cudaSuccess) return MCM_ECUDA;
    const int nb = (int)b->bodies.size();
    std::vector<Saved> saved(nb);
    int st = MCM_OK;
    for (int k = 0; k < nb && !st; ++k) st = save_body(b->bodies[k], saved[k]);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int bestL = b->lanes;
    double bestMs = 1e30;
    if (!st && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) st = MCM_ECUDA;
    const int cand[6] = {2, 4, 8, 16, 32, 64};
    std::vector<mcm_gpu_time> t(nb);
    for (int c = 0; c < 6 && !st; ++c) {
        const int L = std::min(cand[c], nb);
        if (c > 0 && L == std::min(cand[c - 1], nb)) continue;
        b->lanes = L;
        assign_lanes(b);
        for (int k = 0; k < nb && !st; ++k) st = restore_body(b->bodies[k], saved[k]);
        for (int k = 0; k < nb; ++k) t[k] = time_of(saved[k].time);
        if (!st) st = mcm_gpu_batch_run(b, 1, t.data(), nullptr);   // capture + warm-up
        for (int k = 0; k < nb && !st; ++k) st = restore_body(b->bodies[k], saved[k]);
        for (int k = 0; k < nb; ++k) t[k] = time_of(saved[k].time);
        if (st) break;
        cudaEventRecord(e0, b->origin);
        st = mcm_gpu_batch_run(b, nsteps, t.data(), nullptr);
        cudaEventRecord(e1, b->origin);
        if (st) break;
        float f = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&f, e0, e1) != cudaSuccess) {
            st = MCM_ECUDA;
            break;
        }
        const double ms = (double)f / nsteps;
        if (ms < bestMs) { bestMs = ms; bestL = L; }
    }
    b->lanes = bestL;
    assign_lanes(b);
    b->tuned_ms = bestMs;
    for (int k = 0; k < nb; ++k) {
        if (saved[k].snap) {
            const int r = restore_body(b->bodies[k], saved[k]);
            if (!st) st = r;
            cudaFree(saved[k].snap);
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) return st;
    if (lanes) *lanes = bestL;
    if (ms_per_step) *ms_per_step = bestMs;
    return MCM_OK;
}

}  // extern "C"
