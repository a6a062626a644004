// reduce.cu -- grid-level reductions and the device-side time scalars of the
// MCM step: critical timestep minimum (MCM/mcm_calccritts.f90:82-85), the dt
// update (MCM/mcm_solution.f90:58-62) and termination test (:101), the
// per-material energy sums (MCM/mcm_calctotale.f90:27-60) and the coordinate
// bounding box (MCM/mcm_move.f90:25-39).  Block partials are combined in a
// fixed order, so the results do not depend on scheduling.
#include "kernels.h"

namespace mcm {

// One block: minimum over the block partials of k_strain_const / k_init_critts.
// fused == 1 also advances the time scalars on the device.
__global__ void k_critts_reduce(StepArgs a, int nblocks, int fused, int init) {
    __shared__ double sm[32];
    if (a.status->code) return;
    if (a.time->ended >= 2) return;
    double v = 1.0e20;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v = fmin(v, a.red[b]);
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 1.0e20;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmin(m, sm[k]);
        DevTime *t = a.time;
        t->critts = m;
        if (init) return;
        if (a.prm.h_opt) {
            // the largest h of this step's mcm_update_h becomes the next grid's hmax
            // (kept when no particle was at or above its cut-off pressure)
            unsigned long long *bid = reinterpret_cast<unsigned long long *>(a.hmax + 1);
            const unsigned long long b = *bid;
            if (b) a.hmax[0] = __longlong_as_double(static_cast<long long>(b));
            *bid = 0ull;
        }
        if (fused) {
            t->dtold = t->dt;
            double dt = a.prm.tssf * m;
            double lim = 1.1 * t->dtold;
            t->dt = (lim < dt) ? lim : dt;
            t->ptime = t->ptime + t->dt;
            if (t->ptime - t->dt >= t->endtime) t->ended = 1;
        }
    }
}

// Grid of (5*nmat + 6) blocks: block v reduces value v over the partials.
// energy/bbox select which values are reduced.  The bbox is not refreshed in
// the step that terminates the run: there is no position update in it.
__global__ void k_energy_bbox_reduce(StepArgs a, int nblocks, int energy, int bbox) {
    __shared__ double sm[32];
    if (a.status->code || a.time->ended >= 2) return;
    const int nv = 5 * a.nmat + 6;
    const int v = blockIdx.x;
    const bool is_bbox = v >= 5 * a.nmat;
    if (is_bbox && (!bbox || a.time->ended != 0)) return;
    if (!is_bbox && !energy) return;
    const bool is_max = is_bbox && (v - 5 * a.nmat) >= 3;
    double acc = is_bbox ? (is_max ? -1.0e20 : 1.0e20) : 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        double x = a.red[(size_t)b * nv + v];
        acc = is_bbox ? (is_max ? fmax(acc, x) : fmin(acc, x)) : acc + x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        double y = __shfl_xor_sync(0xffffffffu, acc, o);
        acc = is_bbox ? (is_max ? fmax(acc, y) : fmin(acc, y)) : acc + y;
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = is_bbox ? (is_max ? -1.0e20 : 1.0e20) : 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = is_bbox ? (is_max ? fmax(r, sm[k]) : fmin(r, sm[k])) : r + sm[k];
        if (is_bbox) {
            int d = (v - 5 * a.nmat) % 3;
            a.bbox[(is_max ? 3 : 0) + d] = r;
        } else {
            a.energy[v] = r;
        }
    }
}

// Per-material block partials of the energy sums (MCM/mcm_calctotale.f90:
// 33-51) for bodies of several materials, enqueued before the cooperative
// momentum kernels, which then move particles and write only the bounding-box
// partials of the same rows.  Block b sums, material by material, particles
// b*T + tid + k*nblocks*T (T threads) and combines its threads in a fixed
// order, so the sums do not depend on scheduling.
__global__ void k_energy_step_partials(StepArgs a) {
    __shared__ double sm[32];
    if (a.status->code || a.time->ended >= 2) return;
    const int nv = 5 * a.nmat + 6;
    double *out = a.red + (size_t)blockIdx.x * nv;
    const double *const *f = a.F.f;
    for (int m = 1; m <= a.nmat; ++m) {
        double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
            if (a.F.mat[i] != m) continue;
            const double mass = f[FMASS][i], vabs = f[FVABS][i];
            acc[0] += 0.5 * mass * (vabs * vabs);
            acc[1] += f[FE][i];
            acc[2] += mass * fabs(f[FVX][i]);
            acc[3] += mass * fabs(f[FVY][i]);
            acc[4] += mass * fabs(f[FVZ][i]);
        }
        for (int c = 0; c < 5; ++c) {
            double x = acc[c];
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            __syncthreads();
            if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
            __syncthreads();
            if (threadIdx.x == 0) {
                double r = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sm[w];
                out[5 * (m - 1) + c] = r;
            }
        }
    }
}

// Per-material contact forces xcf, ycf, zcf (MCM/mcm_oldacceleration.f90:
// 52-55): one block per material sums mass x repulsion over the particles in
// state order, threads combined in a fixed order.
__global__ void k_contact_forces(StepArgs a, double *out) {
    __shared__ double sm[32];
    const int m = blockIdx.x + 1;
    const double *const *f = a.F.f;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < a.n; i += blockDim.x) {
        if (a.F.mat[i] != m) continue;
        const double mass = f[FMASS][i];
        acc[0] += mass * f[FRPX][i];
        acc[1] += mass * f[FRPY][i];
        acc[2] += mass * f[FRPZ][i];
    }
    for (int c = 0; c < 3; ++c) {
        double x = acc[c];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r += sm[w];
            out[3 * (m - 1) + c] = r;
        }
    }
}

// Totals after the per-material sums (MCM/mcm_calctotale.f90:53-60).
__global__ void k_energy_totals(StepArgs a) {
    if (a.status->code || a.time->ended >= 2) return;
    double ke = 0.0, ie = 0.0;
    for (int m = 0; m < a.nmat; ++m) { ke = ke + a.energy[5 * m]; ie = ie + a.energy[5 * m + 1]; }
    a.energy[5 * a.nmat] = ke;
    a.energy[5 * a.nmat + 1] = ie;
    a.energy[5 * a.nmat + 2] = ke + ie;
}

__global__ void k_set_time(StepArgs a, double dt, double dtold, int set_dtold) {
    a.time->dt = dt;
    if (set_dtold) a.time->dtold = dtold;
}

// End of a fused step: count it and turn "terminated in this step" into
// "terminated" so that later steps are skipped.
__global__ void k_finish_step(StepArgs a) {
    if (a.status->code) return;
    DevTime *t = a.time;
    if (t->ended >= 2) return;
    t->steps_done += 1;
    if (t->ended == 1) t->ended = 2;
}

void launch_critts_reduce(const StepArgs &a, cudaStream_t s, int nblocks) {
    k_critts_reduce<<<1, 1024, 0, s>>>(a, nblocks, a.split_mode ? 0 : 1, 0);
}

void launch_init_critts_reduce(const StepArgs &a, cudaStream_t s, int nblocks) {
    k_critts_reduce<<<1, 1024, 0, s>>>(a, nblocks, 0, 1);
}

void launch_energy_bbox_reduce(const StepArgs &a, cudaStream_t s, int nblocks, int energy, int bbox) {
    k_energy_bbox_reduce<<<5 * a.nmat + 6, 256, 0, s>>>(a, nblocks, energy, bbox);
    if (energy) k_energy_totals<<<1, 1, 0, s>>>(a);
}

void launch_energy_step_partials(const StepArgs &a, cudaStream_t s, int nblocks) {
    k_energy_step_partials<<<nblocks, 256, 0, s>>>(a);
}

void launch_contact_forces(const StepArgs &a, cudaStream_t s, double *out) {
    k_contact_forces<<<a.nmat, 256, 0, s>>>(a, out);
}

void launch_set_time(const StepArgs &a, cudaStream_t s, double dt, double dtold, int set_dtold) {
    k_set_time<<<1, 1, 0, s>>>(a, dt, dtold, set_dtold);
}

void launch_finish_step(const StepArgs &a, cudaStream_t s) { k_finish_step<<<1, 1, 0, s>>>(a); }

}  // namespace mcm
