// step_mixed.cu -- the mixed-precision explicit step.
//
// The pair sums (strain rate, momentum) run in FP32 over FP32 gather records;
// every per-particle field stays FP64, and so do the constitutive update (the
// FP64 fast one), the velocity and position update, the energy sums and the
// critical-timestep minimum.  An FP32 density could not follow a weakly
// compressible fluid, whose per-step density change (~1e-9 relative) is below
// FP32 resolution; FP32 pair terms only carry a relative rounding error.  The
// neighbour search is the shared FP64-exact one, so neighbour sets are those
// of the reference.
//
// Cell-relative positions: the gather records hold each particle's position
// relative to the origin of its cell (FP32, |offset| < one cell), and every
// neighbour-list entry carries the offset of the neighbour's cell from the
// particle's (its 5-bit cell code), so x_i - x_j = (r_i - r_j) - db * cell
// size is formed from small numbers and keeps FP32 relative accuracy at the
// scale of h.  Ghost neighbours (few, near the planes) use FP64 positions.
//
// Compensated sums: 2 lanes share one particle's neighbours, so a lane adds
// about K/2 terms (40) in plain FP32; the two partial sums are combined with
// an error-free TwoSum shuffle step that carries the rounding error of the
// addition, and the result is rounded once to FP64.  Measured on the 2M bar
// (worst field's error against the FP64 step after 205 steps; mixed step
// throughput): 2 lanes plain 1.20e-5, 402 M particle-steps/s; 2 lanes with
// per-lane Kahan sums 1.00e-5, 374 M; 1 lane plain 1.57e-5, 377 M; 1 lane
// Kahan 1.33e-5, 358 M; 4 lanes plain 1.25e-5, 385 M; 16 lanes 6.3e-6, 328 M.
// The error is that of the FP32 pair terms rather than of their sum, and the
// Kahan registers cost occupancy, so the lanes sum plainly.  Two lanes (about
// 40 neighbours in flight per lane, one shuffle level) hide the record-gather
// latency best: strain/momentum 0.78/1.11 ms per step.
#include "nbr_iter.cuh"

namespace mcm {
namespace mixed {

constexpr int L = 2;           // lanes per particle
constexpr float kPiF = 3.14159265358979f;

__device__ __forceinline__ bool skip_step(const StepArgs &a) { return a.status->code || a.time->ended >= 2; }

// ------------------------------------------------------- compensated sums
// Sum of one value per lane over the L lanes of a sub-warp, every addition
// error-free transformed (TwoSum) and the errors added up; every lane gets it.
// c: a correction the lane already carries (the compensation of a Kahan sum).
__device__ __forceinline__ double lane_sum(float s, float c = 0.0f) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) {
        const float s2 = __shfl_xor_sync(0xffffffffu, s, o, L);
        const float c2 = __shfl_xor_sync(0xffffffffu, c, o, L);
        const float t = s + s2;
        const float bp = t - s;
        const float err = (s - (t - bp)) + (s2 - bp);
        s = t;
        c = c + c2 + err;
    }
    return (double)s + (double)c;
}

// ------------------------------------------------------------ geometry
struct Frame {
    double gmin[3], cs[3];
    float csf[3];
    int gl[3];
};
__device__ __forceinline__ Frame make_frame(const DevGrid &g) {
    Frame fr;
    for (int d = 0; d < 3; ++d) {
        fr.gmin[d] = g.gridmin[d];
        fr.cs[d] = 1.0 / g.gridsize[d];
        fr.csf[d] = (float)fr.cs[d];
        fr.gl[d] = g.gridlim[d];
    }
    return fr;
}
__device__ __forceinline__ void frame_origin(const Frame &fr, int key, double o[3]) {
    if (key < 0) { o[0] = o[1] = o[2] = 0.0; return; }
    int b[3];
    cell_coords(key, fr.gl, b[0], b[1], b[2]);
    for (int d = 0; d < 3; ++d) o[d] = fr.gmin[d] + (double)(b[d] - 1) * fr.cs[d];
}

// Offsets of the 27 neighbour cells (cell size times -1, 0, 1 per axis), by code.
__device__ __forceinline__ void fill_offsets(float4 *tab, const Frame &fr) {
    if (threadIdx.x < 27) {
        const int c = threadIdx.x;
        tab[c] = make_float4((float)(c % 3 - 1) * fr.csf[0], (float)((c / 3) % 3 - 1) * fr.csf[1],
                             (float)(c / 9 - 1) * fr.csf[2], 0.0f);
    }
}

// Gather records.  A strain record is 32 bytes {x, y, z, h, vx, vy, vz, V}
// and a momentum record 48 bytes {x, y, z, h, s11, s22, s33, s12 | s13, s23,
// m, rho} in a 64-byte slot, so that one neighbour costs one (strain) or two
// (momentum) 32-byte sectors, each fetched by a single 256-bit or 128-bit load.
struct __align__(32) Rec8 {
    float4 a, b;
};
__device__ __forceinline__ Rec8 ld_rec8(const float4 *p) {
    Rec8 r;
    asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=f"(r.a.x), "=f"(r.a.y), "=f"(r.a.z), "=f"(r.a.w), "=f"(r.b.x), "=f"(r.b.y), "=f"(r.b.z),
                   "=f"(r.b.w)
                 : "l"(p));
    return r;
}
__device__ __forceinline__ float4 ld_rec4(const float4 *p) { return __ldg(p); }

// Cubic B-spline gradient in FP32 (MCM/mcm_gradw.f90:64-101), ih = 1/havg.
__device__ __forceinline__ void gradw_f(float x0, float x1, float x2, float ih, float &d0, float &d1, float &d2) {
    const float r2 = fmaf(x0, x0, fmaf(x1, x1, x2 * x2));
    if (r2 == 0.0f) { d0 = d1 = d2 = 0.0f; return; }
    const float rinv = rsqrtf(r2);
    const float z = r2 * rinv * ih;
    const float const1 = (1.0f / kPiF) * ih * ih * ih;
    float dw;
    if (z < 1.0f) dw = const1 * ((2.25f * z - 3.0f) * z);
    else if (z < 2.0f) { const float tt = 2.0f - z; dw = -0.75f * const1 * (tt * tt); }
    else dw = 0.0f;
    const float f = dw * ih * rinv;
    d0 = f * x0; d1 = f * x1; d2 = f * x2;
}

__device__ __forceinline__ float inv_havg_f(float hi, float hj, float ihi) {
    return (hi == hj) ? ihi : 2.0f / (hi + hj);
}

static inline int nblk(int n, int t) { return (n + t - 1) / t; }

// Kahan (compensated) addition of term to the sum (s, c): c carries the
// low-order part that s lost, so s + c is the sum to about one FP32 rounding
// over all the terms instead of one per addition.  Used by the compensated
// variant of the pair sums (mcm_gpu_config.compensated_sums).
__device__ __forceinline__ void kahan_add(float &s, float &c, float term) {
    const float y = term + c;
    const float t = s + y;
    c = y - (t - s);
    s = t;
}

// ------------------------------------------------------------ strain prep
// MCM/mcm_strain.f90:27-31 (x - v dt/2) and V_j = m_j/rho_j, cell-relative.
__global__ void k_strain_prep(StepArgs a) {
    if (skip_step(a)) return;
    const double dt = a.time->dt;
    const Frame fr = make_frame(*a.grid);
    const double *const *f = a.F.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int i = a.cell_list[p];
        double o[3];
        frame_origin(fr, a.ckey[p], o);
        const double vx = f[FVX][i], vy = f[FVY][i], vz = f[FVZ][i];
        const double xs = f[FX][i] - 0.5 * vx * dt, ys = f[FY][i] - 0.5 * vy * dt, zs = f[FZ][i] - 0.5 * vz * dt;
        a.frec0[2 * (size_t)p] = make_float4((float)(xs - o[0]), (float)(ys - o[1]), (float)(zs - o[2]), (float)f[FH][i]);
        a.frec0[2 * (size_t)p + 1] = make_float4((float)vx, (float)vy, (float)vz, (float)(f[FMASS][i] / f[FRHO][i]));
    }
    if (a.prm.boundary) {
        const int ngp = *a.ngp;
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngp; g += gridDim.x * blockDim.x) {
            a.grec0[g] = make_double4(a.gx[g], a.gy[g], a.gz[g], a.gh[g]);
            a.gfrec1[g] = make_float4((float)a.gvx[g], (float)a.gvy[g], (float)a.gvz[g], (float)(a.gmass[g] / a.grho[g]));
        }
    }
}

// ----------------------------------------------------------- strain rate
// Neighbours a gather lane loads ahead before it uses the first (strain,
// momentum), and the momentum gather's resident blocks per SM.
#ifndef MCM_STRAIN_UNROLL
#define MCM_STRAIN_UNROLL 4
#endif
#ifndef MCM_MOM_UNROLL
#define MCM_MOM_UNROLL 1
#endif
#ifndef MCM_MOM_MINBLOCKS
#define MCM_MOM_MINBLOCKS 4
#endif
constexpr int kUnroll = MCM_STRAIN_UNROLL;

// The list entries base[0 .. 2U) of one particle's two lanes, lane l getting
// entries l, l + 2, ..., l + 2(U - 1) (list order within the lane): each lane
// loads U consecutive entries in 16-byte pieces and the two lanes swap the
// halves the other needs.  A warp's index loads touch 16 rows of the table
// (one per particle), so fewer, wider loads mean fewer L1 wavefronts.  base
// is 16-byte aligned (rows start at multiples of 4 entries); both lanes of
// the pair call this together.
template <int U>
__device__ __forceinline__ void pair_entries(const unsigned *base, int lane, unsigned (&e)[U]) {
    static_assert(L == 2 && U % 4 == 0, "two lanes per particle, 4 entries per 16-byte load");
    const unsigned pm = 3u << (threadIdx.x & 30);
#pragma unroll
    for (int v = 0; v < U / 4; ++v) {
        // lane 0 loads entries 8v .. 8v+3, lane 1 entries 8v+4 .. 8v+7
        const uint4 w = __ldg(reinterpret_cast<const uint4 *>(base + 8 * v + 4 * lane));
        const unsigned r0 = __shfl_xor_sync(pm, lane ? w.x : w.y, 1);
        const unsigned r1 = __shfl_xor_sync(pm, lane ? w.z : w.w, 1);
        e[4 * v + 0] = lane ? r0 : w.x;
        e[4 * v + 1] = lane ? r1 : w.z;
        e[4 * v + 2] = lane ? w.y : r0;
        e[4 * v + 3] = lane ? w.w : r1;
    }
}

// One pair's terms of MCM/mcm_oldstrain.f90:42-53: V_j (v_j - v_i)_n dW/dx_m
// added to gv[3n + m] (KAHAN: compensated, the low parts in gc).
template <bool KAHAN>
__device__ __forceinline__ void strain_term(float dx, float dy, float dz, float hj, float4 vj, float hi, float ihi,
                                            float4 vi, float (&gv)[9], float (&gc)[9]) {
    float d0, d1, d2;
    gradw_f(dx, dy, dz, inv_havg_f(hi, hj, ihi), d0, d1, d2);
    const float t0 = vj.w * (vj.x - vi.x), t1 = vj.w * (vj.y - vi.y), t2 = vj.w * (vj.z - vi.z);
    if (KAHAN) {
        const float tt[3] = {t0, t1, t2}, dd[3] = {d0, d1, d2};
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
            for (int m = 0; m < 3; ++m) kahan_add(gv[3 * n + m], gc[3 * n + m], tt[n] * dd[m]);
    } else {
        gv[0] = fmaf(t0, d0, gv[0]); gv[1] = fmaf(t0, d1, gv[1]); gv[2] = fmaf(t0, d2, gv[2]);
        gv[3] = fmaf(t1, d0, gv[3]); gv[4] = fmaf(t1, d1, gv[4]); gv[5] = fmaf(t1, d2, gv[5]);
        gv[6] = fmaf(t2, d0, gv[6]); gv[7] = fmaf(t2, d1, gv[7]); gv[8] = fmaf(t2, d2, gv[8]);
    }
}

// MCM/mcm_oldstrain.f90:34-64 with FP32 pair sums (KAHAN: compensated per
// lane, the compensation carried into the TwoSum lane combination).
template <bool KAHAN>
__global__ void __launch_bounds__(256, 3) k_strain(StepArgs a) {
    __shared__ float4 offs[27];
    if (skip_step(a)) return;
    const int sub = threadIdx.x / L, lane = threadIdx.x % L;
    const int per = blockDim.x / L;
    const int rounds = (a.n + per * gridDim.x - 1) / (per * gridDim.x);
    const DevGrid g = *a.grid;
    const Frame fr = make_frame(g);
    fill_offsets(offs, fr);
    __syncthreads();
    const double dt = a.time->dt;
    for (int round = 0; round < rounds; ++round) {
        const int t = (round * gridDim.x + blockIdx.x) * per + sub;
        const bool live = t < a.n;
        int nreal = 0, gn = 0, i = 0;
        float4 xi = make_float4(0.f, 0.f, 0.f, 1.f), vi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            nreal = a.nnbr[t];
            gn = a.gnnbr[t];
            const Rec8 r = ld_rec8(a.frec0 + 2 * (size_t)t);
            xi = r.a;
            vi = r.b;
            i = a.cell_list[t];
        }
        const unsigned *spos = a.nidx + (size_t)t * a.nstride;
        double xs[3] = {0.0, 0.0, 0.0};
        if (live && gn > 0) {
            xs[0] = a.F.f[FX][i] - 0.5 * a.F.f[FVX][i] * dt;
            xs[1] = a.F.f[FY][i] - 0.5 * a.F.f[FVY][i] * dt;
            xs[2] = a.F.f[FZ][i] - 0.5 * a.F.f[FVZ][i] * dt;
        }
        const int total = live ? nreal + gn : 0;
        const float ihi = 1.0f / xi.w;
        float gv[9], gc[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) { gv[u] = 0.0f; gc[u] = 0.0f; }
        // real neighbours kUnroll at a time per lane (their list entries and
        // records loaded before any is used, so that several gathers are in
        // flight), then the rest; each lane adds its terms in list order
        int k = lane;
        for (; k - lane + kUnroll * L <= nreal; k += kUnroll * L) {
            unsigned e[kUnroll];
            pair_entries<kUnroll>(spos + (k - lane), lane, e);
            Rec8 r[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) r[u] = ld_rec8(a.frec0 + 2 * (size_t)(e[u] & kPosMask));
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                const float4 o = offs[e[u] >> 26];
                strain_term<KAHAN>((xi.x - r[u].a.x) - o.x, (xi.y - r[u].a.y) - o.y, (xi.z - r[u].a.z) - o.z,
                                   r[u].a.w, r[u].b, xi.w, ihi, vi, gv, gc);
            }
        }
        for (; k < nreal; k += L) {
            const unsigned e = spos[k];
            const float4 o = offs[e >> 26];
            const Rec8 r = ld_rec8(a.frec0 + 2 * (size_t)(e & kPosMask));
            strain_term<KAHAN>((xi.x - r.a.x) - o.x, (xi.y - r.a.y) - o.y, (xi.z - r.a.z) - o.z, r.a.w, r.b, xi.w,
                               ihi, vi, gv, gc);
        }
        for (; k < total; k += L) {
            const int q = a.gnbr[(size_t)(k - nreal) * a.npad + t];
            const double4 xj = a.grec0[q];
            strain_term<KAHAN>((float)(xs[0] - xj.x), (float)(xs[1] - xj.y), (float)(xs[2] - xj.z), (float)xj.w,
                               a.gfrec1[q], xi.w, ihi, vi, gv, gc);
        }
        double r[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) r[u] = lane_sum(gv[u], KAHAN ? gc[u] : 0.0f);
        if (live && lane == 0) {
            // MCM/mcm_oldstrain.f90:56-63
            double *const *f = a.F.f;
            f[FR11][i] = r[0];
            f[FR22][i] = r[4];
            f[FR33][i] = r[8];
            f[FR12][i] = 0.5 * (r[1] + r[3]);
            f[FR13][i] = 0.5 * (r[2] + r[6]);
            f[FR23][i] = 0.5 * (r[5] + r[7]);
            f[FW12][i] = 0.5 * (r[1] - r[3]);
            f[FW13][i] = 0.5 * (r[2] - r[6]);
            f[FW23][i] = 0.5 * (r[5] - r[7]);
            f[FTR][i] = r[0] + r[4] + r[8];
        }
        __syncwarp();
    }
}

// ------------------------------------------- strain rate, rows staged
// The same sums as k_strain<false>, with a particle's neighbour records read
// from shared memory.  A block takes 64 consecutive cell-order positions per
// round; they lie in one row of cells (or two consecutive rows), and their
// neighbours lie in the 9 rows of cells around each: for every such row the
// contiguous range of positions from one cell left of the block's first cell
// to one cell right of its last is a window, copied into shared memory by
// coalesced loads (up to kStageCap records; windows that do not fit are read
// from global memory as in k_strain).  An entry's window follows from its
// cell code, so the lookup is one comparison.  Results are bitwise k_strain's.
constexpr int kStageThreads = 128;
constexpr int kStageCap = 1024;    // strain records of 32 bytes
constexpr int kStageCapM = 896;    // momentum records of 48 bytes

// The windows of one round: for row b (0, or 1 when the block reaches into
// the next row of cells) and each of the 9 rows of cells around it, window
// 9b + r covers positions [lo, lo + len), staged at record offset off.
struct StageWin {
    int lo[18], len[18], off[18];
    int row0;   // row of cells (key / gridlim x) of the block's first position
};

// Computes the windows of the positions [tb, tb + per) and copies the records
// (NF float4 each: record p's first two at src + 2p, a third at src2 + p) of
// those that fit in `cap` records into stage.  Every thread of the block calls
// it; it synchronises.
template <int NF>
__device__ __forceinline__ void stage_rows(const StepArgs &a, int tb, int per, StageWin &W, float4 *stage, int cap,
                                           const float4 *src, const float4 *src2) {
    const int gl0 = a.grid->gridlim[0], gl1 = a.grid->gridlim[1], gl2 = a.grid->gridlim[2];
    if (threadIdx.x < 18) {
        const int w = threadIdx.x;
        int lo = 0, len = 0;
        const int te = min(tb + per, a.n) - 1;
        if (tb < a.n) {
            const int k0 = a.ckey[tb], k1 = a.ckey[te];
            if (k0 >= 0 && k1 >= 0) {
                const int r0 = k0 / gl0, r1 = k1 / gl0;
                const int rr = r0 + (w >= 9 ? 1 : 0);
                if (r1 - r0 <= 1 && rr <= r1) {
                    const int xa = (rr == r0) ? k0 % gl0 + 1 : 1;
                    const int xb = (rr == r1) ? k1 % gl0 + 1 : gl0;
                    const int y = rr % gl1 + 1, z = rr / gl1 + 1;
                    const int rc = w % 9;
                    const int ty = y + rc % 3 - 1, tz = z + rc / 3 - 1;
                    if (ty >= 1 && ty <= gl1 && tz >= 1 && tz <= gl2) {
                        const int xl = xa > 1 ? xa - 1 : 1, xh = xb < gl0 ? xb + 1 : gl0;
                        const int ka = (xl - 1) + gl0 * ((ty - 1) + gl1 * (tz - 1));
                        const int kb = (xh - 1) + gl0 * ((ty - 1) + gl1 * (tz - 1));
                        lo = a.cell_start[ka];
                        len = a.cell_start[kb + 1] - lo;
                    }
                }
            }
        }
        W.lo[w] = lo;
        W.len[w] = len;
    }
    if (threadIdx.x == 0) W.row0 = (tb < a.n && a.ckey[tb] >= 0) ? a.ckey[tb] / gl0 : -1;
    __syncthreads();
    if (threadIdx.x == 0) {
        int off = 0;
        for (int w = 0; w < 18; ++w) {
            if (off + W.len[w] > cap) W.len[w] = 0;   // read from global memory
            W.off[w] = off;
            off += W.len[w];
        }
    }
    __syncthreads();
    for (int w = 0; w < 18; ++w) {
        const int lo = W.lo[w], len = W.len[w], o = W.off[w];
        for (int u = threadIdx.x; u < len; u += blockDim.x)
#pragma unroll
            for (int c = 0; c < NF; ++c)
                stage[NF * (o + u) + c] = c < 2 ? src[2 * (size_t)(lo + u) + c] : src2[lo + u];
    }
    __syncthreads();
}

// First window of position t's row of cells (0 or 9).
__device__ __forceinline__ int stage_base(const StepArgs &a, const StageWin &W, int t) {
    const int kt = a.ckey[t];
    return (kt >= 0 && kt / a.grid->gridlim[0] != W.row0) ? 9 : 0;
}

// Staged record index of neighbour entry e of a particle whose windows start
// at wbase, or -1 when the record was not staged.
__device__ __forceinline__ int stage_index(const StageWin &W, int wbase, unsigned e) {
    const int w = wbase + (int)((e >> 26) / 3u);
    const int u = (int)(e & kPosMask) - W.lo[w];
    return ((unsigned)u < (unsigned)W.len[w]) ? W.off[w] + u : -1;
}

__global__ void __launch_bounds__(kStageThreads, 6) k_strain_staged(StepArgs a) {
    __shared__ float4 offs[27];
    __shared__ float4 stage[2 * kStageCap];
    __shared__ StageWin W;
    if (skip_step(a)) return;
    const int sub = threadIdx.x / L, lane = threadIdx.x % L;
    constexpr int per = kStageThreads / L;
    const int rounds = (a.n + per * gridDim.x - 1) / (per * gridDim.x);
    const DevGrid g = *a.grid;
    const Frame fr = make_frame(g);
    fill_offsets(offs, fr);
    const double dt = a.time->dt;
    for (int round = 0; round < rounds; ++round) {
        const int tb = (round * gridDim.x + blockIdx.x) * per;
        stage_rows<2>(a, tb, per, W, stage, kStageCap, a.frec0, nullptr);
        const int t = tb + sub;
        const bool live = t < a.n;
        int nreal = 0, gn = 0, i = 0, wbase = 0;
        float4 xi = make_float4(0.f, 0.f, 0.f, 1.f), vi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            nreal = a.nnbr[t];
            gn = a.gnnbr[t];
            const Rec8 r = ld_rec8(a.frec0 + 2 * (size_t)t);
            xi = r.a;
            vi = r.b;
            i = a.cell_list[t];
            wbase = stage_base(a, W, t);
        }
        const unsigned *spos = a.nidx + (size_t)t * a.nstride;
        double xs[3] = {0.0, 0.0, 0.0};
        if (live && gn > 0) {
            xs[0] = a.F.f[FX][i] - 0.5 * a.F.f[FVX][i] * dt;
            xs[1] = a.F.f[FY][i] - 0.5 * a.F.f[FVY][i] * dt;
            xs[2] = a.F.f[FZ][i] - 0.5 * a.F.f[FVZ][i] * dt;
        }
        const int total = live ? nreal + gn : 0;
        const float ihi = 1.0f / xi.w;
        float gv[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) gv[u] = 0.0f;
        for (int k = lane; k < total; k += L) {
            float dx, dy, dz, hj;
            float4 vj;
            if (k < nreal) {
                const unsigned e = spos[k];
                const float4 o = offs[e >> 26];
                const int si = stage_index(W, wbase, e);
                float4 xj;
                if (si >= 0) {
                    xj = stage[2 * si];
                    vj = stage[2 * si + 1];
                } else {
                    const Rec8 r = ld_rec8(a.frec0 + 2 * (size_t)(e & kPosMask));
                    xj = r.a;
                    vj = r.b;
                }
                dx = (xi.x - xj.x) - o.x;
                dy = (xi.y - xj.y) - o.y;
                dz = (xi.z - xj.z) - o.z;
                hj = xj.w;
            } else {
                const int q = a.gnbr[(size_t)(k - nreal) * a.npad + t];
                const double4 xj = a.grec0[q];
                vj = a.gfrec1[q];
                dx = (float)(xs[0] - xj.x);
                dy = (float)(xs[1] - xj.y);
                dz = (float)(xs[2] - xj.z);
                hj = (float)xj.w;
            }
            float d0, d1, d2;
            gradw_f(dx, dy, dz, inv_havg_f(xi.w, hj, ihi), d0, d1, d2);
            const float t0 = vj.w * (vj.x - vi.x), t1 = vj.w * (vj.y - vi.y), t2 = vj.w * (vj.z - vi.z);
            gv[0] = fmaf(t0, d0, gv[0]); gv[1] = fmaf(t0, d1, gv[1]); gv[2] = fmaf(t0, d2, gv[2]);
            gv[3] = fmaf(t1, d0, gv[3]); gv[4] = fmaf(t1, d1, gv[4]); gv[5] = fmaf(t1, d2, gv[5]);
            gv[6] = fmaf(t2, d0, gv[6]); gv[7] = fmaf(t2, d1, gv[7]); gv[8] = fmaf(t2, d2, gv[8]);
        }
        double r[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) r[u] = lane_sum(gv[u]);
        if (live && lane == 0) {
            double *const *f = a.F.f;
            f[FR11][i] = r[0];
            f[FR22][i] = r[4];
            f[FR33][i] = r[8];
            f[FR12][i] = 0.5 * (r[1] + r[3]);
            f[FR13][i] = 0.5 * (r[2] + r[6]);
            f[FR23][i] = 0.5 * (r[5] + r[7]);
            f[FW12][i] = 0.5 * (r[1] - r[3]);
            f[FW13][i] = 0.5 * (r[2] - r[6]);
            f[FW23][i] = 0.5 * (r[5] - r[7]);
            f[FTR][i] = r[0] + r[4] + r[8];
        }
        __syncthreads();   // the next round overwrites the windows
    }
}

// Momentum records in three arrays of the 64-byte-per-position buffer:
// position p's first 32 bytes at frec0 + 2p (x y z h, A11 A22 A33 A12), the
// next 16 at frec0 + 2 npad + p (A13 A23 m rho) and the cap model's lower
// triangle at frec0 + 3 npad + p, so that neighbouring positions' records lie
// next to each other in every array.
__device__ __forceinline__ float4 *mom_tail(const StepArgs &a) { return a.frec0 + 2 * (size_t)a.npad; }
__device__ __forceinline__ float4 *mom_lower(const StepArgs &a) { return a.frec0 + 3 * (size_t)a.npad; }

// --------------------------------------------------------- momentum prep
// Records: cell-relative x, h; (sigma - q)/rho^2 (formed in FP64,
// MCM/mcm_oldacceleration.f90:79-80) and m (FP32).  Ghosts: FP64 positions,
// stresses with every off-diagonal negated (MCM/mcm_update_ghost_stress.f90:
// 272-285) over the ghost's own density.
__global__ void k_mom_prep(StepArgs a) {
    if (skip_step(a)) return;
    const Frame fr = make_frame(*a.grid);
    const double *const *f = a.F.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int i = a.cell_list[p];
        double o[3];
        frame_origin(fr, a.ckey[p], o);
        const double rho = f[FRHO][i];
        const double ir2 = 1.0 / (rho * rho);
        const double q = f[FQ][i];
        float4 *rec = a.frec0 + 2 * (size_t)p;
        rec[0] = make_float4((float)(f[FX][i] - o[0]), (float)(f[FY][i] - o[1]), (float)(f[FZ][i] - o[2]),
                             (float)f[FH][i]);
        rec[1] = make_float4((float)((f[FS11][i] - q) * ir2), (float)((f[FS22][i] - q) * ir2),
                                 (float)((f[FS33][i] - q) * ir2), (float)(f[FS12][i] * ir2));
        mom_tail(a)[p] = make_float4((float)(f[FS13][i] * ir2), (float)(f[FS23][i] * ir2), (float)f[FMASS][i], (float)rho);
        // the cap model's lower triangle (21 31 32), read only when a material has it
        if (a.prm.asym)
            mom_lower(a)[p] =
                make_float4((float)(f[FL21][i] * ir2), (float)(f[FL31][i] * ir2), (float)(f[FL32][i] * ir2), 0.0f);
    }
    if (a.prm.boundary) {
        const int ngp = *a.ngp;
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngp; g += gridDim.x * blockDim.x) {
            const int j = a.gpar[g];
            const double rho = a.grho[g];
            const double ir2 = 1.0 / (rho * rho);
            const double q = f[FQ][j];
            a.grec0[g] = make_double4(a.gx[g], a.gy[g], a.gz[g], a.gh[g]);
            a.gfrec1[g] = make_float4((float)((f[FS11][j] - q) * ir2), (float)((f[FS22][j] - q) * ir2),
                                      (float)((f[FS33][j] - q) * ir2), (float)(-f[FS12][j] * ir2));
            a.gfrec2[g] = make_float4((float)(-f[FS13][j] * ir2), (float)(-f[FS23][j] * ir2), (float)a.gmass[g],
                                      (float)rho);
            if (a.prm.asym)
                a.grec3[g] = make_double4(-f[FL21][j] * ir2, -f[FL31][j] * ir2, -f[FL32][j] * ir2, 0.0);
        }
    }
}

__device__ __forceinline__ double block_sum(double v, double *sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sm[k];
    return r;
}

__device__ __forceinline__ double block_minmax(double v, double *sm, bool is_max) {
    for (int o = 16; o > 0; o >>= 1) {
        double y = __shfl_xor_sync(0xffffffffu, v, o);
        v = is_max ? fmax(v, y) : fmin(v, y);
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[w] = v;
    __syncthreads();
    double r = v;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = is_max ? fmax(r, sm[k]) : fmin(r, sm[k]);
    return r;
}

// FP64 velocity and position update (MCM/mcm_update_velocity.f90:29-56,
// MCM/mcm_move.f90:32-40, MCM/mcm_check_sym_pen.f90:27-179 per particle).
__device__ __forceinline__ void integrate(const StepArgs &a, int i, const double acc[3], double dt, double dtold,
                                          double x[3]) {
    double *const *f = a.F.f;
    const double dtn = 0.5 * (dt + dtold);
    double v[3] = {f[FVX][i], f[FVY][i], f[FVZ][i]};
    double vabs = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        if (a.prm.drelax) v[j] = a.prm.drelax_scale * v[j] + acc[j] * dtn;
        else v[j] = v[j] + acc[j] * dtn;
        vabs = vabs + v[j] * v[j];
    }
    vabs = sqrt(vabs);
    x[0] = f[FX][i] + v[0] * dt;
    x[1] = f[FY][i] + v[1] * dt;
    x[2] = f[FZ][i] + v[2] * dt;
    double xo[3] = {x[0], x[1], x[2]};
    if (a.prm.boundary) {
        const DevPlanes &pl = a.prm.planes;
        for (int d = 0; d < 3; ++d) {
            if (pl.code[0][d] == 1 && xo[d] < pl.bx[0][d]) { xo[d] = 2.0 * pl.bx[0][d] - xo[d]; v[d] = -v[d]; }
            if (pl.code[1][d] == 1 && xo[d] > pl.bx[1][d]) { xo[d] = 2.0 * pl.bx[1][d] - xo[d]; v[d] = -v[d]; }
            if (pl.code[0][d] == 2) {
                const double span = pl.bx[1][d] - pl.bx[0][d];
                if (xo[d] < pl.bx[0][d]) xo[d] = xo[d] + span;
                if (xo[d] > pl.bx[1][d]) xo[d] = xo[d] - span;
            }
        }
    }
    f[FVX][i] = v[0]; f[FVY][i] = v[1]; f[FVZ][i] = v[2];
    f[FVABS][i] = vabs;
    f[FX][i] = xo[0]; f[FY][i] = xo[1]; f[FZ][i] = xo[2];
}

// ------------------------------------------------- momentum + integration
// MCM/mcm_oldacceleration.f90:66-89 with FP32 pair sums, then the FP64 tail:
// base acceleration and displacement BCs (MCM/mcm_boundcond.f90), energy
// partials (MCM/mcm_calctotale.f90) and, when integrating, the update.
// Four resident blocks (64 registers) hide the record gathers' latency
// better than three at 80 registers (measured with 16 lanes per particle:
// 1.70 against 2.19 ms per step on the 2M bar).
// STAGED: 128-thread blocks whose rows of neighbour records are staged in
// shared memory as in k_strain_staged (stage_rows); the same sums.
constexpr int kUnrollM = MCM_MOM_UNROLL;

// One pair's term of MCM/mcm_oldacceleration.f90:62-90 for a symmetric sigma:
// a(n) += m_j sum_m (A_j + A_i)(m, n) dW/dx_m, A = (sigma - q I)/rho^2 packed
// as r1 = (11 22 33 12), r2 = (13 23 m_j -).
template <bool KAHAN>
__device__ __forceinline__ void momentum_term(float dx, float dy, float dz, float hj, float4 r1, float4 r2, float hi,
                                              float ihi, float4 r1i, float4 r2i, float (&acc)[3], float (&comp)[3]) {
    float d0, d1, d2;
    gradw_f(dx, dy, dz, inv_havg_f(hi, hj, ihi), d0, d1, d2);
    const float s11 = r1.x + r1i.x, s22 = r1.y + r1i.y, s33 = r1.z + r1i.z;
    const float s12 = r1.w + r1i.w, s13 = r2.x + r2i.x, s23 = r2.y + r2i.y;
    const float mj = r2.z;
    d0 *= mj; d1 *= mj; d2 *= mj;
    if (KAHAN) {
        kahan_add(acc[0], comp[0], fmaf(s11, d0, fmaf(s12, d1, s13 * d2)));
        kahan_add(acc[1], comp[1], fmaf(s12, d0, fmaf(s22, d1, s23 * d2)));
        kahan_add(acc[2], comp[2], fmaf(s13, d0, fmaf(s23, d1, s33 * d2)));
    } else {
        acc[0] = fmaf(s11, d0, fmaf(s12, d1, fmaf(s13, d2, acc[0])));
        acc[1] = fmaf(s12, d0, fmaf(s22, d1, fmaf(s23, d2, acc[1])));
        acc[2] = fmaf(s13, d0, fmaf(s23, d1, fmaf(s33, d2, acc[2])));
    }
}

template <bool ASYM, bool KAHAN, bool STAGED>
__global__ void __launch_bounds__(STAGED ? kStageThreads : 256, STAGED ? 4 : MCM_MOM_MINBLOCKS) k_momentum(StepArgs a, int integrate_flag) {
    __shared__ double sm[32];
    __shared__ float4 offs[27];
    __shared__ float4 stage[STAGED ? 3 * kStageCapM : 1];
    __shared__ StageWin W;
    if (skip_step(a)) return;
    const int sub = threadIdx.x / L, lane = threadIdx.x % L;
    const int per = blockDim.x / L;
    const int rounds = (a.n + per * gridDim.x - 1) / (per * gridDim.x);
    const DevGrid g = *a.grid;
    const Frame fr = make_frame(g);
    fill_offsets(offs, fr);
    __syncthreads();
    const int nm = a.nmat;
    constexpr bool asym = ASYM;   // the cap model: sigma's lower triangle in the record's 4th slot
    double e1[5] = {0, 0, 0, 0, 0};   // sums of material 1 (one-material bodies)
    double xlo[3] = {1.0e20, 1.0e20, 1.0e20}, xhi[3] = {-1.0e20, -1.0e20, -1.0e20};
    const bool do_int = integrate_flag && !a.time->ended;
    for (int round = 0; round < rounds; ++round) {
        const int tb = (round * gridDim.x + blockIdx.x) * per;
        if (STAGED) stage_rows<3>(a, tb, per, W, stage, kStageCapM, a.frec0, a.frec0 + 2 * (size_t)a.npad);
        const int t = tb + sub;
        const bool live = t < a.n;
        int nreal = 0, gn = 0, i = 0, wbase = 0;
        float4 xi = make_float4(0.f, 0.f, 0.f, 1.f), r1i = make_float4(0.f, 0.f, 0.f, 0.f),
               r2i = make_float4(0.f, 0.f, 0.f, 1.f), r3i = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            if (STAGED) wbase = stage_base(a, W, t);
            nreal = a.nnbr[t];
            gn = a.gnnbr[t];
            const Rec8 r = ld_rec8(a.frec0 + 2 * (size_t)t);
            xi = r.a;
            r1i = r.b;
            r2i = ld_rec4(mom_tail(a) + t);
            if (asym) r3i = ld_rec4(mom_lower(a) + t);
            i = a.cell_list[t];
        }
        const unsigned *spos = a.nidx + (size_t)t * a.nstride;
        double xa[3] = {0.0, 0.0, 0.0};
        if (live && gn > 0) { xa[0] = a.F.f[FX][i]; xa[1] = a.F.f[FY][i]; xa[2] = a.F.f[FZ][i]; }
        const int total = live ? nreal + gn : 0;
        const float ihi = 1.0f / xi.w;
        float acc[3] = {0.0f, 0.0f, 0.0f}, comp[3] = {0.0f, 0.0f, 0.0f};
        int k0 = lane;
        if (!STAGED && !asym) {
            // the list entries 8 at a time per particle (4 per lane, in 16-byte
            // loads shared by the two lanes), the records one neighbour at a
            // time; each lane's terms in list order
            for (; k0 - lane + 4 * L <= nreal; k0 += 4 * L) {
                unsigned e[4];
                pair_entries<4>(spos + (k0 - lane), lane, e);
#pragma unroll 1
                for (int u = 0; u < 4; ++u) {
                    const size_t p = e[0] & kPosMask;
                    const float4 o = offs[e[0] >> 26];
                    const Rec8 r = ld_rec8(a.frec0 + 2 * p);
                    const float4 q2 = ld_rec4(mom_tail(a) + p);
                    momentum_term<KAHAN>((xi.x - r.a.x) - o.x, (xi.y - r.a.y) - o.y, (xi.z - r.a.z) - o.z, r.a.w,
                                         r.b, q2, xi.w, ihi, r1i, r2i, acc, comp);
                    e[0] = e[1];
                    e[1] = e[2];
                    e[2] = e[3];
                }
            }
            // real neighbours kUnrollM at a time per lane, loads first (as in
            // k_strain); the terms are added in list order
            for (; k0 + (kUnrollM - 1) * L < nreal; k0 += kUnrollM * L) {
                unsigned e[kUnrollM];
#pragma unroll
                for (int u = 0; u < kUnrollM; ++u) e[u] = spos[k0 + u * L];
                Rec8 r[kUnrollM];
                float4 q2[kUnrollM];
#pragma unroll
                for (int u = 0; u < kUnrollM; ++u) {
                    r[u] = ld_rec8(a.frec0 + 2 * (size_t)(e[u] & kPosMask));
                    q2[u] = ld_rec4(mom_tail(a) + (e[u] & kPosMask));
                }
#pragma unroll
                for (int u = 0; u < kUnrollM; ++u) {
                    const float4 o = offs[e[u] >> 26];
                    momentum_term<KAHAN>((xi.x - r[u].a.x) - o.x, (xi.y - r[u].a.y) - o.y, (xi.z - r[u].a.z) - o.z,
                                         r[u].a.w, r[u].b, q2[u], xi.w, ihi, r1i, r2i, acc, comp);
                }
            }
        }
        for (int k = k0; k < total; k += L) {
            float dx, dy, dz, hj;
            float4 r1, r2, r3;
            if (k < nreal) {
                const unsigned e = spos[k];
                const float4 o = offs[e >> 26];
                const size_t p = e & kPosMask;
                const int si = STAGED ? stage_index(W, wbase, e) : -1;
                float4 xj;
                if (si >= 0) {
                    xj = stage[3 * si];
                    r1 = stage[3 * si + 1];
                    r2 = stage[3 * si + 2];
                } else {
                    const Rec8 r = ld_rec8(a.frec0 + 2 * p);
                    xj = r.a;
                    r1 = r.b;
                    r2 = ld_rec4(mom_tail(a) + p);
                }
                if (asym) r3 = ld_rec4(mom_lower(a) + p);
                dx = (xi.x - xj.x) - o.x;
                dy = (xi.y - xj.y) - o.y;
                dz = (xi.z - xj.z) - o.z;
                hj = xj.w;
            } else {
                const int q = a.gnbr[(size_t)(k - nreal) * a.npad + t];
                const double4 xj = a.grec0[q];
                r1 = a.gfrec1[q];
                r2 = a.gfrec2[q];
                if (asym) {
                    const double4 g3 = a.grec3[q];
                    r3 = make_float4((float)g3.x, (float)g3.y, (float)g3.z, 0.0f);
                }
                dx = (float)(xa[0] - xj.x);
                dy = (float)(xa[1] - xj.y);
                dz = (float)(xa[2] - xj.z);
                hj = (float)xj.w;
            }
            float d0, d1, d2;
            gradw_f(dx, dy, dz, inv_havg_f(xi.w, hj, ihi), d0, d1, d2);
            const float s11 = r1.x + r1i.x, s22 = r1.y + r1i.y, s33 = r1.z + r1i.z;
            const float s12 = r1.w + r1i.w, s13 = r2.x + r2i.x, s23 = r2.y + r2i.y;
            float l21 = s12, l31 = s13, l32 = s23;
            if (asym) { l21 = r3.x + r3i.x; l31 = r3.y + r3i.y; l32 = r3.z + r3i.z; }
            const float mj = r2.z;
            d0 *= mj; d1 *= mj; d2 *= mj;
            // a(n) += m_j sum_m (A_j + A_i)(m,n) dW/dx_m (column n; rows for a symmetric A)
            if (KAHAN) {
                kahan_add(acc[0], comp[0], fmaf(s11, d0, fmaf(l21, d1, l31 * d2)));
                kahan_add(acc[1], comp[1], fmaf(s12, d0, fmaf(s22, d1, l32 * d2)));
                kahan_add(acc[2], comp[2], fmaf(s13, d0, fmaf(s23, d1, s33 * d2)));
            } else {
                acc[0] = fmaf(s11, d0, fmaf(l21, d1, fmaf(l31, d2, acc[0])));
                acc[1] = fmaf(s12, d0, fmaf(s22, d1, fmaf(l32, d2, acc[1])));
                acc[2] = fmaf(s13, d0, fmaf(s23, d1, fmaf(s33, d2, acc[2])));
            }
        }
        double ac[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) ac[c] = lane_sum(acc[c], KAHAN ? comp[c] : 0.0f);
        if (live && lane == 0) {
            double *const *f = a.F.f;
            if (a.prm.contact)   // repulsive contact (MCM/mcm_oldacceleration.f90:49-51)
#pragma unroll
                for (int j = 0; j < 3; ++j) ac[j] = ac[j] + f[FRPX + j][i];
            if (a.prm.baseaccel)
#pragma unroll
                for (int j = 0; j < 3; ++j) ac[j] = ac[j] + a.prm.base_a[j];
            switch (a.F.dispbc[i]) {
                case 1: ac[0] = 0.0; break;
                case 2: ac[1] = 0.0; break;
                case 3: ac[2] = 0.0; break;
                case 4: ac[0] = 0.0; ac[1] = 0.0; break;
                case 5: ac[1] = 0.0; ac[2] = 0.0; break;
                case 6: ac[0] = 0.0; ac[2] = 0.0; break;
                case 7: ac[0] = 0.0; ac[1] = 0.0; ac[2] = 0.0; break;
                default: break;
            }
            if (a.split_mode || a.prm.diag || a.prm.veloc_opt) { f[FAX][i] = ac[0]; f[FAY][i] = ac[1]; f[FAZ][i] = ac[2]; }
            const int mati = a.F.mat[i];
            const double mass = f[FMASS][i], vabs = f[FVABS][i];
            const double vals[5] = {0.5 * mass * (vabs * vabs), f[FE][i], mass * fabs(f[FVX][i]),
                                    mass * fabs(f[FVY][i]), mass * fabs(f[FVZ][i])};
            // one material: sums in registers; several: k_energy_step_partials
            // summed them in a fixed order before this kernel moved anything
            if (nm == 1) {
#pragma unroll
                for (int c = 0; c < 5; ++c) e1[c] += vals[c];
            }
            if (do_int) {
                double xn[3];
                integrate(a, i, ac, a.time->dt, a.time->dtold, xn);
#pragma unroll
                for (int d = 0; d < 3; ++d) { xlo[d] = fmin(xlo[d], xn[d]); xhi[d] = fmax(xhi[d], xn[d]); }
            }
        }
        if (STAGED) __syncthreads();   // the next round overwrites the windows
        else __syncwarp();
    }
    const int stride = 5 * nm + 6;
    double *out = a.red + (size_t)blockIdx.x * stride;
    if (nm == 1) {
        double v[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) v[c] = block_sum(e1[c], sm);
        if (threadIdx.x == 0)
#pragma unroll
            for (int c = 0; c < 5; ++c) out[c] = v[c];
    }
    if (do_int) {
        for (int d = 0; d < 3; ++d) {
            const double lo = block_minmax(xlo[d], sm, false);
            const double hi = block_minmax(xhi[d], sm, true);
            if (threadIdx.x == 0) { out[5 * nm + d] = lo; out[5 * nm + 3 + d] = hi; }
        }
    }
}

// ------------------------------------------------------------ launchers

void launch_strain_prep(const StepArgs &a, cudaStream_t s) {
    int n = a.n > a.ghost_cap ? a.n : a.ghost_cap;
    int b = nblk(n, 256);
    k_strain_prep<<<b < 148 * 16 ? b : 148 * 16, 256, 0, s>>>(a);
}

void launch_strain(const StepArgs &a, cudaStream_t s) {
    if (a.pair_kind == 2 && !a.prm.kahan) {
        int b = nblk(a.n, kStageThreads / L);
        if (b > 148 * 6) b = 148 * 6;
        k_strain_staged<<<b, kStageThreads, 0, s>>>(a);
        return;
    }
    if (a.prm.kahan) {
        k_strain<true><<<pair_blocks_of(a, L, (const void *)k_strain<true>), pair_threads_of(a), 0, s>>>(a);
    } else {
        k_strain<false><<<pair_blocks_of(a, L, (const void *)k_strain<false>), pair_threads_of(a), 0, s>>>(a);
    }
}

void launch_mom_prep(const StepArgs &a, cudaStream_t s) {
    int n = a.n > a.ghost_cap ? a.n : a.ghost_cap;
    int b = nblk(n, 256);
    k_mom_prep<<<b < 148 * 16 ? b : 148 * 16, 256, 0, s>>>(a);
}

int launch_momentum(const StepArgs &a, cudaStream_t s, int integrate_flag) {
    if (a.pair_kind == 2 && !a.prm.kahan) {
        int blocks = nblk(a.n, kStageThreads / L);
        if (blocks > 148 * 4) blocks = 148 * 4;
        if (a.red_blocks > 0 && blocks > a.red_blocks) blocks = a.red_blocks;
        if (a.nmat > 1) launch_energy_step_partials(a, s, blocks);
        if (a.prm.asym) k_momentum<true, false, true><<<blocks, kStageThreads, 0, s>>>(a, integrate_flag);
        else k_momentum<false, false, true><<<blocks, kStageThreads, 0, s>>>(a, integrate_flag);
        return blocks;
    }
    void (*kern)(StepArgs, int) = a.prm.asym ? (a.prm.kahan ? k_momentum<true, true, false> : k_momentum<true, false, false>)
                                             : (a.prm.kahan ? k_momentum<false, true, false> : k_momentum<false, false, false>);
    const int blocks = pair_blocks_of(a, L, (const void *)kern);
    if (a.nmat > 1) launch_energy_step_partials(a, s, blocks);
    kern<<<blocks, pair_threads_of(a), 0, s>>>(a, integrate_flag);
    return blocks;
}


}  // namespace mixed
}  // namespace mcm
