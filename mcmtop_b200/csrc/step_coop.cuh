// step_coop.cuh -- cooperative gather kernels for the FP64 fast path.
//
// L lanes (a sub-warp) work on one particle: each lane takes every L-th entry
// of its neighbour list (see nbr_iter.cuh; consecutive lanes read consecutive
// entries), so L independent record loads are in flight per particle, and
// the partial sums are combined with shuffle reductions (no atomics).  The summation order differs from the
// reference's sequential order; the FP64-exact path keeps that order.
#pragma once
#include "nbr_iter.cuh"
#include "physics.cuh"

namespace mcm {
namespace MCM_FLAVOUR_NS {

template <int L>
__device__ __forceinline__ double sub_sum(double v) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, L);
    return v;
}

// Cubic B-spline gradient with the reciprocal of havg supplied (FP64).
__device__ __forceinline__ void gradw_ih(double x0, double x1, double x2, double ih, double &d0, double &d1,
                                         double &d2) {
    const double r2 = fma(x0, x0, fma(x1, x1, x2 * x2));
    if (r2 == 0.0) { d0 = d1 = d2 = 0.0; return; }
    const double rinv = rsqrt(r2);
    const double rad = r2 * rinv;
    const double z = rad * ih;
    const double const1 = (1.0 / kPi) * ih * ih * ih;
    double dw;
    if (z < 1.0) dw = const1 * ((2.25 * z - 3.0) * z);
    else if (z < 2.0) { const double tt = 2.0 - z; dw = -0.75 * const1 * (tt * tt); }
    else dw = 0.0;
    const double f = dw * ih * rinv;
    d0 = f * x0; d1 = f * x1; d2 = f * x2;
}

__device__ __forceinline__ double kernelw_ih(double x0, double x1, double x2, double ih) {
    const double rad = sqrt(fma(x0, x0, fma(x1, x1, x2 * x2)));
    const double z = rad * ih;
    const double const1 = (1.0 / kPi) * ih * ih * ih;
    if (z < 1.0) return const1 * (((0.75 * z - 1.5) * z) * z + 1.0);
    if (z < 2.0) { const double tt = 2.0 - z; return 0.25 * const1 * (tt * tt * tt); }
    return 0.0;
}

// 1/havg with havg = (h_i + h_j)/2; h_i == h_j in all constant-h runs.
__device__ __forceinline__ double inv_havg(double hi, double hj, double ihi) {
    return (hi == hj) ? ihi : 1.0 / (0.5 * (hi + hj));
}

// Entry k of position t's full list: real neighbours (positions), self
// (disctype 1), ghosts.
struct Entry {
    int kind;   // 0 real position, 1 ghost index
    int idx;
    bool self;
};
__device__ __forceinline__ Entry entry_at(const StepArgs &a, int t, int k, int nreal, int self, const unsigned *list) {
    Entry e;
    if (k < nreal) { e.kind = 0; e.idx = (int)(list[k] & kPosMask); e.self = false; }
    else if (k < nreal + self) { e.kind = 0; e.idx = t; e.self = true; }
    else { e.kind = 1; e.idx = a.gnbr[(size_t)(k - nreal - self) * a.npad + t]; e.self = false; }
    return e;
}

// ----------------------------------------------------------- strain rate
template <int L, int DISC>
__global__ void __launch_bounds__(256, DISC == 0 ? 4 : 1) k_strain_coop(StepArgs a) {
    if (skip_step(a)) return;
    const int sub = threadIdx.x / L, lane = threadIdx.x % L;
    const int per = blockDim.x / L;
    const int rounds = (a.n + per * gridDim.x - 1) / (per * gridDim.x);
    const DevGrid g = *a.grid;
    (void)g;
    for (int round = 0; round < rounds; ++round) {
    const int t = (round * gridDim.x + blockIdx.x) * per + sub;
    const bool live = t < a.n;
    int nreal = 0, gn = 0;
    double4 xi = make_double4(0, 0, 0, 1), vi = make_double4(0, 0, 0, 0);
    if (live) {
        nreal = stored_neighbours(a, t);
        gn = a.gnnbr[t];
        xi = a.rec0[t];
        vi = a.rec1[t];
    }
    const unsigned *spos = a.nidx + (size_t)t * a.nstride;
    const int self = (a.prm.disctype == 1) ? 1 : 0;
    const int total = live ? nreal + self + gn : 0;
    const double ihi = 1.0 / xi.w;
    double gv[9];
#pragma unroll
    for (int u = 0; u < 9; ++u) gv[u] = 0.0;
    if (DISC == 0) {
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double4 vj = e.kind ? a.grec1[e.idx] : a.rec1[e.idx];
            double d[3];
            gradw_ih(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z, inv_havg(xi.w, xj.w, ihi), d[0], d[1], d[2]);
            const double dv[3] = {vj.w * (vj.x - vi.x), vj.w * (vj.y - vi.y), vj.w * (vj.z - vi.z)};
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int m = 0; m < 3; ++m) gv[3 * n + m] = fma(dv[n], d[m], gv[3 * n + m]);
        }
    } else {
        // MCM/mcm_corr_strain.f90:51-134
        double sw = 0.0, sg0 = 0.0, sg1 = 0.0, sg2 = 0.0;
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double Volj = e.kind ? a.grec1[e.idx].w : a.rec1[e.idx].w;
            const double ih = inv_havg(xi.w, xj.w, ihi);
            const double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            double d[3];
            gradw_ih(dx, dy, dz, ih, d[0], d[1], d[2]);
            sw = fma(Volj, kernelw_ih(dx, dy, dz, ih), sw);
            sg0 = fma(Volj, d[0], sg0); sg1 = fma(Volj, d[1], sg1); sg2 = fma(Volj, d[2], sg2);
        }
        sw = sub_sum<L>(sw); sg0 = sub_sum<L>(sg0); sg1 = sub_sum<L>(sg1); sg2 = sub_sum<L>(sg2);
        const double isw2 = 1.0 / (sw * sw);
        double B[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) B[u] = 0.0;
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double Volj = e.kind ? a.grec1[e.idx].w : a.rec1[e.idx].w;
            const double ih = inv_havg(xi.w, xj.w, ihi);
            const double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            double d[3];
            gradw_ih(dx, dy, dz, ih, d[0], d[1], d[2]);
            const double w = kernelw_ih(dx, dy, dz, ih);
            const double cg[3] = {(d[0] * sw - w * sg0) * isw2, (d[1] * sw - w * sg1) * isw2,
                                  (d[2] * sw - w * sg2) * isw2};
            const double xr[3] = {Volj * (xj.x - xi.x), Volj * (xj.y - xi.y), Volj * (xj.z - xi.z)};
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int m = 0; m < 3; ++m) B[3 * n + m] = fma(xr[n], cg[m], B[3 * n + m]);
        }
        double Bm[3][3], invB[3][3];
#pragma unroll
        for (int u = 0; u < 9; ++u) Bm[u / 3][u % 3] = sub_sum<L>(B[u]);
        inverse3(Bm, invB);
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double4 vj = e.kind ? a.grec1[e.idx] : a.rec1[e.idx];
            const double ih = inv_havg(xi.w, xj.w, ihi);
            const double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            double d[3];
            gradw_ih(dx, dy, dz, ih, d[0], d[1], d[2]);
            const double w = kernelw_ih(dx, dy, dz, ih);
            const double cg[3] = {(d[0] * sw - w * sg0) * isw2, (d[1] * sw - w * sg1) * isw2,
                                  (d[2] * sw - w * sg2) * isw2};
            double c2[3];
#pragma unroll
            for (int n = 0; n < 3; ++n) c2[n] = invB[n][0] * cg[0] + invB[n][1] * cg[1] + invB[n][2] * cg[2];
            const double vv[3] = {vj.w * vj.x, vj.w * vj.y, vj.w * vj.z};
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int m = 0; m < 3; ++m) gv[3 * n + m] = fma(vv[n], c2[m], gv[3 * n + m]);
        }
    }
#pragma unroll
    for (int u = 0; u < 9; ++u) gv[u] = sub_sum<L>(gv[u]);
    if (live && lane == 0) {
        const int i = a.cell_list[t];
        double *const *f = a.F.f;
        const double r11 = gv[0], r22 = gv[4], r33 = gv[8];
        f[FR11][i] = r11;
        f[FR22][i] = r22;
        f[FR33][i] = r33;
        f[FR12][i] = 0.5 * (gv[1] + gv[3]);
        f[FR13][i] = 0.5 * (gv[2] + gv[6]);
        f[FR23][i] = 0.5 * (gv[5] + gv[7]);
        f[FW12][i] = 0.5 * (gv[1] - gv[3]);
        f[FW13][i] = 0.5 * (gv[2] - gv[6]);
        f[FW23][i] = 0.5 * (gv[5] - gv[7]);
        f[FTR][i] = r11 + r22 + r33;
    }
    __syncwarp();
    }
}

// ------------------------------------------------- momentum + integration
// Simple SPH: four resident blocks (64 registers) hide the gather latency
// better than three at 80 (2.37 against 2.65 ms per step on the 2M bar, and
// 1.58 against 1.87 ms for the strain gather above).
template <int L, int DISC, bool ASYM>
__global__ void __launch_bounds__(256, DISC == 0 ? 4 : 1) k_momentum_coop(StepArgs a, int integrate) {
    __shared__ double sm[32];
    if (skip_step(a)) return;
    const int sub = threadIdx.x / L, lane = threadIdx.x % L;
    const int per = blockDim.x / L;
    const int rounds = (a.n + per * gridDim.x - 1) / (per * gridDim.x);
    const DevGrid g = *a.grid;
    (void)g;
    const int nm = a.nmat;
    // sums of material 1 in registers; other materials go to the block's partials
    double e1[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double x[3] = {1.0e20, 1.0e20, 1.0e20};
    double xmax[3] = {-1.0e20, -1.0e20, -1.0e20};
    const bool do_int = integrate && !a.time->ended;
    for (int round = 0; round < rounds; ++round) {
    const int t = (round * gridDim.x + blockIdx.x) * per + sub;
    const bool live = t < a.n;
    int nreal = 0, gn = 0;
    double4 xi = make_double4(0, 0, 0, 1), r1i = make_double4(0, 0, 0, 0), r2i = make_double4(0, 0, 0, 1);
    // the cap model leaves sigma asymmetric: its lower triangle (21 31 32)
    constexpr bool asym = ASYM;
    double4 r3i = make_double4(0, 0, 0, 0);
    if (live) {
        nreal = stored_neighbours(a, t);
        gn = a.gnnbr[t];
        xi = a.rec0[t];
        r1i = a.rec1[t];
        r2i = a.rec2[t];
        if (asym) r3i = a.rec3[t];
    }
    const unsigned *spos = a.nidx + (size_t)t * a.nstride;
    const int self = (a.prm.disctype == 1) ? 1 : 0;
    const int total = live ? nreal + self + gn : 0;
    const double ihi = 1.0 / xi.w;
    double acc[3] = {0.0, 0.0, 0.0};
    if (DISC == 0) {
        // MCM/mcm_oldacceleration.f90:66-89: a(n) += m_j sum_m (A_j + A_i)(m,n) dW/dx_m
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double4 r1 = e.kind ? a.grec1[e.idx] : a.rec1[e.idx];
            const double4 r2 = e.kind ? a.grec2[e.idx] : a.rec2[e.idx];
            double d[3];
            gradw_ih(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z, inv_havg(xi.w, xj.w, ihi), d[0], d[1], d[2]);
            const double s11 = r1.x + r1i.x, s22 = r1.y + r1i.y, s33 = r1.z + r1i.z;
            const double s12 = r1.w + r1i.w, s13 = r2.x + r2i.x, s23 = r2.y + r2i.y;
            double l21 = s12, l31 = s13, l32 = s23;
            if (asym) {
                const double4 r3 = e.kind ? a.grec3[e.idx] : a.rec3[e.idx];
                l21 = r3.x + r3i.x; l31 = r3.y + r3i.y; l32 = r3.z + r3i.z;
            }
            const double mj = r2.z;
            acc[0] = fma(mj, s11 * d[0] + l21 * d[1] + l31 * d[2], acc[0]);
            acc[1] = fma(mj, s12 * d[0] + s22 * d[1] + l32 * d[2], acc[1]);
            acc[2] = fma(mj, s13 * d[0] + s23 * d[1] + s33 * d[2], acc[2]);
        }
    } else {
        // MCM/mcm_corr_acceleration.f90:63-161
        double sw = 0.0, sg0 = 0.0, sg1 = 0.0, sg2 = 0.0;
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double4 r2 = e.kind ? a.grec2[e.idx] : a.rec2[e.idx];
            const double Volj = r2.z / r2.w;
            const double ih = inv_havg(xi.w, xj.w, ihi);
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            double d[3];
            gradw_ih(dx, dy, dz, ih, d[0], d[1], d[2]);
            sw = fma(Volj, kernelw_ih(dx, dy, dz, ih), sw);
            sg0 = fma(Volj, d[0], sg0); sg1 = fma(Volj, d[1], sg1); sg2 = fma(Volj, d[2], sg2);
        }
        sw = sub_sum<L>(sw); sg0 = sub_sum<L>(sg0); sg1 = sub_sum<L>(sg1); sg2 = sub_sum<L>(sg2);
        const double isw2 = 1.0 / (sw * sw);
        double B[9];
#pragma unroll
        for (int u = 0; u < 9; ++u) B[u] = 0.0;
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double4 r2 = e.kind ? a.grec2[e.idx] : a.rec2[e.idx];
            const double Volj = r2.z / r2.w;
            const double ih = inv_havg(xi.w, xj.w, ihi);
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            double d[3];
            gradw_ih(dx, dy, dz, ih, d[0], d[1], d[2]);
            const double w = kernelw_ih(dx, dy, dz, ih);
            const double cg[3] = {(d[0] * sw - w * sg0) * isw2, (d[1] * sw - w * sg1) * isw2,
                                  (d[2] * sw - w * sg2) * isw2};
            const double xr[3] = {Volj * dx, Volj * dy, Volj * dz};
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int m = 0; m < 3; ++m) B[3 * n + m] = fma(xr[n], cg[m], B[3 * n + m]);
        }
        double Bm[3][3], invB[3][3];
#pragma unroll
        for (int u = 0; u < 9; ++u) Bm[u / 3][u % 3] = sub_sum<L>(B[u]);
        inverse3(Bm, invB);
        double ds[18];
#pragma unroll
        for (int u = 0; u < 18; ++u) ds[u] = 0.0;
        for (int k = lane; k < total; k += L) {
            const Entry e = entry_at(a, t, k, nreal, self, spos);
            const double4 xj = e.kind ? a.grec0[e.idx] : a.rec0[e.idx];
            const double4 r1 = e.kind ? a.grec1[e.idx] : a.rec1[e.idx];
            const double4 r2 = e.kind ? a.grec2[e.idx] : a.rec2[e.idx];
            const double ih = inv_havg(xi.w, xj.w, ihi);
            const double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            double d[3];
            gradw_ih(dx, dy, dz, ih, d[0], d[1], d[2]);
            const double w = kernelw_ih(dx, dy, dz, ih);
            const double cg[3] = {(d[0] * sw - w * sg0) * isw2, (d[1] * sw - w * sg1) * isw2,
                                  (d[2] * sw - w * sg2) * isw2};
            const double zs = e.self ? 0.0 : 1.0;
            const double dsg[6] = {zs * (r1.x + r1i.x), zs * (r1.y + r1i.y), zs * (r1.z + r1i.z),
                                   zs * (r1.w + r1i.w), zs * (r2.x + r2i.x), zs * (r2.y + r2i.y)};
#pragma unroll
            for (int u = 0; u < 6; ++u)
#pragma unroll
                for (int l = 0; l < 3; ++l) ds[3 * u + l] = fma(dsg[u], cg[l], ds[3 * u + l]);
        }
#pragma unroll
        for (int u = 0; u < 18; ++u) ds[u] = sub_sum<L>(ds[u]);
        // the mass of the last neighbour of the reference order: the last ghost, else self
        double massj = r2i.z;
        if (live && gn > 0) massj = a.grec2[a.gnbr[(size_t)(gn - 1) * a.npad + t]].z;
        else if (live && !self && nreal > 0) massj = a.rec2[spos[nreal - 1] & kPosMask].z;
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int l = 0; l < 3; ++l) acc[n] = fma(massj * ds[3 * sym_index(n, m) + l], invB[l][m], acc[n]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = sub_sum<L>(acc[c]);
    // per-particle tail on lane 0 of each sub-warp
    if (live && lane == 0) {
        const int i = a.cell_list[t];
        double *const *f = a.F.f;
        if (a.prm.contact)   // repulsive contact (MCM/mcm_oldacceleration.f90:49-51)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[j] = acc[j] + f[FRPX + j][i];
        if (a.prm.baseaccel)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[j] = acc[j] + a.prm.base_a[j];
        switch (a.F.dispbc[i]) {
            case 1: acc[0] = 0.0; break;
            case 2: acc[1] = 0.0; break;
            case 3: acc[2] = 0.0; break;
            case 4: acc[0] = 0.0; acc[1] = 0.0; break;
            case 5: acc[1] = 0.0; acc[2] = 0.0; break;
            case 6: acc[0] = 0.0; acc[2] = 0.0; break;
            case 7: acc[0] = 0.0; acc[1] = 0.0; acc[2] = 0.0; break;
            default: break;
        }
        if (a.split_mode || a.prm.diag || a.prm.veloc_opt) { f[FAX][i] = acc[0]; f[FAY][i] = acc[1]; f[FAZ][i] = acc[2]; }
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
            integrate_particle(a, i, acc, a.time->dt, a.time->dtold, xn);
#pragma unroll
            for (int d = 0; d < 3; ++d) { x[d] = fmin(x[d], xn[d]); xmax[d] = fmax(xmax[d], xn[d]); }
        }
    }
    __syncwarp();
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
            double lo = block_minmax(x[d], sm, false);
            double hi = block_minmax(xmax[d], sm, true);
            if (threadIdx.x == 0) { out[5 * nm + d] = lo; out[5 * nm + 3 + d] = hi; }
        }
    }
}

}  // namespace MCM_FLAVOUR_NS
}  // namespace mcm
