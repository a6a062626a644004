// step_fp64.cuh -- FP64 kernels of the MCM explicit step: strain-rate gather
// fused with the constitutive update and the critical-timestep reduction, and
// the momentum gather fused with boundary conditions, energy sums, velocity
// update and position update.
//
// Included by two translation units: MCM_FLAVOUR_EXACT (compiled without
// fused multiply-add; reference expression order and divisions, so the
// result follows the reference arithmetic) and MCM_FLAVOUR_FAST (fused
// multiply-add and reciprocals).  Each thread owns one particle and walks its
// neighbours in the reference order; the sums are sequential, so there are no
// atomics and the FP64-exact flavour accumulates in the reference's order.
#pragma once
#include "nbr_iter.cuh"
#include "physics.cuh"

#ifndef MCM_FLAVOUR_NS
#error "define MCM_FLAVOUR_NS (exact or fast)"
#endif

namespace mcm {
namespace MCM_FLAVOUR_NS {

constexpr double kPi = 3.141592653589793;   // acos(-1) (MCM/mcm_startup.f90:33)

// A step is skipped once an error is raised or after the terminating step
// (time->ended == 2); the terminating step itself (ended == 1) still runs the
// momentum and energy part, as MCM/mcm_solution.f90:69-101 does.
__device__ __forceinline__ bool skip_step(const StepArgs &a) { return a.status->code || a.time->ended >= 2; }

// Cubic B-spline gradient, 3-D (MCM/mcm_gradw.f90:41-103), xij = xi - xj.
__device__ __forceinline__ void gradw(double x0, double x1, double x2, double havg, double &d0, double &d1,
                                      double &d2) {
#if MCM_EXACT
    double const1 = 1.0 / (kPi * havg * havg * havg);
    double const2 = const1 * 0.25;
    double rad = x0 * x0;
    rad = rad + x1 * x1;
    rad = rad + x2 * x2;
    rad = sqrt(rad);
    double z = rad / havg;
    double dw;
    if (z < 1.0) dw = const1 * ((9.0 / 4.0 * z - 3.0) * z);
    else if (z < 2.0) { double t = 2.0 - z; dw = -3.0 * const2 * (t * t); }
    else dw = 0.0;
    if (rad == 0.0) { d0 = d1 = d2 = 0.0; }
    else {
        double den = rad * havg;
        d0 = dw * x0 / den;
        d1 = dw * x1 / den;
        d2 = dw * x2 / den;
    }
#else
    double ih = 1.0 / havg;
    double r2 = fma(x0, x0, fma(x1, x1, x2 * x2));
    double rad = sqrt(r2);
    double z = rad * ih;
    double const1 = (1.0 / kPi) * ih * ih * ih;
    double dw;
    if (z < 1.0) dw = const1 * ((2.25 * z - 3.0) * z);
    else if (z < 2.0) { double t = 2.0 - z; dw = -0.75 * const1 * (t * t); }
    else dw = 0.0;
    if (rad == 0.0) { d0 = d1 = d2 = 0.0; }
    else {
        double f = dw * ih / rad;
        d0 = f * x0; d1 = f * x1; d2 = f * x2;
    }
#endif
}

// Cubic B-spline kernel, 3-D (MCM/mcm_kernel.f90:42-95).
__device__ __forceinline__ double kernelw(double x0, double x1, double x2, double havg) {
#if MCM_EXACT
    double const1 = 1.0 / (kPi * havg * havg * havg);
    double const2 = const1 / 4.0;
    double rad = x0 * x0;
    rad = rad + x1 * x1;
    rad = rad + x2 * x2;
    rad = sqrt(rad);
    double z = rad / havg;
    if (z < 1.0) return const1 * (((0.75 * z - 1.5) * z) * z + 1.0);
    if (z < 2.0) { double t = 2.0 - z; return const2 * (t * t * t); }
    return 0.0;
#else
    double ih = 1.0 / havg;
    double rad = sqrt(fma(x0, x0, fma(x1, x1, x2 * x2)));
    double z = rad * ih;
    double const1 = (1.0 / kPi) * ih * ih * ih;
    if (z < 1.0) return const1 * (((0.75 * z - 1.5) * z) * z + 1.0);
    if (z < 2.0) { double t = 2.0 - z; return 0.25 * const1 * (t * t * t); }
    return 0.0;
#endif
}

// 3x3 inverse with the reference's singular fallback (MCM/mcm_math_func.f90:50-79).
__device__ __forceinline__ void inverse3(const double M[3][3], double inv[3][3]) {
    double sd00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
    double sd01 = M[1][0] * M[2][2] - M[1][2] * M[2][0];
    double sd02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
    double sd10 = M[0][1] * M[2][2] - M[0][2] * M[2][1];
    double sd11 = M[0][0] * M[2][2] - M[0][2] * M[2][0];
    double sd12 = M[0][0] * M[2][1] - M[0][1] * M[2][0];
    double sd20 = M[0][1] * M[1][2] - M[0][2] * M[1][1];
    double sd21 = M[0][0] * M[1][2] - M[0][2] * M[1][0];
    double sd22 = M[0][0] * M[1][1] - M[0][1] * M[1][0];
    double det = M[0][0] * sd00 - M[0][1] * sd01 + M[0][2] * sd02;
    if (fabs(det) < 1.0e-08) {
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) inv[r][c] = (r == c) ? 1.0 : 0.0;
    } else {
        double invdet = 1.0 / det;
        inv[0][0] = sd00 * invdet; inv[0][1] = -sd10 * invdet; inv[0][2] = sd20 * invdet;
        inv[1][0] = -sd01 * invdet; inv[1][1] = sd11 * invdet; inv[1][2] = -sd21 * invdet;
        inv[2][0] = sd02 * invdet; inv[2][1] = -sd12 * invdet; inv[2][2] = sd22 * invdet;
    }
}

// Loads the state one particle's constitutive update reads.  The deviator s
// persists only for model 9 (s(1,2) is never reassigned, MCM/mcm_f3dm9.f90:
// 273-281), alfa only for model 3 and the previous q only for models 1 and 3
// (their energy increment uses it before mcm_aviscosity).
__device__ __forceinline__ void load_state(const StepArgs &a, int i, PState<double> &P, int model) {
    const double *const *f = a.F.f;
    P.mat = a.F.mat[i];
    P.mass = f[FMASS][i]; P.h = f[FH][i]; P.hold = f[FHOLD][i];
    P.rho = f[FRHO][i]; P.e = f[FE][i]; P.p = f[FP][i]; P.c = f[FC][i];
    P.efps = f[FEFPS][i]; P.pcut = f[FPCUT][i]; P.p_cut = f[FPCUT2][i]; P.fail = f[FFAIL][i];
    P.capa = (model == 4) ? f[FCAPA][i] : 0.0;
    P.ptype = 0;
    P.rho0 = a.mats[P.mat - 1].rho;
#pragma unroll
    for (int t = 0; t < 6; ++t) { P.sig[t] = f[FS11 + t][i]; P.s[t] = 0.0; P.alfa[t] = 0.0; }
#pragma unroll
    for (int t = 0; t < 3; ++t) P.sigl[t] = f[FL21 + t][i];
    if (model == 9) {
#pragma unroll
        for (int t = 0; t < 6; ++t) P.s[t] = f[FD11 + t][i];
    }
    if (model == 3) {
#pragma unroll
        for (int t = 0; t < 6; ++t) P.alfa[t] = f[FA11 + t][i];
    }
    P.q = (model == 1 || model == 3) ? f[FQ][i] : 0.0;
    P.etry = 0.0; P.einc = 0.0; P.rhoold = P.rho;
}

__device__ __forceinline__ void store_state(const StepArgs &a, int i, const PState<double> &P, int model) {
    double *const *f = a.F.f;
    f[FH][i] = P.h;
    if (a.prm.h_opt) f[FHOLD][i] = P.hold;
    f[FRHO][i] = P.rho; f[FE][i] = P.e; f[FP][i] = P.p; f[FC][i] = P.c;
    f[FEFPS][i] = P.efps; f[FPCUT][i] = P.pcut; f[FPCUT2][i] = P.p_cut; f[FFAIL][i] = P.fail;
#pragma unroll
    for (int t = 0; t < 6; ++t) f[FS11 + t][i] = P.sig[t];
#pragma unroll
    for (int t = 0; t < 3; ++t) f[FL21 + t][i] = P.sigl[t];
    f[FQ][i] = P.q;
    if (model == 4) {
        f[FCAPA][i] = P.capa;
        a.F.ptype[i] = P.ptype;
    }
    if (a.prm.diag || model == 9) {
#pragma unroll
        for (int t = 0; t < 6; ++t) f[FD11 + t][i] = P.s[t];
    }
    if (model == 3) {
#pragma unroll
        for (int t = 0; t < 6; ++t) f[FA11 + t][i] = P.alfa[t];
    }
    if (a.prm.diag) {
        // rhoupd may have changed rod and the trace (MCM/mcm_rhoupd.f90:35-56)
        f[FR11][i] = P.rod[T11]; f[FR22][i] = P.rod[T22]; f[FR33][i] = P.rod[T33];
        f[FTR][i] = P.tracerod; f[FETRY][i] = P.etry; f[FEINC][i] = P.einc; f[FRHOOLD][i] = P.rhoold;
    }
}

// ------------------------------------------------------------ strain prep
// Gather records for the strain loop: positions shifted back half a step
// (MCM/mcm_strain.f90:27-31) and V_j = m_j/rho_j (MCM/mcm_oldstrain.f90:44).
// Ghosts keep their unshifted positions, as in the reference.
__global__ void k_strain_prep(StepArgs a) {
    if (skip_step(a)) return;
    const double dt = a.time->dt;
    const double *const *f = a.F.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int i = a.cell_list[p];
        double vx = f[FVX][i], vy = f[FVY][i], vz = f[FVZ][i];
        double x = f[FX][i] - 0.5 * vx * dt;
        double y = f[FY][i] - 0.5 * vy * dt;
        double z = f[FZ][i] - 0.5 * vz * dt;
        a.rec0[p] = make_double4(x, y, z, f[FH][i]);
        a.rec1[p] = make_double4(vx, vy, vz, f[FMASS][i] / f[FRHO][i]);
    }
    if (a.prm.boundary) {
        const int ngp = *a.ngp;
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngp; g += gridDim.x * blockDim.x) {
            a.grec0[g] = make_double4(a.gx[g], a.gy[g], a.gz[g], a.gh[g]);
            a.grec1[g] = make_double4(a.gvx[g], a.gvy[g], a.gvz[g], a.gmass[g] / a.grho[g]);
        }
    }
}

template <int DISC>
__device__ __forceinline__ void strain_gather(const StepArgs &a, const DevGrid &g, int t, const double4 xi,
                                              const double4 vi, double gv[3][3]) {
    if (DISC == 0) {
        // MCM/mcm_oldstrain.f90:34-54
        auto body = [&](const double4 xj, const double4 vj) {
            double Volj = vj.w;
            double havg = 0.5 * (xi.w + xj.w);
            double d[3];
            gradw(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z, havg, d[0], d[1], d[2]);
            const double dv[3] = {vj.x - vi.x, vj.y - vi.y, vj.z - vi.z};
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                double tt = Volj * dv[n];
#pragma unroll
                for (int m = 0; m < 3; ++m) gv[n][m] = gv[n][m] + tt * d[m];
            }
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { body(a.rec0[p], a.rec1[p]); }, [&](int q) { body(a.grec0[q], a.grec1[q]); });
    } else {
        // MCM/mcm_corr_strain.f90:51-134 (three passes, kernel centred at i)
        double sum_w = 0.0, sg[3] = {0.0, 0.0, 0.0};
        auto pass1 = [&](const double4 xj, const double4 vj) {
            double Volj = vj.w;
            double havg = 0.5 * (xi.w + xj.w);
            double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            double w = kernelw(dx, dy, dz, havg);
            double d[3];
            gradw(dx, dy, dz, havg, d[0], d[1], d[2]);
            sum_w = sum_w + Volj * w;
#pragma unroll
            for (int l = 0; l < 3; ++l) sg[l] = sg[l] + Volj * d[l];
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { pass1(a.rec0[p], a.rec1[p]); }, [&](int q) { pass1(a.grec0[q], a.grec1[q]); });
        double B[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double sw2 = sum_w * sum_w;
        auto pass2 = [&](const double4 xj, const double4 vj) {
            double Volj = vj.w;
            double havg = 0.5 * (xi.w + xj.w);
            double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            double w = kernelw(dx, dy, dz, havg);
            double d[3];
            gradw(dx, dy, dz, havg, d[0], d[1], d[2]);
            double cg[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) cg[m] = (d[m] * sum_w - w * sg[m]) / sw2;
            const double xr[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int n = 0; n < 3; ++n) B[n][m] = B[n][m] + Volj * xr[n] * cg[m];
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { pass2(a.rec0[p], a.rec1[p]); }, [&](int q) { pass2(a.grec0[q], a.grec1[q]); });
        double invB[3][3];
        inverse3(B, invB);
        auto pass3 = [&](const double4 xj, const double4 vj) {
            double Volj = vj.w;
            double havg = 0.5 * (xi.w + xj.w);
            double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
            double w = kernelw(dx, dy, dz, havg);
            double d[3];
            gradw(dx, dy, dz, havg, d[0], d[1], d[2]);
            double cg[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) cg[m] = (d[m] * sum_w - w * sg[m]) / sw2;
            double c2[3];
#pragma unroll
            for (int n = 0; n < 3; ++n) c2[n] = invB[n][0] * cg[0] + invB[n][1] * cg[1] + invB[n][2] * cg[2];
            const double vv[3] = {vj.x, vj.y, vj.z};
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                double tt = Volj * vv[n];
#pragma unroll
                for (int m = 0; m < 3; ++m) gv[n][m] = gv[n][m] + tt * c2[m];
            }
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { pass3(a.rec0[p], a.rec1[p]); }, [&](int q) { pass3(a.grec0[q], a.grec1[q]); });
    }
}

__device__ __forceinline__ double block_min(double v, double *sm) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : 1.0e300;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// ------------------------------------------------------------ strain rate
// MCM/mcm_oldstrain.f90 / mcm_corr_strain.f90 for the particle at position t:
// rod, spin and trace go to the state's diagnostic arrays, which the
// constitutive kernel reads (this keeps the gather kernel small enough to
// keep many warps resident).
template <int DISC>
__global__ void __launch_bounds__(kRedThreads) k_strain(StepArgs a) {
    if (skip_step(a)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int i = a.cell_list[t];
    const DevGrid g = *a.grid;
    const double4 xi = a.rec0[t], vi = a.rec1[t];
    double gv[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    strain_gather<DISC>(a, g, t, xi, vi, gv);
    double *const *f = a.F.f;
    const double r11 = 0.5 * (gv[0][0] + gv[0][0]);
    const double r22 = 0.5 * (gv[1][1] + gv[1][1]);
    const double r33 = 0.5 * (gv[2][2] + gv[2][2]);
    f[FR11][i] = r11;
    f[FR22][i] = r22;
    f[FR33][i] = r33;
    f[FR12][i] = 0.5 * (gv[0][1] + gv[1][0]);
    f[FR13][i] = 0.5 * (gv[0][2] + gv[2][0]);
    f[FR23][i] = 0.5 * (gv[1][2] + gv[2][1]);
    f[FW12][i] = 0.5 * (gv[0][1] - gv[1][0]);
    f[FW13][i] = 0.5 * (gv[0][2] - gv[2][0]);
    f[FW23][i] = 0.5 * (gv[1][2] - gv[2][1]);
    f[FTR][i] = r11 + r22 + r33;
}

// ------------------------------------------------- variable smoothing length
// MCM/mcm_update_h.f90:25-55 (after mcm_strain, before the constitutive
// update): particles at or above their cut-off pressure take a new h and
// bid it for the next grid's hmax.  h >= 0, so the bit patterns of the
// doubles order like the values and an integer maximum picks the largest.
__device__ __forceinline__ void update_h(const StepArgs &a, int i, PState<double> &P, double dt) {
    if (!(P.p >= P.pcut)) return;
    P.hold = P.h;
    if (a.prm.h_opt == 1) P.h = P.hold * (1.0 + P.tracerod * dt / 3.0);
    else P.h = a.F.f[FH0][i] * pow(P.rho0 / P.rho, 1.0 / 3.0);
    atomicMax(reinterpret_cast<unsigned long long *>(a.hmax + 1),
              static_cast<unsigned long long>(__double_as_longlong(P.h)));
}

// ---------------------------------------------------- constitutive update
// MCM/mcm_rhoupd.f90, mcm_constitutive.f90:29-83 and mcm_calccritts.f90 for
// the particle with state index i, and the forward half-step shift of
// MCM/mcm_strain.f90:56-60 (x - v dt/2 recomputed exactly as k_strain_prep).
// Two resident blocks per SM (128 registers, a few hundred bytes of spills)
// measured faster than one at 154 registers: 0.27 against 0.43 ms per step
// on the 2M bar.
#ifndef MCM_CONST_MINBLOCKS
#define MCM_CONST_MINBLOCKS 2
#endif
__global__ void __launch_bounds__(kRedThreads, MCM_CONST_MINBLOCKS) k_constitutive(StepArgs a) {
    __shared__ double sm[32];
    if (skip_step(a)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const double dt = a.time->dt;
    double crit = 1.0e20;
    int bad = 0;
    if (i < a.n) {
        double *const *f = a.F.f;
        const DevMaterial &M = a.mats[a.F.mat[i] - 1];
        PState<double> P;
        load_state(a, i, P, M.model);
#pragma unroll
        for (int u = 0; u < 6; ++u) P.rod[u] = f[FR11 + u][i];
        P.spin[0] = f[FW12][i];
        P.spin[1] = f[FW13][i];
        P.spin[2] = f[FW23][i];
        P.tracerod = f[FTR][i];
        if (a.prm.h_opt) update_h(a, i, P, dt);
        rhoupd(P, M, dt, 3);
        bad = constitutive_particle(P, M, dt);
        const double vx = f[FVX][i], vy = f[FVY][i], vz = f[FVZ][i];
        const double mindist = (a.prm.tcrit_opt == 2) ? f[FMINDIST][i] : 0.0;
        crit = critts_particle(P, M, a.prm.tcrit_opt, 3, f[FVABS][i], mindist);
        store_state(a, i, P, M.model);
        if (a.prm.diag) f[FCRITTS][i] = crit;
        const double xs = f[FX][i] - 0.5 * vx * dt;
        const double ys = f[FY][i] - 0.5 * vy * dt;
        const double zs = f[FZ][i] - 0.5 * vz * dt;
        f[FX][i] = xs + 0.5 * vx * dt;
        f[FY][i] = ys + 0.5 * vy * dt;
        f[FZ][i] = zs + 0.5 * vz * dt;
    }
    if (bad) raise_status(a.status, bad, i);
    double m = block_min(crit, sm);
    if (threadIdx.x == 0) a.red[blockIdx.x] = m;
}

// ------------------------------------------------------ repulsive contact
// MCM/mcm_rep_contact.f90:37-161 with MCM/mcm_get_j_cont_info.f90:31-58
// (contacttype > 0, called by MCM/mcm_solution.f90:64 before mcm_momentum):
// Monaghan's repulsive acceleration -sum_j m_j (K_i + K_j) f_ij^n grad W_ij
// over the particle's real contacts and then its ghost contacts, for
// particles with at least one real contact (:41); zero for the others.
// Positions are the state's after the strain half-step round trip, ghosts'
// from their creation, as in the reference.  Ghost contacts come from the
// ghost contact list (the reference reads their ids from the real contact
// list past ncont, :48 of mcm_get_j_cont_info.f90, entries no search wrote).
__global__ void k_rep_cont(StepArgs a) {
    if (skip_step(a)) return;
    double *const *f = a.F.f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.n; t += gridDim.x * blockDim.x) {
        const int i = a.cell_list[t];
        double r[3] = {0.0, 0.0, 0.0};
        const int nc = a.ncont[t];
        if (nc > 0) {
            const DevMaterial &M = a.mats[a.F.mat[i] - 1];
            const double ki = M.k_cont, n = M.n_cont;
            const double xi0 = f[FX][i], xi1 = f[FY][i], xi2 = f[FZ][i], hi = f[FH][i];
            const unsigned *list = a.cidx + (size_t)t * a.cstride;
            const int total = nc + a.gncont[t];
            for (int k = 0; k < total; ++k) {
                double xj0, xj1, xj2, hj, mj, kj;
                if (k < nc) {
                    const int j = a.cell_list[list[k] & kPosMask];
                    xj0 = f[FX][j]; xj1 = f[FY][j]; xj2 = f[FZ][j];
                    hj = f[FH][j]; mj = f[FMASS][j];
                    kj = a.mats[a.F.mat[j] - 1].k_cont;
                } else {
                    const int q = a.gcont[(size_t)(k - nc) * a.npad + t];
                    xj0 = a.gx[q]; xj1 = a.gy[q]; xj2 = a.gz[q];
                    hj = a.gh[q]; mj = a.gmass[q];
                    kj = a.mats[a.gmat[q] - 1].k_cont;
                }
                const double havg = 0.5 * (hi + hj);
                // inverse of W at the particle spacing, cubic B-spline (:55-68)
                const double ratio = hj / havg;
                double inv_w;
                if (ratio < 1.0) inv_w = 1.0 / (((0.75 * ratio - 1.5) * ratio) * ratio + 1.0);
                else { const double u = 2.0 - ratio; inv_w = 1.0 / (u * u * u); }
                const double d0 = xi0 - xj0, d1 = xi1 - xj1, d2 = xi2 - xj2;
                double g0, g1, g2;
                gradw(d0, d1, d2, havg, g0, g1, g2);
                // mcm_calc_fij (:129-154); its velocity term is unused
                double rad = d0 * d0;
                rad = rad + d1 * d1;
                rad = rad + d2 * d2;
                rad = sqrt(rad);
                const double z = rad / havg;
                double fij;
                if (z < 1.0) fij = inv_w * (((0.75 * z - 1.5) * z) * z + 1.0);
                else if (z < 2.0) { const double u = 2.0 - z; fij = 0.25 * inv_w * (u * u * u); }
                else fij = 0.0;
                const double mk = mj * ((ki + kj) * pow(fij, n));
                r[0] = r[0] - mk * g0;
                r[1] = r[1] - mk * g1;
                r[2] = r[2] - mk * g2;
            }
        }
        f[FRPX][i] = r[0];
        f[FRPY][i] = r[1];
        f[FRPZ][i] = r[2];
    }
}

// --------------------------------------------------------- momentum prep
// Gather records: x, h; (sigma - q)/rho^2 (MCM/mcm_oldacceleration.f90:79-80);
// mass.  Ghost stresses follow MCM/mcm_update_ghost_stress.f90:28-41 (all
// off-diagonals negated) with the ghost's own density from its creation.
__global__ void k_mom_prep(StepArgs a) {
    if (skip_step(a)) return;
    const double *const *f = a.F.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int i = a.cell_list[p];
        double rho = f[FRHO][i];
        double r2 = rho * rho;
        double q = f[FQ][i];
        a.rec0[p] = make_double4(f[FX][i], f[FY][i], f[FZ][i], f[FH][i]);
        a.rec1[p] = make_double4((f[FS11][i] - q) / r2, (f[FS22][i] - q) / r2, (f[FS33][i] - q) / r2,
                                 (f[FS12][i] - 0.0) / r2);
        a.rec2[p] = make_double4((f[FS13][i] - 0.0) / r2, (f[FS23][i] - 0.0) / r2, f[FMASS][i], rho);
        if (a.prm.asym)
            a.rec3[p] = make_double4((f[FL21][i] - 0.0) / r2, (f[FL31][i] - 0.0) / r2, (f[FL32][i] - 0.0) / r2, 0.0);
    }
    if (a.prm.boundary) {
        const int ngp = *a.ngp;
        for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ngp; g += gridDim.x * blockDim.x) {
            int j = a.gpar[g];
            double rho = a.grho[g];
            double r2 = rho * rho;
            double q = f[FQ][j];
            a.grec0[g] = make_double4(a.gx[g], a.gy[g], a.gz[g], a.gh[g]);
            a.grec1[g] = make_double4((f[FS11][j] - q) / r2, (f[FS22][j] - q) / r2, (f[FS33][j] - q) / r2,
                                      ((-f[FS12][j]) - (-0.0)) / r2);
            a.grec2[g] = make_double4(((-f[FS13][j]) - (-0.0)) / r2, ((-f[FS23][j]) - (-0.0)) / r2, a.gmass[g], rho);
            if (a.prm.asym)
                a.grec3[g] = make_double4(((-f[FL21][j]) - (-0.0)) / r2, ((-f[FL31][j]) - (-0.0)) / r2,
                                          ((-f[FL32][j]) - (-0.0)) / r2, 0.0);
        }
    }
}

__device__ __forceinline__ void sym_from_rec(const double4 &r1, const double4 &r2, double A[3][3]) {
    A[0][0] = r1.x; A[1][1] = r1.y; A[2][2] = r1.z;
    A[0][1] = A[1][0] = r1.w;
    A[0][2] = A[2][0] = r2.x;
    A[1][2] = A[2][1] = r2.y;
}

// The lower triangle from the asymmetric record (cap model, prm.asym).
__device__ __forceinline__ void lower_from_rec(const double4 &r3, double A[3][3]) {
    A[1][0] = r3.x;
    A[2][0] = r3.y;
    A[2][1] = r3.z;
}

template <int DISC>
__device__ __forceinline__ void momentum_gather(const StepArgs &a, const DevGrid &g, int t, double acc[3]) {
    const double4 xi = a.rec0[t];
    double Ai[3][3];
    sym_from_rec(a.rec1[t], a.rec2[t], Ai);
    const bool asym = a.prm.asym != 0;
    if (asym) lower_from_rec(a.rec3[t], Ai);
    if (DISC == 0) {
        // MCM/mcm_oldacceleration.f90:66-89; sigma(m,n) is read as stored,
        // both triangles (they differ for the cap model)
        auto body = [&](const double4 xj, const double4 r1, const double4 r2, const double4 *r3) {
            double havg = 0.5 * (xi.w + xj.w);
            double d[3];
            gradw(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z, havg, d[0], d[1], d[2]);
            double Aj[3][3];
            sym_from_rec(r1, r2, Aj);
            if (r3) lower_from_rec(*r3, Aj);
            const double massj = r2.z;
#pragma unroll
            for (int n = 0; n < 3; ++n) {
                double ds = 0.0;
#pragma unroll
                for (int m = 0; m < 3; ++m) ds = ds + (Aj[m][n] + Ai[m][n]) * d[m];
                acc[n] = acc[n] + massj * ds;
            }
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { body(a.rec0[p], a.rec1[p], a.rec2[p], asym ? &a.rec3[p] : nullptr); },
            [&](int q) { body(a.grec0[q], a.grec1[q], a.grec2[q], asym ? &a.grec3[q] : nullptr); });
    } else {
        // MCM/mcm_corr_acceleration.f90:63-161 (kernel centred at j; the self
        // slot k = nnbr is zeroed; the final sum uses the last neighbour's mass)
        double sum_w = 0.0, sg[3] = {0.0, 0.0, 0.0};
        double massj = 0.0;
        auto pass1 = [&](const double4 xj, const double4 r2) {
            massj = r2.z;
            double Volj = massj / r2.w;
            double havg = 0.5 * (xi.w + xj.w);
            double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            double w = kernelw(dx, dy, dz, havg);
            double d[3];
            gradw(dx, dy, dz, havg, d[0], d[1], d[2]);
            sum_w = sum_w + Volj * w;
#pragma unroll
            for (int l = 0; l < 3; ++l) sg[l] = sg[l] + Volj * d[l];
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { pass1(a.rec0[p], a.rec2[p]); }, [&](int q) { pass1(a.grec0[q], a.grec2[q]); });
        double B[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        const double sw2 = sum_w * sum_w;
        auto pass2 = [&](const double4 xj, const double4 r2) {
            massj = r2.z;
            double Volj = massj / r2.w;
            double havg = 0.5 * (xi.w + xj.w);
            double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            double w = kernelw(dx, dy, dz, havg);
            double d[3];
            gradw(dx, dy, dz, havg, d[0], d[1], d[2]);
            double cg[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) cg[m] = (d[m] * sum_w - w * sg[m]) / sw2;
            const double xr[3] = {dx, dy, dz};
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int n = 0; n < 3; ++n) B[n][m] = B[n][m] + Volj * xr[n] * cg[m];
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool) { pass2(a.rec0[p], a.rec2[p]); }, [&](int q) { pass2(a.grec0[q], a.grec2[q]); });
        double invB[3][3];
        inverse3(B, invB);
        // deltasig(m,n,l) is symmetric in (m,n): keep 6 x 3 accumulators
        double ds[6][3];
#pragma unroll
        for (int u = 0; u < 6; ++u) ds[u][0] = ds[u][1] = ds[u][2] = 0.0;
        auto pass3 = [&](const double4 xj, const double4 r1, const double4 r2, bool self_slot) {
            massj = r2.z;
            double havg = 0.5 * (xi.w + xj.w);
            double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
            double w = kernelw(dx, dy, dz, havg);
            double d[3];
            gradw(dx, dy, dz, havg, d[0], d[1], d[2]);
            double cg[3];
#pragma unroll
            for (int m = 0; m < 3; ++m) cg[m] = (d[m] * sum_w - w * sg[m]) / sw2;
            double Aj[3][3];
            sym_from_rec(r1, r2, Aj);
#pragma unroll
            for (int u = 0; u < 6; ++u) {
                const int m = (u < 3) ? u : (u == 5 ? 1 : 0);
                const int n = (u < 3) ? u : (u == 3 ? 1 : 2);
                double dsig = Aj[m][n] + Ai[m][n];
                if (self_slot) dsig = 0.0;
#pragma unroll
                for (int l = 0; l < 3; ++l) ds[u][l] = ds[u][l] + dsig * cg[l];
            }
        };
        for_each_neighbour(
            a, g, t, [&](int p, bool self) { pass3(a.rec0[p], a.rec1[p], a.rec2[p], self); },
            [&](int q) { pass3(a.grec0[q], a.grec1[q], a.grec2[q], false); });
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
            for (int m = 0; m < 3; ++m)
#pragma unroll
                for (int l = 0; l < 3; ++l) acc[n] = acc[n] + massj * ds[sym_index(n, m)][l] * invB[l][m];
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

// Velocity update (MCM/mcm_update_velocity.f90:29-56) and position update
// (MCM/mcm_move.f90:32-40) of one particle; check_sym_pen is per particle
// because the reference's global test "bbox below the plane" selects exactly
// the particles below it (MCM/mcm_check_sym_pen.f90:27-179).
__device__ __forceinline__ void integrate_particle(const StepArgs &a, int i, const double acc[3], double dt, double dtold,
                                                   double x[3]) {
    double *const *f = a.F.f;
    double dtn = 0.5 * (dt + dtold);
    double v[3] = {f[FVX][i], f[FVY][i], f[FVZ][i]};
    double vabs = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        if (a.prm.drelax) v[j] = a.prm.drelax_scale * v[j] + acc[j] * dtn;
        else v[j] = v[j] + acc[j] * dtn;
        vabs = vabs + v[j] * v[j];
    }
    vabs = sqrt(vabs);
    x[0] = f[FX][i]; x[1] = f[FY][i]; x[2] = f[FZ][i];
#pragma unroll
    for (int j = 0; j < 3; ++j) x[j] = x[j] + v[j] * dt;
    double xo[3] = {x[0], x[1], x[2]};
    if (a.prm.boundary) {
        const DevPlanes &pl = a.prm.planes;
        for (int d = 0; d < 3; ++d) {
            if (pl.code[0][d] == 1 && xo[d] < pl.bx[0][d]) { xo[d] = 2.0 * pl.bx[0][d] - xo[d]; v[d] = -v[d]; }
            if (pl.code[1][d] == 1 && xo[d] > pl.bx[1][d]) { xo[d] = 2.0 * pl.bx[1][d] - xo[d]; v[d] = -v[d]; }
            if (pl.code[0][d] == 2) {
                double dx = pl.bx[1][d] - pl.bx[0][d];
                if (xo[d] < pl.bx[0][d]) xo[d] = xo[d] + dx;
                if (xo[d] > pl.bx[1][d]) xo[d] = xo[d] - dx;
            }
        }
    }
    f[FVX][i] = v[0]; f[FVY][i] = v[1]; f[FVZ][i] = v[2];
    f[FVABS][i] = vabs;
    f[FX][i] = xo[0]; f[FY][i] = xo[1]; f[FZ][i] = xo[2];
}

// ----------------------------------------------- momentum + integration
// Writes a (split path), adds base accelerations and displacement BCs
// (MCM/mcm_boundcond.f90:23-62), block partial energy sums
// (MCM/mcm_calctotale.f90:33-51) and, when integrate is set and the run has
// not terminated, the velocity and position update with block bbox partials.
template <int DISC>
__global__ void __launch_bounds__(kRedThreads) k_momentum(StepArgs a, int integrate) {
    __shared__ double sm[32];
    if (skip_step(a)) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nm = a.nmat;
    double acc[3] = {0.0, 0.0, 0.0};
    int mati = 0;
    double ke = 0.0, ie = 0.0, mo[3] = {0.0, 0.0, 0.0};
    double x[3] = {1.0e20, 1.0e20, 1.0e20};
    double xmax[3] = {-1.0e20, -1.0e20, -1.0e20};
    const bool do_int = integrate && !a.time->ended;
    if (t < a.n) {
        const int i = a.cell_list[t];
        double *const *f = a.F.f;
        const DevGrid g = *a.grid;
        // MCM/mcm_oldacceleration.f90:49-51, mcm_corr_acceleration.f90:45-49
        if (a.prm.contact)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc[j] = acc[j] + f[FRPX + j][i];
        momentum_gather<DISC>(a, g, t, acc);
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
        mati = a.F.mat[i];
        const double mass = f[FMASS][i], vabs = f[FVABS][i];
        ke = 0.5 * mass * (vabs * vabs);
        mo[0] = mass * fabs(f[FVX][i]);
        mo[1] = mass * fabs(f[FVY][i]);
        mo[2] = mass * fabs(f[FVZ][i]);
        ie = f[FE][i];
        if (do_int) {
            double xn[3];
            integrate_particle(a, i, acc, a.time->dt, a.time->dtold, xn);
            x[0] = xn[0]; x[1] = xn[1]; x[2] = xn[2];
            xmax[0] = xn[0]; xmax[1] = xn[1]; xmax[2] = xn[2];
        }
    }
    // per-block partials: [5*nmat energies][6 bbox]
    const int stride = 5 * nm + 6;
    double *out = a.red + (size_t)blockIdx.x * stride;
    for (int m = 1; m <= nm; ++m) {
        bool mine = (mati == m);
        double v0 = block_sum(mine ? ke : 0.0, sm);
        double v1 = block_sum(mine ? ie : 0.0, sm);
        double v2 = block_sum(mine ? mo[0] : 0.0, sm);
        double v3 = block_sum(mine ? mo[1] : 0.0, sm);
        double v4 = block_sum(mine ? mo[2] : 0.0, sm);
        if (threadIdx.x == 0) {
            out[5 * (m - 1) + 0] = v0; out[5 * (m - 1) + 1] = v1;
            out[5 * (m - 1) + 2] = v2; out[5 * (m - 1) + 3] = v3; out[5 * (m - 1) + 4] = v4;
        }
    }
    if (do_int) {
        for (int d = 0; d < 3; ++d) {
            double lo = block_minmax(x[d], sm, false);
            double hi = block_minmax(xmax[d], sm, true);
            if (threadIdx.x == 0) { out[5 * nm + d] = lo; out[5 * nm + 3 + d] = hi; }
        }
    }
}

// Split path: velocity and position update after the host's output phase.
__global__ void __launch_bounds__(kRedThreads) k_update_move(StepArgs a) {
    __shared__ double sm[32];
    if (a.status->code) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double x[3] = {1.0e20, 1.0e20, 1.0e20};
    double xmax[3] = {-1.0e20, -1.0e20, -1.0e20};
    if (i < a.n) {
        double acc[3] = {a.F.f[FAX][i], a.F.f[FAY][i], a.F.f[FAZ][i]};
        double xn[3];
        integrate_particle(a, i, acc, a.time->dt, a.time->dtold, xn);
        x[0] = xmax[0] = xn[0]; x[1] = xmax[1] = xn[1]; x[2] = xmax[2] = xn[2];
    }
    const int stride = 5 * a.nmat + 6;
    double *out = a.red + (size_t)blockIdx.x * stride;
    for (int d = 0; d < 3; ++d) {
        double lo = block_minmax(x[d], sm, false);
        double hi = block_minmax(xmax[d], sm, true);
        if (threadIdx.x == 0) { out[5 * a.nmat + d] = lo; out[5 * a.nmat + 3 + d] = hi; }
    }
}

// ----------------------------------------------------------------- XSPH
// MCM/mcm_update_velocity.f90:29-87 with veloc_opt 1, as three passes over
// the particles: the velocity update, the XSPH sums (which read every
// particle's updated velocity), then the smoothed velocity and the move.
// In a fused run the step that terminates skips all three, like the fused
// momentum kernel.
__global__ void k_velocity(StepArgs a) {
    if (skip_step(a) || a.time->ended) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    double *const *f = a.F.f;
    const double dtn = 0.5 * (a.time->dt + a.time->dtold);
    double vabs = 0.0;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        double v = f[FVX + j][i];
        if (a.prm.drelax) v = a.prm.drelax_scale * v + f[FAX + j][i] * dtn;
        else v = v + f[FAX + j][i] * dtn;
        f[FVX + j][i] = v;
        vabs = vabs + v * v;
    }
    f[FVABS][i] = sqrt(vabs);
}

// Sum over the step's neighbours in reference order: real ones read the
// updated state, ghosts their copies from the start of the step; W takes the
// neighbour's h and V_j = m_j / ((rho_j + rho_i) / 2).
__global__ void k_xsph_sum(StepArgs a) {
    if (skip_step(a) || a.time->ended) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const double *const *f = a.F.f;
    const int i = a.cell_list[t];
    const double xi[3] = {f[FX][i], f[FY][i], f[FZ][i]};
    const double vi[3] = {f[FVX][i], f[FVY][i], f[FVZ][i]};
    const double rhoi = f[FRHO][i];
    double sv[3] = {0.0, 0.0, 0.0};
    auto body = [&](double xj0, double xj1, double xj2, double vj0, double vj1, double vj2, double massj,
                    double rhoj, double hj) {
        const double w = kernelw(xi[0] - xj0, xi[1] - xj1, xi[2] - xj2, hj);
        const double volj = massj / (0.5 * (rhoj + rhoi));
        sv[0] = sv[0] + volj * (vj0 - vi[0]) * w;
        sv[1] = sv[1] + volj * (vj1 - vi[1]) * w;
        sv[2] = sv[2] + volj * (vj2 - vi[2]) * w;
    };
    for_each_neighbour(
        a, *a.grid, t,
        [&](int p, bool) {
            const int j = a.cell_list[p];
            body(f[FX][j], f[FY][j], f[FZ][j], f[FVX][j], f[FVY][j], f[FVZ][j], f[FMASS][j], f[FRHO][j], f[FH][j]);
        },
        [&](int q) { body(a.gx[q], a.gy[q], a.gz[q], a.gvx[q], a.gvy[q], a.gvz[q], a.gmass[q], a.grho[q], a.gh[q]); });
    double *const *fw = a.F.f;
    fw[FXS0][i] = sv[0];
    fw[FXS1][i] = sv[1];
    fw[FXS2][i] = sv[2];
}

__global__ void __launch_bounds__(kRedThreads) k_xsph_move(StepArgs a) {
    __shared__ double sm[32];
    if (skip_step(a) || a.time->ended) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double x[3] = {1.0e20, 1.0e20, 1.0e20};
    double xmax[3] = {-1.0e20, -1.0e20, -1.0e20};
    if (i < a.n) {
        double *const *f = a.F.f;
        const double epsilon = 0.100;
        const double dt = a.time->dt;
        double v[3], xo[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            v[j] = f[FVX + j][i] + epsilon * f[FXS0 + j][i];
            x[j] = f[FX + j][i] + v[j] * dt;
            xmax[j] = x[j];
            xo[j] = x[j];
        }
        if (a.prm.boundary) {
            const DevPlanes &pl = a.prm.planes;
            for (int d = 0; d < 3; ++d) {
                if (pl.code[0][d] == 1 && xo[d] < pl.bx[0][d]) { xo[d] = 2.0 * pl.bx[0][d] - xo[d]; v[d] = -v[d]; }
                if (pl.code[1][d] == 1 && xo[d] > pl.bx[1][d]) { xo[d] = 2.0 * pl.bx[1][d] - xo[d]; v[d] = -v[d]; }
                if (pl.code[0][d] == 2) {
                    double dx = pl.bx[1][d] - pl.bx[0][d];
                    if (xo[d] < pl.bx[0][d]) xo[d] = xo[d] + dx;
                    if (xo[d] > pl.bx[1][d]) xo[d] = xo[d] - dx;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) { f[FVX + j][i] = v[j]; f[FX + j][i] = xo[j]; }
    }
    const int stride = 5 * a.nmat + 6;
    double *out = a.red + (size_t)blockIdx.x * stride;
    for (int d = 0; d < 3; ++d) {
        double lo = block_minmax(x[d], sm, false);
        double hi = block_minmax(xmax[d], sm, true);
        if (threadIdx.x == 0) { out[5 * a.nmat + d] = lo; out[5 * a.nmat + 3 + d] = hi; }
    }
}

// ------------------------------------------------------- initialisation
// Per-particle part of mcm_initial (MCM/mcm_initial.f90:33-69):
// init_boundcond, calcmass (counts in a.red), initvbls, calcrhopc/eoscalc,
// initsigma, initrod, init_h, and the nodal AV with tracerod = 0.
__global__ void k_initial(StepArgs a, int massopt, int init_h_opt, int init_rhoe, const int *nppermat) {
    double *const *f = a.F.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const int mat = a.F.mat[i];
        const DevMaterial &M = a.mats[mat - 1];
        // MCM/mcm_init_boundcond.f90:25-54
        switch (a.F.dispbc[i]) {
            case 1: f[FVX][i] = 0.0; break;
            case 2: f[FVY][i] = 0.0; break;
            case 3: f[FVZ][i] = 0.0; break;
            case 4: f[FVX][i] = 0.0; f[FVY][i] = 0.0; break;
            case 5: f[FVY][i] = 0.0; f[FVZ][i] = 0.0; break;
            case 6: f[FVX][i] = 0.0; f[FVZ][i] = 0.0; break;
            case 7: f[FVX][i] = 0.0; f[FVY][i] = 0.0; f[FVZ][i] = 0.0; break;
            default: break;
        }
        // MCM/mcm_calcmass.f90:129-137
        if (massopt == 0) f[FMASS][i] = M.mass / (double)nppermat[mat - 1];
        // MCM/mcm_initvbls.f90:48-75
        PState<double> P;
        P.mat = mat;
        P.mass = f[FMASS][i];
        P.efps = 0.0; P.fail = 1.0;
        switch (M.model) {
            case 1: case 3: case 4: P.pcut = -9.90E+20; break;
            case 9: P.pcut = M.strinput[0]; break;
            case 10: P.pcut = M.strinput[3]; break;
            default: P.pcut = 0.0;
        }
        double vx = f[FVX][i], vy = f[FVY][i], vz = f[FVZ][i];
        double vabs = 0.0;
        vabs = vabs + vx * vx; vabs = vabs + vy * vy; vabs = vabs + vz * vz;
        f[FVABS][i] = sqrt(vabs);
        // MCM/mcm_calcrhopc.f90:31-95
        P.rho0 = M.rho;
        P.tracerod = 0.0;
        if (init_rhoe == 1) { P.rho = f[FRHO][i]; P.e = f[FE][i]; }
        else { P.rho = 0.0; P.e = 0.0; }
        P.p = 0.0; P.c = 0.0;
        switch (M.model) {
            case 1: case 3:
                if (init_rhoe != 1) { P.rho = P.rho0; P.e = 0.0; }
                P.p = 0.0;
                P.c = sqrt(M.strinput[1] / P.rho);
                break;
            case 4:   // MCM/mcm_calcrhopc.f90:57-67: strinput(10) = cm(5,2), set by mcm_sets4
                if (init_rhoe != 1) { P.rho = P.rho0; P.e = 0.0; }
                P.p = 0.0;
                P.c = sqrt(M.strinput[9] / P.rho);
                break;
            case 9: case 10: {
                const double *ei = M.eosinput;
                switch (M.eos) {
                    case 1:
                        if (init_rhoe != 1) { P.rho = P.rho0 / ei[8]; P.e = ei[7] * P.mass / P.rho; }
                        eos1p(P, M); eos1c(P, M); break;
                    case 4:
                        if (init_rhoe != 1) { P.rho = P.rho0 / ei[7]; P.e = ei[6] * P.mass / P.rho; }
                        eos4p(P, M); eos4c(P, M); break;
                    case 13:
                        if (init_rhoe != 1) { P.rho = P.rho0 / ei[3]; P.e = ei[2] * P.mass / P.rho; }
                        eos13p(P, M); eos13c(P, M); break;
                    case 28:
                        if (init_rhoe != 1) { P.rho = P.rho0 / ei[3]; P.e = ei[2] * P.mass; }
                        eos28p(P, M); eos28c(P, M); break;
                    case 41:
                        if (init_rhoe != 1) { P.rho = P.rho0 / ei[5]; P.e = ei[2] * ei[3] * P.mass / P.rho; }
                        eos41p(P, M, 0.0);
                        if (!eos41c(P, M)) raise_status(a.status, MCM_ECOMPLEX_C, i);
                        break;
                }
                if (M.model == 9) {
                    double pmax = M.strinput[0];
                    if (P.p < pmax) P.p = pmax;
                }
                break;
            }
        }
        f[FRHO][i] = P.rho; f[FE][i] = P.e; f[FP][i] = P.p; f[FC][i] = P.c;
        f[FEFPS][i] = 0.0; f[FFAIL][i] = 1.0; f[FPCUT][i] = P.pcut; f[FPCUT2][i] = 0.0;
        // MCM/mcm_initsigma.f90:26-49
        f[FS11][i] = -P.p; f[FS22][i] = -P.p; f[FS33][i] = -P.p;
        f[FS12][i] = 0.0; f[FS13][i] = 0.0; f[FS23][i] = 0.0;
        f[FL21][i] = 0.0; f[FL31][i] = 0.0; f[FL32][i] = 0.0;
        for (int t = 0; t < 6; ++t) { f[FD11 + t][i] = 0.0; f[FA11 + t][i] = 0.0; f[FR11 + t][i] = 0.0; }
        f[FW12][i] = f[FW13][i] = f[FW23][i] = 0.0;
        // MCM/mcm_init_h.f90:22-48
        if (init_h_opt == 0) f[FH][i] = M.h;
        f[FHOLD][i] = f[FH][i];
        f[FH0][i] = f[FH][i];
        // MCM/mcm_initial.f90:62-69: tracerod = 0 gives q = 0
        f[FQ][i] = 0.0;
        f[FTR][i] = 0.0;
        f[FRHOOLD][i] = P.rho;
        f[FETRY][i] = 0.0; f[FEINC][i] = 0.0; f[FCAPA][i] = 0.0;
        f[FAX][i] = f[FAY][i] = f[FAZ][i] = 0.0;
        f[FCRITTS][i] = 0.0;
    }
}

// Critical timestep of the initial state (MCM/mcm_initial.f90:81).
__global__ void __launch_bounds__(kRedThreads) k_init_critts(StepArgs a) {
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double crit = 1.0e20;
    if (i < a.n) {
        PState<double> P;
        const DevMaterial &M = a.mats[a.F.mat[i] - 1];
        load_state(a, i, P, M.model);
        P.tracerod = a.F.f[FTR][i];
        const double mindist = (a.prm.tcrit_opt == 2) ? a.F.f[FMINDIST][i] : 0.0;
        crit = critts_particle(P, M, a.prm.tcrit_opt, 3, a.F.f[FVABS][i], mindist);
        a.F.f[FCRITTS][i] = crit;
    }
    double m = block_min(crit, sm);
    if (threadIdx.x == 0) a.red[blockIdx.x] = m;
}

}  // namespace MCM_FLAVOUR_NS
}  // namespace mcm

#if !MCM_EXACT
#include "step_coop.cuh"
#endif

namespace mcm {
namespace MCM_FLAVOUR_NS {

// ----------------------------------------------------------- launchers
static inline int nblk(int n, int t) { return (n + t - 1) / t; }
// lanes per particle in the cooperative gathers: 4 lanes (about 20
// neighbours each in flight) hide the gather latency better than 16 (2M bar:
// strain 1.28 against 1.58 ms, momentum 1.70 against 2.37 ms per step)
constexpr int kCoopLanes = 4;
static inline int gs_blocks(int n) { int b = nblk(n, 256); return b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b); }

void launch_strain_prep(const StepArgs &a, cudaStream_t s) {
    k_strain_prep<<<gs_blocks(a.n > a.ghost_cap ? a.n : a.ghost_cap), 256, 0, s>>>(a);
}

void launch_strain(const StepArgs &a, cudaStream_t s) {
#if MCM_EXACT
    int blocks = nblk(a.n, kRedThreads);
    if (a.prm.disctype == 0) k_strain<0><<<blocks, kRedThreads, 0, s>>>(a);
    else k_strain<1><<<blocks, kRedThreads, 0, s>>>(a);
#else
    constexpr int L = kCoopLanes;
    void (*kern)(StepArgs) = a.prm.disctype == 0 ? k_strain_coop<L, 0> : k_strain_coop<L, 1>;
    kern<<<pair_blocks_of(a, L, (const void *)kern), pair_threads_of(a), 0, s>>>(a);
#endif
}

int launch_constitutive(const StepArgs &a, cudaStream_t s) {
    int blocks = nblk(a.n, kRedThreads);
    k_constitutive<<<blocks, kRedThreads, 0, s>>>(a);
    return blocks;
}

void launch_mom_prep(const StepArgs &a, cudaStream_t s) {
    k_mom_prep<<<gs_blocks(a.n > a.ghost_cap ? a.n : a.ghost_cap), 256, 0, s>>>(a);
}

void launch_rep_cont(const StepArgs &a, cudaStream_t s) { k_rep_cont<<<gs_blocks(a.n), 256, 0, s>>>(a); }

int launch_momentum(const StepArgs &a, cudaStream_t s, int integrate) {
#if MCM_EXACT
    int blocks = nblk(a.n, kRedThreads);
    if (a.prm.disctype == 0) k_momentum<0><<<blocks, kRedThreads, 0, s>>>(a, integrate);
    else k_momentum<1><<<blocks, kRedThreads, 0, s>>>(a, integrate);
    return blocks;
#else
    constexpr int L = kCoopLanes;
    void (*kern)(StepArgs, int) = a.prm.disctype != 0 ? k_momentum_coop<L, 1, false>
                                  : (a.prm.asym ? k_momentum_coop<L, 0, true> : k_momentum_coop<L, 0, false>);
    const int blocks = pair_blocks_of(a, L, (const void *)kern);
    if (a.nmat > 1) launch_energy_step_partials(a, s, blocks);
    kern<<<blocks, pair_threads_of(a), 0, s>>>(a, integrate);
    return blocks;
#endif
}

int launch_update_move(const StepArgs &a, cudaStream_t s) {
    int blocks = nblk(a.n, kRedThreads);
    k_update_move<<<blocks, kRedThreads, 0, s>>>(a);
    return blocks;
}

int launch_xsph_move(const StepArgs &a, cudaStream_t s) {
    const int blocks = nblk(a.n, kRedThreads);
    k_velocity<<<blocks, kRedThreads, 0, s>>>(a);
    k_xsph_sum<<<blocks, kRedThreads, 0, s>>>(a);
    k_xsph_move<<<blocks, kRedThreads, 0, s>>>(a);
    return blocks;
}

int launch_initial(const StepArgs &a, cudaStream_t s, int massopt, int init_h_opt, int init_rhoe,
                   const int *nppermat) {
    k_initial<<<gs_blocks(a.n), 256, 0, s>>>(a, massopt, init_h_opt, init_rhoe, nppermat);
    return 0;
}

int launch_init_critts(const StepArgs &a, cudaStream_t s) {
    int blocks = nblk(a.n, kRedThreads);
    k_init_critts<<<blocks, kRedThreads, 0, s>>>(a);
    return blocks;
}

}  // namespace MCM_FLAVOUR_NS
}  // namespace mcm
