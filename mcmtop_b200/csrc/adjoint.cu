// adjoint.cu -- reverse (adjoint) step of the FP64 explicit step.
//
// Scope: disctype 0, model 10 with EOS 41 (the Taylor bar), symmetry and
// periodic planes, fixed smoothing lengths, a prescribed dt schedule (the
// critical-timestep minimum is not differentiated: dt_n is an input), and the
// neighbour lists of each step frozen at their forward values.  One reverse
// step maps the adjoint of the state after step n to the adjoint of the state
// before it, and adds the step's contribution to the material-parameter
// adjoints (G, yield stress, hardening modulus, EOS-41 slope s).
//
// The forward step n (MCM/mcm_solution.f90:37-138) is, per particle:
//   xs = x - v dt_prev/2                      (MCM/mcm_strain.f90:25-29)
//   G_i = sum_j V_j (v_j - v_i) (x) gradW(xs_i - xs_j)   (mcm_oldstrain.f90:34-64)
//   rod, spin, tr = sym G, skew G, tr G
//   (rho, e, p, efps, sigma, q)' = C(rho, e, p, efps, sigma, rod, spin, tr; theta)
//                                             (mcm_rhoupd, mcm_constitutive)
//   a_i = sum_j m_j (S_i + S_j) gradW(x_i - x_j),  S = (sigma' - q' I)/rho'^2
//                                             (mcm_oldacceleration.f90:66-89)
//   v' = v + a (dt + dt_prev)/2,  x' = x + v' dt, plane reflections
//                                             (mcm_update_velocity, mcm_move, mcm_check_sym_pen)
// with ghosts g of parent p: x_g = M_g x_p + c_g, v_g = M_g v_p (M_g = +-1 per
// axis), rho_g = rho_p at neighbour time, S_g = S_p with every off-diagonal
// negated (mcm_update_ghost_stress.f90:28-41).
//
// Reverse kernels (each a gather over the particle's own list; the lists are
// symmetric, i in N(j) <=> j in N(i), so the terms a particle contributes to
// its neighbours' sums are collected from the neighbours' adjoints; only the
// ghost terms, which belong to a parent particle, use atomics):
//   k_adj_move        x', v' -> x, v, a          (reflections by their branch)
//   k_adj_momentum    a -> S (post-constitutive sigma', q', rho'), x, ghost parents
//   k_adj_constitutive  the per-particle vector-Jacobian product of C: one
//                     hand-written reverse pass when every material is model 10
//                     with EOS 41, else forward-mode dual numbers through the same
//                     templated code the step runs (physics.cuh); either way the
//                     derivative is the one of the branch taken (the active
//                     branch of the return map)
//   k_adj_strain      G -> x, v, rho (through V = m/rho), ghost parents
#include "nbr_iter.cuh"
#include "physics.cuh"

namespace mcm {
namespace adj {

constexpr double kPi = 3.14159265358979323846;
#ifndef MCM_ADJ_DIRECTIONS
#define MCM_ADJ_DIRECTIONS 8
#endif
constexpr int kND = MCM_ADJ_DIRECTIONS;   // directions per dual pass
constexpr int kInputs = 20;     // rho e p efps sigma(6) rod(6) spin(3) tr
constexpr int kSeeds = kInputs + kParams;
constexpr int kPasses = (kSeeds + kND - 1) / kND;
using D = Dual<kND>;

// Material constants for the dual passes.  Only the four differentiated
// parameters carry derivatives (strinput(1..3) = G, yield stress, hardening
// modulus of model 10; eosinput(2) = the EOS-41 slope s; the shear modulus g
// that EOS 1 and 4 read is G as well); every other card value is a plain
// double, so that the dual state of a pass stays in registers.  Model 10
// reads strinput[0..7] and EOS 41 eosinput[0..5]; indices beyond the stored
// ones (the 5-row table of models 1 and 3, compiled here but never run: the
// adjoint accepts model 10 only) read the last stored value.
constexpr int kStr = 8, kEos = 8;
struct StrCards {
    double v[kStr];
    D gmod, yield, hard;
    __device__ __forceinline__ D operator[](int k) const {
        return k == 0 ? gmod : (k == 1 ? yield : (k == 2 ? hard : D(v[k < kStr ? k : kStr - 1])));
    }
};
struct EosCards {
    double v[kEos];
    D slope;
    __device__ __forceinline__ D operator[](int k) const { return k == 1 ? slope : D(v[k < kEos ? k : kEos - 1]); }
};
struct DualMat {
    int model, eos, visc_type, pad;
    double rho, av_l, av_q, mass, h, rho_min, rho_max;
    D g;
    StrCards strinput;
    EosCards eosinput;
};

// gradW and its Hessian (symmetric: 11 22 33 12 13 23) at separation r,
// MCM/mcm_gradw.f90:41-103 with havg = (h_i + h_j)/2.
__device__ __forceinline__ void grad_hess(const double r[3], double havg, double g[3], double H[6]) {
    const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
    const double rad = sqrt(r2);
    double F = 0.0, G2 = 0.0;
    if (rad > 0.0) {
        const double z = rad / havg;
        const double c1 = 1.0 / (kPi * havg * havg * havg);
        double dw = 0.0, dwp = 0.0;
        if (z < 1.0) { dw = c1 * (2.25 * z - 3.0) * z; dwp = c1 * (4.5 * z - 3.0); }
        else if (z < 2.0) { const double t = 2.0 - z; dw = -0.75 * c1 * t * t; dwp = 1.5 * c1 * t; }
        F = dw / (rad * havg);
        G2 = (dwp * z - dw) / (r2 * rad * havg);
    }
    g[0] = F * r[0]; g[1] = F * r[1]; g[2] = F * r[2];
    H[0] = F + G2 * r[0] * r[0]; H[1] = F + G2 * r[1] * r[1]; H[2] = F + G2 * r[2] * r[2];
    H[3] = G2 * r[0] * r[1]; H[4] = G2 * r[0] * r[2]; H[5] = G2 * r[1] * r[2];
}

__device__ __forceinline__ void symv(const double S[6], const double v[3], double o[3]) {
    o[0] = S[0] * v[0] + S[3] * v[1] + S[4] * v[2];
    o[1] = S[3] * v[0] + S[1] * v[1] + S[5] * v[2];
    o[2] = S[4] * v[0] + S[5] * v[1] + S[2] * v[2];
}
// d(a . S g)/dS for the 6 stored components of a symmetric S, times w
__device__ __forceinline__ void add_symouter(double Sb[6], const double a[3], const double g[3], double w) {
    Sb[0] += w * a[0] * g[0];
    Sb[1] += w * a[1] * g[1];
    Sb[2] += w * a[2] * g[2];
    Sb[3] += w * (a[0] * g[1] + a[1] * g[0]);
    Sb[4] += w * (a[0] * g[2] + a[2] * g[0]);
    Sb[5] += w * (a[1] * g[2] + a[2] * g[1]);
}
__device__ __forceinline__ double flip(int mask, int d) { return (mask >> d) & 1 ? -1.0 : 1.0; }

// (sigma - q I)/rho^2 of state index i from the post-constitutive fields
__device__ __forceinline__ void stress_over_rho2(const StepArgs &a, int i, double S[6]) {
    const double *const *f = a.F.f;
    const double rho = f[FRHO][i], r2 = rho * rho, q = f[FQ][i];
    S[0] = (f[FS11][i] - q) / r2; S[1] = (f[FS22][i] - q) / r2; S[2] = (f[FS33][i] - q) / r2;
    S[3] = f[FS12][i] / r2; S[4] = f[FS13][i] / r2; S[5] = f[FS23][i] / r2;
}

// ------------------------------------------------------------------ init
__global__ void k_adj_init(StepArgs a, AdjArgs b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        b.yrho[i] = b.rhob[i]; b.ye[i] = b.eb[i]; b.yp[i] = b.pb[i]; b.yefps[i] = b.efpsb[i];
#pragma unroll
        for (int u = 0; u < 6; ++u) b.ysig[u][i] = b.sigb[u][i];
        b.yq[i] = 0.0;
        b.rho0b[i] = 0.0;
    }
}

// ------------------------------------------------- velocity update + move
// MCM/mcm_update_velocity.f90:29-56, MCM/mcm_move.f90:32-40,
// MCM/mcm_check_sym_pen.f90:27-179 reversed.  The acceleration a and x, v
// are the step's values (x after the constitutive round trip).
__global__ void k_adj_move(StepArgs a, AdjArgs b) {
    const double *const *f = a.F.f;
    const double dtn = 0.5 * (b.dt + b.dtold);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double acc[3] = {f[FAX][i], f[FAY][i], f[FAZ][i]};
        double xb[3] = {b.xb[0][i], b.xb[1][i], b.xb[2][i]};
        double vb[3] = {b.vb[0][i], b.vb[1][i], b.vb[2][i]};
        double xo[3];
        const double *pv[3] = {b.pre[FVX], b.pre[FVY], b.pre[FVZ]};
        const double xc[3] = {f[FX][i], f[FY][i], f[FZ][i]};
        for (int d = 0; d < 3; ++d) {
            const double v1 = a.prm.drelax ? a.prm.drelax_scale * pv[d][i] + acc[d] * dtn : pv[d][i] + acc[d] * dtn;
            xo[d] = xc[d] + v1 * b.dt;
        }
        if (a.prm.boundary) {
            const DevPlanes &pl = a.prm.planes;
            for (int d = 0; d < 3; ++d) {
                bool refl = false;
                double x = xo[d];
                if (pl.code[0][d] == 1 && x < pl.bx[0][d]) { x = 2.0 * pl.bx[0][d] - x; refl = !refl; }
                if (pl.code[1][d] == 1 && x > pl.bx[1][d]) { refl = !refl; }
                if (refl) { xb[d] = -xb[d]; vb[d] = -vb[d]; }
            }
        }
        double ab[3];
        for (int d = 0; d < 3; ++d) {
            const double v1b = vb[d] + xb[d] * b.dt;   // x' = x + v' dt
            ab[d] = v1b * dtn;
            vb[d] = a.prm.drelax ? a.prm.drelax_scale * v1b : v1b;
        }
        // MCM/mcm_boundcond.f90: constrained components of a are zeroed
        switch (a.F.dispbc[i]) {
            case 1: ab[0] = 0.0; break;
            case 2: ab[1] = 0.0; break;
            case 3: ab[2] = 0.0; break;
            case 4: ab[0] = 0.0; ab[1] = 0.0; break;
            case 5: ab[1] = 0.0; ab[2] = 0.0; break;
            case 6: ab[0] = 0.0; ab[2] = 0.0; break;
            case 7: ab[0] = 0.0; ab[1] = 0.0; ab[2] = 0.0; break;
            default: break;
        }
        for (int d = 0; d < 3; ++d) { b.ab[d][i] = ab[d]; b.xb[d][i] = xb[d]; b.vb[d][i] = vb[d]; }
    }
}

// ------------------------------------------------------- gather records
// One record per cell-order position holds what a reverse gather reads of a
// neighbour, so that a neighbour costs 4-5 sectors of one or two lines
// instead of one sector in each of 16-18 field arrays.
// momentum: {x y z h} {S11 S22 S33 S12} {S13 S23 m -} {ab_x ab_y ab_z -}
__global__ void k_adj_pack_momentum(StepArgs a, AdjArgs b) {
    const double *const *f = a.F.f;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int i = a.cell_list[p];
        double S[6];
        stress_over_rho2(a, i, S);
        double4 *r = b.rec + (size_t)p * kRecSlots;
        r[0] = make_double4(f[FX][i], f[FY][i], f[FZ][i], f[FH][i]);
        r[1] = make_double4(S[0], S[1], S[2], S[3]);
        r[2] = make_double4(S[4], S[5], f[FMASS][i], 0.0);
        r[3] = make_double4(b.ab[0][i], b.ab[1][i], b.ab[2][i], 0.0);
    }
}
// strain: {xs_x xs_y xs_z h} {v_x v_y v_z V} {G00 G01 G02 G10} {G11 G12 G20 G21} {G22 - - -}
__global__ void k_adj_pack_strain(StepArgs a, AdjArgs b) {
    const double *const *pre = b.pre;
    const double hdt = 0.5 * b.dt_prev;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += gridDim.x * blockDim.x) {
        const int i = a.cell_list[p];
        const double v[3] = {pre[FVX][i], pre[FVY][i], pre[FVZ][i]};
        double4 *r = b.rec + (size_t)p * kRecSlots;
        r[0] = make_double4(pre[FX][i] - hdt * v[0], pre[FY][i] - hdt * v[1], pre[FZ][i] - hdt * v[2], pre[FH][i]);
        r[1] = make_double4(v[0], v[1], v[2], pre[FMASS][i] / pre[FRHO][i]);
        r[2] = make_double4(b.gb[0][i], b.gb[1][i], b.gb[2][i], b.gb[3][i]);
        r[3] = make_double4(b.gb[4][i], b.gb[5][i], b.gb[6][i], b.gb[7][i]);
        r[4] = make_double4(b.gb[8][i], 0.0, 0.0, 0.0);
    }
}

// ----------------------------------------------------------- momentum
// kLanes lanes share a particle: lane l takes neighbours l, l + kLanes, ...;
// the per-particle sums are combined by shuffles and one lane writes them.
constexpr int kLanes = 4;

template <int N>
__device__ __forceinline__ void lane_sum(double (&v)[N]) {
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1)
#pragma unroll
        for (int u = 0; u < N; ++u) v[u] += __shfl_xor_sync(0xffffffffu, v[u], o);
}

__global__ void __launch_bounds__(128) k_adj_momentum(StepArgs a, AdjArgs b) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) / kLanes;
    const int lane = threadIdx.x % kLanes;
    const bool live = t < a.n;
    const double *const *f = a.F.f;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};   // Sb[6], xb[3]
    double *Sb = acc, *xb = acc + 6;
    int i = 0;
    double Si[6] = {0, 0, 0, 0, 0, 0};
    if (live) {
        i = a.cell_list[t];
        const double xi[3] = {f[FX][i], f[FY][i], f[FZ][i]};
        const double hi = f[FH][i], mi = f[FMASS][i];
        stress_over_rho2(a, i, Si);
        const double abi[3] = {b.ab[0][i], b.ab[1][i], b.ab[2][i]};
        const unsigned *list = a.nidx + (size_t)t * a.nstride;
        const int nreal = stored_neighbours(a, t);
        for (int k = lane; k < nreal; k += kLanes) {
            const double4 *rj = b.rec + (size_t)(list[k] & kPosMask) * kRecSlots;
            const double4 q0 = rj[0], q1 = rj[1], q2 = rj[2], q3 = rj[3];
            const double r[3] = {xi[0] - q0.x, xi[1] - q0.y, xi[2] - q0.z};
            double g[3], H[6];
            grad_hess(r, 0.5 * (hi + q0.w), g, H);
            const double Sj[6] = {q1.x, q1.y, q1.z, q1.w, q2.x, q2.y};
            double T[6];
            const double mj = q2.z;
            const double abj[3] = {q3.x, q3.y, q3.z};
            // own sum: a_i += m_j (S_i + S_j) g
            add_symouter(Sb, abi, g, mj);
#pragma unroll
            for (int u = 0; u < 6; ++u) T[u] = mj * (Si[u] + Sj[u]);
            double Ta[3], HTa[3];
            symv(T, abi, Ta);
            symv(H, Ta, HTa);
            // j's sum: a_j += m_i (S_j + S_i) g(x_j - x_i) = -m_i (S_i + S_j) g
            add_symouter(Sb, abj, g, -mi);
#pragma unroll
            for (int u = 0; u < 6; ++u) T[u] = mi * (Si[u] + Sj[u]);
            double Tb[3], HTb[3];
            symv(T, abj, Tb);
            symv(H, Tb, HTb);
            for (int d = 0; d < 3; ++d) xb[d] += HTa[d] - HTb[d];
        }
        const int gn = a.gnnbr[t];
        for (int k = lane; k < gn; k += kLanes) {
            const int q = a.gnbr[(size_t)k * a.npad + t];
            const int p = a.gpar[q];
            const int fl = a.gflip[q];
            const double r[3] = {xi[0] - a.gx[q], xi[1] - a.gy[q], xi[2] - a.gz[q]};
            double g[3], H[6];
            grad_hess(r, 0.5 * (hi + a.gh[q]), g, H);
            // S_g: the parent's sigma', q' over the ghost's density, off-diagonals negated
            const double rg = a.grho[q], r2 = rg * rg, qp = f[FQ][p];
            const double Sg[6] = {(f[FS11][p] - qp) / r2, (f[FS22][p] - qp) / r2, (f[FS33][p] - qp) / r2,
                                  -f[FS12][p] / r2, -f[FS13][p] / r2, -f[FS23][p] / r2};
            const double mg = a.gmass[q];
            add_symouter(Sb, abi, g, mg);
            double T[6], Ta[3], HTa[3];
#pragma unroll
            for (int u = 0; u < 6; ++u) T[u] = mg * (Si[u] + Sg[u]);
            symv(T, abi, Ta);
            symv(H, Ta, HTa);
            for (int d = 0; d < 3; ++d) xb[d] += HTa[d];
            // ghost side, to the parent: S_g, rho_g (the parent's density at neighbour time), x_g
            double Sgb[6] = {0, 0, 0, 0, 0, 0};
            add_symouter(Sgb, abi, g, mg);
            atomicAdd(&b.ysig[0][p], Sgb[0] / r2);
            atomicAdd(&b.ysig[1][p], Sgb[1] / r2);
            atomicAdd(&b.ysig[2][p], Sgb[2] / r2);
            atomicAdd(&b.ysig[3][p], -Sgb[3] / r2);
            atomicAdd(&b.ysig[4][p], -Sgb[4] / r2);
            atomicAdd(&b.ysig[5][p], -Sgb[5] / r2);
            atomicAdd(&b.yq[p], -(Sgb[0] + Sgb[1] + Sgb[2]) / r2);
            double dot = 0.0;
#pragma unroll
            for (int u = 0; u < 6; ++u) dot += Sgb[u] * Sg[u];
            atomicAdd(&b.rho0b[p], -2.0 * dot / rg);
            for (int d = 0; d < 3; ++d) atomicAdd(&b.xb[d][p], -flip(fl, d) * HTa[d]);
        }
    }
    lane_sum(acc);
    if (!live || lane != 0) return;
    // S_i = (sigma' - q' I)/rho'^2 -> sigma', q', rho'
    const double rho = f[FRHO][i], r2 = rho * rho;
    atomicAdd(&b.ysig[0][i], Sb[0] / r2);
    atomicAdd(&b.ysig[1][i], Sb[1] / r2);
    atomicAdd(&b.ysig[2][i], Sb[2] / r2);
    atomicAdd(&b.ysig[3][i], Sb[3] / r2);
    atomicAdd(&b.ysig[4][i], Sb[4] / r2);
    atomicAdd(&b.ysig[5][i], Sb[5] / r2);
    atomicAdd(&b.yq[i], -(Sb[0] + Sb[1] + Sb[2]) / r2);
    double dot = 0.0;
#pragma unroll
    for (int u = 0; u < 6; ++u) dot += Sb[u] * Si[u];
    atomicAdd(&b.yrho[i], -2.0 * dot / rho);
    for (int d = 0; d < 3; ++d) atomicAdd(&b.xb[d][i], xb[d]);
}

// ------------------------------------------------------- constitutive
// Vector-Jacobian product of the per-particle update (rhoupd + model 10 +
// EOS 41 chain) by forward-mode duals, kND input directions per pass.  The
// passes and their seed directions are compile-time constants, so that no
// part of the dual state is addressed through a runtime index (which would
// put it in local memory).

// Sets derivative slot k of seed direction s (inputs, then parameters).
// Every case names its field with a constant index, so a runtime s selects a
// register and does not index the dual state.
__device__ __forceinline__ void seed(PState<D> &P, DualMat &M, int s, int k) {
    switch (s) {
        case 0: P.rho.d[k] = 1.0; break;
        case 1: P.e.d[k] = 1.0; break;
        case 2: P.p.d[k] = 1.0; break;
        case 3: P.efps.d[k] = 1.0; break;
        case 4: P.sig[0].d[k] = 1.0; break;
        case 5: P.sig[1].d[k] = 1.0; break;
        case 6: P.sig[2].d[k] = 1.0; break;
        case 7: P.sig[3].d[k] = 1.0; break;
        case 8: P.sig[4].d[k] = 1.0; break;
        case 9: P.sig[5].d[k] = 1.0; break;
        case 10: P.rod[0].d[k] = 1.0; break;
        case 11: P.rod[1].d[k] = 1.0; break;
        case 12: P.rod[2].d[k] = 1.0; break;
        case 13: P.rod[3].d[k] = 1.0; break;
        case 14: P.rod[4].d[k] = 1.0; break;
        case 15: P.rod[5].d[k] = 1.0; break;
        case 16: P.spin[0].d[k] = 1.0; break;
        case 17: P.spin[1].d[k] = 1.0; break;
        case 18: P.spin[2].d[k] = 1.0; break;
        case 19: P.tracerod.d[k] = 1.0; break;
        case kInputs + 0:                                                     // strinput(1)
            M.strinput.gmod.d[k] = 1.0;
            if (M.model == 10) M.g.d[k] = 1.0;   // mcm_calcg: g = strinput(1) for model 10, 0 for model 9
            break;
        case kInputs + 1: M.strinput.yield.d[k] = 1.0; break;                 // yield stress
        case kInputs + 2: M.strinput.hard.d[k] = 1.0; break;                  // hardening modulus
        case kInputs + 3: M.eosinput.slope.d[k] = 1.0; break;                 // EOS-41 slope s
        default: break;
    }
}

__device__ __forceinline__ void constitutive_pass(int pass, const StepArgs &a, const AdjArgs &b, int i, int mat,
                                                  const DevMaterial &M0, const double (&yb)[11],
                                                  double (&ub)[kInputs], double (&th)[kParams]) {
    const double *const *pre = b.pre;
    const double *const *f = a.F.f;
    DualMat M;
    M.model = M0.model; M.eos = M0.eos; M.visc_type = M0.visc_type; M.pad = 0;
    M.rho = M0.rho; M.av_l = M0.av_l; M.av_q = M0.av_q;
    M.mass = M0.mass; M.h = M0.h; M.rho_min = M0.rho_min; M.rho_max = M0.rho_max;
    M.g = D(M0.g);
#pragma unroll
    for (int k = 0; k < kStr; ++k) M.strinput.v[k] = M0.strinput[k];
#pragma unroll
    for (int k = 0; k < kEos; ++k) M.eosinput.v[k] = M0.eosinput[k];
    M.strinput.gmod = D(M0.strinput[0]);
    M.strinput.yield = D(M0.strinput[1]);
    M.strinput.hard = D(M0.strinput[2]);
    M.eosinput.slope = D(M0.eosinput[1]);
    PState<D> P;
    P.mat = mat;
    P.mass = D(pre[FMASS][i]); P.h = D(pre[FH][i]); P.hold = D(pre[FHOLD][i]);
    P.rho = D(pre[FRHO][i]); P.e = D(pre[FE][i]); P.p = D(pre[FP][i]); P.c = D(pre[FC][i]);
    P.efps = D(pre[FEFPS][i]); P.pcut = D(pre[FPCUT][i]); P.p_cut = D(pre[FPCUT2][i]);
    P.fail = D(pre[FFAIL][i]); P.capa = D(0.0);
    P.rho0 = D(M0.rho);
#pragma unroll
    for (int u = 0; u < 6; ++u) {
        P.sig[u] = D(pre[FS11 + u][i]); P.s[u] = D(0.0); P.alfa[u] = D(0.0);
        P.rod[u] = D(f[FR11 + u][i]);
    }
    P.spin[0] = D(f[FW12][i]); P.spin[1] = D(f[FW13][i]); P.spin[2] = D(f[FW23][i]);
    P.tracerod = D(f[FTR][i]);
    P.q = D(0.0);
#pragma unroll
    for (int k = 0; k < kND; ++k) seed(P, M, pass * kND + k, k);
    sym_lower(P);   // model 10: the lower triangle is the (seeded) upper one
    P.etry = D(0.0); P.einc = D(0.0); P.rhoold = P.rho;
    const D dt = D(b.dt_prev);
    rhoupd(P, M, dt, 3);
    constitutive_particle(P, M, dt);
#pragma unroll
    for (int k = 0; k < kND; ++k) {
        const int s = pass * kND + k;
        if (s >= kSeeds) break;
        const double acc = yb[0] * P.rho.d[k] + yb[1] * P.e.d[k] + yb[2] * P.p.d[k] + yb[3] * P.efps.d[k] +
                           yb[4] * P.sig[0].d[k] + yb[5] * P.sig[1].d[k] + yb[6] * P.sig[2].d[k] +
                           yb[7] * P.sig[3].d[k] + yb[8] * P.sig[4].d[k] + yb[9] * P.sig[5].d[k] +
                           yb[10] * P.q.d[k];
        if (s < kInputs) ub[s] = acc;
        else th[s - kInputs] = acc;
    }
}

// ------------------------------------------- constitutive, reverse mode
// The vector-Jacobian product of the per-particle update for model 10 with
// EOS 41 in one reverse pass (no dual numbers): the forward values of
// rhoupd, the Jaumann rotation, f3dm10, eos41c, nodalav, hieupd, eqos41 and
// stress_up are recomputed with the step's expressions (this translation
// unit has no fused multiply-add, like the dual passes), the branches taken
// are kept, and the adjoints are propagated back through them.  The only
// derivative taken in forward mode is that of the rotation matrix with
// respect to the three spin components.
__device__ __forceinline__ double f_tmax(double a, double b) { return a > b ? a : (b > a ? b : a); }

__device__ __forceinline__ void reverse_m10_eos41(const StepArgs &a, const AdjArgs &b, int i, const DevMaterial &M,
                                                  const double (&yb)[11], double (&ub)[kInputs],
                                                  double (&th)[kParams]) {
    const double *const *pre = b.pre;
    const double *const *f = a.F.f;
    const double dt = b.dt_prev;
    const double third = 1.0 / 3.0;
    const double f30 = (double)1.e-30f, f12 = (double)1.e-12f;
    // ------------------------------------------------------------ forward
    const double mass = pre[FMASS][i], hpart = pre[FH][i], rho0 = M.rho;
    const double rho_in = pre[FRHO][i], e_in = pre[FE][i], efps_in = pre[FEFPS][i];
    const double pcut_in = pre[FPCUT][i], fail_in = pre[FFAIL][i];
    double sg[6], rod[6];
#pragma unroll
    for (int u = 0; u < 6; ++u) { sg[u] = pre[FS11 + u][i]; rod[u] = f[FR11 + u][i]; }
    const double spin[3] = {f[FW12][i], f[FW13][i], f[FW23][i]};
    const double tr_in = f[FTR][i];
    // rhoupd (MCM/mcm_rhoupd.f90:24-56)
    const double rfac = 1.0 - tr_in * dt;
    const double rho_a = rho_in * rfac;
    const bool capped = rho_a > M.rho_max;
    const double rho1 = capped ? rho_a / rfac : rho_a;
    const double tr = capped ? 0.0 : tr_in;
    if (capped) {
        rod[0] = rod[0] - third * tr_in;
        rod[1] = rod[1] - third * tr_in;
        rod[2] = rod[2] - third * tr_in;
    }
    // Jaumann rotation: sp = Q S Q^T (S symmetric, its (3,1) the upper 13)
    double Q[9];
    jaumann_q(spin, dt, Q);
    const double S[9] = {sg[T11], sg[T12], sg[T13], sg[T12], sg[T22], sg[T23], sg[T13], sg[T23], sg[T33]};
    double QS[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) QS[3 * r + c] = Q[3 * r] * S[c] + Q[3 * r + 1] * S[3 + c] + Q[3 * r + 2] * S[6 + c];
    // the six outputs as (row, column) of Q S Q^T, storage order 11 22 33 12 13 23
    constexpr int RR[6] = {0, 1, 2, 0, 0, 1}, RC[6] = {0, 1, 2, 1, 2, 2};
    double sp[6];
#pragma unroll
    for (int u = 0; u < 6; ++u)
        sp[u] = QS[3 * RR[u]] * Q[3 * RC[u]] + QS[3 * RR[u] + 1] * Q[3 * RC[u] + 1] + QS[3 * RR[u] + 2] * Q[3 * RC[u] + 2];
    // f3dm10 (MCM/mcm_f3dm10.f90:28-157)
    const double gg = M.strinput[0], qs = M.strinput[1], qh = M.strinput[2], a1 = M.strinput[4], a2 = M.strinput[5];
    const int ispall = (int)M.strinput[6];
    const double epf = M.strinput[7];
    const double g2 = 2.0 * dt * gg;
    const double davg = third * tr;
    const double p3 = -third * (sp[0] + sp[1] + sp[2]);
    const double mp = f_tmax(0.0, p3);
    const double ak0 = qs + qh * efps_in + (a1 + a2 * p3) * mp;
    double s1[6];
#pragma unroll
    for (int d = 0; d < 3; ++d) s1[d] = sp[d] + p3 + g2 * (rod[d] + davg);
#pragma unroll
    for (int d = 3; d < 6; ++d) s1[d] = sp[d] + 0.5 * g2 * rod[d];
    double scle3 = 1.0, pcut = pcut_in;
    if (ispall == 3) {
        scle3 = 0.5 * (1.0 + (p3 - pcut >= 0.0 ? 1.0 : -1.0));
        pcut = scle3 * pcut;
#pragma unroll
        for (int u = 0; u < 6; ++u) s1[u] = scle3 * s1[u];
    }
    const double aj2 = 0.5 * (s1[0] * s1[0] + s1[1] * s1[1] + s1[2] * s1[2]) + s1[3] * s1[3] + s1[4] * s1[4] + s1[5] * s1[5];
    const double sj2 = sqrt(3.0 * aj2);
    const bool yielding = fail_in == 1.0;
    double thrg = 0.0, den = 0.0, fdv = 0.0, t1 = 0.0, defps = 0.0;
    bool fd_on = false, den_on = false, m_is_sj2 = false;
    if (yielding) {
        thrg = third / gg;
        fd_on = sj2 > ak0;
        fdv = fd_on ? sj2 - ak0 : 0.0;
        den_on = 1.0 > -thrg * qh;
        den = f30 + (den_on ? 1.0 - (-thrg * qh) : 0.0);
        t1 = fdv / den;
        m_is_sj2 = !(t1 < sj2);   // tmin(sj2, t1): sj2 unless t1 < sj2
        defps = thrg * (m_is_sj2 ? sj2 : t1);
    }
    const double efps_out = yielding ? efps_in + defps : efps_in;
    const double xk = ak0 + qh * defps;
    const bool xk_on = !(0.0 > xk);   // tmax(xk, 0): xk unless 0 > xk
    const double ak2 = xk_on ? xk : 0.0;
    const double seps = f30 * gg;
    const bool mx_is_ak = !(sj2 > ak2);   // tmax(ak2, sj2)
    const double mx = mx_is_ak ? ak2 : sj2;
    const double scle = (ak2 + seps) / (mx + seps);
    double s2[6];
#pragma unroll
    for (int u = 0; u < 6; ++u) s2[u] = scle * s1[u];
    const bool broke = epf != 0.0 && efps_out > epf;
    double scle2 = 1.0;
    if (broke) {
#pragma unroll
        for (int u = 0; u < 6; ++u) s2[u] = 0.0;
    }
    if (ispall == 2) {
        const double aj = 0.5 * (s2[0] * s2[0] + s2[1] * s2[1] + s2[2] * s2[2]) + s2[3] * s2[3] + s2[4] * s2[4] +
                          s2[5] * s2[5] + f12;
        const double dj = s2[0] * s2[5] * s2[5] + s2[1] * s2[4] * s2[4] + s2[2] * s2[3] * s2[3] -
                          s2[0] * s2[1] * s2[2] - 2.0 * s2[3] * s2[4] * s2[5];
        double akt = -sqrt(27.0 / aj) * dj * 0.5 / aj;
        const double am = fabs(akt) < 1.0 ? fabs(akt) : (1.0 < fabs(akt) ? 1.0 : fabs(akt));
        akt = akt >= 0.0 ? am : -am;
        const double ywh = acos(akt) * third;
        const double sjp = 2.0 * sqrt(aj * third) * cos(ywh);
        scle2 = 0.5 * (1.0 + (p3 - sjp - pcut >= 0.0 ? 1.0 : -1.0));
        pcut = scle2 * pcut;
#pragma unroll
        for (int u = 0; u < 6; ++u) s2[u] = scle2 * s2[u];
    }
    // eos41c (MCM/mcm_eos41c.f90:31-85): the sound speed of nodalav
    const double cc = M.eosinput[0], sl = M.eosinput[1], gamma0 = M.eosinput[4];
    const double e1 = e_in / mass;
    const double ao = rho0 * (cc * cc);
    const double mu = rho1 / rho0 - 1.0;
    const double gam = gamma0 * rho0 / rho1;
    const double bo = ao * (1.0 + 2.0 * (sl - 1.0));
    const double co = ao * (2.0 * (sl - 1.0) + 3.0 * ((sl - 1.0) * (sl - 1.0)));
    const double fg = gam * mu;
    const double ca1 = ao * (1.0 - fg), cb1 = bo * (2.0 - 1.5 * fg), cc1 = co * (3.0 - 2.0 * fg);
    const bool comp = mu > 0.0;
    const double dpdrho = comp ? (ca1 + cb1 * mu + cc1 * (mu * mu)) / rho0 + gam * e1 : ao * (1.0 - fg) / rho0 + gam * e1;
    const bool at_cut = p3 == pcut;
    const double c2 = at_cut ? cc * cc : dpdrho + (gam * rho1) * (p3 / (rho1 * rho1));
    const double csnd = sqrt(c2);
    // nodalav (MCM/mcm_nodalav.f90:32-47)
    const bool visc = M.visc_type == 1 && tr < 0.0;
    double q = 0.0;
    if (visc) {
        const double ht = hpart * tr;
        q = M.av_l * rho1 * csnd * hpart * fabs(tr) + M.av_q * rho1 * (ht * ht);
    }
    // hieupd (MCM/mcm_hieupd.f90:27-64)
    const double pold = p3;
    const double trq = third * (q + q + q);
    const double volold = mass / rho_in, volnew = mass / rho1;
    double einc = 0.0;
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int t = sym_index(k, l);
            const double de = (k == l) ? rod[t] * (0.5 * (sp[t] + pold + s2[t]) - q + trq) : rod[t] * (0.5 * (sp[t] + s2[t]));
            einc = einc + de;
        }
    const double vavg = 0.5 * (volnew + volold);
    const double dvh = volnew - volold;
    const double etry = e_in + dt * (vavg * einc) - dvh * (0.5 * pold + trq);
    // eqos41 (MCM/mcm_eqos41.f90:32-102)
    const double etry1 = etry / mass;
    const double dvol = mass / rho1 - mass / rho_in;
    const double vol0 = mass / rho0;
    const double ph = comp ? ao * mu + bo * (mu * mu) + co * (mu * mu * mu) : ao * mu;
    const double rg = rho1 * gam;
    const double num = ph * (1.0 - 0.5 * fg) + rg * etry1;
    const double dnm = 1.0 + 0.5 * rho1 * gam * dvol / vol0;
    const double pn = num / dnm;
    const bool clamp = pn < pcut;
    const double rfac2 = 1.0 - tr * dt;
    // ------------------------------------------------------------ reverse
    // outputs: rho, e, p, efps, sigma (11 22 33 12 13 23), q
    double rho1_b = 0.0, rhoin_b = 0.0, ein_b = 0.0, tr_b = 0.0, efps_b = 0.0;
    double gg_b = 0.0, qs_b = 0.0, qh_b = 0.0, sl_b = 0.0;
    double sp_b[6] = {0, 0, 0, 0, 0, 0}, s2_b[6], rod_b[6] = {0, 0, 0, 0, 0, 0};
    double p3_b = 0.0, q_b = yb[10];
    // stress_up: sigma = s - p I
    double p_b = yb[2] - (yb[4] + yb[5] + yb[6]);
#pragma unroll
    for (int u = 0; u < 6; ++u) s2_b[u] = yb[4 + u];
    // eqos41
    double etry_b = 0.0, rg_b = 0.0, dvol_b = 0.0, ph_b = 0.0, fg_b = 0.0, mu_b = 0.0, gam_b = 0.0, bo_b = 0.0,
           co_b = 0.0;
    if (clamp) {
        // p = pcut (no derivative); rho = rho1 / (1 - tr dt); e unchanged
        const double rho_out = rho1 / rfac2;
        rho1_b += yb[0] / rfac2;
        tr_b += (-yb[0] * rho_out / rfac2) * (-dt);
        ein_b += yb[1];
    } else {
        rho1_b += yb[0];
        // e = etry1 mass - dvol pn / 2
        double pn_b = p_b - 0.5 * dvol * yb[1];
        double etry1_b = yb[1] * mass;
        dvol_b += -0.5 * pn * yb[1];
        const double num_b = pn_b / dnm, dnm_b = -pn_b * pn / dnm;
        ph_b += num_b * (1.0 - 0.5 * fg);
        fg_b += -0.5 * ph * num_b;
        rg_b += num_b * etry1 + dnm_b * 0.5 * dvol / vol0;
        etry1_b += num_b * rg;
        dvol_b += dnm_b * 0.5 * rg / vol0;
        etry_b += etry1_b / mass;
    }
    // ph
    if (comp) {
        mu_b += ph_b * (ao + 2.0 * bo * mu + 3.0 * co * (mu * mu));
        bo_b += ph_b * (mu * mu);
        co_b += ph_b * (mu * mu * mu);
    } else {
        mu_b += ph_b * ao;
    }
    // rg = rho1 gam, dvol = m/rho1 - m/rho_in
    rho1_b += rg_b * gam;
    gam_b += rg_b * rho1;
    rho1_b += dvol_b * (-mass / (rho1 * rho1));
    rhoin_b += dvol_b * (mass / (rho_in * rho_in));
    // hieupd: etry = e + dt vavg einc - dvh (pold/2 + trq)
    ein_b += etry_b;
    const double einc_b = etry_b * dt * vavg;
    const double vavg_b = etry_b * dt * einc;
    const double dvh_b = -etry_b * (0.5 * pold + trq);
    double pold_b = -etry_b * dvh * 0.5;
    double trq_b = -etry_b * dvh;
    const double vn_b = dvh_b + 0.5 * vavg_b, vo_b = -dvh_b + 0.5 * vavg_b;
    rho1_b += vn_b * (-mass / (rho1 * rho1));
    rhoin_b += vo_b * (-mass / (rho_in * rho_in));
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        rod_b[d] += einc_b * (0.5 * (sp[d] + pold + s2[d]) - q + trq);
        sp_b[d] += einc_b * 0.5 * rod[d];
        pold_b += einc_b * 0.5 * rod[d];
        s2_b[d] += einc_b * 0.5 * rod[d];
        q_b += -einc_b * rod[d];
        trq_b += einc_b * rod[d];
    }
#pragma unroll
    for (int u = 3; u < 6; ++u) {
        // (k, l) and (l, k): twice rod (sigma + s) / 2
        rod_b[u] += einc_b * (sp[u] + s2[u]);
        sp_b[u] += einc_b * rod[u];
        s2_b[u] += einc_b * rod[u];
    }
    q_b += trq_b;   // trq = (q + q + q) / 3
    p3_b += pold_b;
    // nodalav
    double c_b = 0.0;
    if (visc) {
        const double atr = fabs(tr);
        rho1_b += q_b * (M.av_l * csnd * hpart * atr + M.av_q * (hpart * tr) * (hpart * tr));
        c_b += q_b * M.av_l * rho1 * hpart * atr;
        tr_b += q_b * (-M.av_l * rho1 * csnd * hpart + M.av_q * rho1 * 2.0 * hpart * hpart * tr);
    }
    // eos41c
    if (!at_cut) {
        const double c2_b = csnd > 0.0 ? c_b * 0.5 / csnd : 0.0;
        // c2 = dpdrho + (gam rho1) (p3 / rho1^2)
        const double A = gam * rho1, B = p3 / (rho1 * rho1);
        gam_b += c2_b * B * rho1;
        rho1_b += c2_b * B * gam;
        p3_b += c2_b * A / (rho1 * rho1);
        rho1_b += c2_b * A * (-2.0 * p3 / (rho1 * rho1 * rho1));
        const double e1_b = c2_b * gam;
        gam_b += c2_b * e1;
        ein_b += e1_b / mass;
        if (comp) {
            const double ca1_b = c2_b / rho0, cb1_b = c2_b * mu / rho0, cc1_b = c2_b * (mu * mu) / rho0;
            mu_b += c2_b * (cb1 + 2.0 * cc1 * mu) / rho0;
            fg_b += -ca1_b * ao - 1.5 * cb1_b * bo - 2.0 * cc1_b * co;
            bo_b += cb1_b * (2.0 - 1.5 * fg);
            co_b += cc1_b * (3.0 - 2.0 * fg);
        } else {
            fg_b += -c2_b * ao / rho0;
        }
    }
    // fg = gam mu, gam = gamma0 rho0 / rho1, mu = rho1 / rho0 - 1, bo(s), co(s)
    gam_b += fg_b * mu;
    mu_b += fg_b * gam;
    rho1_b += gam_b * (-gam / rho1);
    rho1_b += mu_b / rho0;
    sl_b += bo_b * 2.0 * ao + co_b * ao * (2.0 + 6.0 * (sl - 1.0));
    // f3dm10, backwards
    double s1_b[6];
#pragma unroll
    for (int u = 0; u < 6; ++u) s1_b[u] = (broke ? 0.0 : scle * scle2 * s2_b[u]);
    double scle_b = 0.0;
    if (!broke) {
#pragma unroll
        for (int u = 0; u < 6; ++u) scle_b += scle2 * s2_b[u] * s1[u];
    }
    // scle = (ak2 + seps) / (mx + seps)
    const double nu_b = scle_b / (mx + seps), de_b = -scle_b * scle / (mx + seps);
    double ak2_b = nu_b, sj2_b = 0.0;
    gg_b += (nu_b + de_b) * f30;
    if (mx_is_ak) ak2_b += de_b; else sj2_b += de_b;
    double ak0_b = 0.0, defps_b = 0.0;
    if (xk_on) { ak0_b += ak2_b; qh_b += ak2_b * defps; defps_b += ak2_b * qh; }
    efps_b += yb[3];   // efps_out = efps_in (+ defps)
    if (yielding) {
        defps_b += yb[3];
        const double m_b = defps_b * thrg;
        double thrg_b = defps_b * (m_is_sj2 ? sj2 : t1);
        double t1_b = 0.0;
        if (m_is_sj2) sj2_b += m_b; else t1_b = m_b;
        const double fd_b = t1_b / den, den_b = -t1_b * t1 / den;
        if (fd_on) { sj2_b += fd_b; ak0_b -= fd_b; }
        if (den_on) { thrg_b += den_b * qh; qh_b += den_b * thrg; }   // den = 1e-30 + 1 + thrg qh
        gg_b += thrg_b * (-thrg / gg);
    }
    // sj2 = sqrt(3 aj2)
    const double aj2_b = sj2 > 0.0 ? sj2_b * 1.5 / sj2 : 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) s1_b[d] += aj2_b * s1[d];
#pragma unroll
    for (int u = 3; u < 6; ++u) s1_b[u] += aj2_b * 2.0 * s1[u];
    // s1 = scle3 (sp + p3 I + g2 (rod + davg I)) on the diagonal, scle3 (sp + g2 rod / 2) off it
    double g2_b = 0.0, davg_b = 0.0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double s0_b = scle3 * s1_b[d];
        sp_b[d] += s0_b;
        p3_b += s0_b;
        g2_b += s0_b * (rod[d] + davg);
        rod_b[d] += s0_b * g2;
        davg_b += s0_b * g2;
    }
#pragma unroll
    for (int u = 3; u < 6; ++u) {
        const double s0_b = scle3 * s1_b[u];
        sp_b[u] += s0_b;
        g2_b += s0_b * 0.5 * rod[u];
        rod_b[u] += s0_b * 0.5 * g2;
    }
    tr_b += davg_b * third;
    gg_b += g2_b * 2.0 * dt;
    // ak0 = qs + qh efps + (a1 + a2 p3) max(0, p3)
    qs_b += ak0_b;
    qh_b += ak0_b * efps_in;
    efps_b += ak0_b * qh;
    p3_b += ak0_b * (a2 * mp + (p3 > 0.0 ? a1 + a2 * p3 : 0.0));
#pragma unroll
    for (int d = 0; d < 3; ++d) sp_b[d] += -third * p3_b;
    // rotation: sp_u = sum_k QS[r][k] Q[c][k]; QS = Q S
    double QS_b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, Q_b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int u = 0; u < 6; ++u)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            QS_b[3 * RR[u] + k] += sp_b[u] * Q[3 * RC[u] + k];
            Q_b[3 * RC[u] + k] += sp_b[u] * QS[3 * RR[u] + k];
        }
    double S_b[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                Q_b[3 * r + j] += QS_b[3 * r + k] * S[3 * j + k];
                S_b[3 * j + k] += QS_b[3 * r + k] * Q[3 * r + j];
            }
    // dQ/dspin by three forward directions
    {
        using D3 = Dual<3>;
        D3 w[3] = {D3(spin[0]), D3(spin[1]), D3(spin[2])};
        w[0].d[0] = 1.0; w[1].d[1] = 1.0; w[2].d[2] = 1.0;
        D3 Qd[9];
        jaumann_q(w, D3(dt), Qd);
        double wb[3] = {0, 0, 0};
#pragma unroll
        for (int u = 0; u < 9; ++u)
#pragma unroll
            for (int k = 0; k < 3; ++k) wb[k] += Q_b[u] * Qd[u].d[k];
        ub[16] = wb[0]; ub[17] = wb[1]; ub[18] = wb[2];
    }
    // rhoupd
    if (capped) {
        // rho1 = (rho_in rfac) / rfac; rod diagonal -= tr_in / 3; tracerod <- 0
        const double ra_b = rho1_b / rfac;
        double rf_b = -rho1_b * rho1 / rfac;
        rhoin_b += ra_b * rfac;
        rf_b += ra_b * rho_in;
        double trin_b = rf_b * (-dt);
        trin_b += -third * (rod_b[0] + rod_b[1] + rod_b[2]);
        tr_b = trin_b;   // the downstream tracerod is the constant 0
    } else {
        rhoin_b += rho1_b * rfac;
        tr_b += rho1_b * (-rho_in * dt);
    }
    // inputs: rho e p efps sigma(6) rod(6) spin(3) tr; sigma (3,1) is read as the upper 13
    ub[0] = rhoin_b;
    ub[1] = ein_b;
    ub[2] = 0.0;   // the incoming pressure is overwritten by f3dm10
    ub[3] = efps_b;
    ub[4] = S_b[0];
    ub[5] = S_b[4];
    ub[6] = S_b[8];
    ub[7] = S_b[1] + S_b[3];
    ub[8] = S_b[2] + S_b[6];
    ub[9] = S_b[5] + S_b[7];
#pragma unroll
    for (int u = 0; u < 6; ++u) ub[10 + u] = rod_b[u];
    ub[19] = tr_b;
    th[0] = gg_b;
    th[1] = qs_b;
    th[2] = qh_b;
    th[3] = sl_b;
}

// REV: one hand-written reverse pass per particle (every material model 10
// with EOS 41); otherwise kPasses dual-number passes.
template <bool REV, int NT>
__global__ void __launch_bounds__(NT) k_adj_constitutive(StepArgs a, AdjArgs b) {
    __shared__ double sth[kParams][NT];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double th[kParams] = {0, 0, 0, 0};
    if (i < a.n) {
        const int mat = a.F.mat[i];
        const DevMaterial &M0 = a.mats[mat - 1];
        double ub[kInputs];
#pragma unroll
        for (int u = 0; u < kInputs; ++u) ub[u] = 0.0;
        const double yb[11] = {b.yrho[i], b.ye[i], b.yp[i], b.yefps[i], b.ysig[0][i], b.ysig[1][i],
                               b.ysig[2][i], b.ysig[3][i], b.ysig[4][i], b.ysig[5][i], b.yq[i]};
        if constexpr (REV) {
            reverse_m10_eos41(a, b, i, M0, yb, ub, th);
        } else {
#pragma unroll 1
            for (int pass = 0; pass < kPasses; ++pass) constitutive_pass(pass, a, b, i, mat, M0, yb, ub, th);
        }
        b.rhob[i] = ub[0] + b.rho0b[i];
        b.eb[i] = ub[1];
        b.pb[i] = ub[2];
        b.efpsb[i] = ub[3];
        for (int u = 0; u < 6; ++u) b.sigb[u][i] = ub[4 + u];
        // rod (11 22 33 12 13 23), spin (12 13 23), tr -> G adjoint (row = velocity component)
        const double *rb = ub + 10, *wb = ub + 16, trb = ub[19];
        b.gb[0][i] = rb[0] + trb;            // G00
        b.gb[4][i] = rb[1] + trb;            // G11
        b.gb[8][i] = rb[2] + trb;            // G22
        b.gb[1][i] = 0.5 * (rb[3] + wb[0]);  // G01
        b.gb[3][i] = 0.5 * (rb[3] - wb[0]);  // G10
        b.gb[2][i] = 0.5 * (rb[4] + wb[1]);  // G02
        b.gb[6][i] = 0.5 * (rb[4] - wb[1]);  // G20
        b.gb[5][i] = 0.5 * (rb[5] + wb[2]);  // G12
        b.gb[7][i] = 0.5 * (rb[5] - wb[2]);  // G21
    }
    // parameter adjoints: block sums, one atomic per block and parameter
    for (int k = 0; k < kParams; ++k) sth[k][threadIdx.x] = th[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        // blocks are small and materials few: sum per material serially
        for (int m = 1; m <= a.nmat; ++m) {
            double s[kParams] = {0, 0, 0, 0};
            bool any = false;
            for (int l = 0; l < (int)blockDim.x; ++l) {
                const int il = blockIdx.x * blockDim.x + l;
                if (il >= a.n || a.F.mat[il] != m) continue;
                any = true;
                for (int k = 0; k < kParams; ++k) s[k] += sth[k][l];
            }
            if (any)
                for (int k = 0; k < kParams; ++k) atomicAdd(&b.theta_b[(m - 1) * kParams + k], s[k]);
        }
    }
}

// ----------------------------------------------------------- strain rate
__device__ __forceinline__ void load_G(const AdjArgs &b, int i, double G[9]) {
#pragma unroll
    for (int u = 0; u < 9; ++u) G[u] = b.gb[u][i];
}

__global__ void __launch_bounds__(128) k_adj_strain(StepArgs a, AdjArgs b) {
    const int t = (blockIdx.x * blockDim.x + threadIdx.x) / kLanes;
    const int lane = threadIdx.x % kLanes;
    const bool live = t < a.n;
    const double *const *pre = b.pre;
    const double hdt = 0.5 * b.dt_prev;
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};   // vb[3], xsb[3], Vb
    double *vb = acc, *xsb = acc + 3;
    int i = 0;
    double Vi = 0.0;
    if (live) {
        i = a.cell_list[t];
        const double vi[3] = {pre[FVX][i], pre[FVY][i], pre[FVZ][i]};
        const double xsi[3] = {pre[FX][i] - hdt * vi[0], pre[FY][i] - hdt * vi[1], pre[FZ][i] - hdt * vi[2]};
        const double hi = pre[FH][i];
        Vi = pre[FMASS][i] / pre[FRHO][i];
        double Gi[9];
        load_G(b, i, Gi);
        const unsigned *list = a.nidx + (size_t)t * a.nstride;
        const int nreal = stored_neighbours(a, t);
        for (int k = lane; k < nreal; k += kLanes) {
            const double4 *rj = b.rec + (size_t)(list[k] & kPosMask) * kRecSlots;
            const double4 q0 = rj[0], q1 = rj[1], q2 = rj[2], q3 = rj[3], q4 = rj[4];
            const double vj[3] = {q1.x, q1.y, q1.z};
            const double r[3] = {xsi[0] - q0.x, xsi[1] - q0.y, xsi[2] - q0.z};
            double g[3], H[6];
            grad_hess(r, 0.5 * (hi + q0.w), g, H);
            const double Vj = q1.w;
            const double dv[3] = {vj[0] - vi[0], vj[1] - vi[1], vj[2] - vi[2]};
            const double Gj[9] = {q2.x, q2.y, q2.z, q2.w, q3.x, q3.y, q3.z, q3.w, q4.x};
            // own sum: G_i += V_j dv (x) g
            double Gig[3], GiTdv[3], Gjg[3], GjTdv[3];
            for (int n = 0; n < 3; ++n) {
                Gig[n] = Gi[3 * n] * g[0] + Gi[3 * n + 1] * g[1] + Gi[3 * n + 2] * g[2];
                Gjg[n] = Gj[3 * n] * g[0] + Gj[3 * n + 1] * g[1] + Gj[3 * n + 2] * g[2];
                GiTdv[n] = Gi[n] * dv[0] + Gi[3 + n] * dv[1] + Gi[6 + n] * dv[2];
                GjTdv[n] = Gj[n] * dv[0] + Gj[3 + n] * dv[1] + Gj[6 + n] * dv[2];
            }
            double HGi[3], HGj[3];
            symv(H, GiTdv, HGi);
            symv(H, GjTdv, HGj);
            for (int d = 0; d < 3; ++d) {
                vb[d] -= Vj * Gig[d];
                // j's sum: G_j += V_i (v_i - v_j) (x) g(xs_j - xs_i) = V_i dv (x) g
                vb[d] -= Vi * Gjg[d];
                xsb[d] += Vj * HGi[d];
                // d/dxs_i of V_i dv (x) g(xs_j - xs_i): -V_i H (G_j^T (v_i - v_j)) = +V_i H (G_j^T dv)
                xsb[d] += Vi * HGj[d];
            }
            // d/dV_i of G_j's term V_i (v_i - v_j) (x) g(xs_j - xs_i) = V_i dv (x) g(r)
            acc[6] += dv[0] * Gjg[0] + dv[1] * Gjg[1] + dv[2] * Gjg[2];
        }
        const int gn = a.gnnbr[t];
        for (int k = lane; k < gn; k += kLanes) {
            const int q = a.gnbr[(size_t)k * a.npad + t];
            const int p = a.gpar[q];
            const int fl = a.gflip[q];
            const double r[3] = {xsi[0] - a.gx[q], xsi[1] - a.gy[q], xsi[2] - a.gz[q]};
            double g[3], H[6];
            grad_hess(r, 0.5 * (hi + a.gh[q]), g, H);
            const double rg = a.grho[q], Vg = a.gmass[q] / rg;
            const double dv[3] = {a.gvx[q] - vi[0], a.gvy[q] - vi[1], a.gvz[q] - vi[2]};
            double Gig[3], GiTdv[3], HGi[3];
            for (int n = 0; n < 3; ++n) {
                Gig[n] = Gi[3 * n] * g[0] + Gi[3 * n + 1] * g[1] + Gi[3 * n + 2] * g[2];
                GiTdv[n] = Gi[n] * dv[0] + Gi[3 + n] * dv[1] + Gi[6 + n] * dv[2];
            }
            symv(H, GiTdv, HGi);
            for (int d = 0; d < 3; ++d) {
                vb[d] -= Vg * Gig[d];
                xsb[d] += Vg * HGi[d];
                // ghost side: v_g = M v_p, x_g = M x_p + c (unshifted, neighbour-time x)
                atomicAdd(&b.vb[d][p], flip(fl, d) * Vg * Gig[d]);
                atomicAdd(&b.xb[d][p], -flip(fl, d) * Vg * HGi[d]);
            }
            const double Vgb = dv[0] * Gig[0] + dv[1] * Gig[1] + dv[2] * Gig[2];
            atomicAdd(&b.rhob[p], -Vgb * Vg / rg);
        }
    }
    lane_sum(acc);
    if (!live || lane != 0) return;
    for (int d = 0; d < 3; ++d) {
        atomicAdd(&b.xb[d][i], xsb[d]);
        atomicAdd(&b.vb[d][i], vb[d] - hdt * xsb[d]);
    }
    atomicAdd(&b.rhob[i], -acc[6] * Vi / pre[FRHO][i]);
}

static inline int nblk(int n, int t) { return (n + t - 1) / t; }

void launch_reverse_momentum(const StepArgs &a, const AdjArgs &b, cudaStream_t s) {
    const int gs = nblk(a.n, 256) < 148 * 8 ? nblk(a.n, 256) : 148 * 8;
    k_adj_init<<<gs, 256, 0, s>>>(a, b);
    k_adj_move<<<gs, 256, 0, s>>>(a, b);
    k_adj_pack_momentum<<<gs, 256, 0, s>>>(a, b);
    k_adj_momentum<<<nblk(a.n, 128 / kLanes), 128, 0, s>>>(a, b);
}
void launch_reverse_constitutive(const StepArgs &a, const AdjArgs &b, cudaStream_t s) {
    if (b.rev) k_adj_constitutive<true, 128><<<nblk(a.n, 128), 128, 0, s>>>(a, b);
    else k_adj_constitutive<false, 64><<<nblk(a.n, 64), 64, 0, s>>>(a, b);
}
void launch_reverse_strain(const StepArgs &a, const AdjArgs &b, cudaStream_t s) {
    const int gs = nblk(a.n, 256) < 148 * 8 ? nblk(a.n, 256) : 148 * 8;
    k_adj_pack_strain<<<gs, 256, 0, s>>>(a, b);
    k_adj_strain<<<nblk(a.n, 128 / kLanes), 128, 0, s>>>(a, b);
}

}  // namespace adj
}  // namespace mcm
