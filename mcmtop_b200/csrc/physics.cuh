// physics.cuh -- per-particle physics of the MCM explicit step as device
// functions.  Templated on the arithmetic type T: T = double for the FP64
// paths, T = float for the constitutive update of the mixed path.  The
// expressions keep the reference's evaluation order (left-to-right, explicit
// parentheses) so that the FP64 translation unit compiled without fused
// multiply-add reproduces the reference arithmetic; single-precision Fortran
// literals appear as float literals cast to T.
#pragma once
#include <type_traits>

#include "common.cuh"
#include "dual.cuh"

namespace mcm {

// Symmetric tensor storage: 0:11 1:22 2:33 3:12 4:13 5:23.
enum { T11 = 0, T22 = 1, T33 = 2, T12 = 3, T13 = 4, T23 = 5 };

template <typename T>
struct PState {
    int mat;
    T mass, h, hold, rho, rho0, rhoold, e, etry, einc, p, c;
    T efps, pcut, p_cut, fail, capa;
    T sig[6], s[6], alfa[6];
    T sigl[3];     // lower triangle of sigma: (2,1), (3,1), (3,2)
    int ptype;     // cap model mode (MCM/mcm_f3dm25.f90:257)
    T rod[6];      // rate of deformation (symmetric)
    T spin[3];     // spin(1,2), spin(1,3), spin(2,3)
    T tracerod;
    T q;           // isotropic nodal artificial viscosity q(k,k)
};

template <typename T>
__device__ __forceinline__ T fdim_t(T x, T y) { return x > y ? x - y : T(0); }
template <typename T>
__device__ __forceinline__ T fsign_t(T a, T b) { return (b >= T(0)) ? fabs(a) : -fabs(a); }
template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return a > b ? a : (b > a ? b : a); }
template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return a < b ? a : (b < a ? b : a); }

// Element (k,l) of a symmetric tensor stored as 6 values.
__device__ __forceinline__ int sym_index(int k, int l) {
    if (k == l) return k;
    int a = k < l ? k : l, b = k < l ? l : k;
    return (a == 0) ? (b == 1 ? T12 : T13) : T23;
}

// ---------------------------------------------------------------- density
// MCM/mcm_rhoupd.f90:24-56
template <typename T, typename Mat>
__device__ __forceinline__ void rhoupd(PState<T> &P, const Mat &M, T dt, int ndim) {
    P.rhoold = P.rho;
    const T othird = T(1.0) / T(3.0);
    P.rho = P.rho * (T(1.0) - P.tracerod * dt);
    for (int rep = 0; rep < 2; ++rep) {
        if (P.rho > T(M.rho_max)) {
            P.rho = P.rho / (T(1.0) - P.tracerod * dt);
            P.rod[T11] = P.rod[T11] - othird * P.tracerod;
            P.rod[T22] = P.rod[T22] - othird * P.tracerod;
            P.rod[T33] = P.rod[T33] - othird * P.tracerod;
            P.tracerod = T(0.0);
            if (rep == 1) P.h = P.hold;
            P.h = T(M.h) * pow(T(M.rho) / P.rho, T(1.0) / T((float)ndim));
        }
    }
}

// --------------------------------------------------------- Jaumann rotation
// The rotation of the exponential map, MCM/mcm_stress_rot1.f90:115-161
// (iorder = 3), row-major: q[3 r + c] = Q(r+1, c+1).
template <typename T>
__device__ __forceinline__ void jaumann_q(const T spin[3], T dt, T q[9]) {
    const T etol = T(1.0e-3f);
    const T z1 = T(1.0) / T(3.0), z2 = T(2.0) / T(15.0), z3 = T(17.0) / T(315.0), z4 = T(62.0) / T(2835.0);
    T dt2 = T(0.5f) * dt;
    T wzz = -dt2 * spin[0];
    T wyy = dt2 * spin[1];
    T wxx = -dt2 * spin[2];
    T wxx2 = wxx * wxx, wyy2 = wyy * wyy, wzz2 = wzz * wzz;
    T qm2 = wxx2 + wyy2 + wzz2;
    T qm = sqrt(qm2);
    T dd = tan(qm * T(0.5));
    T cc;
    if (qm < etol) {
        T aa = qm2 * T(0.25);
        cc = T(0.5) * (T(1.0) + aa * (z1 + aa * (z2 + aa * (z3 + aa * z4))));
    } else {
        cc = dd / qm;
    }
    T bb = T(2.0) * cc / (T(1.0) + dd * dd);
    T aa = bb * cc;
    T q11 = T(1.0) - aa * (wyy2 + wzz2);
    T q22 = T(1.0) - aa * (wxx2 + wzz2);
    T q33 = T(1.0) - aa * (wxx2 + wyy2);
    T q12 = aa * wxx * wyy;
    T q13 = aa * wxx * wzz;
    T q23 = aa * wyy * wzz;
    T q21 = q12, q31 = q13, q32 = q23;
    T bwxx = bb * wxx, bwyy = bb * wyy, bwzz = bb * wzz;
    q[1] = q12 - bwzz;
    q[3] = q21 + bwzz;
    q[2] = q13 + bwyy;
    q[6] = q31 - bwyy;
    q[5] = q23 - bwxx;
    q[7] = q32 + bwxx;
    q[0] = q11;
    q[4] = q22;
    q[8] = q33;
}

// MCM/mcm_stress_rot1.f90:35-199: sigma <- Q sigma Q^T
template <typename T>
__device__ __forceinline__ void stress_rot1(PState<T> &P, T dt) {
    const T s11 = P.sig[T11], s22 = P.sig[T22], s33 = P.sig[T33];
    // the reference reads sigma(1,2), sigma(2,3) and sigma(3,1): the upper
    // triangle except for (3,1) (MCM/mcm_stress_rot1.f90:40-48, 164-172)
    const T s12 = P.sig[T12], s23 = P.sig[T23], s31 = P.sigl[1];
    T q[9];
    jaumann_q(P.spin, dt, q);
    const T q11 = q[0], q12 = q[1], q13 = q[2], q21 = q[3], q22 = q[4], q23 = q[5], q31 = q[6], q32 = q[7], q33 = q[8];
    T qs11 = q11 * s11 + q12 * s12 + q13 * s31;
    T qs12 = q11 * s12 + q12 * s22 + q13 * s23;
    T qs13 = q11 * s31 + q12 * s23 + q13 * s33;
    T qs21 = q21 * s11 + q22 * s12 + q23 * s31;
    T qs22 = q21 * s12 + q22 * s22 + q23 * s23;
    T qs23 = q21 * s31 + q22 * s23 + q23 * s33;
    T qs31 = q31 * s11 + q32 * s12 + q33 * s31;
    T qs32 = q31 * s12 + q32 * s22 + q33 * s23;
    T qs33 = q31 * s31 + q32 * s23 + q33 * s33;
    P.sig[T11] = qs11 * q11 + qs12 * q12 + qs13 * q13;
    P.sig[T22] = qs21 * q21 + qs22 * q22 + qs23 * q23;
    P.sig[T33] = qs31 * q31 + qs32 * q32 + qs33 * q33;
    P.sig[T12] = qs11 * q21 + qs12 * q22 + qs13 * q23;
    P.sig[T23] = qs21 * q31 + qs22 * q32 + qs23 * q33;
    P.sig[T13] = qs11 * q31 + qs12 * q32 + qs13 * q33;
    P.sigl[0] = P.sig[T12];
    P.sigl[1] = P.sig[T13];
    P.sigl[2] = P.sig[T23];
}

// The symmetric writes of the other models (MCM/mcm_f3dm1.f90:58-60,
// mcm_f3dm3.f90:69-71, mcm_stress_up.f90:35-37): lower triangle = upper.
template <typename T>
__device__ __forceinline__ void sym_lower(PState<T> &P) {
    P.sigl[0] = P.sig[T12];
    P.sigl[1] = P.sig[T13];
    P.sigl[2] = P.sig[T23];
}

// ------------------------------------------------------------- EOS: sound speed
// MCM/mcm_eos1c.f90:32-81 (complex c forced to continue)
template <typename T, typename Mat>
__device__ __forceinline__ void eos1c(PState<T> &P, const Mat &M) {
    const auto &ei = M.eosinput;
    T c1 = T(ei[1]), c2 = T(ei[2]), c3 = T(ei[3]), c4 = T(ei[4]), c5 = T(ei[5]), c6 = T(ei[6]);
    T mu = P.rho / P.rho0 - T(1.0);
    T mu_t = tmax(mu, T(0.0));
    T e1 = T(0.0);
    T dmudrho = T(1) / P.rho0;
    T termone = c1 * dmudrho + (c2 * (dmudrho * dmudrho)) + (T(3.0) * c3 * dmudrho) * mu * mu;
    T termtwo = (c5 * dmudrho + c6 * dmudrho * dmudrho) * e1;
    T dpdrho = termone + termtwo;
    T dpde = c4 + c5 * mu + c6 * (mu_t * mu_t);
    T mr = P.mass / P.rho;
    T c_sq = ((T(4.0) / T(3.0)) * T(M.g) / P.rho0 + dpdrho + P.p / P.rho0 * (mr * mr) * dpde);
    if (c_sq > T(0.0)) P.c = sqrt(c_sq);
    else P.c = sqrt(fabs(c_sq));
}

// MCM/mcm_eos4c.f90:33-90
template <typename T, typename Mat>
__device__ __forceinline__ void eos4c(PState<T> &P, const Mat &M) {
    const auto &ei = M.eosinput;
    T c1 = T(ei[0]), s1 = T(ei[1]), s2 = T(ei[2]), s3 = T(ei[3]), gamma = T(ei[4]), a1 = T(ei[5]);
    T e1 = P.e * P.rho0 / P.mass;
    T mu = P.rho / P.rho0 - T(1.0);
    T dpdrho;
    if (mu > T(0.0)) {
        T termone = mu * (T(1.0) - (gamma / T(2.0)));
        T termtwo = (a1 / T(2.0)) * mu * mu;
        T eosnum = mu * P.rho0 * (c1 * c1) * (T(1.0) + termone - termtwo);
        T mu11 = mu / (mu + T(1.0));
        T mu21 = (mu * mu) / (mu + T(1.0));
        T mu22 = (mu * mu) / ((mu + T(1.0)) * (mu + T(1.0)));
        T mu32 = (mu * mu * mu) / ((mu + T(1.0)) * (mu + T(1.0)));
        T mu33 = (mu * mu * mu) / ((mu + T(1.0)) * (mu + T(1.0)) * (mu + T(1.0)));
        T eosden = T(1.0) - (s1 - T(1.0)) * mu - s2 * mu21 - s3 * mu32;
        T termthree = P.rho0 * (c1 * c1) * (T(1.0) + T(2.0) * termone - T(3.0) * termtwo);
        T termfour = T(1.0) - s1 - T(2.0) * s2 * mu11 + s2 * mu22 - T(3.0) * s3 * mu22 + T(2.0) * s3 * mu33;
        dpdrho = (termthree / (eosden * eosden) - T(2.0) * eosnum * termfour / (eosden * eosden * eosden)) / P.rho0 +
                 a1 * e1 / P.rho0;
    } else {
        dpdrho = (c1 * c1) + a1 * e1 / P.rho0;
    }
    T dpde = gamma + a1 * mu;
    T mr = P.mass / P.rho;
    T c_sq = ((T(4.0) / T(3.0)) * T(M.g) / P.rho0 + dpdrho + P.p / P.rho0 * (mr * mr) * dpde);
    if (c_sq > T(0.0)) P.c = sqrt(c_sq);
    else P.c = sqrt(fabs(c_sq));
}

// MCM/mcm_eos13c.f90:29-37
template <typename T, typename Mat>
__device__ __forceinline__ void eos13c(PState<T> &P, const Mat &M) {
    T gamma = T(M.eosinput[0]);
    T e1 = P.e / P.mass;
    P.c = sqrt((gamma - T(1.0)) * gamma * e1);
}

// MCM/mcm_eos28c.f90:28-33
template <typename T, typename Mat>
__device__ __forceinline__ void eos28c(PState<T> &P, const Mat &M) {
    T b = T(M.eosinput[0]), gamma = T(M.eosinput[1]);
    P.c = sqrt(b * gamma / P.rho0);
}

// MCM/mcm_eos41c.f90:31-85.  Returns false when c^2 < 0 (the reference stops).
template <typename T, typename Mat>
__device__ __forceinline__ bool eos41c(PState<T> &P, const Mat &M) {
    const auto &ei = M.eosinput;
    T cc = T(ei[0]), sl = T(ei[1]), gamma0 = T(ei[4]);
    T e1 = P.e / P.mass;
    T ao = P.rho0 * (cc * cc);
    T mu = P.rho / P.rho0 - T(1.0);
    T gamma = gamma0 * P.rho0 / P.rho;
    T bo = ao * (T(1.0) + T(2.0) * (sl - T(1.0)));
    T co = ao * (T(2.0) * (sl - T(1.0)) + T(3.0) * ((sl - T(1.0)) * (sl - T(1.0))));
    T f = gamma * mu;
    T a1 = ao * (T(1.0) - f);
    T b1 = bo * (T(2.0) - T(1.5) * f);
    T c1 = co * (T(3.0) - T(2.0) * f);
    T dpdrho;
    if (mu > T(0.0)) dpdrho = (a1 + b1 * mu + c1 * (mu * mu)) / P.rho0 + gamma * e1;
    else dpdrho = ao * (T(1.0) - f) / P.rho0 + gamma * e1;
    T c2;
    if (P.p == P.pcut) {
        c2 = cc * cc;
    } else {
        T dpdi = gamma * P.rho;
        T didrho = P.p / (P.rho * P.rho);
        dpdrho = dpdrho + dpdi * didrho;
        c2 = dpdrho;
    }
    P.c = sqrt(c2);
    return !(c2 < T(0.0));
}

// MCM/mcm_sueos.f90:24-46
template <typename T, typename Mat>
__device__ __forceinline__ bool sueos(PState<T> &P, const Mat &M) {
    switch (M.eos) {
        case 1: eos1c(P, M); return true;
        case 4: eos4c(P, M); return true;
        case 13: eos13c(P, M); return true;
        case 28: eos28c(P, M); return true;
        case 41: return eos41c(P, M);
    }
    return true;
}

// ------------------------------------------------------------ EOS: pressure
// MCM/mcm_eqos1.f90:32-75
template <typename T, typename Mat>
__device__ __forceinline__ void eqos1(PState<T> &P, const Mat &M, T dt) {
    const auto &ei = M.eosinput;
    T c0 = T(ei[0]), c1 = T(ei[1]), c2 = T(ei[2]), c3 = T(ei[3]), c4 = T(ei[4]), c5 = T(ei[5]), c6 = T(ei[6]);
    T mu = P.rho / P.rho0 - T(1.0);
    T mu_t = tmax(mu, T(0.0));
    T dvol = P.mass / P.rho - P.mass / P.rhoold;
    T vol0 = P.mass / P.rho0;
    T e1try = P.etry / vol0;
    T termone = c0 + (c1 + c3 * (mu * mu)) * mu + c2 * (mu_t * mu_t);
    T termtwo = c4 + c5 * mu + c6 * (mu_t * mu_t);
    P.p = (termone + termtwo * e1try) / (T(1) + termtwo * (dvol / vol0));
    if (P.p < P.pcut) {
        P.p = P.pcut;
        P.rho = P.rho / (T(1.0) - P.tracerod * dt);
    } else {
        P.e = P.etry - T(0.5) * dvol * P.p;
    }
}

// MCM/mcm_eqos4.f90:30-82
template <typename T, typename Mat>
__device__ __forceinline__ void eqos4(PState<T> &P, const Mat &M, T dt) {
    const auto &ei = M.eosinput;
    T c1 = T(ei[0]), s1 = T(ei[1]), s2 = T(ei[2]), s3 = T(ei[3]), gamma = T(ei[4]), a1 = T(ei[5]);
    T mu = P.rho / P.rho0 - T(1.0);
    T dvol = P.mass / P.rho - P.mass / P.rhoold;
    T vol0 = P.mass / P.rho0;
    T e1try = P.etry / vol0;
    if (mu > T(0.0)) {
        T termone = mu * (T(1.0) - (gamma / T(2.0)));
        T termtwo = (a1 / T(2.0)) * mu * mu;
        T eosnum = mu * P.rho0 * (c1 * c1) * (T(1.0) + termone - termtwo);
        T mu21 = (mu * mu) / (mu + T(1.0));
        T mu32 = (mu * mu * mu) / ((mu + T(1.0)) * (mu + T(1.0)));
        T eosden = T(1.0) - (s1 - T(1.0)) * mu - s2 * mu21 - s3 * mu32;
        P.p = (eosnum / (eosden * eosden) + (gamma + a1 * mu) * e1try) /
              (T(1.0) + T(0.5) * (gamma + a1 * mu) * dvol / vol0);
    } else {
        P.p = (P.rho0 * (c1 * c1) * mu + (gamma + a1 * mu) * e1try) / (T(1.0) + T(0.5) * (gamma + a1 * mu) * dvol / vol0);
    }
    if (P.p < P.pcut) {
        P.p = P.pcut;
        P.rho = P.rho / (T(1.0) - P.tracerod * dt);
    } else {
        P.e = P.etry - T(0.5) * dvol * P.p;
    }
}

// MCM/mcm_eqos13.f90:30-46
template <typename T, typename Mat>
__device__ __forceinline__ void eqos13(PState<T> &P, const Mat &M) {
    T gamma_m1 = T(M.eosinput[0]) - T(1.0);
    T e1try = P.etry / P.mass;
    T dvol = P.mass / P.rho - P.mass / P.rhoold;
    P.p = (P.rho * gamma_m1 * e1try) / (T(1.0) + T(0.5) * P.rho * gamma_m1 * dvol / P.mass);
    P.e = P.etry - T(0.5) * dvol * P.p;
}

// MCM/mcm_eqos28.f90:30-45
template <typename T, typename Mat>
__device__ __forceinline__ void eqos28(PState<T> &P, const Mat &M) {
    T b = T(M.eosinput[0]), gamma = T(M.eosinput[1]);
    T dvol = P.mass / P.rho - P.mass / P.rhoold;
    P.p = b * (pow(P.rho / P.rho0, gamma) - T(1.0));
    P.e = P.etry - T(0.5) * dvol * P.p;
}

// MCM/mcm_eqos41.f90:32-102
template <typename T, typename Mat>
__device__ __forceinline__ void eqos41(PState<T> &P, const Mat &M, T dt) {
    const auto &ei = M.eosinput;
    T cc = T(ei[0]), sl = T(ei[1]), gama0 = T(ei[4]);
    T etry1 = P.etry / P.mass;
    T ao = P.rho0 * (cc * cc);
    T mu = P.rho / P.rho0 - T(1.0);
    T dvol = P.mass / P.rho - P.mass / P.rhoold;
    T vol0 = P.mass / P.rho0;
    T gama = gama0 * P.rho0 / P.rho;
    T bo = ao * (T(1.0) + T(2.0) * (sl - T(1.0)));
    T co = ao * (T(2.0) * (sl - T(1.0)) + T(3.0) * ((sl - T(1.0)) * (sl - T(1.0))));
    T f = gama * mu;
    T ph;
    if (mu > T(0.0)) ph = ao * mu + bo * (mu * mu) + co * (mu * mu * mu);
    else ph = ao * mu;
    T pn = (ph * (T(1.0) - T(0.5) * f) + P.rho * gama * etry1) / (T(1.0) + T(0.5) * P.rho * gama * dvol / vol0);
    if (pn < P.pcut) {
        pn = P.pcut;
        P.rho = P.rho / (T(1.0) - P.tracerod * dt);
    } else {
        P.e = etry1 * P.mass - T(0.5) * dvol * pn;
    }
    P.p = pn;
}

// MCM/mcm_eqos.f90:24-55
template <typename T, typename Mat>
__device__ __forceinline__ void eqos(PState<T> &P, const Mat &M, T dt) {
    switch (M.eos) {
        case 1: eqos1(P, M, dt); break;
        case 4: eqos4(P, M, dt); break;
        case 13: eqos13(P, M); break;
        case 28: eqos28(P, M); break;
        case 41: eqos41(P, M, dt); break;
    }
}

// --------------------------------------------------------- EOS: initial state
// MCM/mcm_eos1p.f90:30-47
template <typename T, typename Mat>
__device__ __forceinline__ void eos1p(PState<T> &P, const Mat &M) {
    const auto &ei = M.eosinput;
    T c0 = T(ei[0]), c1 = T(ei[1]), c2 = T(ei[2]), c3 = T(ei[3]), c4 = T(ei[4]), c5 = T(ei[5]), c6 = T(ei[6]);
    T mu = P.rho / P.rho0 - T(1.0);
    T mu_t = tmax(mu, T(0.0));
    T e1 = T(0.0);
    P.p = c0 + (c1 + c3 * (mu * mu)) * mu + c2 * (mu_t * mu_t) + (c4 + c5 * mu + c6 * (mu_t * mu_t)) * e1;
}

// MCM/mcm_eos4p.f90:32-61
template <typename T, typename Mat>
__device__ __forceinline__ void eos4p(PState<T> &P, const Mat &M) {
    const auto &ei = M.eosinput;
    T c1 = T(ei[0]), s1 = T(ei[1]), s2 = T(ei[2]), s3 = T(ei[3]), gamma = T(ei[4]), a1 = T(ei[5]);
    T e1 = P.e * P.rho0 / P.mass;
    T mu = P.rho / P.rho0 - T(1.0);
    if (mu > T(0.0)) {
        T termone = mu * (T(1.0) - (gamma / T(2.0)));
        T termtwo = (a1 / T(2.0)) * mu * mu;
        T eosnum = mu * P.rho0 * (c1 * c1) * (T(1.0) + termone - termtwo);
        T mu21 = (mu * mu) / (mu + T(1.0));
        T mu32 = (mu * mu * mu) / ((mu + T(1.0)) * (mu + T(1.0)));
        T eosden = T(1.0) - (s1 - T(1.0)) * mu - s2 * mu21 - s3 * mu32;
        P.p = eosnum / (eosden * eosden) + (gamma + a1 * mu) * e1;
    } else {
        P.p = P.rho0 * (c1 * c1) * mu + (gamma + a1 * mu) * e1;
    }
}

// MCM/mcm_eos13p.f90:29-35
template <typename T, typename Mat>
__device__ __forceinline__ void eos13p(PState<T> &P, const Mat &M) {
    T gamma = T(M.eosinput[0]);
    T e1 = P.e / P.mass;
    P.p = P.rho * (gamma - T(1.0)) * e1;
}

// MCM/mcm_eos28p.f90:28-33
template <typename T, typename Mat>
__device__ __forceinline__ void eos28p(PState<T> &P, const Mat &M) {
    T B = T(M.eosinput[0]), gamma = T(M.eosinput[1]);
    P.p = B * (pow(P.rho / P.rho0, gamma) - T(1.0));
}

// MCM/mcm_eos41p.f90:31-76 (tracerod and dt are zero at initialisation)
template <typename T, typename Mat>
__device__ __forceinline__ void eos41p(PState<T> &P, const Mat &M, T dt) {
    const auto &ei = M.eosinput;
    T cc = T(ei[0]), sl = T(ei[1]), gamma = T(ei[4]);
    T e1 = P.e / P.mass;
    T ao = P.rho0 * (cc * cc);
    T mu = P.rho / P.rho0 - T(1.0);
    T bo = ao * (T(1.0) + T(2.0) * (sl - T(1.0)));
    T co = ao * (T(2.0) * (sl - T(1.0)) + T(3.0) * ((sl - T(1.0)) * (sl - T(1.0))));
    gamma = gamma * P.rho0 / P.rho;
    T f = gamma * mu;
    T ph;
    if (mu > T(0.0)) ph = ao * mu + bo * (mu * mu) + co * (mu * mu * mu);
    else ph = ao * mu;
    T pn = ph * (T(1.0) - T(0.5) * f) + P.rho * gamma * e1;
    if (pn < P.pcut) {
        pn = P.pcut;
        P.rho = P.rho / (T(1.0) - P.tracerod * dt);
    }
    P.p = pn;
}

// ------------------------------------------------- artificial viscosity
// MCM/mcm_nodalav.f90:32-47 (q is isotropic: only the diagonal is stored)
template <typename T, typename Mat>
__device__ __forceinline__ void nodalav(PState<T> &P, const Mat &M) {
    P.q = T(0.0);
    if (P.tracerod < T(0.0)) {
        T ht = P.h * P.tracerod;
        P.q = T(M.av_l) * P.rho * P.c * P.h * fabs(P.tracerod) + T(M.av_q) * P.rho * (ht * ht);
    }
}

// MCM/mcm_aviscosity.f90:28-39 (other types print an error and leave q)
template <typename T, typename Mat>
__device__ __forceinline__ void aviscosity(PState<T> &P, const Mat &M) {
    if (M.visc_type == 1) nodalav(P, M);
}

// ---------------------------------------------------------- energy updates
// MCM/mcm_hieupd.f90:27-64; de(k,l) summed in column-major order
template <typename T>
__device__ __forceinline__ void hieupd(PState<T> &P, T dt) {
    const T othird = T(1.0) / T(3.0);
    T pold = -othird * (P.sig[T11] + P.sig[T22] + P.sig[T33]);
    T trace_q = othird * (P.q + P.q + P.q);
    T volold = P.mass / P.rhoold;
    T volnew = P.mass / P.rho;
    T eincr = T(0.0);
#pragma unroll
    for (int l = 0; l < 3; ++l) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            int t = sym_index(k, l);
            T qkl = (k == l) ? P.q : T(0.0);
            T de;
            if (k == l) de = P.rod[t] * (T(0.5f) * (P.sig[t] + pold + P.s[t]) - qkl + trace_q);
            else de = P.rod[t] * (T(0.5f) * (P.sig[t] + P.s[t]) - qkl);
            eincr = eincr + de;
        }
    }
    T vavg = T(0.5f) * (volnew + volold);
    eincr = vavg * eincr;
    T dvol = volnew - volold;
    T mean_incr = dvol * (T(0.5f) * pold + trace_q);
    P.etry = P.e + dt * eincr - mean_incr;
}

// MCM/mcm_lieupd.f90:26-33 (dot product in column-major order)
template <typename T>
__device__ __forceinline__ void lieupd(PState<T> &P, T dt) {
    T qpm = T(0.0);
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            T qkl = (k == l) ? P.q : T(0.0);
            qpm = qpm + qkl * P.rod[sym_index(k, l)];
        }
    P.e = P.e + (P.einc - dt * qpm) * P.mass / P.rho;
}

// MCM/mcm_stress_up.f90:28-36
template <typename T>
__device__ __forceinline__ void stress_up(PState<T> &P) {
    P.sig[T11] = P.s[T11] - P.p;
    P.sig[T22] = P.s[T22] - P.p;
    P.sig[T33] = P.s[T33] - P.p;
    P.sig[T12] = P.s[T12];
    P.sig[T13] = P.s[T13];
    P.sig[T23] = P.s[T23];
}

// --------------------------------------------------------------- models
// cm(i,j) of a cm(5,*) view of strinput
template <typename Mat>
__device__ __forceinline__ auto cm5(const Mat &M, int i, int j) { return M.strinput[(i - 1) + 5 * (j - 1)]; }

// MCM/mcm_f3dm1.f90:27-71
template <typename T, typename Mat>
__device__ __forceinline__ void f3dm1(PState<T> &P, const Mat &M, T dt) {
    const T othird = T(1.0) / T(3.0);
    T ym = T(cm5(M, 1, 1)), pr = T(cm5(M, 1, 2)), gg = T(cm5(M, 5, 4));
    T gdt = dt * gg;
    T gd2 = T(2.0) * gdt;
    T blk = dt * ym / ((T(1.0) - T(2.0) * pr));
    T davg = othird * P.tracerod;
    T p_incr = blk * davg;
    T *r = P.rod, *s = P.sig;
    T q = P.q;
    P.einc = (r[T11] * (s[T11] + q) + r[T22] * (s[T22] + q) + r[T33] * (s[T33] + q) +
              T(2.0) * (r[T12] * (s[T12] + T(0.0)) + r[T13] * (s[T13] + T(0.0)) + r[T23] * (s[T23] + T(0.0)))) * dt;
    s[T11] = s[T11] + p_incr + gd2 * (r[T11] - davg);
    s[T22] = s[T22] + p_incr + gd2 * (r[T22] - davg);
    s[T33] = s[T33] + p_incr + gd2 * (r[T33] - davg);
    s[T12] = s[T12] + gd2 * r[T12];
    s[T13] = s[T13] + gd2 * r[T13];
    s[T23] = s[T23] + gd2 * r[T23];
    P.einc = T(0.5) * ((r[T11] * s[T11] + r[T22] * s[T22] + r[T33] * s[T33] +
                        T(2.0) * (r[T12] * s[T12] + r[T13] * s[T13] + r[T23] * s[T23])) * dt + P.einc);
    P.p = -othird * (s[T11] + s[T22] + s[T33]);
}

// MCM/mcm_f3dm3.f90:31-156
template <typename T, typename Mat>
__device__ __forceinline__ void f3dm3(PState<T> &P, const Mat &M, T dt) {
    const T othird = T(1.0) / T(3.0);
    T qh = T(cm5(M, 2, 4)), qb = T(cm5(M, 1, 5)), qs = T(cm5(M, 1, 3)), ym = T(cm5(M, 1, 1)), pr = T(cm5(M, 1, 2));
    T efps_f = T(cm5(M, 2, 6));
    T gg = T(2.0) * T(cm5(M, 5, 4));
    T gdt = dt * gg;
    T qbqh = qb * qh;
    int efps_flag = (int)llround(value_of(cm5(M, 1, 6)));
    T blk = dt * ym / ((T(1.0f) - T(2.0f) * pr));
    T davg = othird * P.tracerod;
    T p_incr = blk * davg;
    P.p = P.p - p_incr;
    T *r = P.rod, *sg = P.sig, *s = P.s, *al = P.alfa;
    T q = P.q;
    P.einc = (r[T11] * (sg[T11] + q) + r[T22] * (sg[T22] + q) + r[T33] * (sg[T33] + q) +
              T(2.0f) * (r[T12] * (sg[T12] + T(0.0)) + r[T13] * (sg[T13] + T(0.0)) + r[T23] * (sg[T23] + T(0.0)))) * dt;
    sg[T11] = sg[T11] + p_incr + gdt * (r[T11] - davg);
    sg[T22] = sg[T22] + p_incr + gdt * (r[T22] - davg);
    sg[T33] = sg[T33] + p_incr + gdt * (r[T33] - davg);
    sg[T12] = sg[T12] + gdt * r[T12];
    sg[T13] = sg[T13] + gdt * r[T13];
    sg[T23] = sg[T23] + gdt * r[T23];
    T k = qs + qbqh * P.efps;
    s[T11] = P.p + sg[T11] - al[T11];
    s[T22] = P.p + sg[T22] - al[T22];
    s[T33] = P.p + sg[T33] - al[T33];
    s[T12] = sg[T12] - al[T12];
    s[T13] = sg[T13] - al[T13];
    s[T23] = sg[T23] - al[T23];
    T j2 = s[T23] * s[T23] + s[T13] * s[T13] + s[T12] * s[T12] - s[T11] * s[T22] - s[T22] * s[T33] - s[T11] * s[T33];
    T k2 = T(3.0f) * j2 - k * k;
    T scle = T(0.5f) * (T(1.0f) + fsign_t(T(1.0f), k2));
    T fac1 = T(1.0f) / (T(1.5f) * gg + qh);
    T fac2 = T(1.5f) * gg;
    T fac3 = (T(1.0f) - qb) * qh;
    T j1 = sqrt(T(3.0f) * fabs(j2)) + T(1.0f) - scle;
    T defps = scle * fac1 * (j1 - k);
    P.efps = P.efps + defps;
    T des = scle * fac2 * defps / j1;
    T depn = scle * fac3 * defps / j1;
#pragma unroll
    for (int t = 0; t < 6; ++t) sg[t] = sg[t] - des * s[t];
#pragma unroll
    for (int t = 0; t < 6; ++t) al[t] = al[t] + depn * s[t];
    if (efps_flag == 1) {
        if (P.efps > efps_f) {
            T press = othird * (sg[T11] + sg[T22] + sg[T33]);
            sg[T11] = press; sg[T22] = press; sg[T33] = press;
            sg[T12] = T(0.0); sg[T13] = T(0.0); sg[T23] = T(0.0);
        }
    }
    P.einc = T(0.5f) * ((r[T11] * sg[T11] + r[T22] * sg[T22] + r[T33] * sg[T33] +
                         T(2.0f) * (r[T12] * sg[T12] + r[T13] * sg[T13] + r[T23] * sg[T23])) * dt + P.einc);
}

// MCM/mcm_f3dm9.f90:26-48 (s(1,2) is never assigned; xmu = cm(2,mat))
template <typename T, typename Mat>
__device__ __forceinline__ void f3dm9(PState<T> &P, const Mat &M) {
    const T othird = T(1.0) / T(3.0);
    T xmu = T(cm5(M, 2, P.mat));
    if (xmu == T(0.0f)) {
#pragma unroll
        for (int t = 0; t < 6; ++t) P.s[t] = T(0.0f);
    } else {
        T davg = -othird * P.tracerod;
        P.s[T11] = xmu * (P.rod[T11] + davg);
        P.s[T22] = xmu * (P.rod[T22] + davg);
        P.s[T33] = xmu * (P.rod[T33] + davg);
        P.s[T13] = xmu * P.rod[T13];
        P.s[T23] = xmu * P.rod[T23];
    }
}

// MCM/mcm_f3dm10.f90:28-157.  `defps` is uninitialised in the reference when
// fail /= 1; it is 0 here.
template <typename T, typename Mat>
__device__ __forceinline__ void f3dm10(PState<T> &P, const Mat &M, T dt) {
    const auto &cm = M.strinput;
    const T othird = T(1.0) / T(3.0);
    T gg = T(cm[0]), qs = T(cm[1]), qh = T(cm[2]), a1 = T(cm[4]), a2 = T(cm[5]);
    int ispall = (int)value_of(cm[6]);
    T epf = T(cm[7]);
    T g2 = T(2.0f) * dt * gg;
    T davg = othird * P.tracerod;
    T *sg = P.sig, *s = P.s, *r = P.rod;
    P.p = -othird * (sg[T11] + sg[T22] + sg[T33]);
    P.p_cut = P.pcut;
    T ak = qs + qh * P.efps + (a1 + a2 * P.p) * tmax(T(0.0), P.p);
    s[T11] = sg[T11] + P.p + g2 * (r[T11] + davg);
    s[T22] = sg[T22] + P.p + g2 * (r[T22] + davg);
    s[T33] = sg[T33] + P.p + g2 * (r[T33] + davg);
    s[T12] = sg[T12] + T(0.5f) * g2 * r[T12];
    s[T13] = sg[T13] + T(0.5f) * g2 * r[T13];
    s[T23] = sg[T23] + T(0.5f) * g2 * r[T23];
    if (ispall == 3) {
        T deltap = P.p - P.p_cut;
        T scle = T(0.50f) * (T(1.0f) + fsign_t(T(1.0f), deltap));
        P.pcut = scle * P.p_cut;
#pragma unroll
        for (int t = 0; t < 6; ++t) s[t] = scle * s[t];
        P.p_cut = P.pcut;
    }
    T aj2 = T(0.5f) * (s[T11] * s[T11] + s[T22] * s[T22] + s[T33] * s[T33]) + s[T12] * s[T12] + s[T13] * s[T13] +
            s[T23] * s[T23];
    T sj2 = sqrt(T(3.0f) * aj2);
    T defps = T(0.0);
    if (P.fail == T(1.0f)) {
        T thrg = othird / gg;
        defps = fdim_t(sj2, ak) / (T(1.e-30f) + fdim_t(T(1.0f), -thrg * qh));
        defps = thrg * tmin(sj2, defps);
        P.efps = P.efps + defps;
    }
    ak = tmax(ak + qh * defps, T(0.0f));
    T seps = T(1.e-30f) * gg;
    T scle = (ak + seps) / (tmax(ak, sj2) + seps);
#pragma unroll
    for (int t = 0; t < 6; ++t) s[t] = scle * s[t];
    if (epf != T(0.0f)) {
        if (P.efps > epf) {
            P.fail = T(0.0f);
#pragma unroll
            for (int t = 0; t < 6; ++t) s[t] = T(0.0f);
        }
    }
    if (ispall == 2) {
        aj2 = T(0.5f) * (s[T11] * s[T11] + s[T22] * s[T22] + s[T33] * s[T33]) + s[T12] * s[T12] + s[T13] * s[T13] +
              s[T23] * s[T23] + T(1.e-12f);
        sj2 = s[T11] * s[T23] * s[T23] + s[T22] * s[T13] * s[T13] + s[T33] * s[T12] * s[T12] -
              s[T11] * s[T22] * s[T33] - T(2.0f) * s[T12] * s[T13] * s[T23];
        T akt = -sqrt(T(27.0f) / aj2) * sj2 * T(0.5f) / aj2;
        akt = fsign_t(tmin(fabs(akt), T(1.0f)), akt);
        T ywh = acos(akt) * othird;
        sj2 = T(2.0f) * sqrt(aj2 * othird) * cos(ywh);
        T davg1 = P.p - sj2 - P.p_cut;
        T scle2 = T(0.50f) * (T(1.0f) + fsign_t(T(1.0f), davg1));
        P.pcut = scle2 * P.p_cut;
#pragma unroll
        for (int t = 0; t < 6; ++t) s[t] = scle2 * s[t];
        P.p_cut = P.pcut;
    }
}

// ---------------------------------------------------------------- cap model
// Model 4, the generalised cap model of MCM/mcm_f3dm25.f90 (f3dm25a :37-827,
// feit :906-966, fcit :968-1038).  f3dm25a has no `implicit none`: its
// undeclared locals are single precision, so they are float here, the
// declared ones double, and mixed expressions are evaluated in the wider kind,
// left to right (this translation unit has no fused multiply-add).  Single-
// precision exp is the correctly rounded float of a double exp.  Quirks kept:
// the local `capa` of :197 is never assigned (static zero), only the upper
// triangle of sigma is written back (:813-815), X0 of the hardening law is
// cm(2,4) while the initial cap used cm(2,5).  The iterated returns (vector
// flag cm(3,5) /= 0) stop the reference when unconverged after 100
// iterations; here the particle reports MCM_ECAP_NOCONV.
namespace cap {

__device__ __forceinline__ float fexp(float x) { return (float)exp((double)x); }
template <typename U> __device__ __forceinline__ U vmin(U a, U b) { return (b < a) ? b : a; }
template <typename U> __device__ __forceinline__ U vmax(U a, U b) { return (a < b) ? b : a; }

struct Const {
    float shear, alpha, theta, gama, beta, r, dDyna, w, z, tcut, fcut;
    double bulk;
    int ltype, ivec;
};

// one failure-surface iteration (feit :923-960)
__device__ __forceinline__ void fail_iter(const Const &C, double &capa, double sig[6], float s[6], float &x1,
                                          float &x2d) {
    float xk = (float)(capa + C.r * (C.alpha - C.gama * exp(-C.beta * capa) + C.theta * capa));
    float dhdk = (float)((C.w * C.dDyna * fexp(-C.dDyna * xk)) *
                         (1.0 + C.r * (C.theta + C.gama * C.beta * exp(-C.beta * capa))));
    float omega = C.theta + C.gama * C.beta * fexp(-C.beta * x1);
    float dcd = (float)(C.shear + 9.0 * C.bulk * (double)(omega * omega));
    float f = x2d - (C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1);
    float delcap = -(3.0f * omega * f / (dcd * dhdk));
    float delam = -(dhdk * delcap / (3.0f * omega));
    capa = capa + delcap;
    float fac1 = C.shear / x2d;
    float fac2 = (float)(3.0 * C.bulk * omega);
    sig[0] = sig[0] - delam * (fac1 * s[0] - fac2);
    sig[1] = sig[1] - delam * (fac1 * s[1] - fac2);
    sig[2] = sig[2] - delam * (fac1 * s[2] - fac2);
    sig[3] = sig[3] - delam * fac1 * s[3];
    sig[4] = sig[4] - delam * fac1 * s[4];
    sig[5] = sig[5] - delam * fac1 * s[5];
    x1 = (float)(sig[0] + sig[1] + sig[2]);
    s[0] = (float)(sig[0] - x1 / 3.0f);
    s[1] = (float)(sig[1] - x1 / 3.0f);
    s[2] = (float)(sig[2] - x1 / 3.0f);
    s[3] = (float)sig[3];
    s[4] = (float)sig[4];
    s[5] = (float)sig[5];
    x2d = sqrtf(0.5f * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
}

// one cap iteration (fcit :986-1022); returns the convergence function of :1023
__device__ __forceinline__ float cap_iter(const Const &C, double &capa, double sig[6], float s[6], float &x1, float &x2d,
                                          float &elcap_out) {
    const float unit = 1.0f;
    float xk = (float)(capa + C.r * (C.alpha - C.gama * exp(-C.beta * capa) + C.theta * capa));
    float dhdk = (float)((C.w * C.dDyna * fexp(-C.dDyna * xk)) *
                         (1.0 + C.r * (C.theta + C.gama * C.beta * exp(-C.beta * capa))));
    float dfdk;
    if (capa >= 0.0) {
        dfdk = (float)(-(2.0f * (fabs((double)x1 - capa) / (double)(C.r * C.r) +
                                 (C.alpha - C.gama * exp(-C.beta * capa) + C.theta * capa) *
                                     (C.theta + C.gama * C.beta * exp(-C.beta * capa)))));
    } else {
        dfdk = (float)(-(((2.0f * xk) * (1.0 + C.r * (C.theta + C.gama * C.beta * exp(-C.beta * capa)))) /
                         (double)(C.r * C.r)));
    }
    float elcap = (float)vmax(capa, (double)(0.0f * unit));
    float omega = vmin(-(2.0f * fabsf(x1 - elcap) / (C.r * C.r)), -1.e-15f * unit);
    float dcd = (float)((4.0f * C.shear * (x2d * x2d)) +
                        9.0 * C.bulk * (double)((2.0f * (x1 - elcap) / (C.r * C.r)) * (2.0f * (x1 - elcap) / (C.r * C.r))));
    float f = x2d * x2d + (x1 - elcap) * (x1 - elcap) / (C.r * C.r) - (xk - elcap) * (xk - elcap) / (C.r * C.r);
    float delcap = -(f / (dfdk + (dcd * dhdk) / (3.0f * omega)));
    float delam = -(dhdk * delcap / (3.0f * omega));
    capa = capa + delcap;
    xk = (float)(capa + C.r * (C.alpha - C.gama * exp(-C.beta * capa) + C.theta * capa));
    float fac1 = 2.0f * C.shear;
    float fac2 = (float)(6.0 * C.bulk * (double)fabsf(x1 - elcap) / (double)(C.r * C.r));
    sig[0] = sig[0] - delam * (fac1 * s[0] + fac2);
    sig[1] = sig[1] - delam * (fac1 * s[1] + fac2);
    sig[2] = sig[2] - delam * (fac1 * s[2] + fac2);
    sig[3] = sig[3] - delam * fac1 * s[3];
    sig[4] = sig[4] - delam * fac1 * s[4];
    sig[5] = sig[5] - delam * fac1 * s[5];
    x1 = (float)(sig[0] + sig[1] + sig[2]);
    s[0] = (float)(sig[0] - x1 / 3.0f);
    s[1] = (float)(sig[1] - x1 / 3.0f);
    s[2] = (float)(sig[2] - x1 / 3.0f);
    s[3] = (float)sig[3];
    s[4] = (float)sig[4];
    s[5] = (float)sig[5];
    x2d = sqrtf(0.5f * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2]) + s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
    elcap_out = elcap;
    return x2d * x2d + (x1 - elcap) * (x1 - elcap) / (C.r * C.r) - (xk - elcap) * (xk - elcap) / (C.r * C.r);
}

}  // namespace cap

// sigma (state convention) <-> the reference's compression-positive
// sig1..sig6 = -(11 22 33 12 13 23); returns 0 or MCM_ECAP_NOCONV
template <typename Mat>
__device__ __noinline__ int f3dm25(PState<double> &P, const Mat &M, double dt) {
    using namespace cap;
    const float unit = 1.0f, third = 1.0f / 3.0f, geop = 0.0f, tol = 1.0e-7f;
    Const C;
    C.bulk = cm5(M, 1, 1);
    C.shear = (float)cm5(M, 1, 2);
    C.alpha = (float)cm5(M, 1, 3);
    C.theta = (float)cm5(M, 1, 4);
    C.gama = (float)cm5(M, 1, 5);
    C.beta = (float)cm5(M, 1, 6);
    C.r = (float)cm5(M, 2, 1);
    C.dDyna = (float)cm5(M, 2, 2);
    C.w = (float)cm5(M, 2, 3);
    const float falfac = (float)cm5(M, 4, 1);
    C.alpha = C.alpha - falfac;
    C.z = (float)cm5(M, 2, 4);
    C.ivec = (cm5(M, 3, 5) != 0.0) ? 0 : 1;
    C.ltype = (int)cm5(M, 2, 6);
    C.tcut = (float)cm5(M, 3, 1);
    C.fcut = (float)cm5(M, 3, 4);
    const float t = vmax(C.fcut, C.tcut + 3.0f * geop);
    const float fet = C.alpha - C.gama * fexp(-C.beta * t) + C.theta * t;
    const float fept = C.gama * C.beta * fexp(-C.beta * t) + C.theta;
    P.capa = vmax(P.capa, (double)cm5(M, 3, 3));
    double sig[6] = {-P.sig[T11], -P.sig[T22], -P.sig[T33], -P.sig[T12], -P.sig[T13], -P.sig[T23]};
    const double dd1 = -P.rod[T11], dd2 = -P.rod[T22], dd3 = -P.rod[T33];
    const double dd4 = -P.rod[T12] / 2.0, dd5 = -P.rod[T13] / 2.0, dd6 = -P.rod[T23] / 2.0;
    const double dd = (dd1 + dd2 + dd3);
    const double davgm = (double)(1.0f / 3.0f) * dd;
    const float dt1 = (float)dt;
    double p = 3.0 * C.bulk * (double)dt1 * davgm;
    const double gdt = dt * (double)C.shear;
    const double gd2 = 2.0 * gdt;
    const float gtr11 = (float)(sig[0] + p + gd2 * (dd1 - davgm));
    const float gtr22 = (float)(sig[1] + p + gd2 * (dd2 - davgm));
    const float gtr33 = (float)(sig[2] + p + gd2 * (dd3 - davgm));
    const float gtr12 = (float)(sig[3] + gd2 * dd4);
    const float gtr23 = (float)(sig[4] + gd2 * dd5);
    const float gtr31 = (float)(sig[5] + gd2 * dd6);
    const float x1tr = gtr11 + gtr22 + gtr33;
    float s[6];
    s[0] = gtr11 - (1.0f / 3.0f) * x1tr;
    s[1] = gtr22 - (1.0f / 3.0f) * x1tr;
    s[2] = gtr33 - (1.0f / 3.0f) * x1tr;
    float x2dtr = 0.5f * (s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.0f * (gtr12 * gtr12 + gtr23 * gtr23 + gtr31 * gtr31));
    x2dtr = sqrtf(x2dtr);
    const float capa_local = 0.0f;
    float fe = C.alpha - C.gama * fexp(-C.beta * capa_local) + C.theta * capa_local;
    const float xkn = capa_local + C.r * fe;
    const float elcapn = (float)vmax(P.capa, (double)(0.0f * unit));
    const float tmises = fabsf(xkn - elcapn) / C.r;
    fe = C.alpha - C.gama * fexp(-C.beta * x1tr) + C.theta * x1tr;
    const float f1tr = x2dtr - vmin(fe, tmises);
    const float tcrit = (float)((double)t - 9.0 * C.bulk / (double)C.shear * (double)(x2dtr - fet) * (double)fept);
    fe = C.alpha - C.gama * fexp(-C.beta * elcapn) + C.theta * elcapn;
    const float fep = C.beta * C.gama * fexp(-C.beta * elcapn) + C.theta;
    const float fc2tr = ((xkn - elcapn) * (xkn - elcapn) - (x1tr - elcapn) * (x1tr - elcapn)) / (C.r * C.r);
    const float f2tr = x2dtr * x2dtr - fc2tr;
    const float x1crt = (float)((double)elcapn - ((double)((x2dtr - fe) * 9.0f) * C.bulk) * (double)fep / (double)C.shear);
    fe = (float)(C.alpha - C.gama * exp(-C.beta * P.capa) + C.theta * P.capa);
    const float capal = (float)vmin((double)(0.0f * unit), P.capa - (double)(tol * fe));
    fe = C.alpha - C.gama * fexp(-C.beta * capal) + C.theta * capal;
    const float xk0 = capal + C.r * fe;
    const float evpn = C.w * (1.0f - fexp(C.dDyna * (C.z - xkn)));
    const float devpb = C.w * (1.0f - fexp(C.dDyna * (C.z - xk0))) - evpn;
    const double capan = P.capa;
    const int ltype = C.ltype;
    int imode = 0;
    if ((x1tr <= t) && (x2dtr <= fet) && (ltype == 1) && (capan > 0.0) && (devpb >= 0.0f)) imode = 2;
    else if ((x1tr <= t) && (x2dtr <= fet) && (ltype == 1) && (capan > 0.0) && (devpb < 0.0f)) imode = 7;
    else if ((x1tr <= t) && (x2dtr <= fet) && ((ltype == 2) || (capan <= 0.0))) imode = 3;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr <= tcrit) && (ltype == 1) && (capan > 0.0) && (devpb >= 0.0f)) imode = 4;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr <= tcrit) && (ltype == 1) && (capan > 0.0) && (devpb < 0.0f)) imode = 6;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr <= tcrit) && ((ltype == 2) || (capan <= 0.0))) imode = 5;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr > tcrit) && (capan >= 0.0)) imode = 10;
    else if ((x1tr <= t) && (x2dtr > fet) && (x1tr > tcrit) && (capan < 0.0)) imode = 8;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr <= tol)) imode = 1;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr > tol) && (x1tr >= x1crt)) imode = 9;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr > tol) && (x1tr < x1crt) && (capan >= 0.0)) imode = 10;
    else if ((x1tr > t) && (x1tr <= elcapn) && (f1tr > tol) && (x1tr < x1crt) && (capan < 0.0)) imode = 8;
    else if ((x1tr > t) && (x1tr > elcapn) && (f2tr < tol)) imode = 1;
    else if ((x1tr > t) && (x1tr > elcapn) && (f2tr >= tol)) imode = 11;
    P.ptype = imode;
    float x1 = 0.0f, x2d = 0.0f, ratio = 0.0f;
    const float sdtr[3] = {s[0], s[1], s[2]};
    auto set_scaled = [&](float rat) {
        sig[0] = (double)(sdtr[0] * rat) + p;
        sig[1] = (double)(sdtr[1] * rat) + p;
        sig[2] = (double)(sdtr[2] * rat) + p;
        sig[3] = (double)(gtr12 * rat);
        sig[4] = (double)(gtr23 * rat);
        sig[5] = (double)(gtr31 * rat);
    };
    auto set_plain = [&]() {
        sig[0] = (double)s[0] + p;
        sig[1] = (double)s[1] + p;
        sig[2] = (double)s[2] + p;
        sig[3] = (double)gtr12;
        sig[4] = (double)gtr23;
        sig[5] = (double)gtr31;
    };
    auto move_cap = [&]() {
        const float x1old = (float)(sig[0] + sig[1] + sig[2]);
        const float devp = (float)(dd - (double)(x1 - x1old) / (3.0 * C.bulk));
        const float xhat = vmin(devpb, devp);
        P.capa = P.capa + (double)devp * ((double)capal - capan) / (double)xhat;
        P.capa = vmax(P.capa, (double)(0.0f * unit));
    };
    int code = 0;
    switch (imode) {
        case 1: x1 = x1tr; x2d = x2dtr; P.capa = capan; p = (double)(third * x1 + geop); set_plain(); break;
        case 2: x1 = t; x2d = x2dtr; P.capa = 0.0; p = (double)(third * x1 + geop); set_plain(); break;
        case 3: x1 = t; x2d = x2dtr; P.capa = capan; p = (double)(third * x1 + geop); set_plain(); break;
        case 4:
            x1 = t; x2d = fet; P.capa = 0.0; p = (double)(third * x1 + geop);
            ratio = x2d / x2dtr; set_scaled(ratio);
            break;
        case 5:
            x1 = t; x2d = fet; P.capa = capan; p = (double)(third * x1 + geop);
            ratio = x2d / x2dtr; set_scaled(ratio);
            break;
        case 6:
            x1 = t; x2d = fet; move_cap(); p = (double)(third * x1 + geop);
            ratio = x2d / x2dtr; set_scaled(ratio);
            break;
        case 7:
            x1 = t; x2d = x2dtr; move_cap(); p = (double)(third * x1 + geop); set_plain();
            break;
        case 8:
            x1 = x1tr;
            fe = C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1;
            x2d = vmin(fe, tmises);
            P.capa = capan;
            ratio = x2d / x2dtr;
            p = (double)(third * x1 + geop);
            set_scaled(ratio);
            break;
        case 9:
            x1 = elcapn;
            x2d = C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1;
            P.capa = capan;
            ratio = x2d / x2dtr;
            p = (double)(third * x1 + geop);
            set_scaled(ratio);
            break;
        case 10: {
            double sg[6] = {gtr11, gtr22, gtr33, gtr12, gtr23, gtr31};
            P.capa = capan;
            x1 = x1tr;
            x2d = x2dtr;
            float si[6];
            for (int k = 0; k < 3; ++k) si[k] = (float)(sg[k] - x1tr / 3.0f);
            for (int k = 3; k < 6; ++k) si[k] = (float)sg[k];
            if (C.ivec == 0) {
                bool conv = false;
                for (int it = 1; it <= 100; ++it) {
                    fail_iter(C, P.capa, sg, si, x1, x2d);
                    const float f = x2d - (C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1);
                    if (fabsf(f) <= 1.0e-8f) { conv = true; break; }
                }
                if (!conv) code = MCM_ECAP_NOCONV;
            } else {
                for (int it = 0; it < 4; ++it) fail_iter(C, P.capa, sg, si, x1, x2d);
            }
            if (x1 > elcapn) x1 = elcapn;
            if ((ltype == 2) || (capan == 0.0)) P.capa = capan;
            if ((double)x1 > P.capa) P.capa = x1;
            if ((ltype == 1) && (capan >= 0.0)) P.capa = vmax(P.capa, (double)(0.0f * unit));
            fe = C.alpha - C.gama * fexp(-C.beta * x1) + C.theta * x1;
            x2d = vmin(fe, tmises);
            ratio = x2d / x2dtr;
            p = (double)(third * x1 + geop);
            set_scaled(ratio);
            break;
        }
        case 11: {
            double sg[6] = {gtr11, gtr22, gtr33, gtr12, gtr23, gtr31};
            P.capa = capan;
            x1 = x1tr;
            x2d = x2dtr;
            float si[6];
            for (int k = 0; k < 3; ++k) si[k] = (float)(sg[k] - x1tr / 3.0f);
            for (int k = 3; k < 6; ++k) si[k] = (float)sg[k];
            float elcap = 0.0f;
            bool done = false;
            const int nit = (C.ivec == 0) ? 100 : 4;
            for (int it = 1; it <= nit; ++it) {
                const float f = cap_iter(C, P.capa, sg, si, x1, x2d, elcap);
                if (C.ivec == 0 && fabsf(f) <= 1.0e-8f) { done = true; break; }
            }
            if (C.ivec == 0 && !done) code = MCM_ECAP_NOCONV;
            if (x1 < elcap) {
                x1 = elcap + fabsf(x1 - elcap);
                sg[0] = (double)(si[0] + x1 / 3.0f);
                sg[1] = (double)(si[1] + x1 / 3.0f);
                sg[2] = (double)(si[2] + x1 / 3.0f);
            }
            for (int k = 0; k < 6; ++k) sig[k] = sg[k];
            break;
        }
        default: break;
    }
    // write-back (:813-827): the upper triangle only; the lower keeps the rotated stress
    P.sig[T11] = -sig[0];
    P.sig[T22] = -sig[1];
    P.sig[T33] = -sig[2];
    P.sig[T12] = -sig[3];
    P.sig[T13] = -sig[4];
    P.sig[T23] = -sig[5];
    P.p = -(1.0 / 3.0) * (P.sig[T11] + P.sig[T22] + P.sig[T33]);
    return code;
}

// -------------------------------------------------------- critical timestep
// MCM/mcm_calccritts.f90:40-78 (per particle)
template <typename T, typename Mat>
__device__ __forceinline__ T critts_particle(const PState<T> &P, const Mat &M, int tcrit_opt, int ndim,
                                             T vabs, T mindist) {
    if (tcrit_opt == 0) {
        T vol = P.mass / P.rho;
        T veae, ae;
        if (ndim == 3) { veae = pow(vol, T(1.0) / T(3.0)); ae = pow(vol, T(2.0) / T(3.0)); }
        else if (ndim == 2) { veae = sqrt(vol); ae = sqrt(vol); }
        else { veae = vol; ae = T(1); }
        T qu = (T(M.av_l) * P.c + T(M.av_q) * P.mass / P.rho * P.tracerod) / ae;
        return veae / (qu + sqrt(qu * qu + P.c * P.c));
    } else if (tcrit_opt == 1) {
        return P.h / (P.c + vabs);
    }
    return mindist / (P.c + vabs);
}

// ------------------------------------------------- constitutive driver
// MCM/mcm_constitutive.f90:29-83 for one particle, after mcm_rhoupd.
// Returns 0, MCM_ECOMPLEX_C (the EOS reported a complex sound speed) or
// MCM_ECAP_NOCONV (the cap model's iterated return did not converge).
template <typename T, typename Mat>
__device__ __forceinline__ int constitutive_particle(PState<T> &P, const Mat &M, T dt) {
    int code = 0;
    switch (M.model) {
        case 1:
            stress_rot1(P, dt); f3dm1(P, M, dt); sym_lower(P); aviscosity(P, M); lieupd(P, dt);
            break;
        case 3:
            stress_rot1(P, dt); f3dm3(P, M, dt); sym_lower(P); aviscosity(P, M); lieupd(P, dt);
            break;
        case 4:
            if constexpr (std::is_same<T, double>::value) {
                stress_rot1(P, dt);
                {
                    // f3dm25 is an out-of-line call: it gets a copy, so that
                    // the caller's state is not address-taken (which would
                    // keep it in local memory for every model)
                    PState<double> Pc = P;
                    code = f3dm25(Pc, M, dt);
                    P = Pc;
                }
                aviscosity(P, M); lieupd(P, dt);
            }
            break;
        case 9:
            stress_rot1(P, dt); f3dm9(P, M);
            if (!sueos(P, M)) code = MCM_ECOMPLEX_C;
            aviscosity(P, M); hieupd(P, dt); eqos(P, M, dt);
            stress_up(P); sym_lower(P);
            break;
        case 10:
            stress_rot1(P, dt); f3dm10(P, M, dt);
            if (!sueos(P, M)) code = MCM_ECOMPLEX_C;
            aviscosity(P, M); hieupd(P, dt); eqos(P, M, dt);
            stress_up(P); sym_lower(P);
            break;
        default: break;
    }
    return code;
}

}  // namespace mcm
