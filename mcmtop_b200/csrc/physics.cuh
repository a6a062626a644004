// physics.cuh -- per-particle physics of the MCM explicit step as device
// functions.  Templated on the arithmetic type T: T = double for the FP64
// paths, T = float for the constitutive update of the mixed path.  The
// expressions keep the reference's evaluation order (left-to-right, explicit
// parentheses) so that the FP64 translation unit compiled without fused
// multiply-add reproduces the reference arithmetic; single-precision Fortran
// literals appear as float literals cast to T.
#pragma once
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
// MCM/mcm_rhoupd.f90:119-151
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
// MCM/mcm_stress_rot1.f90:193-355 (iorder = 3, exponential map)
template <typename T>
__device__ __forceinline__ void stress_rot1(PState<T> &P, T dt) {
    const T etol = T(1.0e-3f);
    const T z1 = T(1.0) / T(3.0), z2 = T(2.0) / T(15.0), z3 = T(17.0) / T(315.0), z4 = T(62.0) / T(2835.0);
    const T s11 = P.sig[T11], s22 = P.sig[T22], s33 = P.sig[T33];
    const T s12 = P.sig[T12], s23 = P.sig[T23], s31 = P.sig[T13];
    T dt2 = T(0.5f) * dt;
    T wzz = -dt2 * P.spin[0];
    T wyy = dt2 * P.spin[1];
    T wxx = -dt2 * P.spin[2];
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
    q12 = q12 - bwzz;
    q21 = q21 + bwzz;
    q13 = q13 + bwyy;
    q31 = q31 - bwyy;
    q23 = q23 - bwxx;
    q32 = q32 + bwxx;
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
}

// ------------------------------------------------------------- EOS: sound speed
// MCM/mcm_eos1c.f90:115-164 (complex c forced to continue)
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

// MCM/mcm_eos13c.f90:219-227
template <typename T, typename Mat>
__device__ __forceinline__ void eos13c(PState<T> &P, const Mat &M) {
    T gamma = T(M.eosinput[0]);
    T e1 = P.e / P.mass;
    P.c = sqrt((gamma - T(1.0)) * gamma * e1);
}

// MCM/mcm_eos28c.f90:305-310
template <typename T, typename Mat>
__device__ __forceinline__ void eos28c(PState<T> &P, const Mat &M) {
    T b = T(M.eosinput[0]), gamma = T(M.eosinput[1]);
    P.c = sqrt(b * gamma / P.rho0);
}

// MCM/mcm_eos41c.f90:240-294.  Returns false when c^2 < 0 (the reference stops).
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

// MCM/mcm_sueos.f90:185-207
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

// MCM/mcm_eqos4.f90:131-183
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

// MCM/mcm_eqos13.f90:258-274
template <typename T, typename Mat>
__device__ __forceinline__ void eqos13(PState<T> &P, const Mat &M) {
    T gamma_m1 = T(M.eosinput[0]) - T(1.0);
    T e1try = P.etry / P.mass;
    T dvol = P.mass / P.rho - P.mass / P.rhoold;
    P.p = (P.rho * gamma_m1 * e1try) / (T(1.0) + T(0.5) * P.rho * gamma_m1 * dvol / P.mass);
    P.e = P.etry - T(0.5) * dvol * P.p;
}

// MCM/mcm_eqos28.f90:343-358
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

// MCM/mcm_eqos.f90:183-214
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
// MCM/mcm_nodalav.f90:76-91 (q is isotropic: only the diagonal is stored)
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
// MCM/mcm_hieupd.f90:119-156; de(k,l) summed in column-major order
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

// MCM/mcm_lieupd.f90:283-290 (dot product in column-major order)
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

// MCM/mcm_stress_up.f90:245-253
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

// MCM/mcm_f3dm3.f90:106-233
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

// MCM/mcm_f3dm9.f90:261-285 (s(1,2) is never assigned; xmu = cm(2,mat))
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
// Returns false if the EOS reported a complex sound speed.
template <typename T, typename Mat>
__device__ __forceinline__ bool constitutive_particle(PState<T> &P, const Mat &M, T dt) {
    bool ok = true;
    switch (M.model) {
        case 1:
            stress_rot1(P, dt); f3dm1(P, M, dt); aviscosity(P, M); lieupd(P, dt);
            break;
        case 3:
            stress_rot1(P, dt); f3dm3(P, M, dt); aviscosity(P, M); lieupd(P, dt);
            break;
        case 9:
            stress_rot1(P, dt); f3dm9(P, M); ok = sueos(P, M); aviscosity(P, M); hieupd(P, dt); eqos(P, M, dt);
            stress_up(P);
            break;
        case 10:
            stress_rot1(P, dt); f3dm10(P, M, dt); ok = sueos(P, M); aviscosity(P, M); hieupd(P, dt); eqos(P, M, dt);
            stress_up(P);
            break;
        default: break;
    }
    return ok;
}

}  // namespace mcm
