// dual.cuh -- forward-mode dual numbers for the per-particle Jacobians of the
// adjoint step.
//
// A Dual<N> carries a value and N directional derivatives.  The templated
// constitutive code (physics.cuh) runs on it unchanged: branches compare
// values, so every derivative is that of the branch the forward step took
// (the active branch of the plastic return map, of the EOS cut-offs, ...).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace mcm {

// keep the built-in overloads visible next to the Dual ones below
using ::acos;
using ::cos;
using ::fabs;
using ::pow;
using ::sqrt;
using ::tan;

template <int N>
struct Dual {
    double v;
    double d[N];
    __host__ __device__ Dual() : v(0.0) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    __host__ __device__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0.0;
    }
    __host__ __device__ explicit operator int() const { return (int)v; }
    __host__ __device__ Dual &operator+=(const Dual &b) { return *this = *this + b; }
    __host__ __device__ Dual &operator-=(const Dual &b) { return *this = *this - b; }
    __host__ __device__ Dual &operator*=(const Dual &b) { return *this = *this * b; }
    __host__ __device__ Dual &operator/=(const Dual &b) { return *this = *this / b; }
    friend __host__ __device__ Dual operator+(const Dual &a, const Dual &b) {
        Dual r;
        r.v = a.v + b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
        return r;
    }
    friend __host__ __device__ Dual operator-(const Dual &a, const Dual &b) {
        Dual r;
        r.v = a.v - b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
        return r;
    }
    friend __host__ __device__ Dual operator-(const Dual &a) {
        Dual r;
        r.v = -a.v;
#pragma unroll
        for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
        return r;
    }
    friend __host__ __device__ Dual operator*(const Dual &a, const Dual &b) {
        Dual r;
        r.v = a.v * b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
        return r;
    }
    friend __host__ __device__ Dual operator/(const Dual &a, const Dual &b) {
        Dual r;
        r.v = a.v / b.v;
        const double ib = 1.0 / b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
        return r;
    }
    friend __host__ __device__ bool operator<(const Dual &a, const Dual &b) { return a.v < b.v; }
    friend __host__ __device__ bool operator>(const Dual &a, const Dual &b) { return a.v > b.v; }
    friend __host__ __device__ bool operator<=(const Dual &a, const Dual &b) { return a.v <= b.v; }
    friend __host__ __device__ bool operator>=(const Dual &a, const Dual &b) { return a.v >= b.v; }
    friend __host__ __device__ bool operator==(const Dual &a, const Dual &b) { return a.v == b.v; }
    friend __host__ __device__ bool operator!=(const Dual &a, const Dual &b) { return a.v != b.v; }
};

// f(a) with f' given: the chain rule on every direction
template <int N>
__host__ __device__ inline Dual<N> dual_chain(const Dual<N> &a, double fv, double fd) {
    Dual<N> r;
    r.v = fv;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = fd * a.d[k];
    return r;
}

template <int N>
__host__ __device__ inline Dual<N> sqrt(const Dual<N> &a) {
    const double s = ::sqrt(a.v);
    return dual_chain(a, s, s > 0.0 ? 0.5 / s : 0.0);
}
template <int N>
__host__ __device__ inline Dual<N> fabs(const Dual<N> &a) {
    return a.v < 0.0 ? -a : a;
}
template <int N>
__host__ __device__ inline Dual<N> tan(const Dual<N> &a) {
    const double t = ::tan(a.v);
    return dual_chain(a, t, 1.0 + t * t);
}
template <int N>
__host__ __device__ inline Dual<N> cos(const Dual<N> &a) {
    return dual_chain(a, ::cos(a.v), -::sin(a.v));
}
template <int N>
__host__ __device__ inline Dual<N> acos(const Dual<N> &a) {
    const double s = 1.0 - a.v * a.v;
    return dual_chain(a, ::acos(a.v), s > 0.0 ? -1.0 / ::sqrt(s) : 0.0);
}
// a^b = exp(b log a); the b-derivative term only where b varies
template <int N>
__host__ __device__ inline Dual<N> pow(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = ::pow(a.v, b.v);
    const double da = (a.v != 0.0) ? b.v * r.v / a.v : 0.0;
    const double db = (a.v > 0.0) ? r.v * ::log(a.v) : 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = da * a.d[k] + db * b.d[k];
    return r;
}

__host__ __device__ inline double value_of(double x) { return x; }
__host__ __device__ inline float value_of(float x) { return x; }
template <int N>
__host__ __device__ inline double value_of(const Dual<N> &x) { return x.v; }

}  // namespace mcm
