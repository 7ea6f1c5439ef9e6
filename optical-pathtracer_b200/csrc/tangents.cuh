// Derivative helpers of the path-replay adjoints (the walks' and the camera paths'): forward-mode
// dual numbers for the local contribution functions, the Fresnel reflectance with its derivative,
// and the derivatives of Snell refraction and of the mirror reflection.
#pragma once

#include "common.cuh"

namespace owec {

// ------------------------------------------------------------------ dual numbers
// A value and its partial derivatives in N variables, FP64. Used to differentiate a path vertex's
// contribution (next-event estimate, emission with MIS) with respect to that vertex's position,
// direction and pdf: the handful of inputs the heights move.
template <int N>
struct Dual {
    double v, d[N];
    __device__ Dual() {}
    __device__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) d[k] = 0;
    }
    __device__ static Dual var(double x, int i) {
        Dual r(x);
        r.d[i] = 1;
        return r;
    }
};

template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) { return a + Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator+(double a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) { return a - Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator-(double a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double a, const Dual<N>& b) { return b * a; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) { return Dual<N>(a) / b; }

// f(a) with f' given: the chain rule on every partial
template <int N>
__device__ __forceinline__ Dual<N> chain(const Dual<N>& a, double f, double fp) {
    Dual<N> r;
    r.v = f;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = fp * a.d[k];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
    const double s = ::sqrt(a.v);
    return chain(a, s, s > 0 ? 0.5 / s : 0.0);
}
template <int N> __device__ __forceinline__ Dual<N> dexp(const Dual<N>& a) {
    const double e = ::exp(a.v);
    return chain(a, e, e);
}
template <int N> __device__ __forceinline__ Dual<N> dabs(const Dual<N>& a) { return a.v < 0 ? -a : a; }

template <int N>
struct DV3 {
    Dual<N> x, y, z;
};
template <int N> __device__ __forceinline__ DV3<N> operator-(const V3<double>& a, const DV3<N>& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int N> __device__ __forceinline__ DV3<N> operator-(const DV3<N>& a, const V3<double>& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int N> __device__ __forceinline__ DV3<N> operator-(const DV3<N>& a, const DV3<N>& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <int N> __device__ __forceinline__ DV3<N> operator/(const DV3<N>& a, const Dual<N>& s) {
    return {a.x / s, a.y / s, a.z / s};
}
template <int N> __device__ __forceinline__ Dual<N> ddot(const DV3<N>& a, const DV3<N>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <int N> __device__ __forceinline__ Dual<N> ddot(const DV3<N>& a, const V3<double>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
// A vector whose components are variables first .. first + 2
template <int N> __device__ __forceinline__ DV3<N> dvar3(const V3<double>& v, int first) {
    return {Dual<N>::var(v.x, first), Dual<N>::var(v.y, first + 1), Dual<N>::var(v.z, first + 2)};
}

// The MIS power heuristic f^2 / (f^2 + g^2) of duals (powerHeuristic).
template <int N> __device__ __forceinline__ Dual<N> dpowerHeuristic(const Dual<N>& f, const Dual<N>& g) {
    const Dual<N> f2 = f * f, g2 = g * g;
    if (f2.v + g2.v == 0) return Dual<N>(0.0);
    return f2 / (f2 + g2);
}

// The Henyey-Greenstein phase of a dual cosine (hgPhase).
template <int N> __device__ __forceinline__ Dual<N> dhgPhase(const Dual<N>& c, double g) {
    const Dual<N> denom = 1.0 + g * g + 2.0 * g * c;
    return (1.0 - g * g) / (4.0 * kPi * denom * dsqrt(denom));
}

// ------------------------------------------------------------------ Fresnel and directions
// Unpolarised Fresnel reflectance and its derivative in cosThetaI (the function of
// src/owe/core/shared/optics.hpp:42-54), eta = n_back / n_front, cosThetaI signed against the
// front normal.
__device__ __forceinline__ void fresnelWithDerivative(double c, double eta, double& R, double& dRdc) {
    double sgn = 1;
    c = fmin(1.0, fmax(-1.0, c));
    if (c < 0) { eta = 1 / eta; c = -c; sgn = -1; }
    const double s2 = (1 - c * c) / (eta * eta);
    if (s2 >= 1) { R = 1; dRdc = 0; return; }
    const double ct = sqrt(fmax(0.0, 1 - s2));
    const double dct = ct > 0 ? (c / (eta * eta)) / ct : 0;
    const double a = eta * c - ct, b = eta * c + ct;
    const double rp = a / b, drp = ((eta - dct) * b - a * (eta + dct)) / (b * b);
    const double e = c - eta * ct, f = c + eta * ct;
    const double rs = e / f, drs = ((1 - eta * dct) * f - e * (1 + eta * dct)) / (f * f);
    R = (rp * rp + rs * rs) / 2;
    dRdc = sgn * (rp * drp + rs * drs);
}

// The derivative of Snell's refracted direction (refractDirection) of unit d at unit normal n, given
// the derivatives dd and dn, from index ni into index nt.
__device__ __forceinline__ V3<double> refractTangent(const V3<double>& d, const V3<double>& n, double ni, double nt,
                                                     const V3<double>& dd, const V3<double>& dn) {
    const bool fr = dot(d, n) < 0;
    const V3<double> nn = fr ? n : -n, dnn = fr ? dn : -dn;
    const double eta = ni / nt, cosi = -dot(d, nn);
    const double dcosi = -(dot(dd, nn) + dot(d, dnn));
    const double kk = 1 - eta * eta * (1 - cosi * cosi), sq = sqrt(fmax(kk, 1e-300));
    const V3<double> u = d * eta + nn * (eta * cosi - sq);
    const double ds = eta * eta * cosi * dcosi / sq;
    const V3<double> du = dd * eta + dnn * (eta * cosi - sq) + nn * (eta * dcosi - ds);
    const double ul = length(u);
    const V3<double> out = u / ul;
    return (du - out * dot(out, du)) / ul;
}

// The derivative of the mirror direction d - 2 (d . n) n.
__device__ __forceinline__ V3<double> reflectTangent(const V3<double>& d, const V3<double>& n, const V3<double>& dd,
                                                     const V3<double>& dn) {
    return dd - n * (2 * (dot(dd, n) + dot(d, dn))) - dn * (2 * dot(d, n));
}

}  // namespace owec
