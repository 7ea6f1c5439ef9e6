// Small vectors and scalar helpers shared by the device kernels and the host runtime.
// V3<T> is instantiated with float (the FP32 bulk of the arithmetic) and double (root refinement,
// ray origins, the all-FP64 instantiation).
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define OWEC_HD __host__ __device__ __forceinline__
// Out of line on the device: a rarely taken branch whose registers would otherwise count against the
// hot loop around it.
#define OWEC_HD_COLD __host__ __device__ __noinline__ inline
#else
#define OWEC_HD inline
#define OWEC_HD_COLD inline
#endif

namespace owec {

constexpr double kPi = 3.14159265358979323846;
constexpr double kInvPi = 0.31830988618379067154;
constexpr uint32_t kNone = 0xFFFFFFFEu;   // "no boundary / no primitive" (the reference's kNone)

template <class T>
struct V3 {
    T x, y, z;
    OWEC_HD V3() : x(0), y(0), z(0) {}
    OWEC_HD V3(T a, T b, T c) : x(a), y(b), z(c) {}
    template <class U>
    OWEC_HD explicit V3(const V3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    OWEC_HD T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    OWEC_HD V3 operator-() const { return {-x, -y, -z}; }
    OWEC_HD V3& operator+=(const V3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    OWEC_HD V3& operator-=(const V3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    OWEC_HD V3& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
};
template <class T> OWEC_HD V3<T> operator+(V3<T> a, const V3<T>& b) { return a += b; }
template <class T> OWEC_HD V3<T> operator-(V3<T> a, const V3<T>& b) { return a -= b; }
template <class T> OWEC_HD V3<T> operator*(V3<T> a, T s) { return a *= s; }
template <class T> OWEC_HD V3<T> operator*(T s, V3<T> a) { return a *= s; }
template <class T> OWEC_HD V3<T> operator/(V3<T> a, T s) { return a * (T(1) / s); }
template <class T> OWEC_HD T dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> OWEC_HD V3<T> cross(const V3<T>& a, const V3<T>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> OWEC_HD T lengthSq(const V3<T>& a) { return dot(a, a); }
template <class T> OWEC_HD T length(const V3<T>& a) { return sqrt(dot(a, a)); }
template <class T> OWEC_HD V3<T> normalize(const V3<T>& a) { return a / length(a); }
template <class T> OWEC_HD T maxAbs(const V3<T>& a) { return fmax(fabs(a.x), fmax(fabs(a.y), fabs(a.z))); }
template <class T> OWEC_HD V3<T> reflect(const V3<T>& d, const V3<T>& n) { return d - n * (T(2) * dot(d, n)); }

template <class T> OWEC_HD T sqr(T x) { return x * x; }
template <class T> OWEC_HD T clampv(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }
template <class T> OWEC_HD T safeSqrt(T x) { return sqrt(x > T(0) ? x : T(0)); }

// Orthonormal basis around a unit vector (Duff et al. 2017), as the reference's
// orthonormalBasis (src/owe/core/shared/warps.hpp:36-43).
template <class T>
OWEC_HD void basis(const V3<T>& n, V3<T>& b1, V3<T>& b2) {
    T sgn = copysign(T(1), n.z);
    T a = T(-1) / (sgn + n.z);
    T b = n.x * n.y * a;
    b1 = V3<T>(T(1) + sgn * n.x * n.x * a, sgn * b, -sgn * n.x);
    b2 = V3<T>(b, sgn + n.y * n.y * a, -n.y);
}

// A shading frame about n (src/owe/core/math.hpp:104-110).
template <class T>
struct Frame {
    V3<T> s, t, n;
    OWEC_HD explicit Frame(const V3<T>& nn) : n(nn) { basis(n, s, t); }
    OWEC_HD V3<T> toLocal(const V3<T>& v) const { return {dot(v, s), dot(v, t), dot(v, n)}; }
    OWEC_HD V3<T> toWorld(const V3<T>& v) const { return s * v.x + t * v.y + n * v.z; }
};

// A rigid transform p' = R p + t, row-major (src/owe/core/math.hpp:114-128).
struct Xform {
    double m[12];
    template <class T>
    OWEC_HD V3<T> point(const V3<T>& p) const {
        return {T(m[0]) * p.x + T(m[1]) * p.y + T(m[2]) * p.z + T(m[3]),
                T(m[4]) * p.x + T(m[5]) * p.y + T(m[6]) * p.z + T(m[7]),
                T(m[8]) * p.x + T(m[9]) * p.y + T(m[10]) * p.z + T(m[11])};
    }
    template <class T>
    OWEC_HD V3<T> vector(const V3<T>& v) const {
        return {T(m[0]) * v.x + T(m[1]) * v.y + T(m[2]) * v.z, T(m[4]) * v.x + T(m[5]) * v.y + T(m[6]) * v.z,
                T(m[8]) * v.x + T(m[9]) * v.y + T(m[10]) * v.z};
    }
};

}  // namespace owec
