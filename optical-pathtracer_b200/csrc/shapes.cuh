// Analytic surfaces in their own frames: spheres, conic and aspheric sags, planes with apertures,
// cylinders, cones, torus patches, round walls, domes and wave surfaces (src/owe/scene/geometry.cpp). Quadric roots
// come from the numerically stable quadratic in precision R and are refined by re-solving from the
// approximate hit in precision Rr (src/owe/core/shared/surfaces.hpp:13-137): with R = float and
// Rr = double this is the selective FP64 step that keeps large-radius lens surfaces exact; with
// R = Rr = float it is the plain FP32 baseline. Aspheres, torus patches and wave surfaces have no
// closed form: their crossings are bracketed along the clipped ray and bisected (or, near a wave
// surface, converged on by Newton's method), in precision Rr.
#pragma once

#include "device_scene.cuh"

namespace owec {

template <class T> struct Tol;
template <> struct Tol<float> {
    static constexpr float refine = 1e-3f, relTol = 1e-6f, tiny = 1e-30f, bisect = 2e-7f, angle = 1e-5f,
                           eps = 1.1920929e-7f;
    static constexpr int bisectSteps = 40;
};
template <> struct Tol<double> {
    static constexpr double refine = 1e-6, relTol = 1e-9, tiny = 1e-300, bisect = 1e-15, angle = 1e-9,
                            eps = 2.220446049250313e-16;
    static constexpr int bisectSteps = 80;
};

// Real roots of a t^2 + b t + c = 0, ascending; returns their count (surfaces.hpp:13-33).
template <class T>
OWEC_HD int solveQuadratic(T a, T b, T c, T& t0, T& t1) {
    t0 = t1 = T(0);
    if (fabs(a) < Tol<T>::tiny || fabs(a) < T(1e-14) * fabs(b)) {
        if (b == T(0)) return 0;
        t0 = t1 = -c / b;
        return 1;
    }
    const T disc = b * b - T(4) * a * c;
    if (disc < T(0)) return 0;
    const T q = -(b + copysign(sqrt(disc), b)) / T(2);
    t0 = q / a;
    t1 = q != T(0) ? c / q : t0;
    if (t0 > t1) { const T tmp = t0; t0 = t1; t1 = tmp; }
    return 2;
}

constexpr int kQuadSag = 0, kQuadSphere = 1, kQuadCylinder = 2, kQuadCone = 3;

// The coefficients of a quadric along o + t d: a sag c (x^2 + y^2) + c (1 + k) z^2 - 2 z
// (qa = c, qb = c (1 + k)), a sphere or an infinite cylinder of radius^2 qa, or a cone
// x^2 + y^2 = (r0 + k (z - z0))^2 (qa = r0, qb = z0, qc = k) (surfaces.hpp:34-72).
template <class T>
OWEC_HD void quadricCoeffs(int kind, T qa, T qb, T qc, const V3<T>& o, const V3<T>& d, T& A, T& B, T& C) {
    if (kind == kQuadCone) {
        const T rho = qa + qc * (o.z - qb);
        A = d.x * d.x + d.y * d.y - qc * qc * d.z * d.z;
        B = T(2) * (o.x * d.x + o.y * d.y - qc * rho * d.z);
        C = o.x * o.x + o.y * o.y - rho * rho;
    } else if (kind == kQuadSag) {
        A = qa * (d.x * d.x + d.y * d.y) + qb * d.z * d.z;
        B = T(2) * (qa * (o.x * d.x + o.y * d.y) + qb * o.z * d.z - d.z);
        C = qa * (o.x * o.x + o.y * o.y) + qb * o.z * o.z - T(2) * o.z;
    } else if (kind == kQuadSphere) {
        A = dot(d, d);
        B = T(2) * dot(o, d);
        C = dot(o, o) - qa;
    } else {
        A = d.x * d.x + d.y * d.y;
        B = T(2) * (o.x * d.x + o.y * d.y);
        C = o.x * o.x + o.y * o.y - qa;
    }
}

// The root t (from precision R) refined in precision Rr, if it may lie in (tmin, tmax) and does
// once refined (refineRoot / mayLieIn / refinedRootIn, surfaces.hpp:75-101).
template <class R, class Rr>
OWEC_HD bool refinedRootIn(int kind, Rr qa, Rr qb, const V3<Rr>& o, const V3<Rr>& d, Rr t, Rr tmin, Rr tmax, Rr& tr,
                           Rr qc = Rr(0)) {
    tr = t;
    const Rr m = Rr(Tol<R>::refine) * (Rr(1) + fabs(t));
    if (t + m <= tmin || t - m >= tmax) return false;
    Rr A, B, C, u0, u1;
    quadricCoeffs(kind, qa, qb, qc, o + d * t, d, A, B, C);
    if (solveQuadratic(A, B, C, u0, u1) != 0) {
        const Rr du = fabs(u0) < fabs(u1) ? u0 : u1;
        if (fabs(du) < m) tr = t + du;
    }
    return tr > tmin && tr < tmax;
}

// A crossing of an analytic surface in its frame.
template <class Rr>
struct AHit {
    Rr t;
    V3<Rr> p, n;
};

// At most two crossings, kept in named members (not an indexed array) so that they stay in
// registers when the count is only known at run time.
template <class Rr>
struct AHits {
    AHit<Rr> h0, h1;
    int n = 0;
    OWEC_HD void add(const AHit<Rr>& h) {
        if (n == 0) h0 = h;
        else h1 = h;
        ++n;
    }
    OWEC_HD const AHit<Rr>& get(int i) const { return i == 0 ? h0 : h1; }
};

// Sphere roots in the geometric form (surfaces.hpp:104-122).
template <class T>
OWEC_HD bool sphereRoots(const V3<T>& o, const V3<T>& d, T R, T& t0, T& t1) {
    const T b = dot(o, d);
    const V3<T> perp = o - d * b;
    const T disc = R * R - dot(perp, perp);
    t0 = t1 = T(0);
    if (disc < T(0)) return false;
    const T c = dot(o, o) - R * R;
    const T q = -b - copysign(sqrt(disc), b);
    t0 = q;
    t1 = q != T(0) ? c / q : q;
    if (t0 > t1) { const T tmp = t0; t0 = t1; t1 = tmp; }
    return true;
}

// Double-double numbers (hi + lo, |lo| at most half an ulp of hi) built from the error-free
// transformations: Knuth's two-sum for a sum, the fused multiply-add for the error of a product.
struct DDouble {
    double hi, lo;
};
OWEC_HD DDouble ddTwoSum(double a, double b) {
    const double s = a + b, v = s - a;
    return {s, (a - (s - v)) + (b - v)};
}
OWEC_HD DDouble ddAdd(const DDouble& a, const DDouble& b) {
    const DDouble s = ddTwoSum(a.hi, b.hi);
    return ddTwoSum(s.hi, s.lo + a.lo + b.lo);
}
OWEC_HD DDouble ddMul(const DDouble& a, const DDouble& b) {
    const double p = a.hi * b.hi;
    return ddTwoSum(p, fma(a.hi, b.hi, -p) + (a.hi * b.lo + a.lo * b.hi));
}
OWEC_HD DDouble ddNeg(const DDouble& a) { return {-a.hi, -a.lo}; }
OWEC_HD double ddValue(const DDouble& a) { return a.hi + a.lo; }

// Whether a ray from od lies near boundary b's sphere against the sphere's size (a planet's surface
// under the camera): there |od - c|^2 - R^2 cancels to nothing in FP64 once od - c is rounded, and
// the reference solves the quadratic in double-double arithmetic (needsNearSphere, intersectNearSphere,
// src/owe/scene/world.cpp:404-438). The same switch, for spheres of kNearSphereMinRadius and more:
// for smaller ones the FP64 roots of a ray leaving the sphere stay within the refined departure
// window, and a scene with a larger one runs the Full instantiations, the only ones that ask.
constexpr double kNearSphereMinRadius = 64.0;
OWEC_HD bool nearSphere(const DBoundary& b, const V3<double>& od) {
    if (b.shape != OWEC_SHAPE_SPHERE || !(b.params[0] >= kNearSphereMinRadius)) return false;
    const double R = b.params[0];
    const V3<double> c(b.toWorld.m[3], b.toWorld.m[7], b.toWorld.m[11]);
    return R > 4096 * fmax(1e-9, fabs(length(od - c) - R));
}

// The sphere's crossings in (tmin, tmax) for such a ray, in the world frame (a sphere's roots do not
// depend on its frame's rotation): od - c exact as a double-double, the quadratic's coefficients in
// double-double, the roots in the numerically stable form. Points and normals in the sphere's local
// frame, as classicCrossings gives them (the normal from the exact od - c; the point converted from
// the world point od + t d). Out of line, its result by value: the callers' own hits stay in registers.
OWEC_HD_COLD AHits<double> nearSphereCrossings(const DBoundary& b, V3<double> od, V3<double> d, double tmin,
                                               double tmax) {
    AHits<double> out;
    const double R = b.params[0];
    const double o[3] = {od.x, od.y, od.z}, dv[3] = {d.x, d.y, d.z};
    const double c[3] = {b.toWorld.m[3], b.toWorld.m[7], b.toWorld.m[11]};
    DDouble rel[3], A{0, 0}, B{0, 0}, C{0, 0};
    for (int k = 0; k < 3; ++k) {
        rel[k] = ddTwoSum(o[k], -c[k]);
        A = ddAdd(A, ddMul({dv[k], 0}, {dv[k], 0}));
        B = ddAdd(B, ddMul(rel[k], {dv[k], 0}));
        C = ddAdd(C, ddMul(rel[k], rel[k]));
    }
    C = ddAdd(C, ddNeg(ddMul({R, 0}, {R, 0})));
    const double disc = ddValue(ddAdd(ddMul(B, B), ddNeg(ddMul(A, C))));
    if (!(disc >= 0)) return out;
    const double bv = ddValue(B), av = ddValue(A);
    const double q = -bv - copysign(sqrt(disc), bv);
    double t0 = q / av, t1 = q != 0 ? ddValue(C) / q : t0;
    if (t0 > t1) { const double tmp = t0; t0 = t1; t1 = tmp; }
    const double ts[2] = {t0, t1};
    for (int i = 0; i < 2; ++i) {
        const double t = ts[i];
        if (!(t > tmin && t < tmax) || (i == 1 && t1 == t0)) continue;
        V3<double> nw;
        nw.x = ddValue(ddAdd(rel[0], ddMul({dv[0], 0}, {t, 0}))) / R;
        nw.y = ddValue(ddAdd(rel[1], ddMul({dv[1], 0}, {t, 0}))) / R;
        nw.z = ddValue(ddAdd(rel[2], ddMul({dv[2], 0}, {t, 0}))) / R;
        out.add({t, b.toLocal.point(od + d * t), normalize(b.toLocal.vector(nw))});
    }
    return out;
}

template <class T>
OWEC_HD bool cylinderRoots(const V3<T>& o, const V3<T>& d, T R, T& t0, T& t1) {
    t0 = t1 = T(0);
    const T A = d.x * d.x + d.y * d.y;
    if (A < Tol<T>::tiny) return false;
    const T b = o.x * d.x + o.y * d.y;
    const T px = o.x - d.x * (b / A), py = o.y - d.y * (b / A);
    const T disc = A * (R * R - (px * px + py * py));
    if (disc < T(0)) return false;
    const T q = -(b + copysign(sqrt(disc), b));
    const T c = o.x * o.x + o.y * o.y - R * R;
    t0 = q / A;
    t1 = q != T(0) ? c / q : t0;
    if (t0 > t1) { const T tmp = t0; t0 = t1; t1 = tmp; }
    return true;
}

template <class T> OWEC_HD T conicSag(T c, T k, T r2) { return c * r2 / (T(1) + safeSqrt(T(1) - (T(1) + k) * c * c * r2)); }
template <class T> OWEC_HD T conicSlope(T c, T k, T r) {
    const T root = safeSqrt(T(1) - (T(1) + k) * c * c * (r * r));
    return root > T(0) ? c * r / root : (c != T(0) ? T(INFINITY) : T(0));
}

// An even asphere's sag z(r) = conic + sum A_{2m} r^{2m} (m >= 2) and its slope dz/dr
// (SagSurface::sag, dsag, src/owe/scene/geometry.cpp:90-103). A: A4, A6, ...
template <class T>
OWEC_HD T asphereSag(T c, T k, const double* A, int nA, T r) {
    const T r2 = r * r;
    T z = conicSag(c, k, r2), rp = r2 * r2;
    for (int i = 0; i < nA; ++i) { z += T(A[i]) * rp; rp *= r2; }
    return z;
}
template <class T>
OWEC_HD T asphereSlope(T c, T k, const double* A, int nA, T r) {
    T s = conicSlope(c, k, r), m = T(4), rp = r * r * r;
    for (int i = 0; i < nA; ++i) { s += T(A[i]) * m * rp; rp *= r * r; m += T(2); }
    return s;
}
// The unit normal (toward +z) of a sag of slope s at radius r of point p (sagNormal, surfaces.hpp:168).
template <class T>
OWEC_HD V3<T> sagNormal(const V3<T>& p, T r, T s) {
    if (r < Tol<T>::tiny) return V3<T>(0, 0, 1);
    return normalize(V3<T>(-s * p.x / r, -s * p.y / r, T(1)));
}

// Clips (ta, tb) to the slab lo <= o + t d <= hi along one axis, and to the infinite cylinder of
// radius R about z; false when nothing remains (clipSlab, clipCylinder, surfaces.hpp:140-157).
template <class T>
OWEC_HD bool clipSlab(T o, T d, T lo, T hi, T& ta, T& tb) {
    if (fabs(d) < Tol<T>::tiny) return o >= lo && o <= hi && ta < tb;
    const T s0 = (lo - o) / d, s1 = (hi - o) / d;
    ta = fmax(ta, fmin(s0, s1));
    tb = fmin(tb, fmax(s0, s1));
    return ta < tb;
}
template <class T>
OWEC_HD bool clipCylinder(const V3<T>& o, const V3<T>& d, T R, T& ta, T& tb) {
    const T a = d.x * d.x + d.y * d.y;
    if (a < Tol<T>::tiny) return o.x * o.x + o.y * o.y <= R * R && ta < tb;
    T q0, q1;
    if (solveQuadratic(a, T(2) * (o.x * d.x + o.y * d.y), o.x * o.x + o.y * o.y - R * R, q0, q1) < 2) return false;
    ta = fmax(ta, q0);
    tb = fmin(tb, q1);
    return ta < tb;
}

// Bisects a sign change of f in [lo, hi] (f(lo) = flo) to the precision's bracket width
// (geometry.cpp:50-64).
template <class T, class F>
OWEC_HD T bisectRoot(const F& f, T lo, T hi, T flo, int steps) {
    for (int it = 0; it < steps && hi - lo > T(Tol<T>::bisect) * (T(1) + fabs(hi)); ++it) {
        const T mid = T(0.5) * (lo + hi);
        const T fm = f(mid);
        if ((fm <= T(0)) == (flo <= T(0))) {
            lo = mid;
            flo = fm;
        } else {
            hi = mid;
        }
    }
    return T(0.5) * (lo + hi);
}

// Torus patch: F < 0 inside the tube, the arc test and the normal away from the arc's centre
// (torusF, torusOnArc, torusNormal, surfaces.hpp:209-225).
template <class T>
OWEC_HD T torusF(T R, T zc, T rho, const V3<T>& p) {
    return sqr(sqrt(p.x * p.x + p.y * p.y) - R) + sqr(p.z - zc) - rho * rho;
}
template <class T>
OWEC_HD bool torusOnArc(T R, T zc, T a0, T a1, const V3<T>& p) {
    const T a = atan2(p.z - zc, sqrt(p.x * p.x + p.y * p.y) - R);
    for (int k = -1; k <= 1; ++k) {
        const T w = a + T(k) * T(2 * kPi);
        if (w >= a0 - T(Tol<T>::angle) && w <= a1 + T(Tol<T>::angle)) return true;
    }
    return false;
}
template <class T>
OWEC_HD V3<T> torusNormal(T R, T zc, const V3<T>& p) {
    const T rho = sqrt(p.x * p.x + p.y * p.y);
    const V3<T> c = rho > T(0) ? V3<T>(p.x * R / rho, p.y * R / rho, zc) : V3<T>(0, 0, zc);
    return normalize(p - c);
}

// Trims: a plane aperture, a round wall's rectangular opening (centred on an azimuth from +y toward
// +x, `width` along the wall, between sill and top) and a dome's slit of constant linear width
// (inPlaneAperture, inWallOpening, domeSolid, surfaces.hpp:232-262).
template <class T>
OWEC_HD bool inPlaneAperture(int kind, T a, T b, T hx, T hy, const V3<T>& p) {
    if (kind == OWEC_APERTURE_DISK) {
        const T r2 = p.x * p.x + p.y * p.y;
        return r2 <= a * a && r2 >= b * b;
    }
    if (kind == OWEC_APERTURE_RECT) return fabs(p.x) <= a && fabs(p.y) <= b;
    if (kind == OWEC_APERTURE_ELLIPSE) return sqr(p.x / a) + sqr(p.y / b) <= T(1);
    return p.x * p.x + p.y * p.y <= a * a && sqr(p.x - hx) + sqr(p.y - hy) >= b * b;
}
template <class T>
OWEC_HD bool inWallOpening(T R, T azimuth, T width, T sill, T top, const V3<T>& p) {
    const T dAz = remainder(atan2(p.x, p.y) - azimuth, T(2 * kPi));
    return fabs(dAz) * R < width / T(2) && p.z > sill && p.z < top;
}
template <class T>
OWEC_HD bool domeSolid(T R, T azimuth, T width, T top, const V3<T>& p) {
    if (p.z < T(0)) return false;
    if (width <= T(0)) return true;
    const T el = asin(fmin(T(1), fmax(T(-1), p.z / R)));
    if (el >= top) return true;
    const T dAz = remainder(atan2(p.x, p.y) - azimuth, T(2 * kPi));
    return fabs(sin(dAz)) * R * cos(el) >= width / T(2) || cos(dAz) < T(0);
}

// The crossings of the shapes every scene had before the trimmed, lathe and aspheric ones: spheres,
// conic sags, disk, rectangle and ellipse apertures and cylinders (the lean traversal's
// analyticCrossings; see there).
template <class R, class Rr>
OWEC_HD int classicCrossings(const DBoundary& b, const V3<Rr>& o, const V3<Rr>& d, Rr tmin, Rr tmax, AHits<Rr>& out) {
    out.n = 0;
    const double* P = b.params;
    switch (b.shape) {
        case OWEC_SHAPE_SPHERE: {
            // Sphere roots in the refinement's precision: a ray leaving a large sphere (a moon, a
            // planet, a dome) has |o| near R, where FP32 loses c = |o|^2 - R^2 entirely, and a root
            // the refinement cannot pull back within its window would survive as a false crossing.
            const Rr Rad = Rr(P[0]);
            Rr t0, t1;
            if (!sphereRoots(o, d, Rad, t0, t1)) return 0;
            const Rr ts[2] = {t0, t1};
            for (int i = 0; i < 2; ++i) {
                Rr tr;
                if (!refinedRootIn<Rr, Rr>(kQuadSphere, Rad * Rad, Rr(0), o, d, ts[i], tmin, tmax, tr)) continue;
                const V3<Rr> p = o + d * tr;
                out.add({tr, p, normalize(p / Rad)});
            }
            break;
        }
        case OWEC_SHAPE_SAG: {
            const Rr c = Rr(P[0]), k = Rr(P[1]), rMax = Rr(P[2]), rMin = Rr(P[3]);
            auto solid = [&](const V3<Rr>& p) {
                const Rr r2 = p.x * p.x + p.y * p.y;
                return r2 <= rMax * rMax && r2 >= rMin * rMin &&
                       (c == Rr(0) || (Rr(1) + k) * c * p.z <= Rr(1) + Rr(Tol<R>::relTol));
            };
            auto normal = [&](const V3<Rr>& p) {
                const Rr r = sqrt(p.x * p.x + p.y * p.y);
                if (r < Tol<Rr>::tiny) return V3<Rr>(0, 0, 1);
                const Rr s = conicSlope(c, k, r);
                return normalize(V3<Rr>(-s * p.x / r, -s * p.y / r, Rr(1)));
            };
            if (c == Rr(0)) {
                if (d.z == Rr(0)) return 0;
                const Rr t = -o.z / d.z;
                if (t <= tmin || t >= tmax) return 0;
                const V3<Rr> p = o + d * t;
                if (!solid(p)) return 0;
                out.add({t, p, normal(p)});
                break;
            }
            R A, B, C, t0, t1;
            quadricCoeffs(kQuadSag, R(c), R(c * (Rr(1) + k)), R(0), V3<R>(o), V3<R>(d), A, B, C);
            if (solveQuadratic(A, B, C, t0, t1) <= 0) return 0;
            const R ts[2] = {t0, t1};
            for (int i = 0; i < 2; ++i) {
                if (i == 1 && t1 == t0) break;
                Rr tr;
                if (!refinedRootIn<R, Rr>(kQuadSag, c, c * (Rr(1) + k), o, d, Rr(ts[i]), tmin, tmax, tr)) continue;
                const V3<Rr> p = o + d * tr;
                if (!solid(p)) continue;
                out.add({tr, p, normal(p)});
            }
            break;
        }
        case OWEC_SHAPE_PLANE: {
            if (d.z == Rr(0)) return 0;
            const Rr t = -o.z / d.z;
            if (t <= tmin || t >= tmax) return 0;
            V3<Rr> p = o + d * t;
            p.z = Rr(0);
            const int ap = int(P[0]);
            const Rr a = Rr(P[1]), bb = Rr(P[2]);
            bool in;
            if (ap == OWEC_APERTURE_DISK) {
                const Rr r2 = p.x * p.x + p.y * p.y;
                in = r2 <= a * a && r2 >= bb * bb;
            } else if (ap == OWEC_APERTURE_RECT) {
                in = fabs(p.x) <= a && fabs(p.y) <= bb;
            } else {
                in = sqr(p.x / a) + sqr(p.y / bb) <= Rr(1);
            }
            if (!in) return 0;
            out.add({t, p, V3<Rr>(0, 0, 1)});
            break;
        }
        case OWEC_SHAPE_CYLINDER: {
            const Rr Rad = Rr(P[0]), z0 = Rr(P[1]), z1 = Rr(P[2]);
            R t0, t1;
            if (!cylinderRoots(V3<R>(o), V3<R>(d), R(P[0]), t0, t1)) return 0;
            const R ts[2] = {t0, t1};
            for (int i = 0; i < 2; ++i) {
                Rr tr;
                if (!refinedRootIn<R, Rr>(kQuadCylinder, Rad * Rad, Rr(0), o, d, Rr(ts[i]), tmin, tmax, tr)) continue;
                const V3<Rr> p = o + d * tr;
                if (p.z < z0 || p.z > z1) continue;
                out.add({tr, p, normalize(V3<Rr>(p.x, p.y, Rr(0)))});
            }
            break;
        }
        default: break;
    }
    if (out.n == 2 && out.h1.t < out.h0.t) { const AHit<Rr> tmp = out.h0; out.h0 = out.h1; out.h1 = tmp; }
    return out.n;
}

// Up to two crossings found numerically, ascending. The root finders below are out of line and
// return by value: they need many registers and run only for the rare aspheres and torus patches,
// so they must not raise the register count of the traversal that inlines analyticCrossings.
template <class Rr>
struct NumericRoots {
    Rr t[2];
    int n;
};

// SagSurface::intersectNumeric (geometry.cpp:138-166): the first sign changes of sag(r) - z over 96
// samples of the ray clipped to the surface's cylinder and z slab, bisected; up to two, each within
// the aperture.
template <class Rr>
__device__ __noinline__ NumericRoots<Rr> asphereRoots(Rr c, Rr k, Rr rMax, Rr rMin, Rr zMin, Rr zMax, const double* A,
                                                      int nA, V3<Rr> o, V3<Rr> d, Rr tmin, Rr tmax) {
    NumericRoots<Rr> r{{Rr(0), Rr(0)}, 0};
    Rr ta = tmin, tb = tmax;
    if (!clipCylinder(o, d, rMax, ta, tb) || !clipSlab(o.z, d.z, zMin, zMax, ta, tb)) return r;
    auto f = [&](Rr t) {
        const V3<Rr> p = o + d * t;
        return asphereSag(c, k, A, nA, sqrt(p.x * p.x + p.y * p.y)) - p.z;
    };
    constexpr int N = 96;
    Rr tPrev = ta, fPrev = f(ta);
    for (int i = 1; i <= N && r.n < 2; ++i) {
        const Rr tCur = ta + (tb - ta) * Rr(i) / Rr(N);
        const Rr fCur = f(tCur);
        if (((fPrev <= Rr(0) && fCur >= Rr(0)) || (fPrev >= Rr(0) && fCur <= Rr(0))) && !(fPrev == Rr(0) && tPrev <= tmin)) {
            const Rr t = bisectRoot(f, tPrev, tCur, fPrev, Tol<Rr>::bisectSteps);
            const V3<Rr> p = o + d * t;
            const Rr r2 = p.x * p.x + p.y * p.y;
            if (t > tmin && t < tmax && r2 <= rMax * rMax && r2 >= rMin * rMin) r.t[r.n++] = t;
        }
        tPrev = tCur;
        fPrev = fCur;
    }
    return r;
}

// TorusPatchShape::intersect (geometry.cpp:581-618): the ray clipped to the patch's slab and
// cylinder, F sampled at 64 steps for sign changes and bisected; a ray leaving the patch starts
// with geometrically growing steps so that its own root and a nearby grazing one fall in different
// brackets. Up to two crossings on the arc a0..a1.
template <class Rr>
__device__ __noinline__ NumericRoots<Rr> torusRoots(Rr R0, Rr zc, Rr rho, Rr a0, Rr a1, Rr rMax, Rr zMin, Rr zMax, V3<Rr> o,
                                                    V3<Rr> d, Rr tmin, Rr tmax, bool departed) {
    NumericRoots<Rr> r{{Rr(0), Rr(0)}, 0};
    Rr ta = tmin, tb = tmax;
    const Rr pad = Rr(1e-9) * (Rr(1) + rMax + fabs(zMax));
    if (!clipSlab(o.z, d.z, zMin - pad, zMax + pad, ta, tb) || !clipCylinder(o, d, rMax + pad, ta, tb)) return r;
    auto F = [&](Rr t) { return torusF(R0, zc, rho, o + d * t); };
    constexpr int N = 64;
    Rr tPrev = ta, fPrev = F(ta);
    int sample = 1;
    Rr firstStep = !departed ? tb - ta
                             : fmin((tb - ta) / Rr(N), fmax(ldexp((tb - ta) / Rr(N), -60),
                                                            Rr(64) * Rr(Tol<Rr>::eps) * (Rr(1) + fabs(ta))));
    for (int guard = 0; sample <= N && guard < N + 64 && r.n < 2; ++guard) {
        const Rr uniform = ta + (tb - ta) * Rr(sample) / Rr(N);
        const Rr tCur = fmin(uniform, ta + firstStep);
        if (tCur == uniform) ++sample;
        else firstStep = fmin(tb - ta, firstStep * Rr(2));
        const Rr fCur = F(tCur);
        if ((fPrev <= Rr(0)) != (fCur <= Rr(0)) || fCur == Rr(0)) {
            const Rr t = bisectRoot(F, tPrev, tCur, fPrev, 100);
            if (t > tmin && t < tmax && torusOnArc(R0, zc, a0, a1, o + d * t)) r.t[r.n++] = t;
        }
        tPrev = tCur;
        fPrev = fCur;
    }
    return r;
}

// ------------------------------------------------------------------ liquid waves
// A wave surface z = h(x, y) (WaveSurface, src/owe/scene/geometry.hpp:90-140): h = w(x) w(y) sum of
// a_i sin(k_i . (x, y) + phase_i) over |x| <= halfX, |y| <= halfY, w a smoothstep taper to zero
// within `margin` of the edges; or that sum sampled at nodes as a bicubic Hermite spline. The
// device record: params = halfX, halfY, margin (clamped to the half sizes), the number of waves;
// ext = the amplitude bound, the slope bound, the node spacings in x and y (0: the analytic sum);
// data = the node counts in x and y, the waves as (amplitude, kx, ky, phase), then the nodes row by
// row from (-halfX, -halfY), each (h, dh/dx, dh/dy, d2h/dxdy).

// The taper w(u) toward the edges at +-half within `margin`, and dw/du (waveTaper,
// src/owe/core/shared/surfaces.hpp:177-192).
template <class T>
OWEC_HD void waveTaper(T u, T half, T margin, T& w, T& dw) {
    w = T(1);
    dw = T(0);
    if (!(margin > T(0))) return;
    const T e = half - fabs(u);
    if (e >= margin) return;
    if (e <= T(0)) {
        w = T(0);
        return;
    }
    const T s = e / margin;
    w = s * s * (T(3) - T(2) * s);
    dw = (u < T(0) ? T(6) : T(-6)) * s * (T(1) - s) / margin;
}

// The tapered wave sum at (x, y) with its derivatives dh/dx, dh/dy and d2h/dxdy; zero outside the
// rectangle (WaveSurface::analytic, geometry.cpp:223-242). waves: nW (amplitude, kx, ky, phase).
template <class T>
OWEC_HD void waveAnalytic(const double* waves, int nW, T hx, T hy, T margin, T x, T y, T& h, T& gx, T& gy, T& gxy) {
    h = gx = gy = gxy = T(0);
    if (fabs(x) > hx || fabs(y) > hy) return;
    T g = T(0), sx = T(0), sy = T(0), sxy = T(0);
    for (int i = 0; i < nW; ++i) {
        const T a = T(waves[4 * i]), kx = T(waves[4 * i + 1]), ky = T(waves[4 * i + 2]);
        const T arg = kx * x + ky * y + T(waves[4 * i + 3]);
        const T s = sin(arg), c = cos(arg);
        g += a * s;
        sx += a * c * kx;
        sy += a * c * ky;
        sxy -= a * s * kx * ky;
    }
    T wx, dwx, wy, dwy;
    waveTaper(x, hx, margin, wx, dwx);
    waveTaper(y, hy, margin, wy, dwy);
    h = wx * wy * g;
    gx = dwx * wy * g + wx * wy * sx;
    gy = wx * dwy * g + wx * wy * sy;
    gxy = dwx * dwy * g + dwx * wy * sy + wx * dwy * sx + wx * wy * sxy;
}

// The cubic Hermite bases on [0, 1] at u: value bases p0, p1 and slope bases q0, q1 of the two ends,
// and their derivatives.
template <class T>
OWEC_HD void hermiteBasis(T u, T p[2], T q[2], T dp[2], T dq[2]) {
    const T u2 = u * u, u3 = u2 * u;
    p[0] = T(2) * u3 - T(3) * u2 + T(1);
    p[1] = T(3) * u2 - T(2) * u3;
    q[0] = u3 - T(2) * u2 + u;
    q[1] = u3 - u2;
    dp[0] = T(6) * u2 - T(6) * u;
    dp[1] = T(6) * u - T(6) * u2;
    dq[0] = T(3) * u2 - T(4) * u + T(1);
    dq[1] = T(3) * u2 - T(2) * u;
}

// The wave surface's height and gradient at local (x, y), zero outside its rectangle
// (WaveSurface::height, geometry.cpp:244-270).
template <class T>
OWEC_HD void waveHeight(const DBoundary& b, const double* data, T x, T y, T& h, T& gx, T& gy) {
    const T hx = T(b.params[0]), hy = T(b.params[1]);
    const int nW = int(b.params[3]);
    if (b.ext[2] == 0) {
        T gxy;
        waveAnalytic(data + 2, nW, hx, hy, T(b.params[2]), x, y, h, gx, gy, gxy);
        return;
    }
    h = gx = gy = T(0);
    if (fabs(x) > hx || fabs(y) > hy) return;
    const int nx = int(data[0]), ny = int(data[1]);
    const double* nodes = data + 2 + 4 * nW;
    const T dx = T(b.ext[2]), dy = T(b.ext[3]);
    const T fx = (x + hx) / dx, fy = (y + hy) / dy;
    const int i = min(max(int(fx), 0), nx - 2), j = min(max(int(fy), 0), ny - 2);
    T P[2], Q[2], dP[2], dQ[2], Pv[2], Qv[2], dPv[2], dQv[2];
    hermiteBasis(fx - T(i), P, Q, dP, dQ);
    hermiteBasis(fy - T(j), Pv, Qv, dPv, dQv);
    T f = T(0), fu = T(0), fv = T(0);
    for (int bj = 0; bj < 2; ++bj)
        for (int ai = 0; ai < 2; ++ai) {
            const double* n = nodes + 4 * (size_t(j + bj) * nx + (i + ai));
            const T c0 = T(n[0]), cu = T(n[1]) * dx, cv = T(n[2]) * dy, cuv = T(n[3]) * dx * dy;
            f += c0 * P[ai] * Pv[bj] + cu * Q[ai] * Pv[bj] + cv * P[ai] * Qv[bj] + cuv * Q[ai] * Qv[bj];
            fu += c0 * dP[ai] * Pv[bj] + cu * dQ[ai] * Pv[bj] + cv * dP[ai] * Qv[bj] + cuv * dQ[ai] * Qv[bj];
            fv += c0 * P[ai] * dPv[bj] + cu * Q[ai] * dPv[bj] + cv * P[ai] * dQv[bj] + cuv * Q[ai] * dQv[bj];
        }
    h = f;
    gx = fu / dx;
    gy = fv / dy;
}

template <class T>
OWEC_HD V3<T> waveNormal(const DBoundary& b, const double* data, const V3<T>& p) {
    T h, gx, gy;
    waveHeight(b, data, p.x, p.y, h, gx, gy);
    return normalize(V3<T>(-gx, -gy, T(1)));
}

// WaveSurface::intersect (geometry.cpp:278-344): the ray clipped to the surface's box is marched in
// steps |f| / L, f = z - h along the ray and L its Lipschitz bound along the ray, so that no crossing
// is stepped over; near the surface Newton's method converges on the crossing being approached; a
// sign change within a minimum step is bisected. A crossing within depWindow (plus its own error)
// along the normal of a ray leaving this surface is the departure and skipped. The first accepted
// crossing is returned, and a second only when the first lies within nearWindow of the origin along
// its normal, where the caller's region rule may still reject it.
template <class Rr>
__device__ __noinline__ NumericRoots<Rr> waveRoots(const DBoundary& b, const double* data, V3<Rr> o, V3<Rr> d, Rr tmin,
                                                   Rr tmax, Rr depWindow, Rr nearWindow) {
    NumericRoots<Rr> r{{Rr(0), Rr(0)}, 0};
    const Rr hx = Rr(b.params[0]), hy = Rr(b.params[1]), amp = Rr(b.ext[0]), slope = Rr(b.ext[1]);
    Rr ta = tmin, tb = tmax;
    if (!clipSlab(o.x, d.x, -hx, hx, ta, tb) || !clipSlab(o.y, d.y, -hy, hy, ta, tb) || !clipSlab(o.z, d.z, -amp, amp, ta, tb))
        return r;
    const Rr L = fabs(d.z) + slope * sqrt(d.x * d.x + d.y * d.y);
    const Rr tol = Rr(sizeof(Rr) == 8 ? 1e-12 : 1e-6) * (Rr(1) + fmax(fmax(hx, hy), amp));
    auto f = [&](Rr t, Rr& dfdt) {
        const V3<Rr> p = o + d * t;
        Rr h, gx, gy;
        waveHeight(b, data, p.x, p.y, h, gx, gy);
        dfdt = d.z - gx * d.x - gy * d.y;
        return p.z - h;
    };
    auto value = [&](Rr t) {
        Rr dfdt;
        return f(t, dfdt);
    };
    Rr t = ta, dfdt;
    Rr ft = f(t, dfdt);
    if (t <= tmin && fabs(ft) < tol) {  // starting on the surface it leaves
        t = tmin + tol / fmax(L, Rr(1e-30));
        ft = f(t, dfdt);
    }
    const Rr minStep = Rr(1e-7) * (tb - ta), nearSurface = Rr(1e-6) * (amp + tol);
    // Records crossing tr; true when the search is over.
    auto record = [&](Rr tr) {
        const V3<Rr> p = o + d * tr;
        if (!(tr > tmin && tr < tmax) || fabs(p.x) > hx || fabs(p.y) > hy) return false;
        Rr h, gx, gy;
        waveHeight(b, data, p.x, p.y, h, gx, gy);
        const Rr gl = sqrt(Rr(1) + gx * gx + gy * gy);
        const Rr along = fabs(tr * (d.z - gx * d.x - gy * d.y)) / gl;  // |t d.n|
        if (depWindow > Rr(0) && along <= depWindow + fabs(p.z - h) / gl) return false;
        if (r.n == 1 && fabs(tr - r.t[0]) <= Rr(1e3) * tol) return false;  // the same crossing again
        r.t[r.n++] = tr;
        return r.n == 2 || along > nearWindow;
    };
    for (int i = 0; i < 4096 && t < tb; ++i) {
        Rr step = fmax(fabs(ft) / L, minStep);
        if (fabs(ft) < nearSurface) {
            Rr tn = t;
            for (int k = 0; k < 8; ++k) {
                const Rr fn = f(tn, dfdt);
                const V3<Rr> p = o + d * tn;
                const Rr arithmeticTol = Rr(8) * Rr(Tol<Rr>::eps) *
                                         fmax(fmax(Rr(1e-12), amp), fmax(fmax(fabs(p.x), fabs(p.y)), fabs(p.z)));
                if (fabs(fn) < arithmeticTol || fabs(dfdt) < Rr(1e-12)) break;
                tn -= fn / dfdt;
            }
            if (tn >= t - Rr(1e3) * tol && fabs(value(tn)) < Rr(1e3) * tol && record(tn)) return r;
            step = fmax(minStep, Rr(2) * fabs(ft) / L);  // a grazing approach: move past it
        }
        const Rr tn = fmin(t + step, tb);
        const Rr fn = f(tn, dfdt);
        if ((fn < Rr(0)) != (ft < Rr(0)) && record(bisectRoot(value, t, tn, ft, Tol<Rr>::bisectSteps))) return r;
        t = tn;
        ft = fn;
    }
    return r;
}

// The quadric crossings of a shape: roots t0 <= t1 in precision R, each refined in precision Rr and
// kept when it lies in (tmin, tmax) and solid(p) accepts it (firstRefinedHit, geometry.cpp:32-48,
// for both roots).
template <class R, class Rr, bool SkipDouble = false, class Solid, class Normal>
OWEC_HD void quadricHits(int kind, Rr qa, Rr qb, Rr qc, const V3<Rr>& o, const V3<Rr>& d, R t0, R t1, Rr tmin, Rr tmax,
                         const Solid& solid, const Normal& normal, AHits<Rr>& out) {
    const R ts[2] = {t0, t1};
    for (int i = 0; i < 2; ++i) {
        if (SkipDouble && i == 1 && t1 == t0) break;  // a sag's double root counts once
        Rr tr;
        if (!refinedRootIn<R, Rr>(kind, qa, qb, o, d, Rr(ts[i]), tmin, tmax, tr, qc)) continue;
        const V3<Rr> p = o + d * tr;
        if (!solid(p)) continue;
        out.add({tr, p, normal(p)});
    }
}

// The crossings of every shape (analyticCrossings with Full).
template <class R, class Rr>
OWEC_HD int fullCrossings(const DBoundary& b, const double* data, const V3<Rr>& o, const V3<Rr>& d, Rr tmin, Rr tmax,
                          bool departed, AHits<Rr>& out, Rr depWindow, Rr nearWindow) {
    out.n = 0;
    const double* P = b.params;
    switch (b.shape) {
        case OWEC_SHAPE_SPHERE: {  // roots in the refinement's precision, as classicCrossings
            const Rr Rad = Rr(P[0]);
            Rr t0, t1;
            if (!sphereRoots(o, d, Rad, t0, t1)) return 0;
            quadricHits<Rr, Rr>(kQuadSphere, Rad * Rad, Rr(0), Rr(0), o, d, t0, t1, tmin, tmax,
                                [](const V3<Rr>&) { return true; }, [&](const V3<Rr>& p) { return normalize(p / Rad); },
                                out);
            break;
        }
        case OWEC_SHAPE_DOME: {
            const Rr Rad = Rr(P[0]), az = Rr(P[1]), w = Rr(P[2]), top = Rr(P[3]);
            Rr t0, t1;
            if (!sphereRoots(o, d, Rad, t0, t1)) return 0;
            quadricHits<Rr, Rr>(kQuadSphere, Rad * Rad, Rr(0), Rr(0), o, d, t0, t1, tmin, tmax,
                               [&](const V3<Rr>& p) { return domeSolid(Rad, az, w, top, p); },
                               [](const V3<Rr>& p) { return normalize(p); }, out);
            break;
        }
        case OWEC_SHAPE_SAG: {
            const Rr c = Rr(P[0]), k = Rr(P[1]), rMax = Rr(P[2]), rMin = Rr(P[3]);
            const int nA = int(b.dataCount);
            auto accept = [&](const V3<Rr>& p) {
                const Rr r2 = p.x * p.x + p.y * p.y;
                return r2 <= rMax * rMax && r2 >= rMin * rMin;
            };
            auto normal = [&](const V3<Rr>& p) {
                const Rr r = sqrt(p.x * p.x + p.y * p.y);
                return sagNormal(p, r, nA ? asphereSlope(c, k, data, nA, r) : conicSlope(c, k, r));
            };
            if (nA > 0) {
                const NumericRoots<Rr> r = asphereRoots<Rr>(c, k, rMax, rMin, Rr(b.ext[0]), Rr(b.ext[1]), data, nA, o, d, tmin, tmax);
                for (int i = 0; i < r.n; ++i) {
                    const V3<Rr> p = o + d * r.t[i];
                    out.add({r.t[i], p, normal(p)});
                }
                break;
            }
            auto solid = [&](const V3<Rr>& p) {
                return accept(p) && (c == Rr(0) || (Rr(1) + k) * c * p.z <= Rr(1) + Rr(Tol<R>::relTol));
            };
            if (c == Rr(0)) {
                if (d.z == Rr(0)) return 0;
                const Rr t = -o.z / d.z;
                if (t <= tmin || t >= tmax) return 0;
                const V3<Rr> p = o + d * t;
                if (!solid(p)) return 0;
                out.add({t, p, normal(p)});
                break;
            }
            R A, B, C, t0, t1;
            quadricCoeffs(kQuadSag, R(c), R(c * (Rr(1) + k)), R(0), V3<R>(o), V3<R>(d), A, B, C);
            if (solveQuadratic(A, B, C, t0, t1) <= 0) return 0;
            quadricHits<R, Rr, true>(kQuadSag, c, c * (Rr(1) + k), Rr(0), o, d, t0, t1, tmin, tmax, solid, normal, out);
            break;
        }
        case OWEC_SHAPE_PLANE: {
            if (d.z == Rr(0)) return 0;
            const Rr t = -o.z / d.z;
            if (t <= tmin || t >= tmax) return 0;
            V3<Rr> p = o + d * t;
            p.z = Rr(0);
            const int ap = int(P[0]);
            const bool hole = ap == OWEC_APERTURE_DISK_HOLE && b.dataCount >= 2;
            if (!inPlaneAperture(ap, Rr(P[1]), Rr(P[2]), hole ? Rr(data[0]) : Rr(0), hole ? Rr(data[1]) : Rr(0), p))
                return 0;
            out.add({t, p, V3<Rr>(0, 0, 1)});
            break;
        }
        case OWEC_SHAPE_CYLINDER:
        case OWEC_SHAPE_ROUND_WALL: {
            const bool wall = b.shape == OWEC_SHAPE_ROUND_WALL;
            const Rr Rad = Rr(P[0]), z0 = wall ? Rr(0) : Rr(P[1]), z1 = wall ? Rr(P[1]) : Rr(P[2]);
            const int openings = wall ? int(b.dataCount / 4) : 0;
            R t0, t1;
            if (!cylinderRoots(V3<R>(o), V3<R>(d), R(P[0]), t0, t1)) return 0;
            auto solid = [&](const V3<Rr>& p) {
                if (p.z < z0 || p.z > z1) return false;
                for (int i = 0; i < openings; ++i)
                    if (inWallOpening(Rad, Rr(data[4 * i]), Rr(data[4 * i + 1]), Rr(data[4 * i + 2]), Rr(data[4 * i + 3]), p))
                        return false;
                return true;
            };
            quadricHits<R, Rr>(kQuadCylinder, Rad * Rad, Rr(0), Rr(0), o, d, t0, t1, tmin, tmax, solid,
                               [](const V3<Rr>& p) { return normalize(V3<Rr>(p.x, p.y, Rr(0))); }, out);
            break;
        }
        case OWEC_SHAPE_CONE: {
            // x^2 + y^2 = (r0 + k (z - z0))^2 on the nappe where r0 + k (z - z0) >= 0 (ConeShape,
            // geometry.cpp:519-538), z0 < z1 after ordering the ends
            const bool swap = P[1] > P[3];
            const Rr r0 = Rr(swap ? P[2] : P[0]), z0 = Rr(swap ? P[3] : P[1]);
            const Rr r1 = Rr(swap ? P[0] : P[2]), z1 = Rr(swap ? P[1] : P[3]);
            const Rr k = (r1 - r0) / (z1 - z0);
            R A, B, C, t0, t1;
            quadricCoeffs(kQuadCone, R(r0), R(z0), R(k), V3<R>(o), V3<R>(d), A, B, C);
            if (solveQuadratic(A, B, C, t0, t1) <= 0) return 0;
            quadricHits<R, Rr>(kQuadCone, r0, z0, k, o, d, t0, t1, tmin, tmax,
                               [&](const V3<Rr>& p) { return p.z >= z0 && p.z <= z1 && r0 + k * (p.z - z0) >= Rr(0); },
                               [&](const V3<Rr>& p) { return normalize(V3<Rr>(p.x, p.y, -(r0 + k * (p.z - z0)) * k)); },
                               out);
            break;
        }
        case OWEC_SHAPE_TORUS: {
            const NumericRoots<Rr> r = torusRoots<Rr>(Rr(P[0]), Rr(P[1]), Rr(P[2]), Rr(P[3]), Rr(b.ext[3]), Rr(b.ext[0]),
                                                      Rr(b.ext[1]), Rr(b.ext[2]), o, d, tmin, tmax, departed);
            for (int i = 0; i < r.n; ++i) {
                const V3<Rr> p = o + d * r.t[i];
                out.add({r.t[i], p, torusNormal(Rr(P[0]), Rr(P[1]), p)});
            }
            break;
        }
        case OWEC_SHAPE_WAVES: {
            const NumericRoots<Rr> r = waveRoots<Rr>(b, data, o, d, tmin, tmax, departed ? depWindow : Rr(0), nearWindow);
            for (int i = 0; i < r.n; ++i) {
                const V3<Rr> p = o + d * r.t[i];
                out.add({r.t[i], p, waveNormal(b, data, p)});
            }
            break;
        }
        default: break;
    }
    if (out.n == 2 && out.h1.t < out.h0.t) { const AHit<Rr> tmp = out.h0; out.h0 = out.h1; out.h1 = tmp; }
    return out.n;
}

// Up to two crossings of boundary b's shape by the local ray (o, d) in (tmin, tmax), ascending,
// each inside the shape's trim. data: the shape's run of the scene's shape data. departed: the ray
// leaves this boundary (a torus patch then resolves the start of its bracket finely; a wave surface
// skips the crossings within depWindow of the origin along their normal). nearWindow: the origin's
// error along a surface normal (a wave surface looks for a second crossing only behind a first one
// within it). Returns how many. Full = false compiles only the spheres, conic sags, plain apertures
// and cylinders: the kernels of a scene without the other shapes keep the registers they need for
// those alone.
template <class R, class Rr, bool Full>
OWEC_HD int analyticCrossings(const DBoundary& b, const double* data, const V3<Rr>& o, const V3<Rr>& d, Rr tmin, Rr tmax,
                              bool departed, AHits<Rr>& out, Rr depWindow = Rr(0), Rr nearWindow = Rr(0)) {
    if constexpr (Full) return fullCrossings<R, Rr>(b, data, o, d, tmin, tmax, departed, out, depWindow, nearWindow);
    else return classicCrossings<R, Rr>(b, o, d, tmin, tmax, out);
}

// The unit normal of a shape found by a numeric crossing (aspheres, torus patches, wave surfaces) at
// local point p.
template <class Rr>
OWEC_HD V3<Rr> numericNormal(const DBoundary& b, const double* data, const V3<Rr>& p) {
    const double* P = b.params;
    if (b.shape == OWEC_SHAPE_TORUS) return torusNormal(Rr(P[0]), Rr(P[1]), p);
    if (b.shape == OWEC_SHAPE_WAVES) return waveNormal(b, data, p);
    const Rr r = sqrt(p.x * p.x + p.y * p.y);
    return sagNormal(p, r, asphereSlope(Rr(P[0]), Rr(P[1]), data, int(b.dataCount), r));
}
// Whether boundary b's crossings are found numerically (no closed form).
OWEC_HD bool numericShape(const DBoundary& b) {
    return b.shape == OWEC_SHAPE_TORUS || b.shape == OWEC_SHAPE_WAVES || (b.shape == OWEC_SHAPE_SAG && b.dataCount > 0);
}

// Watertight line-triangle crossing test (Woop, Benthin and Wald 2013), edges included, as the
// reference's lineCrossesTriangle (surfaces.hpp:272-290): in a frame sheared so the line runs
// along an axis, the side of each edge is a 2-D cross product of that edge's own vertices.
template <class T>
struct ShearedRay {
    V3<T> X, Y;  // a point's sheared coordinates are dot(X, p) and dot(Y, p)
};
template <class T>
OWEC_HD ShearedRay<T> shearRay(const V3<T>& d) {
    const T dx = fabs(d.x), dy = fabs(d.y), dz = fabs(d.z);
    const int kz = dx > dy ? (dx > dz ? 0 : 2) : (dy > dz ? 1 : 2);
    const int kx = kz == 2 ? 0 : kz + 1;
    const int ky = kx == 2 ? 0 : kx + 1;
    const T sx = d[kx] / d[kz], sy = d[ky] / d[kz];
    ShearedRay<T> s;
    s.X = V3<T>(kx == 0 ? T(1) : (kz == 0 ? -sx : T(0)), kx == 1 ? T(1) : (kz == 1 ? -sx : T(0)),
                kx == 2 ? T(1) : (kz == 2 ? -sx : T(0)));
    s.Y = V3<T>(ky == 0 ? T(1) : (kz == 0 ? -sy : T(0)), ky == 1 ? T(1) : (kz == 1 ? -sy : T(0)),
                ky == 2 ? T(1) : (kz == 2 ? -sy : T(0)));
    return s;
}
template <class T>
OWEC_HD T shearDot(const V3<T>& k, const V3<T>& p) {
    return fma(k.z, p.z, fma(k.y, p.y, k.x * p.x));
}
template <class T>
OWEC_HD bool lineCrossesTriangle(const ShearedRay<T>& s, const V3<T>& a, const V3<T>& b, const V3<T>& c) {
    const T ax = shearDot(s.X, a), ay = shearDot(s.Y, a);
    const T bx = shearDot(s.X, b), by = shearDot(s.Y, b);
    const T cx = shearDot(s.X, c), cy = shearDot(s.Y, c);
    const T u = cx * by - cy * bx, v = ax * cy - ay * cx, w = bx * ay - by * ax;
    if ((u < T(0) || v < T(0) || w < T(0)) && (u > T(0) || v > T(0) || w > T(0))) return false;
    return u + v + w != T(0);
}
// A triangle's normal from its two shorter edges (surfaces.hpp:265-270).
template <class T>
OWEC_HD V3<T> triangleNormal(const V3<T>& v0, const V3<T>& v1, const V3<T>& v2) {
    const V3<T> a = v1 - v0, b = v2 - v0, c = v2 - v1;
    const T la = dot(a, a), lb = dot(b, b), lc = dot(c, c);
    if (lc >= la && lc >= lb) return cross(a, b);
    return la >= lb ? cross(b, c) : cross(a, c);
}

}  // namespace owec
