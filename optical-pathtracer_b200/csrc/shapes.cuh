// Analytic surfaces in their own frames: spheres, conic sags, planes with apertures and cylinders.
// Roots come from the numerically stable quadratic in precision R and are refined by re-solving
// from the approximate hit in precision Rr (src/owe/core/shared/surfaces.hpp:13-137): with
// R = float and Rr = double this is the selective FP64 step that keeps large-radius lens surfaces
// exact; with R = Rr = float it is the plain FP32 baseline.
#pragma once

#include "device_scene.cuh"

namespace owec {

template <class T> struct Tol;
template <> struct Tol<float> {
    static constexpr float refine = 1e-3f, relTol = 1e-6f, tiny = 1e-30f;
};
template <> struct Tol<double> {
    static constexpr double refine = 1e-6, relTol = 1e-9, tiny = 1e-300;
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

constexpr int kQuadSag = 0, kQuadSphere = 1, kQuadCylinder = 2;

template <class T>
OWEC_HD void quadricCoeffs(int kind, T qa, T qb, const V3<T>& o, const V3<T>& d, T& A, T& B, T& C) {
    if (kind == kQuadSag) {
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
OWEC_HD bool refinedRootIn(int kind, Rr qa, Rr qb, const V3<Rr>& o, const V3<Rr>& d, Rr t, Rr tmin, Rr tmax, Rr& tr) {
    tr = t;
    const Rr m = Rr(Tol<R>::refine) * (Rr(1) + fabs(t));
    if (t + m <= tmin || t - m >= tmax) return false;
    Rr A, B, C, u0, u1;
    quadricCoeffs(kind, qa, qb, o + d * t, d, A, B, C);
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

// Up to two crossings of boundary b's shape by the local ray (o, d) in (tmin, tmax), ascending,
// each inside the shape's trim. Returns how many.
template <class R, class Rr>
OWEC_HD int analyticCrossings(const DBoundary& b, const V3<Rr>& o, const V3<Rr>& d, Rr tmin, Rr tmax, AHits<Rr>& out) {
    out.n = 0;
    const double* P = b.params;
    switch (b.shape) {
        case OWEC_SHAPE_SPHERE: {
            const Rr Rad = Rr(P[0]);
            R t0, t1;
            if (!sphereRoots(V3<R>(o), V3<R>(d), R(P[0]), t0, t1)) return 0;
            const R ts[2] = {t0, t1};
            for (int i = 0; i < 2; ++i) {
                Rr tr;
                if (!refinedRootIn<R, Rr>(kQuadSphere, Rad * Rad, Rr(0), o, d, Rr(ts[i]), tmin, tmax, tr)) continue;
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
            quadricCoeffs(kQuadSag, R(c), R(c * (Rr(1) + k)), V3<R>(o), V3<R>(d), A, B, C);
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
