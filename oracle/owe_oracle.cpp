// CPU restatement of the reference engine's camera-path transport (IEEE double), over the same
// scene description the CUDA backend takes (include/owec.h).
//
// TEST INFRASTRUCTURE ONLY. This file is the oracle the tests check the CUDA backend against (and
// which they pin against the reference engine itself, oracle/_ref). Nothing in the product loads or
// calls it; bench.py runs it only as the timed CPU baseline when the reference could not be built.
//
// It restates, function by function (citations are to the reference's files):
//   PCG32 streams and uniforms        src/owe/core/sampling.hpp:11-51, core/shared/warps.hpp:12-30
//   spectra, index models, CIE fit    src/owe/core/spectrum.cpp:131-167, core/medium.cpp:45-60,
//                                     core/shared/spectra.hpp:10-61, core/wavelengths.hpp:32-84
//   shapes                            src/owe/scene/geometry.cpp:115-166, 391-480, 503-515,
//                                     src/owe/scene/mesh.cpp:50-97, core/shared/surfaces.hpp
//   World::intersect (contacts)       src/owe/scene/world.cpp:440-582
//   light table, light sampling       src/owe/scene/world.cpp:285-377, transport/transport.cpp:35-70
//   optics and scattering             src/owe/core/shared/optics.hpp, transport/scattering.cpp:65-222
//   Tracer::radiance and helpers      src/owe/transport/transport.cpp:72-529
//   detectors, the pass loop          src/owe/scene/detector.cpp:61-148, backends/cpu/cpu_backend.cpp:52-94
//
//   Tracer::walk                      src/owe/transport/transport.cpp:531-595
//
// Shapes the scene description does not carry (waves, lathe patches, domes, walls, aspheres) and
// environment maps, textures and aim guides are not restated; the double-double near-sphere solve
// of world.cpp:384-438 (planet-sized spheres) is not either.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "owec.h"

namespace oracle {

constexpr double Pi = 3.14159265358979323846, InvPi = 1.0 / Pi;
constexpr double Inf = std::numeric_limits<double>::infinity();
constexpr uint32_t kNone = 0xFFFFFFFEu;
constexpr int NW = 4;
constexpr double kRefine = 1e-6, kRelTol = 1e-9, kTiny = 1e-300, kGrazing = 1e-12;

// ------------------------------------------------------------------ vectors
struct V {
    double x = 0, y = 0, z = 0;
    V() = default;
    V(double a, double b, double c) : x(a), y(b), z(c) {}
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V operator+(V a, V b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V operator-(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V operator-(V a) { return {-a.x, -a.y, -a.z}; }
inline V operator*(V a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V operator/(V a, double s) { return a * (1.0 / s); }
inline double dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V cross(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(V a) { return std::sqrt(dot(a, a)); }
inline V unit(V a) { return a / len(a); }
inline double maxAbs(V a) { return std::max({std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}); }
inline V reflectV(V d, V n) { return d - n * (2.0 * dot(d, n)); }
inline double sq(double x) { return x * x; }
inline double clampd(double x, double lo, double hi) { return std::min(hi, std::max(lo, x)); }
inline double safeSqrt(double x) { return std::sqrt(std::max(0.0, x)); }
inline double contactError(double scale) { return 64 * std::numeric_limits<double>::epsilon() * std::max(1e-12, scale); }

void basis(V n, V& b1, V& b2) {
    const double sgn = std::copysign(1.0, n.z), a = -1 / (sgn + n.z), b = n.x * n.y * a;
    b1 = {1 + sgn * n.x * n.x * a, sgn * b, -sgn * n.x};
    b2 = {b, sgn + n.y * n.y * a, -n.y};
}
struct Frame {
    V s, t, n;
    explicit Frame(V nn) : n(nn) { basis(n, s, t); }
    V toLocal(V v) const { return {dot(v, s), dot(v, t), dot(v, n)}; }
    V toWorld(V v) const { return s * v.x + t * v.y + n * v.z; }
};
struct Xf {
    double m[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    V point(V p) const {
        return {m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
                m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]};
    }
    V vec(V v) const {
        return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z,
                m[8] * v.x + m[9] * v.y + m[10] * v.z};
    }
    V translation() const { return {m[3], m[7], m[11]}; }
    Xf inverse() const {
        Xf r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) r.m[4 * i + j] = m[4 * j + i];
        for (int i = 0; i < 3; ++i) r.m[4 * i + 3] = -(r.m[4 * i] * m[3] + r.m[4 * i + 1] * m[7] + r.m[4 * i + 2] * m[11]);
        return r;
    }
};

// ------------------------------------------------------------------ random numbers
uint64_t mixBits(uint64_t v) {
    v ^= v >> 31;
    v *= 0x7fb5d329728ea185ULL;
    v ^= v >> 27;
    v *= 0x81dadef4bc2dd44dULL;
    v ^= v >> 33;
    return v;
}
uint64_t hashCombine(uint64_t a, uint64_t b) { return mixBits(a ^ (mixBits(b) + 0x9e3779b97f4a7c15ULL)); }
struct Rng {
    uint64_t s = 0, inc = 1;
    Rng(uint64_t seed, uint64_t stream) {
        s = 0;
        inc = (stream << 1u) | 1u;
        next();
        s += seed;
        next();
    }
    uint32_t next() {
        const uint64_t old = s;
        s = old * 6364136223846793005ULL + inc;
        const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u), rot = uint32_t(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31u));
    }
    double uniform() {
        const uint64_t a = next() >> 5, b = next() >> 6;
        return (double(a) * 67108864.0 + double(b)) * (1.0 / 9007199254740992.0);
    }
};
// two and three uniforms, the last drawn first
struct D2 { double u1, u2; explicit D2(Rng& r) { u2 = r.uniform(); u1 = r.uniform(); } };
struct D3 { double u1, u2, u3; explicit D3(Rng& r) { u3 = r.uniform(); u2 = r.uniform(); u1 = r.uniform(); } };

// ------------------------------------------------------------------ spectra
constexpr double LMin = 360, LMax = 830;
double lobe(double x, double mu, double s1, double s2) {
    const double t = (x - mu) / (x < mu ? s1 : s2);
    return std::exp(-0.5 * t * t);
}
double cieX(double l) { return 1.056 * lobe(l, 599.8, 37.9, 31.0) + 0.362 * lobe(l, 442.0, 16.0, 26.7) - 0.065 * lobe(l, 501.1, 20.4, 26.2); }
double cieY(double l) { return 0.821 * lobe(l, 568.8, 46.9, 40.5) + 0.286 * lobe(l, 530.9, 16.3, 31.1); }
double cieZ(double l) { return 1.217 * lobe(l, 437.0, 11.8, 36.0) + 0.681 * lobe(l, 459.0, 26.0, 13.8); }
template <class F>
double simpsonVisible(F f) {
    const int n = int((LMax - LMin) * 2);
    const double h = (LMax - LMin) / n;
    double s = f(LMin) + f(LMax);
    for (int i = 1; i < n; ++i) s += f(LMin + i * h) * ((i & 1) ? 4 : 2);
    return s * h / 3;
}
double cieYIntegral() {
    static const double v = simpsonVisible(cieY);
    return v;
}
double planck(double lnm, double T) {
    const double c1 = 1.191042972e8, c2 = 1.438776877e4, l = lnm * 1e-3, l2 = l * l;
    return 1e6 * c1 / (l2 * l2 * l * (std::exp(c2 / (l * T)) - 1));
}

struct Scene;

struct Spec {
    int kind = OWEC_SPEC_CONSTANT;
    double a = 0, scale = 1;
    std::vector<double> l, v;
    double eval(double lam) const {
        if (kind == OWEC_SPEC_CONSTANT) return a;
        if (kind == OWEC_SPEC_BLACKBODY) return scale * planck(lam, a);
        if (lam <= l.front()) return scale * v.front();
        if (lam >= l.back()) return scale * v.back();
        const size_t i = size_t(std::upper_bound(l.begin(), l.end(), lam) - l.begin());
        const double t = (lam - l[i - 1]) / (l[i] - l[i - 1]);
        return scale * (v[i - 1] * (1 - t) + v[i] * t);
    }
    bool isZero() const { return kind == OWEC_SPEC_CONSTANT && a == 0; }
    double luminance() const { return simpsonVisible([&](double x) { return eval(x) * cieY(x); }) / cieYIntegral(); }
};

double ciddor(double l2) {
    const double s2 = 1 / l2;
    return 1 + 0.05792105 / (238.0185 - s2) + 0.00167917 / (57.362 - s2);
}

struct Medium {
    owec_medium d{};
    Spec table;  // tabulated index
    Spec absorption, scattering;
    bool absorbs() const { return !absorption.isZero(); }
    bool scatters() const { return !scattering.isZero(); }
    double n(double lam) const {
        const double l = lam * 1e-3, l2 = l * l;
        double v;
        switch (d.index_kind) {
            case OWEC_INDEX_CONSTANT: v = d.coef_a[0]; break;
            case OWEC_INDEX_CAUCHY: v = d.coef_a[0] + d.coef_a[1] / l2 + d.coef_a[2] / (l2 * l2); break;
            case OWEC_INDEX_SELLMEIER: {
                double s = 1;
                for (int i = 0; i < d.n_terms; ++i) s += d.coef_a[i] * l2 / (l2 - d.coef_b[i]);
                v = std::sqrt(s);
                break;
            }
            case OWEC_INDEX_CIDDOR: v = ciddor(l2); break;
            default: v = table.eval(lam); break;
        }
        return d.rel_air ? v * ciddor(l2) : v;
    }
};

// ------------------------------------------------------------------ rays, boxes
struct Ray {
    V o, d;
    uint32_t depB = kNone, hint = kNone;
    V depN;
    uint32_t depP = kNone;
    double depErr = 0;
    bool forwardOnly = false;
    V at(double t) const { return o + d * t; }
};
struct Box {
    V lo{Inf, Inf, Inf}, hi{-Inf, -Inf, -Inf};
    void expand(V p) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    void expand(const Box& b) { expand(b.lo); expand(b.hi); }
    bool valid() const { return lo.x <= hi.x && lo.y <= hi.y && lo.z <= hi.z; }
    V extent() const { return hi - lo; }
    V corner(int i) const { return {(i & 1) ? hi.x : lo.x, (i & 2) ? hi.y : lo.y, (i & 4) ? hi.z : lo.z}; }
};
// RaySlabs (src/owe/core/math.hpp:187-205)
struct Slabs {
    double o[3], inv[3];
    bool neg[3];
    explicit Slabs(const Ray& r) {
        for (int a = 0; a < 3; ++a) { o[a] = r.o[a]; inv[a] = 1.0 / r.d[a]; neg[a] = inv[a] < 0; }
    }
    bool hit(const Box& b, double tmin, double tmax, double& tEnter) const {
        for (int a = 0; a < 3; ++a) {
            const double t0 = ((neg[a] ? b.hi[a] : b.lo[a]) - o[a]) * inv[a];
            const double t1 = ((neg[a] ? b.lo[a] : b.hi[a]) - o[a]) * inv[a] * (1.0 + 4e-16);
            tmin = t0 > tmin ? t0 : tmin;
            tmax = t1 < tmax ? t1 : tmax;
            if (tmin > tmax) return false;
        }
        tEnter = tmin;
        return true;
    }
};

// ------------------------------------------------------------------ quadrics
int solveQuadratic(double a, double b, double c, double& t0, double& t1) {
    t0 = t1 = 0;
    if (std::fabs(a) < kTiny || std::fabs(a) < 1e-14 * std::fabs(b)) {
        if (b == 0) return 0;
        t0 = t1 = -c / b;
        return 1;
    }
    const double disc = b * b - 4 * a * c;
    if (disc < 0) return 0;
    const double q = -(b + std::copysign(std::sqrt(disc), b)) / 2;
    t0 = q / a;
    t1 = q != 0 ? c / q : t0;
    if (t0 > t1) std::swap(t0, t1);
    return 2;
}
enum QKind { QSag, QSphere, QCyl };
void qcoeffs(QKind k, double qa, double qb, V o, V d, double& A, double& B, double& C) {
    if (k == QSag) {
        A = qa * (d.x * d.x + d.y * d.y) + qb * d.z * d.z;
        B = 2 * (qa * (o.x * d.x + o.y * d.y) + qb * o.z * d.z - d.z);
        C = qa * (o.x * o.x + o.y * o.y) + qb * o.z * o.z - 2 * o.z;
    } else if (k == QSphere) {
        A = dot(d, d);
        B = 2 * dot(o, d);
        C = dot(o, o) - qa;
    } else {
        A = d.x * d.x + d.y * d.y;
        B = 2 * (o.x * d.x + o.y * d.y);
        C = o.x * o.x + o.y * o.y - qa;
    }
}
bool refinedRootIn(QKind k, double qa, double qb, V o, V d, double t, double tmin, double tmax, double& tr) {
    tr = t;
    const double m = kRefine * (1 + std::fabs(t));
    if (t + m <= tmin || t - m >= tmax) return false;
    double A, B, C, u0, u1;
    qcoeffs(k, qa, qb, o + d * t, d, A, B, C);
    if (solveQuadratic(A, B, C, u0, u1) != 0) {
        const double du = std::fabs(u0) < std::fabs(u1) ? u0 : u1;
        if (std::fabs(du) < m) tr = t + du;
    }
    return tr > tmin && tr < tmax;
}

struct LocalHit {
    double t = Inf;
    V p, n;
    uint32_t prim = 0;
    double error = 0;
};

// ------------------------------------------------------------------ meshes (own binary BVH)
struct Mesh {
    std::vector<V> pos;
    std::vector<std::array<uint32_t, 3>> tri;
    std::vector<double> cdf;
    double area = 0;
    struct Node { Box box; uint32_t start, count, right; };
    std::vector<Node> nodes;
    std::vector<uint32_t> order;
    Box bounds;

    static V triNormal(V v0, V v1, V v2) {
        const V a = v1 - v0, b = v2 - v0, c = v2 - v1;
        const double la = dot(a, a), lb = dot(b, b), lc = dot(c, c);
        if (lc >= la && lc >= lb) return cross(a, b);
        return la >= lb ? cross(b, c) : cross(a, c);
    }
    void build() {
        std::vector<Box> boxes(tri.size());
        std::vector<V> cent(tri.size());
        cdf.resize(tri.size());
        double acc = 0;
        for (size_t i = 0; i < tri.size(); ++i) {
            const V &a = pos[tri[i][0]], &b = pos[tri[i][1]], &c = pos[tri[i][2]];
            boxes[i].expand(a);
            boxes[i].expand(b);
            boxes[i].expand(c);
            const double pad = 1e-12 * (1 + maxAbs(boxes[i].hi) + maxAbs(boxes[i].lo));
            boxes[i].lo = boxes[i].lo - V(pad, pad, pad);
            boxes[i].hi = boxes[i].hi + V(pad, pad, pad);
            cent[i] = (boxes[i].lo + boxes[i].hi) * 0.5;
            acc += 0.5 * len(cross(b - a, c - a));
            cdf[i] = acc;
            bounds.expand(boxes[i]);
        }
        area = acc;
        order.resize(tri.size());
        for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
        nodes.clear();
        nodes.reserve(2 * tri.size() + 1);
        // median split on the longest axis of the centroids, leaves of up to 4
        struct Item { uint32_t node, b, e; };
        std::vector<Item> stack{{0, 0, uint32_t(tri.size())}};
        nodes.push_back({});
        while (!stack.empty()) {
            Item it = stack.back();
            stack.pop_back();
            Box bx, cb;
            for (uint32_t k = it.b; k < it.e; ++k) { bx.expand(boxes[order[k]]); cb.expand(cent[order[k]]); }
            nodes[it.node].box = bx;
            if (it.e - it.b <= 4) {
                nodes[it.node].start = it.b;
                nodes[it.node].count = it.e - it.b;
                continue;
            }
            const V ext = cb.extent();
            const int ax = ext.x > ext.y ? (ext.x > ext.z ? 0 : 2) : (ext.y > ext.z ? 1 : 2);
            const uint32_t mid = (it.b + it.e) / 2;
            std::nth_element(order.begin() + it.b, order.begin() + mid, order.begin() + it.e,
                             [&](uint32_t p, uint32_t q) { return cent[p][ax] < cent[q][ax]; });
            const uint32_t l = uint32_t(nodes.size());
            nodes.push_back({});
            const uint32_t r = uint32_t(nodes.size());
            nodes.push_back({});
            nodes[it.node].count = 0;
            nodes[it.node].start = l;
            nodes[it.node].right = r;
            stack.push_back({r, mid, it.e});
            stack.push_back({l, it.b, mid});
        }
    }
    // Woop-Benthin-Wald watertight crossing (surfaces.hpp:272-290)
    static bool crosses(V o, V d, V v0, V v1, V v2) {
        const double dx = std::fabs(d.x), dy = std::fabs(d.y), dz = std::fabs(d.z);
        const int kz = dx > dy ? (dx > dz ? 0 : 2) : (dy > dz ? 1 : 2);
        const int kx = kz == 2 ? 0 : kz + 1, ky = kx == 2 ? 0 : kx + 1;
        const double sx = d[kx] / d[kz], sy = d[ky] / d[kz];
        const V a = v0 - o, b = v1 - o, c = v2 - o;
        const double ax = a[kx] - sx * a[kz], ay = a[ky] - sy * a[kz];
        const double bx = b[kx] - sx * b[kz], by = b[ky] - sy * b[kz];
        const double cx = c[kx] - sx * c[kz], cy = c[ky] - sy * c[kz];
        const double u = cx * by - cy * bx, v = ax * cy - ay * cx, w = bx * ay - by * ax;
        if ((u < 0 || v < 0 || w < 0) && (u > 0 || v > 0 || w > 0)) return false;
        return u + v + w != 0;
    }
    // MeshShape::sameFace (mesh.cpp:50-71)
    bool sameFace(uint32_t first, uint32_t second) const {
        if (first >= tri.size() || second >= tri.size()) return false;
        if (first == second) return true;
        const auto &a = tri[first], &b = tri[second];
        auto shared = [&](uint32_t v) {
            for (uint32_t u : a)
                if (pos[v].x == pos[u].x && pos[v].y == pos[u].y && pos[v].z == pos[u].z) return true;
            return false;
        };
        int n = 0;
        for (uint32_t v : b) n += shared(v);
        if (n < 2) return false;
        const V na = cross(pos[a[1]] - pos[a[0]], pos[a[2]] - pos[a[0]]);
        if (dot(na, cross(pos[b[1]] - pos[b[0]], pos[b[2]] - pos[b[0]])) <= 0) return false;
        for (uint32_t v : b)
            if (!shared(v) && dot(na, pos[v] - pos[a[0]]) != 0) return false;
        return true;
    }
    // MeshShape::intersect (mesh.cpp:73-97)
    bool intersect(const Ray& r, double tmin, double tmax, LocalHit& h) const {
        if (nodes.empty()) return false;
        const Slabs rs(r);
        bool found = false;
        double best = tmax, te;
        struct E { uint32_t n; double t; };
        E stack[128];
        int sp = 0;
        if (!rs.hit(nodes[0].box, tmin, best, te)) return false;
        uint32_t cur = 0;
        for (;;) {
            const Node& nd = nodes[cur];
            bool descend = false;
            if (nd.count > 0) {
                for (uint32_t k = 0; k < nd.count; ++k) {
                    const uint32_t i = order[nd.start + k];
                    const V &v0 = pos[tri[i][0]], &v1 = pos[tri[i][1]], &v2 = pos[tri[i][2]];
                    if (!crosses(r.o, r.d, v0, v1, v2)) continue;
                    const V n = unit(triNormal(v0, v1, v2)), tv = r.o - v0;
                    const double tt = -dot(tv, n) / dot(r.d, n);
                    if (!(tt > tmin && tt < best)) continue;
                    if (sameFace(r.depP, i) && std::fabs(dot(tv, n)) <= r.depErr) continue;
                    best = tt;
                    found = true;
                    h.t = tt;
                    h.prim = i;
                }
            } else {
                uint32_t a = nd.start, b = nd.right;
                double t0, t1;
                const bool h0 = rs.hit(nodes[a].box, tmin, best, t0), h1 = rs.hit(nodes[b].box, tmin, best, t1);
                if (h0 && h1) {
                    if (t1 < t0) { std::swap(a, b); std::swap(t0, t1); }
                    if (sp < 128) stack[sp++] = {b, t1};
                    cur = a;
                    descend = true;
                } else if (h0 || h1) {
                    cur = h0 ? a : b;
                    descend = true;
                }
            }
            if (descend) continue;
            while (sp > 0 && stack[sp - 1].t > best) --sp;
            if (sp == 0) break;
            cur = stack[--sp].n;
        }
        if (!found) return false;
        const auto& t = tri[h.prim];
        h.p = r.at(h.t);
        h.n = unit(triNormal(pos[t[0]], pos[t[1]], pos[t[2]]));
        h.error = std::fabs(dot(h.p - pos[t[0]], h.n));
        return true;
    }
};

// ------------------------------------------------------------------ shapes
struct Shape {
    int kind;
    double P[4];
    std::shared_ptr<Mesh> mesh;
    double zMin = 0, zMax = 0;

    bool canSample() const {
        if (kind == OWEC_SHAPE_MESH) return mesh->area > 0;
        if (kind == OWEC_SHAPE_SAG) return P[0] == 0;
        return true;
    }
    double area() const {
        switch (kind) {
            case OWEC_SHAPE_SPHERE: return 4 * Pi * P[0] * P[0];
            case OWEC_SHAPE_PLANE: {
                const int ap = int(P[0]);
                if (ap == OWEC_APERTURE_DISK) return Pi * (P[1] * P[1] - P[2] * P[2]);
                if (ap == OWEC_APERTURE_RECT) return 4 * P[1] * P[2];
                return Pi * P[1] * P[2];
            }
            case OWEC_SHAPE_SAG: return Pi * (P[2] * P[2] - P[3] * P[3]);
            case OWEC_SHAPE_CYLINDER: return 2 * Pi * P[0] * (std::max(P[1], P[2]) - std::min(P[1], P[2]));
            default: return mesh->area;
        }
    }
    Box bounds() const {
        Box b;
        switch (kind) {
            case OWEC_SHAPE_SPHERE: b.expand(V(-P[0], -P[0], -P[0])); b.expand(V(P[0], P[0], P[0])); break;
            case OWEC_SHAPE_SAG: b.expand(V(-P[2], -P[2], zMin)); b.expand(V(P[2], P[2], zMax)); break;
            case OWEC_SHAPE_PLANE: {
                const double ex = P[1], ey = int(P[0]) == OWEC_APERTURE_DISK ? P[1] : P[2];
                const double pad = 1e-9 * (1 + std::max(ex, ey));
                b.expand(V(-ex, -ey, -pad));
                b.expand(V(ex, ey, pad));
                break;
            }
            case OWEC_SHAPE_CYLINDER:
                b.expand(V(-P[0], -P[0], std::min(P[1], P[2])));
                b.expand(V(P[0], P[0], std::max(P[1], P[2])));
                break;
            default: b = mesh->bounds; break;
        }
        return b;
    }
    bool sameFace(uint32_t a, uint32_t b) const { return kind == OWEC_SHAPE_MESH ? mesh->sameFace(a, b) : true; }

    static double conicSlope(double c, double k, double r) {
        const double root = safeSqrt(1 - (1 + k) * c * c * (r * r));
        return root > 0 ? c * r / root : (c != 0 ? Inf : 0.0);
    }
    V sagNormal(V p) const {
        const double r = std::sqrt(p.x * p.x + p.y * p.y);
        if (r < kTiny) return {0, 0, 1};
        const double s = conicSlope(P[0], P[1], r);
        return unit(V(-s * p.x / r, -s * p.y / r, 1));
    }
    template <class Solid, class Normal>
    bool firstRefined(const Ray& r, QKind k, double qa, double qb, double t0, double t1, double tmin, double tmax,
                      Solid solid, Normal normal, LocalHit& h) const {
        for (double t : {t0, t1}) {
            double tr;
            if (!refinedRootIn(k, qa, qb, r.o, r.d, t, tmin, tmax, tr)) continue;
            const V p = r.at(tr);
            if (!solid(p)) continue;
            h.t = tr;
            h.p = p;
            h.n = normal(p);
            h.prim = 0;
            return true;
        }
        return false;
    }
    bool intersect(const Ray& r, double tmin, double tmax, LocalHit& h) const {
        switch (kind) {
            case OWEC_SHAPE_SPHERE: {
                const double R = P[0], b = dot(r.o, r.d);
                const V perp = r.o - r.d * b;
                const double disc = R * R - dot(perp, perp);
                if (disc < 0) return false;
                const double c = dot(r.o, r.o) - R * R, q = -b - std::copysign(std::sqrt(disc), b);
                double t0 = q, t1 = q != 0 ? c / q : q;
                if (t0 > t1) std::swap(t0, t1);
                return firstRefined(r, QSphere, R * R, 0, t0, t1, tmin, tmax, [](V) { return true; },
                                    [&](V p) { return unit(p / R); }, h);
            }
            case OWEC_SHAPE_SAG: {
                const double c = P[0], k = P[1], rMax = P[2], rMin = P[3];
                auto solid = [&](V p) {
                    const double r2 = p.x * p.x + p.y * p.y;
                    return r2 <= rMax * rMax && r2 >= rMin * rMin && (c == 0 || (1 + k) * c * p.z <= 1 + kRelTol);
                };
                if (c == 0) {
                    if (r.d.z == 0) return false;
                    const double t = -r.o.z / r.d.z;
                    if (t <= tmin || t >= tmax || !solid(r.at(t))) return false;
                    h.t = t;
                    h.p = r.at(t);
                    h.n = sagNormal(h.p);
                    h.prim = 0;
                    return true;
                }
                double A, B, C, t0, t1;
                qcoeffs(QSag, c, c * (1 + k), r.o, r.d, A, B, C);
                return solveQuadratic(A, B, C, t0, t1) > 0 &&
                       firstRefined(r, QSag, c, c * (1 + k), t0, t1, tmin, tmax, solid, [&](V p) { return sagNormal(p); }, h);
            }
            case OWEC_SHAPE_PLANE: {
                if (r.d.z == 0) return false;
                const double t = -r.o.z / r.d.z;
                if (t <= tmin || t >= tmax) return false;
                V p = r.at(t);
                p.z = 0;
                const int ap = int(P[0]);
                bool in;
                if (ap == OWEC_APERTURE_DISK) {
                    const double r2 = p.x * p.x + p.y * p.y;
                    in = r2 <= P[1] * P[1] && r2 >= P[2] * P[2];
                } else if (ap == OWEC_APERTURE_RECT) {
                    in = std::fabs(p.x) <= P[1] && std::fabs(p.y) <= P[2];
                } else {
                    in = sq(p.x / P[1]) + sq(p.y / P[2]) <= 1;
                }
                if (!in) return false;
                h.t = t;
                h.p = p;
                h.n = {0, 0, 1};
                h.prim = 0;
                return true;
            }
            case OWEC_SHAPE_CYLINDER: {
                const double R = P[0], z0 = std::min(P[1], P[2]), z1 = std::max(P[1], P[2]);
                const double A = r.d.x * r.d.x + r.d.y * r.d.y;
                if (A < kTiny) return false;
                const double b = r.o.x * r.d.x + r.o.y * r.d.y;
                const double px = r.o.x - r.d.x * (b / A), py = r.o.y - r.d.y * (b / A);
                const double disc = A * (R * R - (px * px + py * py));
                if (disc < 0) return false;
                const double q = -(b + std::copysign(std::sqrt(disc), b)), c = r.o.x * r.o.x + r.o.y * r.o.y - R * R;
                double t0 = q / A, t1 = q != 0 ? c / q : t0;
                if (t0 > t1) std::swap(t0, t1);
                return firstRefined(r, QCyl, R * R, 0, t0, t1, tmin, tmax,
                                    [&](V p) { return p.z >= z0 && p.z <= z1; },
                                    [](V p) { return unit(V(p.x, p.y, 0)); }, h);
            }
            default: return mesh->intersect(r, tmin, tmax, h);
        }
    }
    void sampleArea(double u1, double u2, double u3, V& p, V& n) const {
        n = {0, 0, 1};
        switch (kind) {
            case OWEC_SHAPE_SPHERE: {
                const double z = 1 - 2 * u1, rr = safeSqrt(1 - z * z), phi = 2 * Pi * u2;
                n = {rr * std::cos(phi), rr * std::sin(phi), z};
                p = n * P[0];
                return;
            }
            case OWEC_SHAPE_PLANE: {
                const int ap = int(P[0]);
                if (ap == OWEC_APERTURE_DISK) {
                    const double rr = std::sqrt(P[2] * P[2] + u1 * (P[1] * P[1] - P[2] * P[2])), phi = 2 * Pi * u2;
                    p = {rr * std::cos(phi), rr * std::sin(phi), 0};
                } else if (ap == OWEC_APERTURE_RECT) {
                    p = {(2 * u1 - 1) * P[1], (2 * u2 - 1) * P[2], 0};
                } else {
                    const double rr = std::sqrt(u1), phi = 2 * Pi * u2;
                    p = {P[1] * rr * std::cos(phi), P[2] * rr * std::sin(phi), 0};
                }
                return;
            }
            case OWEC_SHAPE_SAG: {
                const double rr = std::sqrt(P[3] * P[3] + u1 * (P[2] * P[2] - P[3] * P[3])), phi = 2 * Pi * u2;
                p = {rr * std::cos(phi), rr * std::sin(phi), 0};
                return;
            }
            case OWEC_SHAPE_CYLINDER: {
                const double phi = 2 * Pi * u1;
                n = {std::cos(phi), std::sin(phi), 0};
                p = {P[0] * n.x, P[0] * n.y, P[1] + u2 * (P[2] - P[1])};
                return;
            }
            default: {
                const auto& cdf = mesh->cdf;
                size_t i = size_t(std::lower_bound(cdf.begin(), cdf.end(), u3 * mesh->area) - cdf.begin());
                if (i >= mesh->tri.size()) i = mesh->tri.size() - 1;
                const auto& t = mesh->tri[i];
                const double su = std::sqrt(u1), b0 = 1 - su, b1 = u2 * su;
                p = mesh->pos[t[0]] * b0 + mesh->pos[t[1]] * b1 + mesh->pos[t[2]] * (1 - b0 - b1);
                n = unit(Mesh::triNormal(mesh->pos[t[0]], mesh->pos[t[1]], mesh->pos[t[2]]));
                return;
            }
        }
    }
    uint32_t sampledPrimitive(double u) const {
        if (kind != OWEC_SHAPE_MESH) return 0;
        const auto& cdf = mesh->cdf;
        if (cdf.empty()) return ~0u;
        return uint32_t(std::min(size_t(std::lower_bound(cdf.begin(), cdf.end(), u * mesh->area) - cdf.begin()),
                                 cdf.size() - 1));
    }
    static bool areaToSolidAngle(V ref, V p, V n, double area, double& pdfW) {
        pdfW = 0;
        const V w = p - ref;
        const double d2 = dot(w, w);
        if (!(d2 > 0)) return false;
        const double cosL = std::fabs(dot(n, w)) / std::sqrt(d2);
        if (cosL <= kGrazing) return false;
        pdfW = d2 / (cosL * area);
        return true;
    }
    static double sphereConeSize(V ref, double R) {
        const double dc2 = dot(ref, ref);
        if (dc2 <= R * R * (1 + kRelTol)) return 0;
        const double s2 = R * R / dc2;
        return s2 / (1 + safeSqrt(1 - s2));
    }
    bool sampleFrom(V ref, double u1, double u2, double u3, V& p, V& n, double& pdfW) const {
        if (kind == OWEC_SHAPE_SPHERE) {
            const double omc = sphereConeSize(ref, P[0]);
            if (omc != 0) {
                const V axis = -ref / len(ref);
                V s, t;
                basis(axis, s, t);
                const double omcT = u1 * omc, cosT = 1 - omcT, sinT = safeSqrt(omcT * (2 - omcT)), phi = 2 * Pi * u2;
                const V w = s * (sinT * std::cos(phi)) + t * (sinT * std::sin(phi)) + axis * cosT;
                LocalHit h;
                Ray rr;
                rr.o = ref;
                rr.d = w;
                if (intersect(rr, 0, Inf, h)) p = h.p;
                else p = unit(ref + w * dot(-ref, w)) * P[0];
                n = unit(p);
                pdfW = 1 / (2 * Pi * omc);
                return true;
            }
        }
        if (!canSample() || area() <= 0) return false;
        sampleArea(u1, u2, u3, p, n);
        return areaToSolidAngle(ref, p, n, area(), pdfW);
    }
    double pdfFrom(V ref, V p, V n) const {
        if (kind == OWEC_SHAPE_SPHERE) {
            const double omc = sphereConeSize(ref, P[0]);
            if (omc != 0) return 1 / (2 * Pi * omc);
        }
        double pdfW;
        return canSample() && area() > 0 && areaToSolidAngle(ref, p, n, area(), pdfW) ? pdfW : 0;
    }
};

// ------------------------------------------------------------------ world
struct Boundary {
    Shape shape;
    Xf toWorld, toLocal;
    Box worldBox;
    uint32_t front, back, optics;
    int emission;
    int light = -1;
};
struct Hit {
    double t = Inf;
    V p, n, pLocal, nLocal;
    uint32_t boundary = kNone, prim = 0;
    double error = 0;
    bool ambiguous = false;
};
struct Light { int kind; uint32_t boundary; double power; };

struct Scene {
    std::vector<Spec> spectra;
    std::vector<Medium> media;
    std::vector<uint32_t> regionMedium;
    std::vector<owec_optics> optics;
    std::vector<owec_emission> emissions;
    std::vector<Boundary> boundaries;
    Box bounds;
    std::vector<Light> lights;
    std::vector<double> lightPdf, lightCdf;
    // environment
    int skyModel = OWEC_SKY_NONE, skySpec = -1, sunSpec = -1;
    bool hasSun = false;
    V sunDir{0, 0, 1};
    double sunRadius = 0, sunShare = 0;
    // detector
    owec_detector det{};
    V fwd, right, up;
    double tanX = 1, tanY = 1;
    uint32_t detRegion = 0;
    Xf sensorXf;
    V sensorN;

    const Medium& mediumOf(uint32_t r) const { return media[regionMedium[r]]; }
    double indexOf(uint32_t r, double l) const { return mediumOf(r).n(l); }
    double specEval(int i, double l) const { return i < 0 ? 0.0 : spectra[size_t(i)].eval(l); }
    double sceneRadius() const { return bounds.valid() ? std::max(1e-3, 0.5 * len(bounds.extent())) : 1.0; }
    double sunCos() const { return std::cos(sunRadius); }
    double sunSolidAngle() const { return 2 * Pi * (1 - std::cos(sunRadius)); }
    double sun(V d, double l) const { return hasSun && dot(d, sunDir) >= std::cos(sunRadius) ? specEval(sunSpec, l) : 0; }
    double sky(V, double l) const { return skyModel == OWEC_SKY_UNIFORM ? specEval(skySpec, l) : 0; }

    // World::buildLightTable (world.cpp:285-350)
    void buildLights() {
        lights.clear();
        for (size_t i = 0; i < boundaries.size(); ++i) {
            Boundary& b = boundaries[i];
            b.light = -1;
            if (b.emission < 0 || !b.shape.canSample() || !emissions[size_t(b.emission)].nee) continue;
            const owec_emission& e = emissions[size_t(b.emission)];
            const double sides = (e.front ? 1 : 0) + (e.back ? 1 : 0);
            const double p = std::max(1e-12, spectra[size_t(e.radiance)].luminance()) * b.shape.area() * Pi * sides;
            b.light = int(lights.size());
            lights.push_back({0, uint32_t(i), p});
        }
        if (hasSun) {
            const double R = sceneRadius();
            lights.push_back({1, kNone, std::max(1e-12, spectra[size_t(sunSpec)].luminance()) * sunSolidAngle() * Pi * R * R});
        }
        double total = 0, bp = 0, nearP = 0, farP = 0;
        for (auto& l : lights) {
            total += l.power;
            if (l.kind == 0) {
                bp += l.power;
                (emissions[size_t(boundaries[l.boundary].emission)].distant ? farP : nearP) += l.power;
            }
        }
        double share = hasSun && bp > 0 ? clampd(sunShare, 0, 0.999) : 0;
        if (farP > 0 && hasSun && share == 0) share = 0.5;
        lightPdf.clear();
        lightCdf.clear();
        double acc = 0;
        for (auto& l : lights) {
            double p = total > 0 ? l.power / total : 0;
            if (share > 0) p = l.kind == 1 ? share : (1 - share) * l.power / bp;
            if (farP > 0 && l.kind == 0) {
                const bool distant = emissions[size_t(boundaries[l.boundary].emission)].distant;
                p = (1 - share) * (nearP > 0 ? 0.5 : 1) * l.power / (distant ? farP : nearP);
            }
            lightPdf.push_back(p);
            acc += p;
            lightCdf.push_back(acc);
        }
        if (!lightCdf.empty()) lightCdf.back() = 1.0;
    }
    size_t pickLight(double u) const {
        const size_t i = size_t(std::upper_bound(lightCdf.begin(), lightCdf.end(), u) - lightCdf.begin());
        return std::min(i, lights.size() - 1);
    }

    // firstCrossing and NearestCrossing (world.cpp:440-550)
    struct Candidate {
        LocalHit lh;
        double error = 0;
        bool matches = false, unresolved = false;
    };
    bool firstCrossing(const Boundary& b, uint32_t i, const Ray& ray, const Slabs& rs, double worldScale, double tm,
                       Candidate& c) const {
        Ray lr;
        lr.o = b.toLocal.point(ray.o);
        lr.d = b.toLocal.vec(ray.d);
        const double scale = std::max({worldScale, maxAbs(lr.o), maxAbs(b.toWorld.translation()),
                                       maxAbs(b.shape.bounds().extent())});
        const double anchorError = std::max(ray.depErr, contactError(scale));
        c.error = anchorError;
        const bool isMesh = b.shape.kind == OWEC_SHAPE_MESH;
        const bool knownMeshDeparture = isMesh && i == ray.depB && ray.depP < b.shape.mesh->tri.size();
        if (i == ray.depB) {
            lr.depP = ray.depP;
            lr.depN = b.toLocal.vec(ray.depN);
        }
        if (knownMeshDeparture) {
            const auto& t = b.shape.mesh->tri[ray.depP];
            const auto& pos = b.shape.mesh->pos;
            const V nrm = unit(cross(pos[t[1]] - pos[t[0]], pos[t[2]] - pos[t[0]]));
            lr.o = lr.o - nrm * dot(lr.o - pos[t[0]], nrm);
        }
        lr.depErr = c.error;
        const bool spawned = ray.depB != kNone;
        const double tmin = ray.forwardOnly || knownMeshDeparture ? std::nextafter(0.0, -Inf) : (spawned ? -c.error : 0.0);
        double tEnter;
        if (!rs.hit(b.worldBox, tmin, tm, tEnter)) return false;
        auto solve = [&](double lo) {
            c.lh.error = 0;
            const bool ok = b.shape.intersect(lr, lo, tm, c.lh);
            c.error = anchorError + c.lh.error;
            return ok;
        };
        if (!solve(tmin)) return false;
        V n;
        auto incidence = [&] {
            n = b.toWorld.vec(c.lh.n);
            const uint32_t inc = dot(ray.d, n) < 0 ? b.front : b.back;
            c.matches = ray.hint == kNone || inc == ray.hint;
        };
        incidence();
        auto excluded = [&] {
            const bool ownNear = std::fabs(c.lh.t * dot(ray.d, unit(n))) <= c.error;
            return spawned && ((std::fabs(c.lh.t) <= c.error && !c.matches) ||
                               (ownNear && !isMesh && i == ray.depB && (b.front == b.back || dot(ray.depN, ray.depN) > 0) &&
                                dot(ray.d, n) * dot(ray.d, ray.depN) >= 0));
        };
        for (int retry = 0; excluded(); ++retry) {
            if (retry == 8) { c.unresolved = true; break; }
            if (!solve(std::max(0.0, c.lh.t))) return false;
            incidence();
        }
        return true;
    }
    struct Nearest {
        bool found = false, ambiguous = false, readout = false;
        uint32_t boundary = kNone;
        Candidate best;
        bool offer(uint32_t i, const Candidate& c, double t, bool isReadout, bool hinted) {
            const bool tie = found && std::fabs(t - best.lh.t) <= std::max(c.error, best.error);
            if (tie && c.matches && best.matches && isReadout != readout) {
                if (isReadout) return false;
                ambiguous = false;
            } else if (tie && hinted && c.matches && best.matches && i != boundary) ambiguous = true;
            if (tie && best.matches && !c.matches) return false;
            if (!tie) ambiguous = false;
            bool replace = !found || !tie;
            if (found && tie) {
                if (c.matches != best.matches) replace = c.matches;
                else if (isReadout != readout) replace = readout;
                else replace = i < boundary;
            }
            if (replace) {
                best = c;
                best.lh.t = t;
                boundary = i;
                readout = isReadout;
                found = true;
                ambiguous = ambiguous || c.unresolved;
            }
            return true;
        }
    };
    // World::intersect (world.cpp:553-582); boundaries offered near-first by their box entry.
    bool intersect(const Ray& ray, double tmax, Hit& hit) const {
        Nearest nearest;
        const Slabs rs(ray);
        const double worldScale = std::max(1e-12, maxAbs(ray.o));
        const double broad = std::max(ray.depErr, contactError(std::max(worldScale, maxAbs(bounds.extent()))));
        std::vector<std::pair<double, uint32_t>> cand;
        cand.reserve(boundaries.size());
        for (uint32_t i = 0; i < boundaries.size(); ++i) {
            double te;
            if (rs.hit(boundaries[i].worldBox, -broad, tmax, te)) cand.push_back({te, i});
        }
        std::sort(cand.begin(), cand.end());
        double tm = tmax;
        for (auto& [te, i] : cand) {
            if (te > tm) continue;
            const Boundary& b = boundaries[i];
            Candidate c;
            if (!firstCrossing(b, i, ray, rs, worldScale, tm, c)) continue;
            const bool readout = optics[b.optics].type == OWEC_SURF_DETECTOR && b.front == b.back;
            if (!nearest.offer(i, c, std::max(0.0, c.lh.t), readout, ray.hint != kNone)) continue;
            tm = std::min(tmax, nearest.best.lh.t + std::max(c.error, nearest.best.error));
        }
        if (!nearest.found) return false;
        const Boundary& b = boundaries[nearest.boundary];
        const LocalHit& lh = nearest.best.lh;
        hit.t = lh.t;
        hit.pLocal = lh.p;
        hit.nLocal = lh.n;
        hit.p = b.toWorld.point(lh.p);
        hit.n = unit(b.toWorld.vec(lh.n));
        hit.boundary = nearest.boundary;
        hit.prim = lh.prim;
        hit.error = nearest.best.error;
        hit.ambiguous = nearest.ambiguous;
        return true;
    }
    Ray spawn(const Hit& h, V dir, uint32_t region) const {
        Ray r;
        r.o = h.p;
        r.d = dir;
        r.depB = h.boundary;
        r.hint = region;
        r.depN = h.n;
        r.depP = h.prim;
        r.depErr = h.error;
        return r;
    }
};

// ------------------------------------------------------------------ optics (optics.hpp, scattering.cpp)
double fresnelDielectric(double cosI, double eta) {
    cosI = clampd(cosI, -1, 1);
    if (cosI < 0) { eta = 1 / eta; cosI = -cosI; }
    const double s2 = (1 - cosI * cosI) / (eta * eta);
    if (s2 >= 1) return 1;
    const double cosT = safeSqrt(1 - s2);
    const double a = (eta * cosI - cosT) / (eta * cosI + cosT), b = (cosI - eta * cosT) / (cosI + eta * cosT);
    return (a * a + b * b) / 2;
}
bool refractDir(V d, V n, double ni, double nt, V& out) {
    const V nn = dot(d, n) < 0 ? n : -n;
    const double cosi = -dot(d, nn), eta = ni / nt, k = 1 - eta * eta * (1 - cosi * cosi);
    out = d;
    if (k < 0) return false;
    out = unit(d * eta + nn * (eta * cosi - std::sqrt(k)));
    return true;
}
struct Iface {
    const owec_optics* o;
    V n, p;
    double nFront = 1, nBack = 1, lambda = 550, floorP = 0, albedo = 1;
    double condN = 0, condK = 0;  // conductor n, k at lambda
};
struct Sample {
    V wi;
    double weight = 0, pdf = 0;
    bool delta = false, transmitted = false;
    double R = 0, T = 0;
};
bool isDelta(const owec_optics& o) {
    if (o.type == OWEC_SURF_DIELECTRIC || o.type == OWEC_SURF_CONDUCTOR) return o.roughness < 1e-3;
    return o.type == OWEC_SURF_MIRROR;
}

// complex arithmetic as (re, im) pairs
struct Cx { double re, im; };
Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
Cx cdiv(Cx a, Cx b) { const double d = b.re * b.re + b.im * b.im; return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d}; }
Cx csqrt(Cx z) {
    const double r = std::sqrt(z.re * z.re + z.im * z.im);
    return {std::sqrt(std::max(0.0, (r + z.re) / 2)), std::copysign(std::sqrt(std::max(0.0, (r - z.re) / 2)), z.im)};
}
// Reflectance of a conductor of complex relative index eta (optics.hpp:69-79).
double fresnelConductor(double c, Cx eta) {
    c = clampd(c, 0, 1);
    const Cx s2 = cdiv({1 - c * c, 0}, cmul(eta, eta));
    const Cx ct = csqrt({1 - s2.re, -s2.im});
    const Cx ec{eta.re * c, eta.im * c}, ect = cmul(eta, ct);
    const Cx rp = cdiv({ec.re - ct.re, ec.im - ct.im}, {ec.re + ct.re, ec.im + ct.im});
    const Cx rs = cdiv({c - ect.re, -ect.im}, {c + ect.re, ect.im});
    return (rp.re * rp.re + rp.im * rp.im + rs.re * rs.re + rs.im * rs.im) / 2;
}

// GGX (Trowbridge-Reitz) with visible-normal sampling (optics.hpp:104-246).
double ggxAlpha(double r) { return std::max(r, 1e-4); }
double ggxD(double a, V m) {
    const double c2 = m.z * m.z;
    if (c2 <= 0) return 0;
    const double c4 = c2 * c2;
    if (c4 < 1e-16) return 0;
    const double e = (1 - c2) / c2 / (a * a);
    return 1 / (Pi * a * a * c4 * sq(1 + e));
}
double ggxLambda(double a, V w) {
    const double c2 = w.z * w.z;
    if (c2 <= 0) return 0;
    return (std::sqrt(1 + a * a * ((1 - c2) / c2)) - 1) / 2;
}
double ggxG1(double a, V w) { return 1 / (1 + ggxLambda(a, w)); }
double ggxG(double a, V wo, V wi) { return 1 / (1 + ggxLambda(a, wo) + ggxLambda(a, wi)); }
double ggxPdf(double a, V w, V m) { return w.z == 0 ? 0 : ggxG1(a, w) / std::fabs(w.z) * ggxD(a, m) * std::fabs(dot(w, m)); }
V ggxSampleWm(double a, V w, double u1, double u2) {
    V wh = unit(V(a * w.x, a * w.y, w.z));
    if (wh.z < 0) wh = -wh;
    const V T1 = wh.z < 0.99999 ? unit(cross(V(0, 0, 1), wh)) : V(1, 0, 0);
    const V T2 = cross(wh, T1);
    const double r = std::sqrt(u1), phi = 2 * Pi * u2;
    const double px = r * std::cos(phi);
    double py = r * std::sin(phi);
    const double h = std::sqrt(std::max(0.0, 1 - px * px)), s = (1 + wh.z) / 2;
    py = (1 - s) * h + s * py;
    const double pz = safeSqrt(1 - px * px - py * py);
    const V nh = T1 * px + T2 * py + wh * pz;
    return unit(V(a * nh.x, a * nh.y, std::max(1e-6, nh.z)));
}
bool sameHemi(V a, V b) { return a.z * b.z > 0; }
bool refractLocal(V wi, V n, double eta, double& etap, V& wt) {
    double cosI = dot(n, wi);
    etap = 1;
    wt = wi;
    if (cosI < 0) { eta = 1 / eta; cosI = -cosI; n = -n; }
    const double s2 = std::max(0.0, 1 - cosI * cosI) / (eta * eta);
    if (s2 >= 1) return false;
    const double cosT = safeSqrt(1 - s2);
    wt = -wi / eta + n * (cosI / eta - cosT);
    etap = eta;
    return true;
}
struct Lobe { V wi; double weight = 0, pdf = 0; bool transmitted = false; double R = 0, T = 0; };
bool sampleRoughDielectric(double a, V wo, double eta, double uc, double u1, double u2, bool radiance, Lobe& s) {
    const V wm = ggxSampleWm(a, wo, u1, u2);
    const double R = fresnelDielectric(dot(wo, wm), eta), T = 1 - R;
    s = Lobe{};
    s.wi = wo;
    s.R = R;
    s.T = T;
    if (uc < R / (R + T)) {
        s.wi = reflectV(-wo, wm);
        if (!sameHemi(wo, s.wi)) return false;
        s.pdf = ggxPdf(a, wo, wm) / (4 * std::fabs(dot(wo, wm))) * R / (R + T);
        const double f = ggxD(a, wm) * ggxG(a, wo, s.wi) * R / (4 * std::fabs(s.wi.z) * std::fabs(wo.z));
        s.weight = f * std::fabs(s.wi.z) / s.pdf;
    } else {
        double etap;
        V wi;
        if (!refractLocal(wo, wm, eta, etap, wi)) return false;
        if (sameHemi(wo, wi) || wi.z == 0) return false;
        s.wi = wi;
        s.transmitted = true;
        const double den = sq(dot(wi, wm) + dot(wo, wm) / etap);
        s.pdf = ggxPdf(a, wo, wm) * (std::fabs(dot(wi, wm)) / den) * T / (R + T);
        double ft = T * ggxD(a, wm) * ggxG(a, wo, wi) * std::fabs(dot(wi, wm) * dot(wo, wm) / (wi.z * wo.z * den));
        if (radiance) ft /= sq(etap);
        s.weight = ft * std::fabs(wi.z) / s.pdf;
    }
    return std::isfinite(s.weight) && s.pdf > 0;
}
double evalRoughDielectric(double a, V wo, V wi, double eta, bool radiance, double& pdf) {
    pdf = 0;
    const double co = wo.z, ci = wi.z;
    if (co == 0 || ci == 0) return 0;
    const bool refl = co * ci > 0;
    double etap = 1;
    if (!refl) etap = co > 0 ? eta : 1 / eta;
    V wm = wi * etap + wo;
    if (dot(wm, wm) == 0) return 0;
    wm = unit(wm);
    if (wm.z < 0) wm = -wm;
    if (dot(wm, wi) * ci < 0 || dot(wm, wo) * co < 0) return 0;
    const double R = fresnelDielectric(dot(wo, wm), eta), T = 1 - R;
    if (refl) {
        pdf = ggxPdf(a, wo, wm) / (4 * std::fabs(dot(wo, wm))) * R / (R + T);
        return ggxD(a, wm) * ggxG(a, wo, wi) * R / std::fabs(4 * ci * co);
    }
    const double den = sq(dot(wi, wm) + dot(wo, wm) / etap);
    pdf = ggxPdf(a, wo, wm) * std::fabs(dot(wi, wm)) / den * T / (R + T);
    double ft = ggxD(a, wm) * T * ggxG(a, wo, wi) * std::fabs(dot(wi, wm) * dot(wo, wm) / (den * ci * co));
    if (radiance) ft /= sq(etap);
    return ft;
}
bool sampleRoughConductor(double a, V w, Cx eta, double tint, double u1, double u2, Lobe& s) {
    const V wm = ggxSampleWm(a, w, u1, u2);
    s = Lobe{};
    s.wi = reflectV(-w, wm);
    s.R = fresnelConductor(std::fabs(dot(w, wm)), eta) * tint;
    if (s.wi.z <= 0) return false;
    s.pdf = ggxPdf(a, w, wm) / (4 * std::fabs(dot(w, wm)));
    if (!(s.pdf > 0)) return false;
    const double f = ggxD(a, wm) * s.R * ggxG(a, w, s.wi) / (4 * s.wi.z * w.z);
    s.weight = f * s.wi.z / s.pdf;
    return std::isfinite(s.weight);
}
double evalRoughConductor(double a, V wo, V wi, Cx eta, double tint, double& pdf) {
    pdf = 0;
    V wm = wo + wi;
    if (dot(wm, wm) == 0) return 0;
    wm = unit(wm);
    const double F = fresnelConductor(std::fabs(dot(wo, wm)), eta) * tint;
    pdf = ggxPdf(a, wo, wm) / (4 * std::fabs(dot(wo, wm)));
    return ggxD(a, wm) * F * ggxG(a, wo, wi) / (4 * wi.z * wo.z);
}
Cx conductorEta(const Iface& it, double nMed) { return {it.condN / nMed, it.condK / nMed}; }

// sampleScatter (scattering.cpp:65-145)
bool sampleScatter(const Iface& it, V d, double uc, double u1, double u2, bool radiance, Sample& s) {
    const Frame fr(it.n);
    const V wo = fr.toLocal(-d);
    const bool fromFront = wo.z > 0;
    s = Sample{};
    const owec_optics& o = *it.o;
    auto fromLobe = [&](const Lobe& l) {
        s.wi = fr.toWorld(l.wi);
        s.weight = l.weight;
        s.pdf = l.pdf;
        s.transmitted = l.transmitted;
        s.R = l.R;
        s.T = l.T;
    };
    switch (o.type) {
        case OWEC_SURF_DIELECTRIC: {
            const double eta = it.nBack / it.nFront;
            if (o.roughness >= 1e-3 && eta != 1) {
                Lobe l;
                if (!sampleRoughDielectric(ggxAlpha(o.roughness), wo, eta, uc, u1, u2, radiance, l)) return false;
                fromLobe(l);
                return true;
            }
            const double ni = fromFront ? it.nFront : it.nBack, nt = fromFront ? it.nBack : it.nFront;
            const double R = fresnelDielectric(wo.z, eta);
            const double pR = it.floorP > 0 && R < 1 ? clampd(R, it.floorP, 1 - it.floorP) : R;
            s.R = R;
            s.T = 1 - R;
            s.delta = true;
            if (uc < pR) {
                s.wi = fr.toWorld(V(-wo.x, -wo.y, wo.z));
                s.weight = R / pR;
                return s.weight > 0;
            }
            if (!refractDir(d, it.n, ni, nt, s.wi)) return false;
            s.weight = (1 - R) / (1 - pR) * (radiance ? sq(ni / nt) : 1.0);
            s.transmitted = true;
            return true;
        }
        case OWEC_SURF_DIFFUSE: {
            if (!fromFront && o.back_absorbs) return false;
            if (it.albedo <= 0) return false;
            const double a = 2 * u1 - 1, b = 2 * u2 - 1;
            double dx = 0, dy = 0;
            if (!(a == 0 && b == 0)) {
                double r, phi;
                if (std::fabs(a) > std::fabs(b)) { r = a; phi = (Pi / 4) * (b / a); }
                else { r = b; phi = Pi / 2 - (Pi / 4) * (a / b); }
                dx = r * std::cos(phi);
                dy = r * std::sin(phi);
            }
            V w(dx, dy, safeSqrt(1 - dx * dx - dy * dy));
            if (!fromFront) w.z = -w.z;
            s.wi = fr.toWorld(w);
            s.pdf = std::fabs(w.z) * InvPi;
            s.weight = it.albedo;
            s.R = it.albedo;
            return s.pdf > 0;
        }
        case OWEC_SURF_MIRROR:
            if (!fromFront && o.back_absorbs) return false;
            s.wi = fr.toWorld(V(-wo.x, -wo.y, wo.z));
            s.weight = it.albedo;
            s.delta = true;
            s.R = s.weight;
            return s.weight > 0;
        case OWEC_SURF_CONDUCTOR: {
            if (!fromFront && o.back_absorbs) return false;
            const Cx eta = conductorEta(it, fromFront ? it.nFront : it.nBack);
            const V w = fromFront ? wo : V(wo.x, wo.y, -wo.z);
            if (o.roughness < 1e-3) {
                s.wi = fr.toWorld(V(-wo.x, -wo.y, wo.z));
                s.weight = fresnelConductor(w.z, eta) * it.albedo;
                s.delta = true;
                s.R = s.weight;
                return s.weight > 0;
            }
            Lobe l;
            if (!sampleRoughConductor(ggxAlpha(o.roughness), w, eta, it.albedo, u1, u2, l)) return false;
            if (!fromFront) l.wi.z = -l.wi.z;
            fromLobe(l);
            return true;
        }
        default: return false;
    }
}
// evalScatter (scattering.cpp:147-172)
double evalScatter(const Iface& it, V d, V wiW, double& pdf, bool radiance = true) {
    pdf = 0;
    const owec_optics& o = *it.o;
    if (isDelta(o)) return 0;
    const Frame fr(it.n);
    V wo = fr.toLocal(-d), wi = fr.toLocal(wiW);
    const bool fromFront = wo.z > 0;
    switch (o.type) {
        case OWEC_SURF_DIFFUSE:
            if (!fromFront && o.back_absorbs) return 0;
            if (!sameHemi(wo, wi)) return 0;
            pdf = std::fabs(wi.z) * InvPi;
            return it.albedo * InvPi;
        case OWEC_SURF_CONDUCTOR: {
            if (!fromFront && o.back_absorbs) return 0;
            if (!sameHemi(wo, wi)) return 0;
            if (!fromFront) { wo.z = -wo.z; wi.z = -wi.z; }
            return evalRoughConductor(ggxAlpha(o.roughness), wo, wi, conductorEta(it, fromFront ? it.nFront : it.nBack),
                                      it.albedo, pdf);
        }
        case OWEC_SURF_DIELECTRIC:
            return evalRoughDielectric(ggxAlpha(o.roughness), wo, wi, it.nBack / it.nFront, radiance, pdf);
        default: return 0;
    }
}

// ------------------------------------------------------------------ the tracer (transport.cpp)
struct Stats { uint64_t paths = 0, segments = 0, inconsistencies = 0, leaks = 0; };
using S4 = std::array<double, NW>;
struct WL {
    S4 lambda{}, pdf{};
    bool secTerminated() const { return pdf[1] == 0 && pdf[2] == 0 && pdf[3] == 0; }
    void terminateSecondary() {
        if (secTerminated()) return;
        for (int i = 1; i < NW; ++i) pdf[size_t(i)] = 0;
        pdf[0] /= NW;
    }
};
struct Endpoint {
    V p;
    uint32_t region = kNone, boundary = kNone;
    V normal;
    uint32_t primitive = kNone;
    double error = 0;
};

struct Tracer {
    const Scene& w;
    int maxDepth, rrDepth;
    double floorP;

    Iface makeInterface(const Hit& h, double lambda) const {
        const Boundary& b = w.boundaries[h.boundary];
        Iface it;
        it.o = &w.optics[b.optics];
        it.n = h.n;
        it.p = h.p;
        it.nFront = w.indexOf(b.front, lambda);
        it.nBack = w.indexOf(b.back, lambda);
        it.lambda = lambda;
        it.floorP = floorP;
        it.albedo = it.o->reflectance >= 0 ? w.specEval(it.o->reflectance, lambda) : 1.0;
        it.condN = w.specEval(it.o->conductor_n, lambda);
        it.condK = w.specEval(it.o->conductor_k, lambda);
        return it;
    }
    Iface atWavelength(const Iface& base, const Hit& h, double lambda) const {
        Iface it = base;
        const Boundary& b = w.boundaries[h.boundary];
        it.nFront = w.indexOf(b.front, lambda);
        it.nBack = w.indexOf(b.back, lambda);
        it.lambda = lambda;
        it.albedo = it.o->reflectance >= 0 ? w.specEval(it.o->reflectance, lambda) : 1.0;
        it.condN = w.specEval(it.o->conductor_n, lambda);
        it.condK = w.specEval(it.o->conductor_k, lambda);
        return it;
    }
    double secondaryWeight(const Iface& it, V d, const Sample& s) const {
        if (!s.delta) {
            double pdf;
            const double f = evalScatter(it, d, s.wi, pdf);
            return s.pdf > 0 ? f * std::fabs(dot(s.wi, it.n)) / s.pdf : 0.0;
        }
        if (it.o->type == OWEC_SURF_DIELECTRIC) return s.weight;
        if (it.o->type == OWEC_SURF_MIRROR) return it.albedo;
        if (it.o->type == OWEC_SURF_CONDUCTOR) {
            const bool fromFront = dot(d, it.n) < 0;
            return fresnelConductor(std::fabs(dot(d, it.n)), conductorEta(it, fromFront ? it.nFront : it.nBack)) * it.albedo;
        }
        return 0;
    }

    struct LightSample {
        V wi;
        double dist = Inf, pdf = 0;
        S4 Le{};
        uint32_t boundary = kNone, region = kNone;
        Hit endpoint;
    };
    bool sampleLightFrom(V p, const WL& wl, Rng& rng, LightSample& ls) const {
        if (w.lights.empty()) return false;
        const size_t li = w.pickLight(rng.uniform());
        const double sel = w.lightPdf[li];
        const Light& L = w.lights[li];
        const double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
        if (L.kind == 1) {
            const double cosT = (1 - u1) + u1 * w.sunCos(), sinT = safeSqrt(1 - cosT * cosT), phi = 2 * Pi * u2;
            ls.wi = Frame(w.sunDir).toWorld(V(std::cos(phi) * sinT, std::sin(phi) * sinT, cosT));
            for (int i = 0; i < NW; ++i) ls.Le[size_t(i)] = w.specEval(w.sunSpec, wl.lambda[size_t(i)]);
            ls.pdf = sel / w.sunSolidAngle();
            return true;
        }
        const Boundary& b = w.boundaries[L.boundary];
        V pL, nL;
        double pdfW;
        if (!b.shape.sampleFrom(b.toLocal.point(p), u1, u2, u3, pL, nL, pdfW)) return false;
        Hit& e = ls.endpoint;
        e.p = b.toWorld.point(pL);
        e.n = unit(b.toWorld.vec(nL));
        e.boundary = L.boundary;
        e.prim = b.shape.sampledPrimitive(u3);
        e.error = contactError(std::max({maxAbs(e.p), maxAbs(pL), maxAbs(b.toWorld.translation()),
                                         maxAbs(b.shape.bounds().extent())}));
        const V dv = e.p - p;
        ls.dist = len(dv);
        if (!(ls.dist > 0)) return false;
        ls.wi = dv / ls.dist;
        const owec_emission& em = w.emissions[size_t(b.emission)];
        const double cosL = dot(e.n, -ls.wi);
        const bool lit = (cosL > 0 && em.front) || (cosL < 0 && em.back);
        for (int i = 0; i < NW; ++i) ls.Le[size_t(i)] = lit ? w.specEval(em.radiance, wl.lambda[size_t(i)]) : 0.0;
        ls.pdf = sel * pdfW;
        ls.boundary = L.boundary;
        ls.region = cosL > 0 ? b.front : b.back;
        return true;
    }
    S4 sigmaT(const Medium& m, const WL& wl) const {
        S4 r{};
        for (int i = 0; i < NW; ++i) r[size_t(i)] = m.absorption.eval(wl.lambda[size_t(i)]) + m.scattering.eval(wl.lambda[size_t(i)]);
        return r;
    }
    // Tracer::transmittance (transport.cpp:237-285)
    S4 transmittance(const Endpoint& start, V dir, double dist, const WL& wl, uint32_t* finalRegion,
                     const Endpoint* endpoint) const {
        uint32_t region = start.region;
        S4 Tr{1, 1, 1, 1};
        Ray ray;
        ray.o = start.p;
        ray.d = dir;
        ray.depB = start.boundary;
        ray.hint = region;
        ray.depN = start.normal;
        ray.depP = start.primitive;
        ray.depErr = start.error;
        double remaining = dist;
        const double endError = endpoint ? std::max(endpoint->error, contactError(std::max({dist, maxAbs(endpoint->p), maxAbs(start.p)}))) : 0;
        const double margin = std::isinf(dist) || endpoint ? 0 : 1e-7 * dist + 1e-12;
        auto finish = [&](const S4& v) { if (finalRegion) *finalRegion = region; return v; };
        const S4 zero{};
        for (int guard = 0; guard < 256; ++guard) {
            Hit h;
            const double tmax = std::isinf(remaining) ? Inf : (endpoint ? remaining + endError : remaining - margin);
            if (tmax <= 0) return finish(Tr);
            ray.hint = region;
            const bool found = w.intersect(ray, tmax, h);
            const double seg = found ? std::min(h.t, remaining) : remaining;
            const Medium& m = w.mediumOf(region);
            if (m.absorbs() || m.scatters()) {
                if (std::isinf(seg)) return zero;
                const S4 st = sigmaT(m, wl);
                for (int i = 0; i < NW; ++i) Tr[size_t(i)] *= std::exp(-st[size_t(i)] * seg);
            }
            if (!found) {
                if (std::isinf(dist) && region != 0) return zero;
                return finish(Tr);
            }
            bool endpointFace = endpoint && h.boundary == endpoint->boundary;
            if (endpointFace) endpointFace = w.boundaries[h.boundary].shape.sameFace(endpoint->primitive, h.prim);
            if (endpointFace && !h.ambiguous && std::fabs(h.t - remaining) <= endError && dot(h.n, endpoint->normal) > 0 &&
                region == endpoint->region)
                return finish(Tr);
            if (endpoint && dot(h.p - endpoint->p, dir) > 0) return finish(Tr);
            const Boundary& b = w.boundaries[h.boundary];
            const uint32_t incident = dot(dir, h.n) < 0 ? b.front : b.back;
            if (incident != region || h.ambiguous) return zero;
            if (w.optics[b.optics].type != OWEC_SURF_NULL) return zero;
            region = dot(dir, h.n) < 0 ? b.back : b.front;
            ray = w.spawn(h, dir, region);
            if (!std::isinf(remaining)) remaining -= h.t;
        }
        return finish(zero);
    }
    // Tracer::connectionTransmittance (transport.cpp:287-308)
    S4 connectionTransmittance(Endpoint source, const Endpoint& target, const WL& wl) const {
        const V delta = source.p - target.p;
        const double distance = len(delta);
        const S4 zero{};
        if (!(distance > 0)) return zero;
        const V direction = delta / distance;
        const double error = contactError(std::max({distance, maxAbs(source.p), maxAbs(target.p)}));
        if (source.boundary != kNone) {
            const Boundary& b = w.boundaries[source.boundary];
            const V pl = b.toLocal.point(source.p);
            source.error = std::max(source.error, contactError(std::max({maxAbs(source.p), maxAbs(pl),
                                                                       maxAbs(b.toWorld.translation()),
                                                                       maxAbs(b.shape.bounds().extent())})));
        }
        Hit contact;
        Ray proof;
        proof.o = source.p;
        proof.d = -direction;
        proof.depB = source.boundary;
        proof.hint = source.region;
        proof.depN = source.normal;
        proof.depP = source.primitive;
        proof.depErr = source.error;
        proof.forwardOnly = true;
        if (w.intersect(proof, std::max(error, source.error), contact)) {
            if (contact.ambiguous || w.optics[w.boundaries[contact.boundary].optics].type != OWEC_SURF_NULL) return zero;
        }
        uint32_t arrival = kNone;
        const S4 tr = transmittance(target, direction, distance, wl, &arrival, &source);
        return arrival == source.region ? tr : zero;
    }
    double lightPdf(V ref, const Hit& h) const {
        const Boundary& b = w.boundaries[h.boundary];
        if (b.light < 0) return 0;
        return w.lightPdf[size_t(b.light)] * b.shape.pdfFrom(b.toLocal.point(ref), h.pLocal, h.nLocal);
    }
    static double powerHeuristic(double f, double g) {
        const double a = f * f, b = g * g;
        if (std::isinf(a)) return 1;
        if (a + b == 0) return 0;
        return a / (a + b);
    }
    static double hgPhase(double c, double g) {
        const double den = 1 + g * g + 2 * g * c;
        return (1 - g * g) / (4 * Pi * den * std::sqrt(std::max(den, kTiny)));
    }
    // Tracer::directLighting (transport.cpp:323-348)
    S4 directLighting(const Hit& hit, const Iface* surface, V d, const WL& wl, Rng& rng, double g, uint32_t region) const {
        const S4 zero{};
        LightSample ls;
        if (!sampleLightFrom(hit.p, wl, rng, ls)) return zero;
        bool leZero = true;
        for (double v : ls.Le) leZero = leZero && v == 0;
        if (leZero || ls.pdf <= 0) return zero;
        S4 f{};
        double pdfS = 0, cosF = 1;
        uint32_t startRegion = region;
        if (!surface) {
            pdfS = hgPhase(dot(-d, ls.wi), g);
            f.fill(pdfS);
        } else {
            bool fz = true;
            for (int i = 0; i < NW; ++i) {
                if (wl.pdf[size_t(i)] == 0) continue;
                double pdf;
                f[size_t(i)] = evalScatter(i == 0 ? *surface : atWavelength(*surface, hit, wl.lambda[size_t(i)]), d, ls.wi, pdf);
                if (i == 0) pdfS = pdf;
                fz = fz && f[size_t(i)] == 0;
            }
            if (fz) return zero;
            cosF = std::fabs(dot(ls.wi, hit.n));
            const Boundary& b = w.boundaries[hit.boundary];
            startRegion = dot(ls.wi, hit.n) > 0 ? b.front : b.back;
        }
        Endpoint start;
        start.p = hit.p;
        start.region = startRegion;
        if (surface) {
            start.boundary = hit.boundary;
            start.normal = hit.n;
            start.primitive = hit.prim;
            start.error = hit.error;
        }
        S4 Tr;
        if (std::isfinite(ls.dist)) {
            Endpoint src;
            src.p = ls.endpoint.p;
            src.region = ls.region;
            src.boundary = ls.endpoint.boundary;
            src.normal = ls.endpoint.n;
            src.primitive = ls.endpoint.prim;
            src.error = ls.endpoint.error;
            Tr = connectionTransmittance(src, start, wl);
        } else {
            Tr = transmittance(start, ls.wi, Inf, wl, nullptr, nullptr);
        }
        bool tz = true;
        for (double v : Tr) tz = tz && v == 0;
        if (tz) return zero;
        const double wmis = powerHeuristic(ls.pdf, pdfS);
        S4 out{};
        for (int i = 0; i < NW; ++i) out[size_t(i)] = f[size_t(i)] * Tr[size_t(i)] * ls.Le[size_t(i)] * (cosF * wmis / ls.pdf);
        return out;
    }

    // Tracer::walk (transport.cpp:531-595), without the record: the last event's kind, boundary,
    // point and throughput. kind: 0 escape, 1 detect/diffuse/absorb (the walk ends on matter),
    // 2 the event budget ran out, 3 the scattering sample failed.
    struct WalkEnd { int kind = 0; uint32_t boundary = kNone; V p; double beta = 0; int events = 0; };
    WalkEnd walk(Ray ray, uint32_t region, double lambda, bool primary, Rng& rng, int maxEvents) const {
        WalkEnd end;
        double beta = 1;
        for (int ev = 0; ev < maxEvents; ++ev) {
            ++end.events;
            Hit hit;
            ray.hint = region;
            if (!w.intersect(ray, Inf, hit)) { end.kind = 0; end.beta = beta; return end; }
            const Medium& med = w.mediumOf(region);
            if (med.absorbs()) beta *= std::exp(-med.absorption.eval(lambda) * hit.t);
            const Boundary& b = w.boundaries[hit.boundary];
            const bool fromFront = dot(ray.d, hit.n) < 0;
            const uint32_t inc = fromFront ? b.front : b.back, other = fromFront ? b.back : b.front;
            region = inc;
            const owec_optics& o = w.optics[b.optics];
            if (o.type == OWEC_SURF_NULL) {
                region = other;
                ray = w.spawn(hit, ray.d, region);
                continue;
            }
            if (o.type == OWEC_SURF_ABSORBER || o.type == OWEC_SURF_DETECTOR || (primary && o.type == OWEC_SURF_DIFFUSE)) {
                end.kind = 1;
                end.boundary = hit.boundary;
                end.p = hit.p;
                end.beta = beta;
                return end;
            }
            const Iface it = makeInterface(hit, lambda);
            Sample s;
            bool ok;
            if (primary && o.type == OWEC_SURF_DIELECTRIC) {
                const D2 u(rng);
                ok = sampleScatter(it, ray.d, 1.0, u.u1, u.u2, false, s);
                if (!ok) {
                    const D2 v(rng);
                    ok = sampleScatter(it, ray.d, 0.0, v.u1, v.u2, false, s);
                }
                if (ok && s.delta) s.weight = s.transmitted ? s.T : s.R;
            } else {
                const D3 u(rng);
                ok = sampleScatter(it, ray.d, u.u1, u.u2, u.u3, false, s);
            }
            if (!ok) { end.kind = 3; end.beta = 0; return end; }
            beta *= s.weight;
            if (s.transmitted) region = other;
            ray = w.spawn(hit, s.wi, region);
        }
        end.kind = 2;
        end.beta = beta;
        return end;
    }

    // Tracer::radiance (transport.cpp:473-529)
    S4 radiance(Ray ray, uint32_t region, WL& wl, Rng& rng, Stats& st) const {
        S4 L{}, beta{1, 1, 1, 1};
        for (int i = 1; i < NW; ++i)
            if (wl.pdf[size_t(i)] == 0) beta[size_t(i)] = 0;
        bool specular = true;
        double prevPdf = 0;
        V prevP = ray.o;
        st.paths++;
        auto add = [&](const S4& v) { for (int i = 0; i < NW; ++i) L[size_t(i)] += v[size_t(i)]; };
        auto survives = [&]() {
            double q = beta[0];
            for (double b : beta) q = std::max(q, b);
            q = std::min(1.0, q);
            if (rng.uniform() >= q) return false;
            for (double& b : beta) b *= 1 / q;
            return true;
        };
        for (int depth = 0;; ++depth) {
            Hit hit;
            ray.hint = region;
            const bool found = w.intersect(ray, Inf, hit);
            st.segments++;
            const Medium& med = w.mediumOf(region);
            // sampleMedium
            const double seg = found ? hit.t : Inf;
            int event = 0;
            double t = 0;
            if (med.scatters()) {
                const S4 sT = sigmaT(med, wl);
                t = -std::log(1 - rng.uniform()) / sT[0];
                if (t < seg) {
                    const double pdf0 = sT[0] * std::exp(-sT[0] * t);
                    for (int i = 0; i < NW; ++i)
                        beta[size_t(i)] *= med.scattering.eval(wl.lambda[size_t(i)]) * std::exp(-sT[size_t(i)] * t) / pdf0;
                    event = 1;
                } else if (std::isinf(seg)) {
                    event = 2;
                } else {
                    const double p0 = std::exp(-sT[0] * seg);
                    for (int i = 0; i < NW; ++i) beta[size_t(i)] *= std::exp(-sT[size_t(i)] * seg) / p0;
                }
            } else if (med.absorbs()) {
                if (std::isinf(seg)) event = 2;
                else
                    for (int i = 0; i < NW; ++i) beta[size_t(i)] *= std::exp(-med.absorption.eval(wl.lambda[size_t(i)]) * seg);
            }
            if (event == 2) break;
            if (event == 1) {
                // scatterInMedium
                const V p = ray.at(t);
                if (depth >= maxDepth) break;
                Hit mh;
                mh.p = p;
                const S4 dl = directLighting(mh, nullptr, ray.d, wl, rng, med.d.g, region);
                S4 c{};
                for (int i = 0; i < NW; ++i) c[size_t(i)] = beta[size_t(i)] * dl[size_t(i)];
                add(c);
                const D2 u(rng);
                const double g = med.d.g;
                double cosT;
                if (std::fabs(g) < 1e-3) cosT = 1 - 2 * u.u1;
                else cosT = -1 / (2 * g) * (1 + g * g - sq((1 - g * g) / (1 + g - 2 * g * u.u1)));
                const double sinT = safeSqrt(1 - cosT * cosT), phi = 2 * Pi * u.u2;
                const V wo = -ray.d;
                V s, tt;
                basis(wo, s, tt);
                const V wi = s * (sinT * std::cos(phi)) + tt * (sinT * std::sin(phi)) + wo * cosT;
                prevPdf = hgPhase(dot(wo, wi), g);
                specular = false;
                prevP = p;
                Ray nr;
                nr.o = p;
                nr.d = wi;
                ray = nr;
                if (!(depth < rrDepth || survives())) break;
                continue;
            }
            if (!found) {
                if (region == 0) {
                    // skyMet
                    S4 sky{}, sun{};
                    bool sunZero = true;
                    for (int i = 0; i < NW; ++i) {
                        sky[size_t(i)] = w.sky(ray.d, wl.lambda[size_t(i)]);
                        sun[size_t(i)] = w.sun(ray.d, wl.lambda[size_t(i)]);
                        sunZero = sunZero && sun[size_t(i)] == 0;
                    }
                    double sunPdf = 0;
                    if (w.hasSun) sunPdf = w.lightPdf.back() / w.sunSolidAngle();
                    const double wm = (specular || sunZero) ? 1.0 : powerHeuristic(prevPdf, sunPdf);
                    S4 c{};
                    for (int i = 0; i < NW; ++i) c[size_t(i)] = beta[size_t(i)] * (sky[size_t(i)] + sun[size_t(i)] * wm);
                    add(c);
                } else {
                    st.leaks++;
                }
                break;
            }
            // meetBoundary
            const Boundary& b = w.boundaries[hit.boundary];
            const bool fromFront = dot(ray.d, hit.n) < 0;
            const uint32_t inc = fromFront ? b.front : b.back, other = fromFront ? b.back : b.front;
            if (inc != region || hit.ambiguous) {
                st.inconsistencies++;
                region = inc;
            }
            if (hit.ambiguous) break;
            // emissionMet
            if (b.emission >= 0) {
                const owec_emission& e = w.emissions[size_t(b.emission)];
                if (fromFront ? e.front : e.back) {
                    double wm = 1;
                    if (!specular) {
                        const double pl = lightPdf(prevP, hit);
                        if (pl > 0) wm = powerHeuristic(prevPdf, pl);
                    }
                    S4 c{};
                    for (int i = 0; i < NW; ++i) c[size_t(i)] = beta[size_t(i)] * w.specEval(e.radiance, wl.lambda[size_t(i)]) * wm;
                    add(c);
                }
            }
            const owec_optics& o = w.optics[b.optics];
            if (o.type == OWEC_SURF_NULL) {
                region = other;
                ray = w.spawn(hit, ray.d, region);
                if (depth >= 4 * maxDepth) break;
                continue;
            }
            if (o.type == OWEC_SURF_ABSORBER || o.type == OWEC_SURF_DETECTOR) break;
            if (depth >= maxDepth) break;
            // scatterAtSurface
            const Iface it = makeInterface(hit, wl.lambda[0]);
            if (o.type == OWEC_SURF_DIELECTRIC && !wl.secTerminated()) {
                for (int i = 1; i < NW; ++i) {
                    if (wl.pdf[size_t(i)] == 0) continue;
                    const Iface o2 = atWavelength(it, hit, wl.lambda[size_t(i)]);
                    const double a = it.nBack / it.nFront, c = o2.nBack / o2.nFront;
                    if (std::fabs(a - c) > 1e-12 * std::fabs(a)) {
                        wl.terminateSecondary();
                        for (int j = 1; j < NW; ++j)
                            if (wl.pdf[size_t(j)] == 0) beta[size_t(j)] = 0;
                        break;
                    }
                }
            }
            if (!isDelta(o)) {
                const S4 dl = directLighting(hit, &it, ray.d, wl, rng, 0, region);
                S4 c{};
                for (int i = 0; i < NW; ++i) c[size_t(i)] = beta[size_t(i)] * dl[size_t(i)];
                add(c);
            }
            const D3 u(rng);
            Sample s;
            const bool ok = sampleScatter(it, ray.d, u.u1, u.u2, u.u3, true, s);
            if (!ok || s.weight <= 0) break;
            beta[0] *= s.weight;
            for (int i = 1; i < NW; ++i)
                if (wl.pdf[size_t(i)] != 0) beta[size_t(i)] *= secondaryWeight(atWavelength(it, hit, wl.lambda[size_t(i)]), ray.d, s);
            if (s.transmitted) region = other;
            specular = s.delta;
            prevPdf = s.pdf;
            prevP = hit.p;
            ray = w.spawn(hit, s.wi, region);
            if (depth >= rrDepth && !survives()) break;
        }
        return L;
    }
};

// ------------------------------------------------------------------ scene from a description
std::unique_ptr<Scene> build(const owec_scene_desc& d) {
    auto sc = std::make_unique<Scene>();
    auto spec = [&](int i) {
        Spec s;
        const owec_spectrum& o = d.spectra[i];
        s.kind = o.kind;
        s.a = o.a;
        s.scale = o.scale;
        if (o.kind == OWEC_SPEC_TABULATED)
            for (int k = 0; k < o.table_count; ++k) {
                s.l.push_back(d.spectrum_table[2 * (o.table_offset + k)]);
                s.v.push_back(d.spectrum_table[2 * (o.table_offset + k) + 1]);
            }
        return s;
    };
    for (uint32_t i = 0; i < d.n_spectra; ++i) sc->spectra.push_back(spec(int(i)));
    for (uint32_t i = 0; i < d.n_media; ++i) {
        Medium m;
        m.d = d.media[i];
        if (m.d.index_table >= 0) m.table = spec(m.d.index_table);
        if (m.d.absorption >= 0) m.absorption = spec(m.d.absorption);
        if (m.d.scattering >= 0) m.scattering = spec(m.d.scattering);
        sc->media.push_back(m);
    }
    sc->regionMedium.assign(d.region_medium, d.region_medium + d.n_regions);
    sc->optics.assign(d.optics, d.optics + d.n_optics);
    sc->emissions.assign(d.emissions, d.emissions + d.n_emissions);
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& ob = d.boundaries[i];
        Boundary b;
        b.shape.kind = ob.shape;
        for (int k = 0; k < 4; ++k) b.shape.P[k] = ob.params[k];
        if (ob.shape == OWEC_SHAPE_MESH) {
            auto m = std::make_shared<Mesh>();
            const owec_mesh& om = d.meshes[ob.mesh];
            for (uint64_t v = 0; v < om.vertex_count; ++v) {
                const double* p = d.vertices + 3 * (om.vertex_offset + v);
                m->pos.push_back({p[0], p[1], p[2]});
            }
            for (uint64_t t = 0; t < om.tri_count; ++t) {
                const uint32_t* q = d.triangles + 3 * (om.tri_offset + t);
                m->tri.push_back({q[0], q[1], q[2]});
            }
            m->build();
            b.shape.mesh = m;
        }
        if (ob.shape == OWEC_SHAPE_SAG) {  // the sag's z slab (geometry.cpp:74-90)
            const double c = ob.params[0], k = ob.params[1], rMax = ob.params[2], rMin = ob.params[3];
            double zMin = Inf, zMax = -Inf;
            for (int s = 0; s <= 512; ++s) {
                const double r = rMin + (rMax - rMin) * s / 512, r2 = r * r;
                const double z = c * r2 / (1 + safeSqrt(1 - (1 + k) * c * c * r2));
                zMin = std::min(zMin, z);
                zMax = std::max(zMax, z);
            }
            const double pad = 1e-9 + 1e-3 * (zMax - zMin);
            b.shape.zMin = zMin - pad;
            b.shape.zMax = zMax + pad;
        }
        for (int k = 0; k < 12; ++k) b.toWorld.m[k] = ob.to_world[k];
        b.toLocal = b.toWorld.inverse();
        const Box lb = b.shape.bounds();
        for (int c = 0; c < 8; ++c) b.worldBox.expand(b.toWorld.point(lb.corner(c)));
        sc->bounds.expand(b.worldBox);
        b.front = ob.front;
        b.back = ob.back;
        b.optics = ob.optics;
        b.emission = ob.emission;
        sc->boundaries.push_back(std::move(b));
    }
    sc->skyModel = d.env.sky_model;
    sc->skySpec = d.env.sky_radiance;
    sc->hasSun = d.env.has_sun != 0;
    sc->sunDir = unit(V(d.env.sun_dir[0], d.env.sun_dir[1], d.env.sun_dir[2]));
    sc->sunRadius = d.env.sun_angular_radius;
    sc->sunSpec = d.env.sun_radiance;
    sc->sunShare = d.env.sun_nee_share;
    sc->buildLights();
    sc->det = d.detector;
    if (d.detector.kind == OWEC_DETECTOR_OBSERVER) {
        const V pos(d.detector.position[0], d.detector.position[1], d.detector.position[2]);
        sc->fwd = unit(V(d.detector.look_at[0], d.detector.look_at[1], d.detector.look_at[2]) - pos);
        V u(d.detector.up[0], d.detector.up[1], d.detector.up[2]);
        if (std::fabs(dot(unit(u), sc->fwd)) > 0.9999) u = std::fabs(sc->fwd.z) < 0.9 ? V(0, 0, 1) : V(0, 1, 0);
        sc->right = unit(cross(sc->fwd, u));
        sc->up = cross(sc->right, sc->fwd);
        sc->tanY = std::tan(0.5 * d.detector.fov_y);
        sc->tanX = sc->tanY * double(d.detector.width) / double(d.detector.height);
        sc->detRegion = d.detector.region;
    } else {
        const Boundary& b = sc->boundaries[d.detector.boundary];
        sc->sensorXf = b.toWorld;
        sc->sensorN = unit(b.toWorld.vec(V(0, 0, 1)));
        sc->detRegion = b.front;
    }
    return sc;
}

// One pass of spp samples per pixel over pixels [first, last) (CpuRenderer::pass).
void pass(const Scene& sc, const owec_settings& s, int spp, int passIndex, int threads, uint64_t first, uint64_t last,
          double* xyz, double* samples, Stats& total) {
    Tracer tr{sc, s.max_depth, s.rr_depth, clampd(s.fresnel_floor, 0, 0.49)};
    const int W = sc.det.width, H = sc.det.height;
    threads = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
    std::vector<Stats> st(static_cast<size_t>(threads));
    std::atomic<uint64_t> next{first};
    const double invY = 1.0 / (NW * cieYIntegral());
    auto worker = [&](int tid) {
        for (;;) {
            const uint64_t pixel = next.fetch_add(1);
            if (pixel >= last) break;
            const int x = int(pixel % uint64_t(W)), y = int(pixel / uint64_t(W));
            Rng rng(hashCombine(s.seed, pixel), uint64_t(passIndex));
            double acc[3] = {0, 0, 0};
            const double rot = rng.uniform();
            for (int si = 0; si < spp; ++si) {
                double u = (si + rng.uniform()) / spp + rot;
                u -= std::floor(u);
                WL wl;
                if (s.wavelength_mode == OWEC_WAVELENGTHS_UNIFORM1) {
                    wl.lambda.fill(s.lambda_min + (s.lambda_max - s.lambda_min) * u);
                    wl.pdf.fill(0);
                    wl.pdf[0] = 1.0 / ((s.lambda_max - s.lambda_min) * NW);
                } else {
                    for (int i = 0; i < NW; ++i) {
                        double up = u + double(i) / NW;
                        if (up >= 1) up -= 1;
                        const double l = clampd(538 - 138.888889 * std::atanh(0.85691062 - 1.82750197 * up), LMin, LMax);
                        wl.lambda[size_t(i)] = l;
                        wl.pdf[size_t(i)] = (l < LMin || l > LMax) ? 0 : 0.0039398042 / sq(std::cosh(0.0072 * (l - 538)));
                    }
                }
                double px = x + rng.uniform(), py = y + rng.uniform();
                if (sc.det.pixel_sigma > 0) {
                    const D2 g(rng);
                    const double r = std::sqrt(-2 * std::log(1 - g.u1)), phi = 2 * Pi * g.u2;
                    px += r * std::cos(phi) * sc.det.pixel_sigma;
                    py += r * std::sin(phi) * sc.det.pixel_sigma;
                }
                Ray ray;
                double weight = 0;
                if (sc.det.kind == OWEC_DETECTOR_OBSERVER) {
                    const double sx = (2 * px / W - 1) * sc.tanX, sy = (1 - 2 * py / H) * sc.tanY;
                    ray.o = V(sc.det.position[0], sc.det.position[1], sc.det.position[2]);
                    ray.d = unit(sc.right * sx + sc.up * sy + sc.fwd);
                    weight = 1;
                } else {
                    if (px < 0 || py < 0 || px >= W || py >= H) continue;
                    const V pl((2 * px / W - 1) * sc.det.half_x, (1 - 2 * py / H) * sc.det.half_y, 0);
                    ray.o = sc.sensorXf.point(pl);
                    const D2 g(rng);
                    const double a = 2 * g.u1 - 1, b = 2 * g.u2 - 1;
                    double dx = 0, dy = 0;
                    if (!(a == 0 && b == 0)) {
                        double r, phi;
                        if (std::fabs(a) > std::fabs(b)) { r = a; phi = (Pi / 4) * (b / a); }
                        else { r = b; phi = Pi / 2 - (Pi / 4) * (a / b); }
                        dx = r * std::cos(phi);
                        dy = r * std::sin(phi);
                    }
                    ray.d = Frame(sc.sensorN).toWorld(V(dx, dy, safeSqrt(1 - dx * dx - dy * dy)));
                    ray.depB = sc.det.boundary;
                    ray.hint = sc.detRegion;
                    ray.depN = sc.sensorN;
                    ray.forwardOnly = true;
                    weight = Pi;
                }
                const S4 L = tr.radiance(ray, sc.detRegion, wl, rng, st[size_t(tid)]);
                double c[3] = {0, 0, 0};
                bool any = false;
                for (int i = 0; i < NW; ++i) {
                    const double Li = L[size_t(i)] * weight;
                    if (wl.pdf[size_t(i)] == 0 || Li == 0) continue;
                    any = true;
                    const double wv = Li / wl.pdf[size_t(i)] * invY, l = wl.lambda[size_t(i)];
                    c[0] += wv * cieX(l);
                    c[1] += wv * cieY(l);
                    c[2] += wv * cieZ(l);
                }
                if (!any || !std::isfinite(c[0] + c[1] + c[2])) continue;
                for (int k = 0; k < 3; ++k) acc[k] += c[k];
            }
            for (int k = 0; k < 3; ++k) xyz[3 * pixel + k] += acc[k];
            if (samples) samples[pixel] += spp;
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker, t);
    worker(0);
    for (auto& t : pool) t.join();
    for (auto& s2 : st) {
        total.paths += s2.paths;
        total.segments += s2.segments;
        total.inconsistencies += s2.inconsistencies;
        total.leaks += s2.leaks;
    }
}

thread_local std::string g_error;

}  // namespace oracle

extern "C" {

const char* oweport_last_error(void) { return oracle::g_error.c_str(); }

void* oweport_scene_create(const owec_scene_desc* desc) {
    try {
        return oracle::build(*desc).release();
    } catch (const std::exception& e) {
        oracle::g_error = e.what();
        return nullptr;
    }
}

void oweport_scene_destroy(void* s) { delete static_cast<oracle::Scene*>(s); }

int oweport_render(void* scene, const owec_settings* s, int spp, int passes, int first_pass, int threads,
                   uint64_t pixel_begin, uint64_t pixel_end, double* xyz, double* samples, owec_stats* stats) {
    try {
        const auto& sc = *static_cast<const oracle::Scene*>(scene);
        const uint64_t npix = uint64_t(sc.det.width) * uint64_t(sc.det.height);
        const uint64_t end = pixel_end == 0 ? npix : std::min(pixel_end, npix);
        oracle::Stats total;
        for (int p = 0; p < passes; ++p) oracle::pass(sc, *s, spp, first_pass + p, threads, pixel_begin, end, xyz, samples, total);
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->paths = total.paths;
            stats->segments = total.segments;
            stats->inconsistencies = total.inconsistencies;
            stats->leaks = total.leaks;
        }
        return 0;
    } catch (const std::exception& e) {
        oracle::g_error = e.what();
        return -1;
    }
}

int oweport_cast_rays(void* scene, uint64_t n, const double* o, const double* d, int threads, uint32_t* boundary,
                      uint32_t* prim, double* t) {
    try {
        const auto& sc = *static_cast<const oracle::Scene*>(scene);
        threads = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
        std::vector<std::thread> pool;
        auto work = [&](int k) {
            for (uint64_t i = uint64_t(k); i < n; i += uint64_t(threads)) {
                oracle::Ray r;
                r.o = {o[3 * i], o[3 * i + 1], o[3 * i + 2]};
                r.d = {d[3 * i], d[3 * i + 1], d[3 * i + 2]};
                oracle::Hit h;
                if (sc.intersect(r, oracle::Inf, h)) {
                    boundary[i] = h.boundary;
                    prim[i] = h.prim;
                    t[i] = h.t;
                } else {
                    boundary[i] = oracle::kNone;
                    prim[i] = 0;
                    t[i] = oracle::Inf;
                }
            }
        };
        for (int k = 1; k < threads; ++k) pool.emplace_back(work, k);
        work(0);
        for (auto& th : pool) th.join();
        return 0;
    } catch (const std::exception& e) {
        oracle::g_error = e.what();
        return -1;
    }
}

// Forward walks, emitted and binned as owec_walk describes them (include/owec.h). bins receive the
// sum of the binned walks' throughput times their splat weights; stats: [walks, binned, escaped,
// events].
int oweport_walk(void* scene, const owec_walk_desc* w, uint64_t first, uint64_t n, int threads, double* bins,
                 uint64_t* stats) {
    using namespace oracle;
    try {
        const auto& sc = *static_cast<const Scene*>(scene);
        Tracer tr{sc, 64, 6, 0};
        const V axis = unit(V(w->axis[0], w->axis[1], w->axis[2]));
        V S, T;
        basis(axis, S, T);
        const double cosMax = std::cos(w->extent);
        const Boundary& target = sc.boundaries.at(w->target);
        threads = threads > 0 ? threads : int(std::max(1u, std::thread::hardware_concurrency()));
        const size_t nb = size_t(w->width) * w->height;
        std::vector<std::vector<double>> part(size_t(threads), std::vector<double>(nb, 0.0));
        std::vector<std::array<uint64_t, 4>> st(size_t(threads), {0, 0, 0, 0});
        auto work = [&](int t) {
            const uint64_t b = n * uint64_t(t) / uint64_t(threads), e = n * uint64_t(t + 1) / uint64_t(threads);
            for (uint64_t k = b; k < e; ++k) {
                Rng rng(hashCombine(w->seed, first + k), w->stream);
                const double lambda = w->lambda_min + (w->lambda_max - w->lambda_min) * rng.uniform();
                const D2 u(rng);
                Ray ray;
                ray.o = V(w->position[0], w->position[1], w->position[2]);
                if (w->source_kind == OWEC_SOURCE_POINT) {
                    const double cosT = (1 - u.u1) + u.u1 * cosMax, sinT = safeSqrt(1 - cosT * cosT), phi = 2 * Pi * u.u2;
                    ray.d = S * (std::cos(phi) * sinT) + T * (std::sin(phi) * sinT) + axis * cosT;
                } else if (w->source_kind == OWEC_SOURCE_COLLIMATED) {
                    const double a = 2 * u.u1 - 1, bb = 2 * u.u2 - 1;
                    double dx = 0, dy = 0;
                    if (!(a == 0 && bb == 0)) {
                        double r, phi;
                        if (std::fabs(a) > std::fabs(bb)) { r = a; phi = (Pi / 4) * (bb / a); }
                        else { r = bb; phi = Pi / 2 - (Pi / 4) * (a / bb); }
                        dx = r * std::cos(phi);
                        dy = r * std::sin(phi);
                    }
                    ray.o = ray.o + (S * dx + T * dy) * w->extent;
                    ray.d = axis;
                } else {
                    ray.o = ray.o + (S * (2 * u.u1 - 1) + T * (2 * u.u2 - 1)) * w->extent;
                    ray.d = axis;
                }
                const Tracer::WalkEnd end = tr.walk(ray, w->region, lambda, w->mode == OWEC_WALK_PRIMARY_TRANSMISSION, rng,
                                                    w->max_events);
                st[size_t(t)][0]++;
                st[size_t(t)][3] += uint64_t(end.events);
                if (end.kind == 0) { st[size_t(t)][2]++; continue; }
                if (end.kind != 1 || end.boundary != w->target) continue;
                const V pl = target.toLocal.point(end.p);
                const double fx = (pl.x / w->half_x + 1) * 0.5 * w->width, fy = (1 - pl.y / w->half_y) * 0.5 * w->height;
                bool any = false;
                if (w->splat == OWEC_SPLAT_NEAREST) {
                    if (fx >= 0 && fy >= 0 && fx < w->width && fy < w->height) {
                        part[size_t(t)][size_t(int(fy)) * w->width + size_t(int(fx))] += end.beta;
                        any = true;
                    }
                } else {
                    const double gx = fx - 0.5, gy = fy - 0.5;
                    const int x0 = int(std::floor(gx)), y0 = int(std::floor(gy));
                    const double ax = gx - x0, ay = gy - y0;
                    for (int j = 0; j < 2; ++j)
                        for (int i = 0; i < 2; ++i) {
                            const int xi = x0 + i, yj = y0 + j;
                            if (xi < 0 || yj < 0 || xi >= w->width || yj >= w->height) continue;
                            part[size_t(t)][size_t(yj) * w->width + size_t(xi)] += end.beta * (i ? ax : 1 - ax) * (j ? ay : 1 - ay);
                            any = true;
                        }
                }
                if (any) st[size_t(t)][1]++;
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
        for (size_t i = 0; i < nb; ++i)
            for (int t = 0; t < threads; ++t) bins[i] += part[size_t(t)][i];
        for (int k = 0; k < 4; ++k) {
            stats[k] = 0;
            for (int t = 0; t < threads; ++t) stats[k] += st[size_t(t)][size_t(k)];
        }
        return 0;
    } catch (const std::exception& e) {
        oracle::g_error = e.what();
        return -1;
    }
}

// The light-selection probabilities of the restated light table.
int oweport_light_pdfs(void* scene, double* out, int max, int* n) {
    const auto& sc = *static_cast<const oracle::Scene*>(scene);
    *n = int(sc.lightPdf.size());
    for (int i = 0; i < std::min(max, *n); ++i) out[i] = sc.lightPdf[size_t(i)];
    return 0;
}

}  // extern "C"
