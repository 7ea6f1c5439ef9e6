// Host runtime of the CUDA backend and its C ABI (include/owec.h).
//
// A context owns one stream and everything on the device: the flattened scene, the wide BVH, the
// path state of a batch of samples, the queues and the film. owec_upload_scene restates the parts of
// World::build the kernels need (src/owe/scene/world.cpp:263-350: frames, world boxes, the scene
// radius and the light table) and converts the geometry to camera-relative FP32. owec_pass runs
// batches of one-sample sub-passes through the wavefront loop and folds them into the film.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "bvh_build.hpp"
#include "owec.h"
#include "particle.hpp"
#include "spectral.cuh"
#include "path_adjoint.hpp"
#include "peaks.hpp"
#include "walk.hpp"
#include "wavefront.hpp"

using namespace owec;

namespace {

thread_local std::string g_error = "no error";

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& w) : std::runtime_error(w), code(c) {}
};

// ------------------------------------------------------------------ host restatements of World::build parts
double hostCieY(double l) { return cieY(l); }

// Composite Simpson over [360, 830] nm in 0.5 nm steps (spectrum.cpp:10-17).
template <class F>
double integrateVisible(F f) {
    const int n = int((kLambdaMax - kLambdaMin) * 2);
    const double h = (kLambdaMax - kLambdaMin) / n;
    double s = f(kLambdaMin) + f(kLambdaMax);
    for (int i = 1; i < n; ++i) s += f(kLambdaMin + i * h) * ((i & 1) ? 4 : 2);
    return s * h / 3;
}

double cieYIntegralHost() {
    static const double v = integrateVisible([](double l) { return hostCieY(l); });
    return v;
}

double evalSpectrumHost(const owec_scene_desc& d, int32_t idx, double l) {
    if (idx < 0) return 0;
    const owec_spectrum& s = d.spectra[idx];
    if (s.kind == OWEC_SPEC_CONSTANT) return s.a;
    if (s.kind == OWEC_SPEC_BLACKBODY) return s.scale * planck(l, s.a);
    const double* t = d.spectrum_table + 2 * s.table_offset;
    const int n = s.table_count;
    if (l <= t[0]) return s.scale * t[1];
    if (l >= t[2 * (n - 1)]) return s.scale * t[2 * (n - 1) + 1];
    int i = 1;
    while (i < n && t[2 * i] <= l) ++i;
    const double u = (l - t[2 * (i - 1)]) / (t[2 * i] - t[2 * (i - 1)]);
    return s.scale * (t[2 * (i - 1) + 1] * (1 - u) + t[2 * i + 1] * u);
}

// Spectrum::luminance (spectrum.cpp:165-167).
double luminanceHost(const owec_scene_desc& d, int32_t idx) {
    return integrateVisible([&](double l) { return evalSpectrumHost(d, idx, l) * hostCieY(l); }) / cieYIntegralHost();
}

struct Box {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void expand(const double p[3]) {
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    bool valid() const { return lo[0] <= hi[0] && lo[1] <= hi[1] && lo[2] <= hi[2]; }
};

void xfPoint(const double m[12], const double p[3], double out[3]) {
    for (int i = 0; i < 3; ++i) out[i] = m[4 * i] * p[0] + m[4 * i + 1] * p[1] + m[4 * i + 2] * p[2] + m[4 * i + 3];
}

// The sag's z range over the aperture (SagSurface's constructor, geometry.cpp:70-88); A: the even
// asphere terms A4, A6, ...
void sagZRange(double c, double k, double rMax, double rMin, const double* A, uint32_t nA, double& zMin, double& zMax) {
    zMin = INFINITY;
    zMax = -INFINITY;
    const int N = 512;
    for (int i = 0; i <= N; ++i) {
        const double r = rMin + (rMax - rMin) * i / N;
        const double r2 = r * r;
        double z = c * r2 / (1 + std::sqrt(std::max(0.0, 1 - (1 + k) * c * c * r2)));
        double rp = r2 * r2;
        for (uint32_t j = 0; j < nA; ++j) { z += A[j] * rp; rp *= r2; }
        zMin = std::min(zMin, z);
        zMax = std::max(zMax, z);
    }
    const double pad = 1e-9 + 1e-3 * (zMax - zMin);
    zMin -= pad;
    zMax += pad;
}

// A torus patch's extent (TorusPatchShape's constructor, geometry.cpp:557-577): ext = rMax, zMin,
// zMax of the arc a0..a1 of radius rho about (R, zc), and the arc's upper end.
void torusExtent(double R, double zc, double rho, double a0, double a1, double ext[4]) {
    const double lo = std::min(a0, a1), hi = std::max(a0, a1);
    double rMax = -INFINITY, zMin = INFINITY, zMax = -INFINITY;
    auto add = [&](double a) {
        rMax = std::max(rMax, R + rho * std::cos(a));
        const double z = zc + rho * std::sin(a);
        zMin = std::min(zMin, z);
        zMax = std::max(zMax, z);
    };
    add(lo);
    add(hi);
    for (int k = -4; k <= 4; ++k) {  // the extremes of cos and sin inside the range
        const double a = k * kPi / 2;
        if (a > lo && a < hi) add(a);
    }
    ext[0] = rMax;
    ext[1] = zMin;
    ext[2] = zMax;
    ext[3] = hi;
}

// A wave surface's derived record (WaveSurface's constructor, geometry.cpp:190-221): the margin
// clamped to the half sizes, the amplitude bound (the sum of |a|), the slope bound (the sum of |a| k,
// plus the taper's share), and, for a sampled surface, the node spacings, the nodes (h, dh/dx,
// dh/dy, d2h/dxdy, row by row) and the slope bound tightened to the nodes' largest slope plus the
// curvature bound over half a cell diagonal. P: halfX, halfY, margin; D: nodes x, nodes y, waves.
struct WaveSetup {
    double margin = 0, amp = 0, slope = 0, dx = 0, dy = 0;
    std::vector<double> nodes;
};
WaveSetup waveSetup(const double* P, const double* D, uint32_t count) {
    WaveSetup w;
    const double hx = P[0], hy = P[1];
    w.margin = std::max(0.0, std::min({P[2], hx, hy}));
    const int nW = int((count - 2) / 4);
    const double* waves = D + 2;
    double slope = 0, curvature = 0;
    for (int i = 0; i < nW; ++i) {
        const double a = std::fabs(waves[4 * i]), k = std::hypot(waves[4 * i + 1], waves[4 * i + 2]);
        w.amp += a;
        slope += a * k;
        curvature += a * k * k;
    }
    const double taper = w.margin > 0 ? 1.5 * std::sqrt(2.0) / w.margin : 0;
    w.slope = slope + w.amp * taper;
    const int nx = int(D[0]), ny = int(D[1]);
    if (nx == 0) return w;
    w.dx = 2 * hx / (nx - 1);
    w.dy = 2 * hy / (ny - 1);
    w.nodes.resize(size_t(4) * nx * ny);
    double nodeSlope = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            double* n = w.nodes.data() + 4 * (size_t(j) * nx + i);
            waveAnalytic<double>(waves, nW, hx, hy, w.margin, -hx + i * w.dx, -hy + j * w.dy, n[0], n[1], n[2], n[3]);
            nodeSlope = std::max(nodeSlope, std::hypot(n[1], n[2]));
        }
    const double hessian = curvature + 2 * taper * slope + (w.margin > 0 ? 6 * w.amp / (w.margin * w.margin) : 0);
    w.slope = std::min(w.slope, 1.05 * (nodeSlope + hessian * 0.5 * std::hypot(w.dx, w.dy)));
    return w;
}

// A shape's bounds in its frame (Shape::bounds of the reference's shapes).
Box localBounds(const owec_scene_desc& d, const owec_boundary& b) {
    Box bx;
    const double* P = b.params;
    auto put = [&](double x0, double y0, double z0, double x1, double y1, double z1) {
        const double a[3] = {x0, y0, z0}, c[3] = {x1, y1, z1};
        bx.expand(a);
        bx.expand(c);
    };
    switch (b.shape) {
        case OWEC_SHAPE_SPHERE: put(-P[0], -P[0], -P[0], P[0], P[0], P[0]); break;
        case OWEC_SHAPE_SAG: {
            double zMin, zMax;
            sagZRange(P[0], P[1], P[2], P[3], d.shape_data + b.data_offset, b.data_count, zMin, zMax);
            put(-P[2], -P[2], zMin, P[2], P[2], zMax);
            break;
        }
        case OWEC_SHAPE_CONE: {
            const double R = std::max(P[0], P[2]);
            put(-R, -R, std::min(P[1], P[3]), R, R, std::max(P[1], P[3]));
            break;
        }
        case OWEC_SHAPE_TORUS: {
            double ext[4];
            torusExtent(P[0], P[1], P[2], P[3], d.shape_data[b.data_offset], ext);
            put(-ext[0], -ext[0], ext[1], ext[0], ext[0], ext[2]);
            break;
        }
        case OWEC_SHAPE_ROUND_WALL: put(-P[0], -P[0], 0, P[0], P[0], P[1]); break;
        case OWEC_SHAPE_DOME: put(-P[0], -P[0], 0, P[0], P[0], P[0]); break;
        case OWEC_SHAPE_WAVES: {
            double amp = 0;
            for (uint32_t i = 2; i + 3 < b.data_count; i += 4) amp += std::fabs(d.shape_data[b.data_offset + i]);
            put(-P[0], -P[1], -amp, P[0], P[1], amp);
            break;
        }
        case OWEC_SHAPE_PLANE: {
            const int ap = int(P[0]);
            const double ex = P[1], ey = (ap == OWEC_APERTURE_DISK || ap == OWEC_APERTURE_DISK_HOLE) ? P[1] : P[2];
            const double pad = 1e-9 * (1 + std::max(ex, ey));
            put(-ex, -ey, -pad, ex, ey, pad);
            break;
        }
        case OWEC_SHAPE_CYLINDER: put(-P[0], -P[0], std::min(P[1], P[2]), P[0], P[0], std::max(P[1], P[2])); break;
        case OWEC_SHAPE_MESH: {
            const owec_mesh& m = d.meshes[b.mesh];
            for (uint64_t t = 0; t < m.tri_count; ++t) {
                const uint32_t* tri = d.triangles + 3 * (m.tri_offset + t);
                Box tb;
                for (int k = 0; k < 3; ++k) tb.expand(d.vertices + 3 * (m.vertex_offset + tri[k]));
                const double pad = 1e-12 * (1 + std::max({std::fabs(tb.hi[0]), std::fabs(tb.hi[1]), std::fabs(tb.hi[2])}) +
                                            std::max({std::fabs(tb.lo[0]), std::fabs(tb.lo[1]), std::fabs(tb.lo[2])}));
                for (int k = 0; k < 3; ++k) { tb.lo[k] -= pad; tb.hi[k] += pad; }
                bx.expand(tb.lo);
                bx.expand(tb.hi);
            }
            break;
        }
    }
    return bx;
}

Box worldBox(const Box& local, const double m[12]) {
    Box w;
    for (int i = 0; i < 8; ++i) {
        const double c[3] = {(i & 1) ? local.hi[0] : local.lo[0], (i & 2) ? local.hi[1] : local.lo[1],
                             (i & 4) ? local.hi[2] : local.lo[2]};
        double p[3];
        xfPoint(m, c, p);
        w.expand(p);
    }
    return w;
}

double shapeArea(const owec_scene_desc& d, const owec_boundary& b, bool& canSample) {
    const double* P = b.params;
    canSample = true;
    switch (b.shape) {
        case OWEC_SHAPE_SPHERE: return 4 * kPi * P[0] * P[0];
        case OWEC_SHAPE_PLANE: {
            const int ap = int(P[0]);
            if (ap == OWEC_APERTURE_DISK_HOLE) {  // no area sampler (PlaneShape::canSample)
                canSample = false;
                return kPi * (P[1] * P[1] - P[2] * P[2]);
            }
            if (ap == OWEC_APERTURE_DISK) return kPi * (P[1] * P[1] - P[2] * P[2]);
            if (ap == OWEC_APERTURE_RECT) return 4 * P[1] * P[2];
            return kPi * P[1] * P[2];
        }
        case OWEC_SHAPE_SAG:
            canSample = P[0] == 0 && b.data_count == 0;  // only a flat sag has an area sampler
            return kPi * (P[2] * P[2] - P[3] * P[3]);
        case OWEC_SHAPE_CYLINDER: return 2 * kPi * P[0] * std::fabs(P[2] - P[1]);
        default: canSample = false; return 0;  // emitting meshes are not sampled by next-event estimation here
    }
}

// A primitive's box in FP32, padded outward by a relative 1e-6 (so the FP32 traversal of rays
// rounded to FP32 stays conservative) and rounded outward.
void padPrimBox(const double lo[3], const double hi[3], float4& flo, float4& fhi) {
    double ext = 0, mag = 0;
    for (int k = 0; k < 3; ++k) {
        ext = std::max(ext, hi[k] - lo[k]);
        mag = std::max({mag, std::fabs(lo[k]), std::fabs(hi[k])});
    }
    const double pad = 1e-6 * (mag + ext) + 1e-9;
    flo = make_float4(std::nextafter(float(lo[0] - pad), -INFINITY), std::nextafter(float(lo[1] - pad), -INFINITY),
                      std::nextafter(float(lo[2] - pad), -INFINITY), 0.f);
    fhi = make_float4(std::nextafter(float(hi[0] + pad), INFINITY), std::nextafter(float(hi[1] + pad), INFINITY),
                      std::nextafter(float(hi[2] + pad), INFINITY), 0.f);
}

// Whether the scene has contacts the lean traversal would resolve differently from the reference:
// faces of two boundaries in one plane (bodies that touch, a sheet under a box), or parallel faces
// closer than the FP32 anchor error `tol` (plates thinner than it). Mesh triangles and plane shapes
// are keyed by their world plane (the normal, signed so its largest component is positive, rounded
// to 1e-6, then the offset); neighbours in key order with the same normal are compared.
bool hasContacts(const owec_scene_desc& d, double tol) {
    struct Plane {
        int64_t k[3];
        double off;
        uint32_t boundary;
        bool flipped;  // the face's normal points against the key's
    };
    std::vector<Plane> planes;
    auto add = [&](double n[3], const double p[3], uint32_t b) {
        const double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (!(l > 0)) return;
        int big = 0;
        for (int k = 1; k < 3; ++k)
            if (std::fabs(n[k]) > std::fabs(n[big])) big = k;
        const double s = (n[big] < 0 ? -1.0 : 1.0) / l;
        Plane pl;
        for (int k = 0; k < 3; ++k) pl.k[k] = int64_t(std::llround(n[k] * s * 1e6));
        pl.off = (n[0] * p[0] + n[1] * p[1] + n[2] * p[2]) * s;
        pl.boundary = b;
        pl.flipped = n[big] < 0;
        planes.push_back(pl);
    };
    std::vector<double> sphere;  // centre and radius of every sphere, with its boundary
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        const double* m = b.to_world;
        if (b.shape == OWEC_SHAPE_MESH) {
            const owec_mesh& me = d.meshes[b.mesh];
            for (uint64_t t = 0; t < me.tri_count; ++t) {
                const uint32_t* tri = d.triangles + 3 * (me.tri_offset + t);
                double w[3][3];
                for (int k = 0; k < 3; ++k) xfPoint(m, d.vertices + 3 * (me.vertex_offset + tri[k]), w[k]);
                const double e1[3] = {w[1][0] - w[0][0], w[1][1] - w[0][1], w[1][2] - w[0][2]};
                const double e2[3] = {w[2][0] - w[0][0], w[2][1] - w[0][1], w[2][2] - w[0][2]};
                double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
                add(n, w[0], i);
            }
        } else if (b.shape == OWEC_SHAPE_PLANE) {
            double n[3] = {m[2], m[6], m[10]};
            const double c[3] = {m[3], m[7], m[11]};
            add(n, c, i);
        } else if (b.shape == OWEC_SHAPE_SPHERE) {
            sphere.insert(sphere.end(), {m[3], m[7], m[11], b.params[0], double(i)});
        }
    }
    std::sort(planes.begin(), planes.end(), [](const Plane& a, const Plane& b) {
        if (a.k[0] != b.k[0]) return a.k[0] < b.k[0];
        if (a.k[1] != b.k[1]) return a.k[1] < b.k[1];
        if (a.k[2] != b.k[2]) return a.k[2] < b.k[2];
        return a.off < b.off;
    });
    for (size_t i = 1; i < planes.size(); ++i) {
        const Plane &a = planes[i - 1], &b = planes[i];
        if (a.k[0] != b.k[0] || a.k[1] != b.k[1] || a.k[2] != b.k[2]) continue;
        const double gap = b.off - a.off;
        if (gap > tol) continue;
        if (a.boundary != b.boundary) return true;  // two bodies' faces in one plane
        // a body thinner than the anchor error: its two faces, facing apart (adjacent faces of a
        // smooth mesh that are nearly coplanar face the same way)
        if (a.flipped != b.flipped && gap > 1e-12 * (1 + std::fabs(a.off))) return true;
    }
    for (size_t i = 0; i < sphere.size(); i += 5)
        for (size_t j = i + 5; j < sphere.size(); j += 5) {
            const double dc = std::sqrt(sqr(sphere[i] - sphere[j]) + sqr(sphere[i + 1] - sphere[j + 1]) +
                                        sqr(sphere[i + 2] - sphere[j + 2]));
            if (std::fabs(sphere[i + 3] - sphere[j + 3]) <= tol && dc <= tol) return true;  // one sphere twice
        }
    return false;
}

void invertRigid(const double m[12], double out[12]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[4 * i + j] = m[4 * j + i];
    for (int i = 0; i < 3; ++i)
        out[4 * i + 3] = -(out[4 * i] * m[3] + out[4 * i + 1] * m[7] + out[4 * i + 2] * m[11]);
}

}  // namespace

// ------------------------------------------------------------------ the context
struct owec_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t passStart = nullptr, passStop = nullptr;
    std::vector<cudaEvent_t> travEvents;
    int numSMs = 148;
    char name[256] = {0};

    // scene (host)
    bool hasScene = false, bvhDirty = true;
    owec_scene_desc descCopy{};
    std::vector<owec_spectrum> spectra;
    std::vector<double> table;
    std::vector<owec_medium> media;
    std::vector<uint32_t> regionMedium;
    std::vector<owec_optics> optics;
    std::vector<owec_emission> emissions;
    std::vector<DBoundary> boundaries;
    std::vector<DLight> lights;
    std::vector<float4> primLo, primHi, triRecs;
    std::vector<uint32_t> triBase;       // first primitive of each mesh boundary
    std::vector<uint64_t> triCount;      // its triangle count
    std::vector<double> tri64;
    uint32_t nTriangles = 0, nPrims = 0;
    bool hasNull = false;
    DeviceScene ds{};
    DBuf<DeviceScene> dScene;  // ds's copy on the device (DeviceScene::self), allocated when the context opens
    bool contacts = false;  // touching bodies or plates thinner than the FP32 anchor error
    // particles: the sky's share of the emitted power and the disc distant light leaves from
    double pSky = 0, discRadius = 1, discCentre[3] = {0, 0, 0};

    // scene (device)
    DBuf<owec_spectrum> dSpectra;
    DBuf<double> dTable;
    DBuf<owec_medium> dMedia;
    DBuf<uint32_t> dRegionMedium;
    DBuf<owec_optics> dOptics;
    DBuf<owec_emission> dEmissions;
    DBuf<DBoundary> dBoundaries;
    DBuf<DLight> dLights;
    std::vector<double> shapeData;  // the scene's shape data, then the nodes of sampled wave surfaces
    DBuf<double> dShapeData;
    DBuf<float4> dPrimLo, dPrimHi, dTri;
    DBuf<double> dTri64;
    BvhScratch scratch;
    DBuf<WideNode> dNodes;
    DBuf<uint32_t> dLeafOrder;
    DBuf<PrimRec> dPrims;
    DBuf<PrimRec64> dPrims64;
    uint32_t nNodes = 0;
    bool prims64Ready = false;

    // rendering
    owec_settings settings{1, 64, 6, OWEC_WAVELENGTHS_HERO4, OWEC_PRECISION_MIXED, 380, 780, 0, OWEC_INTEGRATOR_PATH, 0};
    uint64_t passCount = 0;  // samples per pixel accumulated (the PCG32 stream of the next sample)
    DBuf<double> dFilm, dComp, dSamples;
    DBuf<double> dResolved;  // owec_resolve's per-pixel XYZ, read back in one copy
    // owec_resolve_async: two device images (XYZ, then samples) that a copy stream reads back while
    // later passes run, each read-back ordered after its image by an event
    cudaStream_t copyStream = nullptr;
    cudaEvent_t resolvedEv[2] = {nullptr, nullptr};
    DBuf<double> dResolvedAsync[2];
    int asyncSlot = 0;
    DBuf<unsigned long long> dSplat;  // the light integrator's film: fixed-point splat sums
    double particles = 0;             // particles emitted into it
    DBuf<uint8_t> dPathRay, dPathSpec, dPathAux, dHit, dShadow;
    DBuf<uint32_t> dQueue0, dQueue1, dQueueSurf, dQueueSurfSimple, dQueueShadow, dCounts;
    DBuf<uint8_t> dShadowVis;  // per shadow-queue entry: 0 blocked, 1 clear, 2 fault
    DBuf<uint32_t> dShadowPixel;  // light integrator: the pixel of each queued connection
    DBuf<StatCounters> dStats;
    DBuf<unsigned long long> dTravCounters;
    // while counting: the query counter after each closest-hit launch of the last pass
    static constexpr int kLaunchLog = 256;
    DBuf<unsigned long long> dLaunchQueries;
    int launchQueryCount = 0;
    // the inconsistent-crossing log (owec_inconsistency_log)
    DBuf<double> dEventLog;
    DBuf<uint32_t> dEventLogCount;
    uint32_t eventLogCap = 0;
    uint32_t capacity = 0;
    double lastPassSeconds = 0, lastIntersectSeconds = 0, lastShadowSeconds = 0, lastIntersectLaunches = 0;
    uint32_t* hostCounts = nullptr;  // pinned

    // the heightfield the adjoint differentiates
    HeightfieldParams hf{kNone, nullptr, {0, 0, 1}};
    uint64_t hfVertices = 0;
    double lastPathAdjointSeconds = 0;
    DBuf<uint32_t> dHfTris;
    struct MeshCopy {
        std::vector<double> verts;    // shape-frame vertices as uploaded
        std::vector<uint32_t> tris;
    };
    std::vector<MeshCopy> meshes;    // per boundary (empty for analytic ones)
    double lastWalkSeconds = 0, lastAdjointSeconds = 0;

    // forward light walks
    owec_walk_desc walk{};
    bool hasWalk = false;
    uint64_t walks = 0;
    DBuf<unsigned long long> dWalkBins, dWalkStats;
};

namespace {

template <class F>
int guarded(F&& f) {
    try {
        f();
        return OWEC_OK;
    } catch (const Error& e) {
        g_error = e.what();
        return e.code;
    } catch (const CudaError& e) {
        g_error = e.what();
        return e.code == cudaErrorMemoryAllocation ? OWEC_E_NOMEM : OWEC_E_CUDA;
    } catch (const std::bad_alloc&) {
        g_error = "host allocation failed";
        return OWEC_E_NOMEM;
    } catch (const std::exception& e) {
        g_error = e.what();
        return OWEC_E_INVALID;
    }
}

void require(bool ok, const std::string& why, int code = OWEC_E_INVALID) {
    if (!ok) throw Error(code, why);
}

void checkLaunch() {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError(e, std::string("kernel launch: ") + cudaGetErrorString(e));
}

void validateDesc(const owec_scene_desc& d) {
    require(d.abi_version == OWEC_ABI_VERSION, "scene description ABI version mismatch");
    require(d.n_regions >= 1 && d.region_medium, "a scene needs its ambient region");
    for (uint32_t r = 0; r < d.n_regions; ++r) require(d.region_medium[r] < d.n_media, "region medium out of range");
    auto specOk = [&](int32_t s) { return s < 0 || uint32_t(s) < d.n_spectra; };
    for (uint32_t i = 0; i < d.n_spectra; ++i) {
        const owec_spectrum& s = d.spectra[i];
        require(s.kind >= OWEC_SPEC_CONSTANT && s.kind <= OWEC_SPEC_BLACKBODY, "unknown spectrum kind");
        if (s.kind == OWEC_SPEC_TABULATED)
            require(s.table_count >= 1 && uint64_t(s.table_offset) + s.table_count <= d.n_spectrum_table,
                    "tabulated spectrum out of the table");
    }
    for (uint32_t i = 0; i < d.n_media; ++i) {
        const owec_medium& m = d.media[i];
        require(m.index_kind >= OWEC_INDEX_CONSTANT && m.index_kind <= OWEC_INDEX_TABULATED, "unknown index model");
        require(m.index_kind != OWEC_INDEX_SELLMEIER || (m.n_terms >= 1 && m.n_terms <= OWEC_MAX_SELLMEIER_TERMS),
                "Sellmeier needs 1 to 4 terms");
        require(specOk(m.absorption) && specOk(m.scattering), "medium spectrum out of range");
        require(m.index_kind != OWEC_INDEX_TABULATED || (m.index_table >= 0 && specOk(m.index_table)),
                "tabulated index needs a spectrum");
    }
    for (uint32_t i = 0; i < d.n_optics; ++i) {
        const owec_optics& o = d.optics[i];
        require(o.type >= OWEC_SURF_NULL && o.type <= OWEC_SURF_DETECTOR, "unknown surface type");
        require(specOk(o.reflectance) && specOk(o.conductor_n) && specOk(o.conductor_k), "optics spectrum out of range");
        require(o.texture >= OWEC_TEXTURE_NONE && o.texture <= OWEC_TEXTURE_MARBLE, "unknown texture");
        require(o.texture == OWEC_TEXTURE_NONE ||
                    (o.type == OWEC_SURF_DIFFUSE && o.reflectance >= 0 && o.texture_b >= 0 && specOk(o.texture_b) &&
                     o.texture_c >= 0 && specOk(o.texture_c) && o.texture_scale > 0),
                "a texture needs a Lambertian surface, its three spectra and a positive scale");
        if (o.aim_share != 0) {
            const double nl = std::sqrt(o.aim_normal[0] * o.aim_normal[0] + o.aim_normal[1] * o.aim_normal[1] +
                                        o.aim_normal[2] * o.aim_normal[2]);
            require(o.type == OWEC_SURF_DIFFUSE && o.aim_share > 0 && o.aim_share <= 1 && o.aim_radius > 0 && nl > 0 &&
                        std::isfinite(o.aim_center[0] + o.aim_center[1] + o.aim_center[2]),
                    "an aim guide needs a Lambertian surface, a share in (0, 1], a disk radius and a normal");
        }
    }
    for (uint32_t i = 0; i < d.n_emissions; ++i) require(specOk(d.emissions[i].radiance) && d.emissions[i].radiance >= 0,
                                                          "emission needs a radiance spectrum");
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        require(b.shape >= OWEC_SHAPE_SPHERE && b.shape <= OWEC_SHAPE_WAVES, "unknown shape");
        require(b.data_count == 0 || (d.shape_data && uint64_t(b.data_offset) + b.data_count <= d.n_shape_data),
                "shape data out of range");
        const double* P = b.params;
        const double* D = b.data_count ? d.shape_data + b.data_offset : nullptr;
        switch (b.shape) {
            case OWEC_SHAPE_SPHERE: require(P[0] > 0, "sphere: radius must be positive"); break;
            case OWEC_SHAPE_PLANE:
                require(P[0] >= OWEC_APERTURE_DISK && P[0] <= OWEC_APERTURE_DISK_HOLE, "plane: unknown aperture");
                if (int(P[0]) == OWEC_APERTURE_DISK_HOLE)
                    require(b.data_count == 2 && P[1] > 0 && P[2] > 0 && std::hypot(D[0], D[1]) + P[2] < P[1],
                            "disk with hole: the hole must lie inside the disk");
                break;
            case OWEC_SHAPE_CONE:
                require(std::fabs(P[3] - P[1]) > 0 && P[0] >= 0 && P[2] >= 0, "cone: needs z0 != z1 and radii >= 0");
                break;
            case OWEC_SHAPE_TORUS: {
                require(b.data_count == 1, "torus patch: its data is the arc's end angle");
                require(P[2] > 0 && std::fabs(D[0] - P[3]) <= kPi + 1e-12, "torus patch: invalid arc");
                double rMin = INFINITY;
                for (double a : {std::min(P[3], D[0]), std::max(P[3], D[0])}) rMin = std::min(rMin, P[0] + P[2] * std::cos(a));
                for (int k = -4; k <= 4; ++k) {
                    const double a = k * kPi / 2;
                    if (a > std::min(P[3], D[0]) && a < std::max(P[3], D[0])) rMin = std::min(rMin, P[0] + P[2] * std::cos(a));
                }
                require(rMin >= -1e-12 * P[2], "torus patch: the arc crosses the axis");
                break;
            }
            case OWEC_SHAPE_ROUND_WALL:
                require(P[0] > 0 && P[1] > 0 && b.data_count % 4 == 0, "round wall: radius, height and openings");
                break;
            case OWEC_SHAPE_DOME: require(P[0] > 0, "dome: radius must be positive"); break;
            case OWEC_SHAPE_WAVES: {
                require(P[0] > 0 && P[1] > 0 && std::isfinite(P[0]) && std::isfinite(P[1]) && P[2] >= 0,
                        "wave surface: positive half sizes and a margin >= 0");
                require(b.data_count >= 2 && (b.data_count - 2) % 4 == 0,
                        "wave surface: its data is the node counts and (amplitude, kx, ky, phase) per wave");
                const double nx = D[0], ny = D[1];
                const bool analytic = nx == 0 && ny == 0;
                const bool sampled = nx == std::floor(nx) && ny == std::floor(ny) && nx >= 2 && ny >= 2 && nx <= 4096 &&
                                     ny <= 4096;
                require(analytic || sampled, "wave surface: node counts are 0 (analytic) or 2..4096");
                for (uint32_t k = 2; k < b.data_count; ++k) require(std::isfinite(D[k]), "wave surface: waves must be finite");
                break;
            }
            default: break;
        }
        require(b.front < d.n_regions && b.back < d.n_regions, "boundary region out of range");
        require(b.optics < d.n_optics, "boundary optics out of range");
        require(b.emission < 0 || uint32_t(b.emission) < d.n_emissions, "boundary emission out of range");
        if (b.shape == OWEC_SHAPE_MESH) {
            require(b.mesh >= 0 && uint32_t(b.mesh) < d.n_meshes, "mesh index out of range");
            const owec_mesh& m = d.meshes[b.mesh];
            require(m.vertex_offset + m.vertex_count <= d.n_vertices && m.tri_offset + m.tri_count <= d.n_triangles,
                    "mesh out of the vertex or triangle arrays");
            for (uint64_t t = 0; t < m.tri_count; ++t)
                for (int k = 0; k < 3; ++k)
                    require(d.triangles[3 * (m.tri_offset + t) + k] < m.vertex_count, "triangle index out of range");
        }
        if (b.shape == OWEC_SHAPE_SAG) {
            const double c = b.params[0], k = b.params[1], rMax = b.params[2], rMin = b.params[3];
            require(rMax > 0 && rMin >= 0 && rMin < rMax, "sag surface: invalid aperture radii");
            require(1 - (1 + k) * c * c * rMax * rMax >= 0, "sag surface: aperture exceeds the conic's domain");
        }
        if ((d.optics[b.optics].type == OWEC_SURF_DIELECTRIC || d.optics[b.optics].type == OWEC_SURF_NULL))
            require(!d.media[d.region_medium[b.front]].opaque && !d.media[d.region_medium[b.back]].opaque,
                    "a transmissive boundary borders an opaque medium");
    }
    const owec_detector& det = d.detector;
    require(det.width > 0 && det.height > 0 && uint64_t(det.width) * det.height <= (1ull << 28),
            "detector resolution out of range");
    require(det.kind == OWEC_DETECTOR_OBSERVER || det.kind == OWEC_DETECTOR_SENSOR, "unknown detector kind");
    if (det.kind == OWEC_DETECTOR_SENSOR) {
        require(det.boundary < d.n_boundaries, "sensor boundary out of range");
        require(det.half_x > 0 && det.half_y > 0, "sensor needs a size");
    } else {
        require(det.region < d.n_regions, "observer region out of range (the engine locates it before flattening)");
        require(det.fov_y > 0 && det.fov_y < kPi, "observer field of view out of range");
        require(det.pupil_radius >= 0 && !(det.focus_distance < 0) && det.guide_radius >= 0 && det.guide_share >= 0 &&
                    det.guide_share < 1, "observer: pupil, focus or guide out of range");
    }
    require(d.env.sky_model == OWEC_SKY_NONE || d.env.sky_model == OWEC_SKY_UNIFORM || d.env.sky_model == OWEC_SKY_GRADIENT,
            "unknown sky model");
    require(d.env.sky_model != OWEC_SKY_GRADIENT ||
                (d.env.sky_radiance >= 0 && d.env.sky_horizon >= 0 && specOk(d.env.sky_horizon) && d.env.sky_ground >= 0 &&
                 specOk(d.env.sky_ground)),
            "a gradient sky needs its zenith, horizon and ground spectra");
    require(specOk(d.env.sky_radiance) && specOk(d.env.sun_radiance), "environment spectrum out of range");
}

void uploadScene(owec_ctx& c, const owec_scene_desc& d) {
    validateDesc(d);
    cudaStream_t s = c.stream;
    c.spectra.assign(d.spectra, d.spectra + d.n_spectra);
    c.table.assign(d.spectrum_table, d.spectrum_table + 2 * d.n_spectrum_table);
    c.media.assign(d.media, d.media + d.n_media);
    c.regionMedium.assign(d.region_medium, d.region_medium + d.n_regions);
    c.optics.assign(d.optics, d.optics + d.n_optics);
    c.emissions.assign(d.emissions, d.emissions + d.n_emissions);
    c.shapeData.assign(d.shape_data, d.shape_data + (d.shape_data ? d.n_shape_data : 0));

    // The camera-relative origin: the one given, the observer's position, or the sensor's centre.
    double origin[3];
    if (d.frame_origin_set) {
        for (int k = 0; k < 3; ++k) origin[k] = d.frame_origin[k];
    } else if (d.detector.kind == OWEC_DETECTOR_OBSERVER) {
        for (int k = 0; k < 3; ++k) origin[k] = d.detector.position[k];
    } else {
        const double* m = d.boundaries[d.detector.boundary].to_world;
        origin[0] = m[3]; origin[1] = m[7]; origin[2] = m[11];
    }

    // Boundaries: frames relative to the origin, world boxes, emitter areas.
    Box scene;
    c.boundaries.resize(d.n_boundaries);
    std::vector<Box> wboxes(d.n_boundaries);
    c.hasNull = false;
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        DBoundary& db = c.boundaries[i];
        db.shape = b.shape;
        db.emission = b.emission;
        db.front = b.front;
        db.back = b.back;
        db.optics = b.optics;
        db.light = -1;
        for (int k = 0; k < 12; ++k) db.toWorld.m[k] = b.to_world[k];
        wboxes[i] = worldBox(localBounds(d, b), b.to_world);
        scene.expand(wboxes[i].lo);
        scene.expand(wboxes[i].hi);
        db.toWorld.m[3] -= origin[0];
        db.toWorld.m[7] -= origin[1];
        db.toWorld.m[11] -= origin[2];
        invertRigid(db.toWorld.m, db.toLocal.m);
        for (int k = 0; k < 4; ++k) db.params[k] = b.params[k];
        db.dataOffset = b.data_offset;
        db.dataCount = b.data_count;
        for (double& e : db.ext) e = 0;
        if (b.shape == OWEC_SHAPE_SAG && b.data_count) {
            sagZRange(b.params[0], b.params[1], b.params[2], b.params[3], d.shape_data + b.data_offset, b.data_count,
                      db.ext[0], db.ext[1]);
        } else if (b.shape == OWEC_SHAPE_TORUS) {
            torusExtent(b.params[0], b.params[1], b.params[2], b.params[3], d.shape_data[b.data_offset], db.ext);
            db.params[3] = std::min(b.params[3], d.shape_data[b.data_offset]);
        } else if (b.shape == OWEC_SHAPE_WAVES) {
            const WaveSetup w = waveSetup(b.params, d.shape_data + b.data_offset, b.data_count);
            db.params[2] = w.margin;
            db.params[3] = double((b.data_count - 2) / 4);
            db.ext[0] = w.amp;
            db.ext[1] = w.slope;
            db.ext[2] = w.dx;
            db.ext[3] = w.dy;
            if (!w.nodes.empty()) {  // the record and its nodes, appended to the device copy of the data
                require(c.shapeData.size() + b.data_count + w.nodes.size() < (1ull << 32), "wave surface: too many nodes");
                db.dataOffset = uint32_t(c.shapeData.size());
                db.dataCount = uint32_t(b.data_count + w.nodes.size());
                c.shapeData.insert(c.shapeData.end(), d.shape_data + b.data_offset, d.shape_data + b.data_offset + b.data_count);
                c.shapeData.insert(c.shapeData.end(), w.nodes.begin(), w.nodes.end());
            }
        }
        bool canSample = false;
        db.area = shapeArea(d, b, canSample);
        if (!canSample) db.area = 0;
        db.scale = 0;
        for (int k = 0; k < 3; ++k) db.scale = std::max(db.scale, wboxes[i].hi[k] - wboxes[i].lo[k]);
        if (d.optics[b.optics].type == OWEC_SURF_NULL) c.hasNull = true;
    }
    double sceneRadius = 1.0, center[3] = {0, 0, 0};
    if (scene.valid()) {
        double e2 = 0;
        for (int k = 0; k < 3; ++k) {
            e2 += (scene.hi[k] - scene.lo[k]) * (scene.hi[k] - scene.lo[k]);
            center[k] = 0.5 * (scene.lo[k] + scene.hi[k]) - origin[k];
        }
        sceneRadius = std::max(1e-3, 0.5 * std::sqrt(e2));
    }

    // The light table (World::buildLightTable, world.cpp:285-350; no environment map here).
    c.lights.clear();
    std::vector<double> power;
    std::vector<int> distant;
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        if (b.emission < 0) continue;
        const owec_emission& e = d.emissions[b.emission];
        bool canSample = false;
        const double area = shapeArea(d, b, canSample);
        if (!canSample || !(area > 0) || !e.nee) continue;
        const double sides = (e.front ? 1 : 0) + (e.back ? 1 : 0);
        c.boundaries[i].light = int(c.lights.size());
        c.lights.push_back(DLight{kLightBoundary, i, 0, 0});
        power.push_back(std::max(1e-12, luminanceHost(d, e.radiance)) * area * kPi * sides);
        distant.push_back(e.distant);
    }
    const double cosMax = std::cos(d.env.sun_angular_radius);
    const double sunSolid = 2 * kPi * (1 - cosMax);
    if (d.env.has_sun) {
        c.lights.push_back(DLight{kLightSun, kNone, 0, 0});
        power.push_back(std::max(1e-12, luminanceHost(d, d.env.sun_radiance)) * sunSolid * kPi * sceneRadius * sceneRadius);
        distant.push_back(0);
    }
    double total = 0, boundaryPower = 0, nearbyPower = 0, distantPower = 0;
    for (size_t l = 0; l < c.lights.size(); ++l) {
        total += power[l];
        if (c.lights[l].kind == kLightBoundary) {
            boundaryPower += power[l];
            (distant[l] ? distantPower : nearbyPower) += power[l];
        }
    }
    double share = d.env.has_sun && boundaryPower > 0 ? std::min(0.999, std::max(0.0, d.env.sun_nee_share)) : 0;
    if (distantPower > 0 && d.env.has_sun && share == 0) share = 0.5;
    double acc = 0, sunSel = 0;
    for (size_t l = 0; l < c.lights.size(); ++l) {
        double p = total > 0 ? power[l] / total : 0;
        if (share > 0) p = c.lights[l].kind == kLightSun ? share : (1 - share) * power[l] / boundaryPower;
        if (distantPower > 0 && c.lights[l].kind == kLightBoundary) {
            const double groupShare = nearbyPower > 0 ? 0.5 : 1;
            p = (1 - share) * groupShare * power[l] / (distant[l] ? distantPower : nearbyPower);
        }
        c.lights[l].pdf = p;
        acc += p;
        c.lights[l].cdf = acc;
        if (c.lights[l].kind == kLightSun) sunSel = p;
    }
    if (!c.lights.empty()) c.lights.back().cdf = 1.0;

    // Particles: the sky's share of the emitted power (World::computeEnvironmentPower for the
    // uniform sky, world.cpp:352-368: its mean over 400..700 nm, times pi R^2 4 pi) and the disc the
    // sun and the sky shine from, about the scene's centre.
    double skyPower = 0;
    if (d.env.sky_model != OWEC_SKY_NONE && d.env.sky_radiance >= 0) {
        // the sky's mean over 16 x 32 directions and 400..700 nm (computeEnvironmentPower)
        double upv[3] = {d.env.sky_up[0], d.env.sky_up[1], d.env.sky_up[2]};
        const double ul = std::sqrt(upv[0] * upv[0] + upv[1] * upv[1] + upv[2] * upv[2]);
        for (int k = 0; k < 3; ++k) upv[k] = ul > 0 ? upv[k] / ul : (k == 2 ? 1.0 : 0.0);
        auto sky = [&](const double dir[3], double l) {
            if (d.env.sky_model == OWEC_SKY_UNIFORM) return evalSpectrumHost(d, d.env.sky_radiance, l);
            const double c = dir[0] * upv[0] + dir[1] * upv[1] + dir[2] * upv[2];
            if (c < 0) return evalSpectrumHost(d, d.env.sky_ground, l);
            const double t = std::pow(c, 0.45);
            return evalSpectrumHost(d, d.env.sky_horizon, l) * (1 - t) + evalSpectrumHost(d, d.env.sky_radiance, l) * t;
        };
        double sum = 0;
        int n = 0;
        for (int i = 0; i < 16; ++i)
            for (int j = 0; j < 32; ++j) {
                const double z = 1 - 2 * (i + 0.5) / 16, r = std::sqrt(std::max(0.0, 1 - z * z));
                const double phi = 2 * kPi * (j + 0.5) / 32;
                const double dir[3] = {r * std::cos(phi), r * std::sin(phi), z};
                double y = 0;
                for (double l = 400; l <= 700; l += 50) y += sky(dir, l);
                sum += y / 7;
                ++n;
            }
        skyPower = std::max(0.0, sum / n) * kPi * sceneRadius * sceneRadius * 4 * kPi;
    }
    const double emitted = skyPower + (c.lights.empty() ? 0.0 : total);
    c.pSky = emitted > 0 ? skyPower / emitted : 0;
    c.discRadius = sceneRadius * 1.001;
    for (int k = 0; k < 3; ++k) c.discCentre[k] = center[k];

    // Primitives: every mesh triangle (camera-relative FP32, and FP64 for the all-FP64 mode), then
    // every analytic boundary as one primitive of its own world box.
    c.triRecs.clear();
    c.tri64.clear();
    c.primLo.clear();
    c.primHi.clear();
    auto asF = [](uint32_t v) { float f; std::memcpy(&f, &v, 4); return f; };
    c.triBase.assign(d.n_boundaries, 0);
    c.triCount.assign(d.n_boundaries, 0);
    c.hf = HeightfieldParams{kNone, nullptr, {0, 0, 1}};
    c.meshes.assign(d.n_boundaries, owec_ctx::MeshCopy{});
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        if (b.shape != OWEC_SHAPE_MESH) continue;
        const owec_mesh& m = d.meshes[b.mesh];
        c.triBase[i] = uint32_t(c.primLo.size());
        c.triCount[i] = m.tri_count;
        c.meshes[i].verts.assign(d.vertices + 3 * m.vertex_offset, d.vertices + 3 * (m.vertex_offset + m.vertex_count));
        c.meshes[i].tris.assign(d.triangles + 3 * m.tri_offset, d.triangles + 3 * (m.tri_offset + m.tri_count));
        double rel[12];
        std::memcpy(rel, c.boundaries[i].toWorld.m, sizeof(rel));
        for (uint64_t t = 0; t < m.tri_count; ++t) {
            const uint32_t* tri = d.triangles + 3 * (m.tri_offset + t);
            double w[3][3];
            for (int k = 0; k < 3; ++k) xfPoint(rel, d.vertices + 3 * (m.vertex_offset + tri[k]), w[k]);
            const uint32_t ids[3] = {i, uint32_t(t), kPrimTriangle};
            double lo[3], hi[3];
            for (int k = 0; k < 3; ++k) {
                c.triRecs.push_back(make_float4(float(w[k][0]), float(w[k][1]), float(w[k][2]), asF(ids[k])));
                for (int a = 0; a < 3; ++a) c.tri64.push_back(w[k][a]);
            }
            for (int a = 0; a < 3; ++a) {
                // the box of the FP32 vertices (what the FP32 traversal tests), padded outward
                float f0 = float(w[0][a]), f1 = float(w[1][a]), f2 = float(w[2][a]);
                lo[a] = std::min({double(f0), double(f1), double(f2), w[0][a], w[1][a], w[2][a]});
                hi[a] = std::max({double(f0), double(f1), double(f2), w[0][a], w[1][a], w[2][a]});
            }
            float4 flo, fhi;
            padPrimBox(lo, hi, flo, fhi);
            c.primLo.push_back(flo);
            c.primHi.push_back(fhi);
        }
    }
    c.nTriangles = uint32_t(c.primLo.size());
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        if (d.boundaries[i].shape == OWEC_SHAPE_MESH) continue;
        const uint32_t ids[3] = {i, 0u, kPrimAnalytic};
        for (int k = 0; k < 3; ++k) {
            c.triRecs.push_back(make_float4(0.f, 0.f, 0.f, asF(ids[k])));
            for (int a = 0; a < 3; ++a) c.tri64.push_back(0.0);
        }
        double lo[3], hi[3];
        for (int k = 0; k < 3; ++k) { lo[k] = wboxes[i].lo[k] - origin[k]; hi[k] = wboxes[i].hi[k] - origin[k]; }
        float4 flo, fhi;
        padPrimBox(lo, hi, flo, fhi);
        c.primLo.push_back(flo);
        c.primHi.push_back(fhi);
    }
    c.nPrims = uint32_t(c.primLo.size());

    // The detector (IdealObserver::prepare, detector.cpp:46-59; SurfaceSensor::prepare, :102-111).
    DDetector det{};
    const owec_detector& dd = d.detector;
    det.kind = dd.kind;
    det.width = dd.width;
    det.height = dd.height;
    det.sigma = dd.pixel_sigma;
    if (dd.kind == OWEC_DETECTOR_OBSERVER) {
        double f[3], u[3] = {dd.up[0], dd.up[1], dd.up[2]};
        double fl = 0;
        for (int k = 0; k < 3; ++k) { f[k] = dd.look_at[k] - dd.position[k]; fl += f[k] * f[k]; }
        fl = std::sqrt(fl);
        require(fl > 0, "observer looks at its own position");
        for (double& x : f) x /= fl;
        const double ul = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        if (std::fabs((u[0] * f[0] + u[1] * f[1] + u[2] * f[2]) / ul) > 0.9999) {
            u[0] = 0; u[1] = 0; u[2] = 0;
            if (std::fabs(f[2]) < 0.9) u[2] = 1; else u[1] = 1;
        }
        double r[3] = {f[1] * u[2] - f[2] * u[1], f[2] * u[0] - f[0] * u[2], f[0] * u[1] - f[1] * u[0]};
        const double rl = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        for (double& x : r) x /= rl;
        const double up[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
        for (int k = 0; k < 3; ++k) {
            det.fwd[k] = f[k];
            det.right[k] = r[k];
            det.up[k] = up[k];
            det.pos[k] = dd.position[k] - origin[k];
        }
        det.tanY = std::tan(0.5 * dd.fov_y);
        det.tanX = det.tanY * double(dd.width) / double(dd.height);
        det.region = dd.region;
        det.pupil = dd.pupil_radius;
        det.focus = dd.focus_distance > 0 && std::isfinite(dd.focus_distance) ? dd.focus_distance : INFINITY;
        det.guideR = dd.pupil_radius > 0 ? dd.guide_radius : 0;
        det.guideShare = dd.guide_share;
        for (int k = 0; k < 3; ++k) det.guideC[k] = dd.guide_center[k] - origin[k];
    } else {
        const owec_boundary& b = d.boundaries[dd.boundary];
        require(d.optics[b.optics].type == OWEC_SURF_DETECTOR || d.optics[b.optics].type == OWEC_SURF_DIFFUSE,
                "sensor boundary is not a detector surface");
        det.boundary = dd.boundary;
        det.halfX = dd.half_x;
        det.halfY = dd.half_y;
        double nrm[3] = {b.to_world[2], b.to_world[6], b.to_world[10]};
        const double nl = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
        for (int k = 0; k < 3; ++k) det.normal[k] = nrm[k] / nl;
        det.region = b.front;
        det.flipX = dd.flip_x != 0;
        det.flipY = dd.flip_y != 0;
        if (dd.has_aim) {
            const double al = std::sqrt(dd.aim_normal[0] * dd.aim_normal[0] + dd.aim_normal[1] * dd.aim_normal[1] +
                                        dd.aim_normal[2] * dd.aim_normal[2]);
            require(al > 0 && dd.aim_radius > 0 && dd.aim_share > 0 && dd.aim_share <= 1,
                    "sensor aim: needs a normal, a radius and a share in (0, 1]");
            require(dd.focus_share >= 0 && dd.focus_share < 1 && (dd.focus_share == 0 || dd.focus_radius > 0),
                    "sensor aim: focus share in [0, 1) with a radius");
            det.aimR = dd.aim_radius;
            det.aimShare = dd.aim_share;
            det.focusR = dd.focus_radius;
            det.focusShare = dd.focus_share;
            for (int k = 0; k < 3; ++k) {
                det.aimC[k] = dd.aim_center[k] - origin[k];
                det.aimN[k] = dd.aim_normal[k] / al;
                det.focusC[k] = dd.focus_center[k] - origin[k];
            }
        }
    }

    // Aim guides in the camera-relative frame, with unit normals.
    for (owec_optics& o : c.optics) {
        if (!(o.aim_share > 0)) continue;
        const double nl = std::sqrt(o.aim_normal[0] * o.aim_normal[0] + o.aim_normal[1] * o.aim_normal[1] +
                                    o.aim_normal[2] * o.aim_normal[2]);
        for (int k = 0; k < 3; ++k) {
            o.aim_center[k] -= origin[k];
            o.aim_normal[k] /= nl;
        }
    }

    // Upload.
    c.dSpectra.upload(c.spectra.data(), c.spectra.size(), s);
    if (c.table.empty()) c.table.assign(2, 0.0);  // never empty, so its device pointer is valid
    c.dTable.upload(c.table.data(), c.table.size(), s);
    c.dMedia.upload(c.media.data(), c.media.size(), s);
    c.dRegionMedium.upload(c.regionMedium.data(), c.regionMedium.size(), s);
    c.dOptics.upload(c.optics.data(), c.optics.size(), s);
    c.dEmissions.upload(c.emissions.data(), c.emissions.size(), s);
    c.dBoundaries.upload(c.boundaries.data(), c.boundaries.size(), s);
    c.dLights.upload(c.lights.data(), c.lights.size(), s);
    c.dShapeData.upload(c.shapeData.data(), c.shapeData.size(), s);
    c.dPrimLo.upload(c.primLo.data(), c.primLo.size(), s);
    c.dPrimHi.upload(c.primHi.data(), c.primHi.size(), s);
    c.dTri.upload(c.triRecs.data(), c.triRecs.size(), s);
    OWEC_CUDA(cudaStreamSynchronize(s));  // the host vectors above may change after this call

    DeviceScene& ds = c.ds;
    ds = DeviceScene{};
    if (c.eventLogCap > 0) {  // an enabled event log outlasts a scene upload
        ds.eventLog = c.dEventLog.get();
        ds.eventLogCount = c.dEventLogCount.get();
        ds.eventLogCap = c.eventLogCap;
    }
    ds.spectra = c.dSpectra.get();
    ds.table = c.dTable.get();
    ds.media = c.dMedia.get();
    ds.regionMedium = c.dRegionMedium.get();
    ds.optics = c.dOptics.get();
    ds.emissions = c.dEmissions.get();
    ds.boundaries = c.dBoundaries.get();
    ds.lights = c.dLights.get();
    ds.shapeData = c.dShapeData.get();
    ds.fullFeatures = 0;
    for (uint32_t i = 0; i < d.n_boundaries; ++i) {
        const owec_boundary& b = d.boundaries[i];
        if (b.shape == OWEC_SHAPE_CONE || b.shape == OWEC_SHAPE_TORUS || b.shape == OWEC_SHAPE_ROUND_WALL ||
            b.shape == OWEC_SHAPE_DOME || b.shape == OWEC_SHAPE_WAVES || (b.shape == OWEC_SHAPE_SAG && b.data_count > 0) ||
            (b.shape == OWEC_SHAPE_PLANE && int(b.params[0]) == OWEC_APERTURE_DISK_HOLE))
            ds.fullFeatures = 1;
        // a sphere of planetary size (the reference's scenes have 1.7e6 m and more; their lab-sized
        // spheres stay under 50): rays near it take the double-double solve, in the Full instantiation
        // only, so that the lean traversal's registers stay those of a scene without one
        if (b.shape == OWEC_SHAPE_SPHERE && b.params[0] >= kNearSphereMinRadius) ds.fullFeatures = 1;
    }
    for (uint32_t i = 0; i < d.n_optics; ++i)
        if (d.optics[i].texture != OWEC_TEXTURE_NONE || d.optics[i].aim_share > 0) ds.fullFeatures = 1;
    // contacts: resolved as the reference does by the contact-resolving instantiation; the tolerance
    // is the FP32 anchor error over the scene's extent
    c.contacts = hasContacts(d, 1e-5 * std::max(2 * sceneRadius, 1e-3));
    if (c.contacts) ds.fullFeatures = 1;
    {
        auto participates = [&](int32_t spectrum) {
            return spectrum >= 0 && !(d.spectra[spectrum].kind == OWEC_SPEC_CONSTANT && d.spectra[spectrum].a == 0.0);
        };
        bool simple = !c.hasNull && !ds.fullFeatures;
        for (uint32_t i = 0; i < d.n_boundaries && simple; ++i) {
            const int32_t t = d.optics[d.boundaries[i].optics].type;
            simple = t == OWEC_SURF_DIFFUSE || t == OWEC_SURF_ABSORBER || t == OWEC_SURF_DETECTOR;
        }
        for (uint32_t r = 0; r < d.n_regions && simple; ++r) {
            const owec_medium& m = d.media[d.region_medium[r]];
            simple = !participates(m.absorption) && !participates(m.scattering);
        }
        ds.simpleOptics = simple ? 1 : 0;
    }
    ds.nRegions = d.n_regions;
    ds.nBoundaries = d.n_boundaries;
    ds.nLights = uint32_t(c.lights.size());
    ds.nMedia = d.n_media;
    ds.skyModel = d.env.sky_model;
    ds.skySpectrum = d.env.sky_radiance;
    ds.skyHorizon = d.env.sky_horizon;
    ds.skyGround = d.env.sky_ground;
    {
        const double* u = d.env.sky_up;
        double ul = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        for (int k = 0; k < 3; ++k) ds.skyUp[k] = ul > 0 ? u[k] / ul : (k == 2 ? 1.0 : 0.0);
    }
    ds.hasSun = d.env.has_sun;
    ds.sunSpectrum = d.env.sun_radiance;
    double sl = std::sqrt(d.env.sun_dir[0] * d.env.sun_dir[0] + d.env.sun_dir[1] * d.env.sun_dir[1] +
                          d.env.sun_dir[2] * d.env.sun_dir[2]);
    if (!(sl > 0)) sl = 1;
    for (int k = 0; k < 3; ++k) {
        ds.sunDir[k] = d.env.sun_dir[k] / sl;
        ds.sceneCenter[k] = center[k];
        ds.origin[k] = origin[k];
    }
    ds.sunCosMax = cosMax;
    ds.sunSolidAngle = sunSolid;
    ds.sunSelectPdf = sunSel;
    ds.sceneRadius = sceneRadius;
    ds.det = det;
    ds.cieYIntegral = cieYIntegralHost();
    ds.contactScale = sceneRadius;
    c.hasScene = true;
    c.bvhDirty = true;
    c.prims64Ready = false;
    // a new scene has no heightfield until owec_set_heightfield names one of its boundaries
    c.hf.boundary = kNone;
    c.hfVertices = 0;
    c.passCount = 0;
    c.dFilm.release();
    c.dComp.release();
    c.dSamples.release();
    c.dSplat.release();
    c.particles = 0;
}

void ensurePrims64(owec_ctx& c);

void buildBvh(owec_ctx& c) {
    require(c.hasScene, "no scene uploaded", OWEC_E_STATE);
    if (c.nPrims == 0) {
        // nothing to meet (a sky or a sun alone): no tree, and every traversal misses at once
        // (Traversal::run returns before it reads a node when the tree is empty)
        c.nNodes = 0;
        c.ds.nodes = nullptr;
        c.ds.prims = nullptr;
        c.ds.prims64 = nullptr;
        c.ds.nNodes = 0;
        c.ds.nPrims = 0;
        c.bvhDirty = false;
        c.prims64Ready = true;
        return;
    }
    c.nNodes = buildWideBvh(c.dPrimLo.get(), c.dPrimHi.get(), c.nPrims, c.scratch, c.dNodes, c.dLeafOrder, c.stream);
    c.dPrims.reserve(c.nPrims);
    launchMaterialize(c.dLeafOrder.get(), c.nPrims, c.dTri.get(), nullptr, c.dPrims.get(), nullptr, c.stream);
    checkLaunch();
    OWEC_CUDA(cudaStreamSynchronize(c.stream));
    c.ds.nodes = c.dNodes.get();
    c.ds.prims = c.dPrims.get();
    c.ds.nNodes = c.nNodes;
    c.ds.nPrims = c.nPrims;
    c.bvhDirty = false;
    c.prims64Ready = false;
    if (c.settings.precision != OWEC_PRECISION_FP32) ensurePrims64(c);
}

void ensurePrims64(owec_ctx& c) {
    if (c.prims64Ready || c.nPrims == 0) return;
    c.dTri64.upload(c.tri64.data(), c.tri64.size(), c.stream);
    c.dPrims64.reserve(c.nPrims);
    launchMaterialize(c.dLeafOrder.get(), c.nPrims, c.dTri.get(), c.dTri64.get(), c.dPrims.get(), c.dPrims64.get(),
                      c.stream);
    checkLaunch();
    OWEC_CUDA(cudaStreamSynchronize(c.stream));
    c.ds.prims64 = c.dPrims64.get();
    c.prims64Ready = true;
}

// Copies the scene description to its device copy, which the out-of-line traversal functions read
// (DeviceScene::self); every launch follows one. A copy from pageable memory: ds may change as soon
// as this returns.
void publishScene(owec_ctx& c) {
    c.ds.self = c.dScene.get();
    OWEC_CUDA(cudaMemcpyAsync(c.dScene.get(), &c.ds, sizeof(DeviceScene), cudaMemcpyHostToDevice, c.stream));
}

void ensureReady(owec_ctx& c) {
    require(c.hasScene, "no scene uploaded", OWEC_E_STATE);
    if (c.bvhDirty) buildBvh(c);
    // FP64 vertices: the traversal's in the FP64 mode, the refined triangle distances in the mixed one
    if (c.settings.precision != OWEC_PRECISION_FP32) ensurePrims64(c);
    publishScene(c);
}

void ensureFilm(owec_ctx& c) {
    const size_t np = size_t(c.ds.det.width) * c.ds.det.height;
    if (c.settings.integrator == OWEC_INTEGRATOR_LIGHT && c.dSplat.size() != np * kSplatWordsPerPixel) {
        c.dSplat.resize(np * kSplatWordsPerPixel);
        OWEC_CUDA(cudaMemsetAsync(c.dSplat.get(), 0, c.dSplat.bytes(), c.stream));
        c.particles = 0;
    }
    if (c.dFilm.size() != 3 * np) {
        c.dFilm.resize(3 * np);
        c.dComp.resize(3 * np);
        c.dSamples.resize(np);
        OWEC_CUDA(cudaMemsetAsync(c.dFilm.get(), 0, c.dFilm.bytes(), c.stream));
        OWEC_CUDA(cudaMemsetAsync(c.dComp.get(), 0, c.dComp.bytes(), c.stream));
        OWEC_CUDA(cudaMemsetAsync(c.dSamples.get(), 0, c.dSamples.bytes(), c.stream));
    }
}

// The path state and queues for `cap` paths in flight (grown, never shrunk).
template <int M>
PathBuffers<ModeR<M>> pathState(owec_ctx& c, uint32_t cap, Queues& q) {
    using R = ModeR<M>;
    // every buffer whose record depends on the precision is checked: a context may switch modes
    if (c.capacity < cap || c.dPathRay.bytes() < size_t(cap) * sizeof(PathRay<R>) ||
        c.dPathSpec.bytes() < size_t(cap) * sizeof(PathSpec<R>) ||
        c.dShadow.bytes() < size_t(cap) * sizeof(ShadowRay<R>)) {
        c.dPathRay.resize(size_t(cap) * sizeof(PathRay<R>));
        c.dPathSpec.resize(size_t(cap) * sizeof(PathSpec<R>));
        c.dPathAux.resize(size_t(cap) * sizeof(PathAux));
        c.dHit.resize(size_t(cap) * sizeof(HitRec));
        c.dShadow.resize(size_t(cap) * sizeof(ShadowRay<R>));
        c.dQueue0.resize(cap);
        c.dQueue1.resize(cap);
        c.dQueueSurf.resize(cap);
        c.dQueueSurfSimple.resize(cap);
        c.dShadowVis.resize(cap);
        c.dQueueShadow.resize(cap);
        c.capacity = cap;
    }
    q = Queues{{c.dQueue0.get(), c.dQueue1.get()}, c.dQueueSurf.get(), c.dQueueShadow.get(), c.dCounts.get(),
               c.dQueueSurfSimple.get()};
    return PathBuffers<R>{reinterpret_cast<PathRay<R>*>(c.dPathRay.get()), reinterpret_cast<PathSpec<R>*>(c.dPathSpec.get()),
                          reinterpret_cast<PathAux*>(c.dPathAux.get()), reinterpret_cast<HitRec*>(c.dHit.get()),
                          reinterpret_cast<ShadowRay<R>*>(c.dShadow.get())};
}

// Blocks per SM of the grid-stride medium and surface kernels of the camera paths.
#ifndef OWEC_SHADING_GRID
#define OWEC_SHADING_GRID 8
#endif

// The bounces of one batch of camera paths already generated into pb: intersect, medium, surface
// and shadow kernels per bounce until the active queue is empty. The kernels read their queue
// lengths on the device, so the bounces are queued without a look at the host: maxDepth + 1 of
// them first (a path without null boundaries ends by then), then four at a time until the queue
// is empty. The host waits once per batch, not once per bounce. With timed, CUDA events around the
// intersect and shadow launches add their device seconds to travSeconds.
template <int M>
void runBounces(owec_ctx& c, const PassParams& pp, PathBuffers<ModeR<M>>& pb, Queues& q, StatCounters* st, int grid,
                bool timed, double travSeconds[2], int& evUsed, int& intersectLaunches) {
    cudaStream_t s = c.stream;
    int cur = 0;
    int nextCheck = pp.maxDepth + 1;
    for (int bounce = 0; bounce < 4 * pp.maxDepth + 8; ++bounce) {
        if (bounce == nextCheck) {
            OWEC_CUDA(cudaMemcpyAsync(c.hostCounts, c.dCounts.get(), 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
            OWEC_CUDA(cudaStreamSynchronize(s));
            if (c.hostCounts[cur] == 0) break;
            nextCheck = bounce + 4;
        }
        // the next-bounce queue and the per-bounce queues start empty
        OWEC_CUDA(cudaMemsetAsync(c.dCounts.get() + (cur ^ 1), 0, sizeof(uint32_t), s));
        OWEC_CUDA(cudaMemsetAsync(c.dCounts.get() + 2, 0, 5 * sizeof(uint32_t), s));  // + fetch counters, simple queue
        if (timed && size_t(evUsed + 4) > c.travEvents.size())
            for (int k = 0; k < 4; ++k) {
                cudaEvent_t e;
                OWEC_CUDA(cudaEventCreate(&e));
                c.travEvents.push_back(e);
            }
        if (timed) OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed], s));
        launchIntersect<M>(c.ds, pb, q, cur, st, c.dCounts.get() + 4, grid, s);
        ++intersectLaunches;
        if (c.ds.travCounters && c.launchQueryCount < owec_ctx::kLaunchLog)
            OWEC_CUDA(cudaMemcpyAsync(c.dLaunchQueries.get() + c.launchQueryCount++, c.ds.travCounters,
                                      sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
        if (timed) OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed + 1], s));
        checkLaunch();
        launchMedium<M>(c.ds, pp, pb, q, cur, st, c.numSMs * OWEC_SHADING_GRID, s);
        launchSurface<M>(c.ds, pp, pb, q, cur, st, c.numSMs * OWEC_SHADING_GRID, s);
        if (timed) OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed + 2], s));
        launchShadow<M>(c.ds, pp, pb, q, st, c.dCounts.get() + 5, c.dShadowVis.get(), grid, s);
        if (timed) OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed + 3], s));
        checkLaunch();
        if (timed) evUsed += 4;
        OWEC_CUDA(cudaMemsetAsync(c.dCounts.get() + cur, 0, sizeof(uint32_t), s));
        cur ^= 1;
        if (timed && evUsed >= 256) {  // fold the timings in before reusing the events
            OWEC_CUDA(cudaStreamSynchronize(s));
            for (int e = 0; e < evUsed; e += 2) {
                float ms = 0;
                OWEC_CUDA(cudaEventElapsedTime(&ms, c.travEvents[e], c.travEvents[e + 1]));
                travSeconds[(e >> 1) & 1] += ms * 1e-3;
            }
            evUsed = 0;
        }
    }
}

template <int M>
void runPass(owec_ctx& c, int spp) {
    using R = ModeR<M>;
    const uint32_t nPix = uint32_t(c.ds.det.width) * uint32_t(c.ds.det.height);
    // Paths in flight: enough to fill the GPU several times over (2M+), within the state budget.
    const uint32_t target = std::max<uint32_t>(nPix, 1u << 21);
    uint32_t perBatch = std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(spp), target / nPix));
    const uint32_t cap = perBatch * nPix;
    Queues q;
    PathBuffers<R> pb = pathState<M>(c, cap, q);
    PassParams pp{};
    pp.seed = c.settings.seed;
    pp.maxDepth = c.settings.max_depth;
    pp.rrDepth = c.settings.rr_depth;
    pp.wavelengthMode = c.settings.wavelength_mode;
    pp.lambdaMin = float(c.settings.lambda_min);
    pp.lambdaMax = float(c.settings.lambda_max);
    pp.fresnelFloor = float(std::min(0.49, std::max(0.0, c.settings.fresnel_floor)));
    pp.nPixels = nPix;
    pp.anyHitShadows = c.hasNull ? 0 : 1;
    const int grid = c.numSMs * 8;
    cudaStream_t s = c.stream;
    double travSeconds[2] = {0, 0};
    int intersectLaunches = 0;
    OWEC_CUDA(cudaEventRecord(c.passStart, s));
    int evUsed = 0;
    for (int done = 0; done < spp;) {
        const uint32_t S = std::min<uint32_t>(perBatch, uint32_t(spp - done));
        pp.nPaths = S * nPix;
        pp.streamBase = uint32_t(c.passCount + done);
        OWEC_CUDA(cudaMemsetAsync(c.dCounts.get(), 0, 8 * sizeof(uint32_t), s));
        launchGenerate<M>(c.ds, pp, pb, q, c.dStats.get(), s);
        checkLaunch();
        runBounces<M>(c, pp, pb, q, c.dStats.get(), grid, true, travSeconds, evUsed, intersectLaunches);
        launchFilm<M>(c.ds, pp, pb, c.dFilm.get(), c.dComp.get(), c.dSamples.get(), S, s);
        checkLaunch();
        done += int(S);
    }
    OWEC_CUDA(cudaEventRecord(c.passStop, s));
    OWEC_CUDA(cudaEventSynchronize(c.passStop));
    for (int e = 0; e < evUsed; e += 2) {
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, c.travEvents[e], c.travEvents[e + 1]));
        travSeconds[(e >> 1) & 1] += ms * 1e-3;  // pairs alternate: intersect, shadow
    }
    float passMs = 0;
    OWEC_CUDA(cudaEventElapsedTime(&passMs, c.passStart, c.passStop));
    c.lastPassSeconds = passMs * 1e-3;
    c.lastIntersectSeconds = travSeconds[0];
    c.lastShadowSeconds = travSeconds[1];
    c.lastIntersectLaunches = intersectLaunches;
    c.passCount += uint64_t(spp);
}

// A pass of the light integrator: width x height x spp particles, through the wavefront in batches
// of up to 2^21 (the particle index, not the batch, keys a particle's stream).
template <int M>
void runParticles(owec_ctx& c, int spp) {
    using R = ModeR<M>;
    const DDetector& det = c.ds.det;
    const uint64_t nPix = uint64_t(det.width) * uint64_t(det.height);
    const uint64_t total = nPix * uint64_t(spp);
    const uint32_t cap = uint32_t(std::min<uint64_t>(total, 1u << 21));
    Queues q;
    PathBuffers<R> pb = pathState<M>(c, cap, q);
    c.dShadowPixel.reserve(cap);
    const SplatTarget film{c.dSplat.get(), c.dShadowPixel.get()};
    ParticleParams P{};
    P.seed = c.settings.seed;
    P.stream = c.passCount;
    P.maxDepth = c.settings.max_depth;
    P.rrDepth = c.settings.rr_depth;
    P.wavelengthMode = c.settings.wavelength_mode;
    P.lambdaMin = float(c.settings.lambda_min);
    P.lambdaMax = float(c.settings.lambda_max);
    P.fresnelFloor = float(std::min(0.49, std::max(0.0, c.settings.fresnel_floor)));
    P.pSky = c.pSky;
    P.discRadius = c.discRadius;
    for (int k = 0; k < 3; ++k) P.discCentre[k] = c.discCentre[k];
    P.pixelArea = det.kind == OWEC_DETECTOR_OBSERVER ? (2 * det.tanX / det.width) * (2 * det.tanY / det.height)
                                                     : (2 * det.halfX / det.width) * (2 * det.halfY / det.height);
    PassParams pp{};
    pp.anyHitShadows = c.hasNull ? 0 : 1;
    const int grid = c.numSMs * 8;
    cudaStream_t s = c.stream;
    uint32_t* counts = c.dCounts.get();
    double travSeconds[2] = {0, 0};
    int intersectLaunches = 0, evUsed = 0;
    OWEC_CUDA(cudaEventRecord(c.passStart, s));
    // nothing emits: the estimate is zero, but the particles still count
    const bool emits = c.pSky > 0 || !c.lights.empty();
    for (uint64_t first = 0; emits && first < total; first += cap) {
        const uint32_t n = uint32_t(std::min<uint64_t>(cap, total - first));
        P.first = first;
        OWEC_CUDA(cudaMemsetAsync(counts, 0, 8 * sizeof(uint32_t), s));
        launchEmit<M>(c.ds, P, pb, q, c.dStats.get(), film, n, s);
        launchConnect<M>(c.ds, pp, pb, q, c.dStats.get(), counts + 5, c.dShadowVis.get(), film, grid, s);
        checkLaunch();
        int cur = 0;
        // as the camera paths: bounces queued without a host wait, the queue looked at once the
        // depth cap is reached and every four bounces after it
        int nextCheck = P.maxDepth + 1;
        for (int bounce = 0; bounce < 4 * P.maxDepth + 8; ++bounce) {
            if (bounce == nextCheck) {
                OWEC_CUDA(cudaMemcpyAsync(c.hostCounts, counts, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                OWEC_CUDA(cudaStreamSynchronize(s));
                if (c.hostCounts[cur] == 0) break;
                nextCheck = bounce + 4;
            }
            OWEC_CUDA(cudaMemsetAsync(counts + (cur ^ 1), 0, sizeof(uint32_t), s));
            OWEC_CUDA(cudaMemsetAsync(counts + 2, 0, 5 * sizeof(uint32_t), s));  // shadow queue, fetch counters
            if (size_t(evUsed + 4) > c.travEvents.size())
                for (int k = 0; k < 4; ++k) {
                    cudaEvent_t e;
                    OWEC_CUDA(cudaEventCreate(&e));
                    c.travEvents.push_back(e);
                }
            OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed], s));
            launchIntersect<M>(c.ds, pb, q, cur, c.dStats.get(), counts + 4, grid, s);
            ++intersectLaunches;
            OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed + 1], s));
            launchParticleEvent<M>(c.ds, P, pb, q, cur, c.dStats.get(), film, grid, s);
            OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed + 2], s));
            launchConnect<M>(c.ds, pp, pb, q, c.dStats.get(), counts + 5, c.dShadowVis.get(), film, grid, s);
            OWEC_CUDA(cudaEventRecord(c.travEvents[evUsed + 3], s));
            checkLaunch();
            evUsed += 4;
            OWEC_CUDA(cudaMemsetAsync(counts + cur, 0, sizeof(uint32_t), s));
            cur ^= 1;
            if (evUsed >= 256) {  // fold the timings in before reusing the events
                OWEC_CUDA(cudaStreamSynchronize(s));
                for (int e = 0; e < evUsed; e += 2) {
                    float ms = 0;
                    OWEC_CUDA(cudaEventElapsedTime(&ms, c.travEvents[e], c.travEvents[e + 1]));
                    travSeconds[(e >> 1) & 1] += ms * 1e-3;
                }
                evUsed = 0;
            }
        }
    }
    OWEC_CUDA(cudaEventRecord(c.passStop, s));
    OWEC_CUDA(cudaEventSynchronize(c.passStop));
    for (int e = 0; e < evUsed; e += 2) {
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, c.travEvents[e], c.travEvents[e + 1]));
        travSeconds[(e >> 1) & 1] += ms * 1e-3;  // pairs alternate: intersect, connections
    }
    float ms = 0;
    OWEC_CUDA(cudaEventElapsedTime(&ms, c.passStart, c.passStop));
    c.lastPassSeconds = ms * 1e-3;
    c.lastIntersectSeconds = travSeconds[0];
    c.lastShadowSeconds = travSeconds[1];
    c.lastIntersectLaunches = intersectLaunches;
    c.particles += double(total);
    c.passCount += uint64_t(spp);
}

// The camera-path adjoint in two phases per batch of paths: the wavefront runs the batch and stops
// each path at its first surface event on the heightfield, leaving its state there (a checkpoint);
// the derivative replay then resumes only those paths. Paths that never meet the heightfield carry
// no derivative and so cost one forward pass's work and nothing more.
// Returns the number of camera paths the first phase generated; freeDuring receives the device's free
// memory while the phases' buffers are still held.
template <int M>
uint64_t runAdjointCheckpointed(owec_ctx& c, PassParams pp, uint64_t firstPass, int spp, const PathAdjointTargets& t,
                                bool fixedDecisions, size_t& freeDuring, double& replaySeconds) {
    using R = ModeR<M>;
    const uint32_t nPix = pp.nPixels;
    const uint32_t target = std::max<uint32_t>(nPix, 1u << 21);
    const uint32_t perBatch = std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(spp), target / nPix));
    const uint32_t cap = perBatch * nPix;
    Queues q;
    PathBuffers<R> pb = pathState<M>(c, cap, q);
    // every path checkpoints at most once (it ends there)
    DBuf<uint8_t> ckpt(size_t(cap) * pathCheckpointBytes(M));
    DBuf<uint32_t> ckptCount(1);
    DBuf<StatCounters> st(1);  // the phase's own counters: the context's transport statistics stay the forward's
    OWEC_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(StatCounters), c.stream));
    pp.ckptBoundary = c.hf.boundary;
    pp.ckptCount = ckptCount.get();
    pp.ckpt = ckpt.get();
    const int grid = c.numSMs * 8;
    double unusedSeconds[2] = {0, 0};
    int unusedEvents = 0, unusedLaunches = 0;
    cudaEvent_t replayStart, replayStop;
    OWEC_CUDA(cudaEventCreate(&replayStart));
    OWEC_CUDA(cudaEventCreate(&replayStop));
    for (int done = 0; done < spp;) {
        const uint32_t S = std::min<uint32_t>(perBatch, uint32_t(spp - done));
        pp.nPaths = S * nPix;
        pp.streamBase = uint32_t(firstPass + uint64_t(done));
        OWEC_CUDA(cudaMemsetAsync(c.dCounts.get(), 0, 8 * sizeof(uint32_t), c.stream));
        OWEC_CUDA(cudaMemsetAsync(ckptCount.get(), 0, sizeof(uint32_t), c.stream));
        launchGenerate<M>(c.ds, pp, pb, q, st.get(), c.stream);
        checkLaunch();
        runBounces<M>(c, pp, pb, q, st.get(), grid, false, unusedSeconds, unusedEvents, unusedLaunches);
        OWEC_CUDA(cudaEventRecord(replayStart, c.stream));
        launchPathAdjoint(M, c.ds, pp, c.hf, t, fixedDecisions, ckpt.get(), ckptCount.get(), grid, c.stream);
        checkLaunch();
        OWEC_CUDA(cudaEventRecord(replayStop, c.stream));
        OWEC_CUDA(cudaEventSynchronize(replayStop));
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, replayStart, replayStop));
        replaySeconds += ms * 1e-3;
        done += int(S);
    }
    cudaEventDestroy(replayStart);
    cudaEventDestroy(replayStop);
    StatCounters hs{};
    OWEC_CUDA(cudaMemcpyAsync(&hs, st.get(), sizeof(StatCounters), cudaMemcpyDeviceToHost, c.stream));
    OWEC_CUDA(cudaStreamSynchronize(c.stream));
    size_t total = 0;
    OWEC_CUDA(cudaMemGetInfo(&freeDuring, &total));
    return hs.paths;
}

}  // namespace

// ------------------------------------------------------------------ adjoint scratch that is never allocated
// owec_walk_adjoint_noalloc's scratch: the loss gradient per bin, the height-gradient accumulator and
// the walk counters, in one array that is part of the library image. Every GPU that loads the
// library holds these 10.5 MB until the process exits; every call of that entry point shares them.
constexpr size_t kNoAllocMaxBins = 512 * 512;      // walk film bins (width x height)
constexpr size_t kNoAllocMaxHeights = 1u << 20;    // heightfield vertices
constexpr size_t kNoAllocStatsWords = 8;           // walk counters (5 used)
static __device__ __align__(256) double gAdjointScratch[kNoAllocMaxBins + kNoAllocMaxHeights + kNoAllocStatsWords];

namespace {

// The device address of gAdjointScratch on the current device. In host code the array's name is only
// a host-side stand-in, so the address is asked of the runtime. It is asked on every call, not kept:
// a host application that resets the device (cudaDeviceReset) or tears its primary context down
// gets the module loaded again at another address, and a kept pointer would then point at freed
// memory. The first request on a device also loads the array onto it.
double* adjointScratch() {
    void* p = nullptr;
    OWEC_CUDA(cudaGetSymbolAddress(&p, gAdjointScratch));
    return static_cast<double*>(p);
}

}  // namespace

// ------------------------------------------------------------------ the C ABI
extern "C" {

const char* owec_last_error(void) { return g_error.c_str(); }
int owec_abi_version(void) { return OWEC_ABI_VERSION; }

int owec_open(int device, owec_ctx** out) {
    return guarded([&] {
        require(out != nullptr, "owec_open: null output");
        *out = nullptr;
        int count = 0;
        const cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0) throw Error(OWEC_E_CUDA, "no CUDA device available");
        if (device < 0) OWEC_CUDA(cudaGetDevice(&device));
        require(device < count, "device index out of range");
        OWEC_CUDA(cudaSetDevice(device));
        auto c = std::make_unique<owec_ctx>();
        c->device = device;
        cudaDeviceProp prop;
        OWEC_CUDA(cudaGetDeviceProperties(&prop, device));
        c->numSMs = prop.multiProcessorCount;
        std::snprintf(c->name, sizeof(c->name), "%s", prop.name);
        OWEC_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        OWEC_CUDA(cudaEventCreate(&c->passStart));
        OWEC_CUDA(cudaEventCreate(&c->passStop));
        OWEC_CUDA(cudaMallocHost(&c->hostCounts, 8 * sizeof(uint32_t)));
        c->dCounts.resize(8);
        c->dStats.resize(1);
        c->dScene.resize(1);
        OWEC_CUDA(cudaMemsetAsync(c->dStats.get(), 0, sizeof(StatCounters), c->stream));
        configureKernels();
        OWEC_CUDA(cudaStreamSynchronize(c->stream));
        *out = c.release();
    });
}

int owec_close(owec_ctx* ctx) {
    if (!ctx) return OWEC_OK;
    return guarded([&] {
        cudaSetDevice(ctx->device);
        cudaStreamSynchronize(ctx->stream);
        if (ctx->copyStream) {
            cudaStreamSynchronize(ctx->copyStream);
            for (int k = 0; k < 2; ++k) cudaEventDestroy(ctx->resolvedEv[k]);
            cudaStreamDestroy(ctx->copyStream);
        }
        for (cudaEvent_t e : ctx->travEvents) cudaEventDestroy(e);
        cudaEventDestroy(ctx->passStart);
        cudaEventDestroy(ctx->passStop);
        cudaFreeHost(ctx->hostCounts);
        cudaStream_t s = ctx->stream;
        delete ctx;  // frees the device buffers
        cudaStreamDestroy(s);
    });
}

int owec_device_name(owec_ctx* ctx, char* buf, size_t len) {
    return guarded([&] {
        require(ctx && buf && len > 0, "owec_device_name: bad arguments");
        std::snprintf(buf, len, "%s", ctx->name);
    });
}

int owec_upload_scene(owec_ctx* ctx, const owec_scene_desc* scene) {
    return guarded([&] {
        require(ctx && scene, "owec_upload_scene: null argument");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        uploadScene(*ctx, *scene);
    });
}

int owec_build_bvh(owec_ctx* ctx) {
    return guarded([&] {
        require(ctx != nullptr, "owec_build_bvh: null context");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        buildBvh(*ctx);
    });
}

int owec_bvh_info(owec_ctx* ctx, uint64_t info[6]) {
    return guarded([&] {
        require(ctx && info, "owec_bvh_info: null argument");
        require(!ctx->bvhDirty, "the BVH is not built", OWEC_E_STATE);
        info[0] = ctx->nNodes;
        info[1] = ctx->nPrims;
        info[2] = ctx->nTriangles;
        info[3] = uint64_t(ctx->nNodes) * sizeof(WideNode);
        info[4] = uint64_t(ctx->nPrims) * sizeof(PrimRec);
        info[5] = ctx->nPrims - ctx->nTriangles;
    });
}

int owec_set_settings(owec_ctx* ctx, const owec_settings* s) {
    return guarded([&] {
        require(ctx && s, "owec_set_settings: null argument");
        require(s->max_depth >= 0 && s->max_depth <= 4096 && s->rr_depth >= 0, "depth out of range");
        require(s->wavelength_mode == OWEC_WAVELENGTHS_HERO4 || s->wavelength_mode == OWEC_WAVELENGTHS_UNIFORM1,
                "unknown wavelength mode");
        require(s->precision >= OWEC_PRECISION_MIXED && s->precision <= OWEC_PRECISION_FP64, "unknown precision mode");
        require(s->wavelength_mode != OWEC_WAVELENGTHS_UNIFORM1 ||
                    (s->lambda_min > 0 && s->lambda_max > s->lambda_min), "bad wavelength range");
        require(s->integrator == OWEC_INTEGRATOR_PATH || s->integrator == OWEC_INTEGRATOR_LIGHT,
                "unknown integrator (expected path or light)", OWEC_E_UNSUPPORTED);
        const bool estimatorChange = std::memcmp(s, &ctx->settings, sizeof(owec_settings)) != 0;
        ctx->settings = *s;
        if (estimatorChange) {
            ctx->passCount = 0;
            ctx->dFilm.release();
            ctx->dComp.release();
            ctx->dSamples.release();
            ctx->dSplat.release();
            ctx->particles = 0;
        }
    });
}

int owec_pass(owec_ctx* ctx, int spp) {
    return guarded([&] {
        require(ctx != nullptr, "owec_pass: null context");
        if (spp <= 0) return;
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureReady(*ctx);
        ensureFilm(*ctx);
        if (ctx->settings.integrator == OWEC_INTEGRATOR_LIGHT) {
            switch (ctx->settings.precision) {
                case OWEC_PRECISION_MIXED: runParticles<OWEC_PRECISION_MIXED>(*ctx, spp); break;
                case OWEC_PRECISION_FP32: runParticles<OWEC_PRECISION_FP32>(*ctx, spp); break;
                default: runParticles<OWEC_PRECISION_FP64>(*ctx, spp); break;
            }
            return;
        }
        switch (ctx->settings.precision) {
            case OWEC_PRECISION_MIXED: runPass<OWEC_PRECISION_MIXED>(*ctx, spp); break;
            case OWEC_PRECISION_FP32: runPass<OWEC_PRECISION_FP32>(*ctx, spp); break;
            default: runPass<OWEC_PRECISION_FP64>(*ctx, spp); break;
        }
    });
}

int owec_resolve(owec_ctx* ctx, double* xyz, double* samples) {
    return guarded([&] {
        require(ctx != nullptr, "owec_resolve: null context");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureFilm(*ctx);
        const size_t np = size_t(ctx->ds.det.width) * ctx->ds.det.height;
        if (ctx->settings.integrator == OWEC_INTEGRATOR_LIGHT) {
            if (xyz) {
                ctx->dResolved.reserve(3 * np);
                launchResolveSplats(ctx->dSplat.get(), uint32_t(np), ctx->particles > 0 ? 1.0 / ctx->particles : 0.0,
                                    ctx->dResolved.get(), ctx->stream);
                checkLaunch();
                OWEC_CUDA(cudaMemcpyAsync(xyz, ctx->dResolved.get(), 3 * np * 8, cudaMemcpyDeviceToHost, ctx->stream));
                OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
            }
            if (samples) std::fill(samples, samples + np, ctx->particles / double(np));
            return;
        }
        if (xyz) {
            ctx->dResolved.reserve(3 * np);
            launchResolve(ctx->dFilm.get(), ctx->dComp.get(), ctx->dSamples.get(), uint32_t(np), ctx->dResolved.get(),
                          ctx->stream);
            checkLaunch();
            OWEC_CUDA(cudaMemcpyAsync(xyz, ctx->dResolved.get(), 3 * np * 8, cudaMemcpyDeviceToHost, ctx->stream));
        }
        if (samples)
            OWEC_CUDA(cudaMemcpyAsync(samples, ctx->dSamples.get(), np * 8, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int owec_resolve_async(owec_ctx* ctx, double* xyz, double* samples) {
    return guarded([&] {
        require(ctx != nullptr, "owec_resolve_async: null context");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureFilm(*ctx);
        if (!ctx->copyStream) {
            OWEC_CUDA(cudaStreamCreateWithFlags(&ctx->copyStream, cudaStreamNonBlocking));
            for (int k = 0; k < 2; ++k) OWEC_CUDA(cudaEventCreateWithFlags(&ctx->resolvedEv[k], cudaEventDisableTiming));
        }
        const size_t np = size_t(ctx->ds.det.width) * ctx->ds.det.height;
        const int slot = ctx->asyncSlot;
        ctx->asyncSlot ^= 1;
        DBuf<double>& img = ctx->dResolvedAsync[slot];
        // the slot's previous read-back (two calls ago) must end before its image is overwritten or
        // resized; in a render loop it ended during the pass since
        OWEC_CUDA(cudaStreamSynchronize(ctx->copyStream));
        img.reserve(4 * np);
        const bool light = ctx->settings.integrator == OWEC_INTEGRATOR_LIGHT;
        if (xyz) {
            if (light)
                launchResolveSplats(ctx->dSplat.get(), uint32_t(np), ctx->particles > 0 ? 1.0 / ctx->particles : 0.0,
                                    img.get(), ctx->stream);
            else
                launchResolve(ctx->dFilm.get(), ctx->dComp.get(), ctx->dSamples.get(), uint32_t(np), img.get(), ctx->stream);
            checkLaunch();
        }
        if (samples && !light)
            OWEC_CUDA(cudaMemcpyAsync(img.get() + 3 * np, ctx->dSamples.get(), np * 8, cudaMemcpyDeviceToDevice,
                                      ctx->stream));
        if (samples && light) std::fill(samples, samples + np, ctx->particles / double(np));
        // the read-back waits for the image, not for the passes queued after it
        OWEC_CUDA(cudaEventRecord(ctx->resolvedEv[slot], ctx->stream));
        OWEC_CUDA(cudaStreamWaitEvent(ctx->copyStream, ctx->resolvedEv[slot], 0));
        if (xyz) OWEC_CUDA(cudaMemcpyAsync(xyz, img.get(), 3 * np * 8, cudaMemcpyDeviceToHost, ctx->copyStream));
        if (samples && !light)
            OWEC_CUDA(cudaMemcpyAsync(samples, img.get() + 3 * np, np * 8, cudaMemcpyDeviceToHost, ctx->copyStream));
    });
}

int owec_resolve_wait(owec_ctx* ctx) {
    return guarded([&] {
        require(ctx != nullptr, "owec_resolve_wait: null context");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        if (ctx->copyStream) OWEC_CUDA(cudaStreamSynchronize(ctx->copyStream));
    });
}

int owec_read_film(owec_ctx* ctx, double* xyz_sums, double* samples) {
    return guarded([&] {
        require(ctx != nullptr, "owec_read_film: null context");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureFilm(*ctx);
        const size_t np = size_t(ctx->ds.det.width) * ctx->ds.det.height;
        if (ctx->settings.integrator == OWEC_INTEGRATOR_LIGHT) {
            if (xyz_sums) {
                ctx->dResolved.reserve(3 * np);
                launchResolveSplats(ctx->dSplat.get(), uint32_t(np), 1.0 / double(np), ctx->dResolved.get(), ctx->stream);
                checkLaunch();
                OWEC_CUDA(cudaMemcpyAsync(xyz_sums, ctx->dResolved.get(), 3 * np * 8, cudaMemcpyDeviceToHost,
                                          ctx->stream));
                OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
            }
            if (samples) std::fill(samples, samples + np, ctx->particles / double(np));
            return;
        }
        if (xyz_sums) {
            std::vector<double> film(3 * np), comp(3 * np);
            OWEC_CUDA(cudaMemcpyAsync(film.data(), ctx->dFilm.get(), 3 * np * 8, cudaMemcpyDeviceToHost, ctx->stream));
            OWEC_CUDA(cudaMemcpyAsync(comp.data(), ctx->dComp.get(), 3 * np * 8, cudaMemcpyDeviceToHost, ctx->stream));
            OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
            for (size_t i = 0; i < 3 * np; ++i) xyz_sums[i] = film[i] - comp[i];
        }
        if (samples) {
            OWEC_CUDA(cudaMemcpyAsync(samples, ctx->dSamples.get(), np * 8, cudaMemcpyDeviceToHost, ctx->stream));
            OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        }
    });
}

int owec_read_film_device(owec_ctx* ctx, double* xyz_sums_dev, double* samples_dev) {
    return guarded([&] {
        require(ctx != nullptr, "owec_read_film_device: null context");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        require(ctx->settings.integrator == OWEC_INTEGRATOR_PATH,
                "owec_read_film_device reads the path integrator's film", OWEC_E_UNSUPPORTED);
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureFilm(*ctx);
        const size_t np = size_t(ctx->ds.det.width) * ctx->ds.det.height;
        if (xyz_sums_dev) {
            launchFoldFilm(ctx->dFilm.get(), ctx->dComp.get(), xyz_sums_dev, 3 * np, ctx->stream);
            checkLaunch();
        }
        if (samples_dev)
            OWEC_CUDA(cudaMemcpyAsync(samples_dev, ctx->dSamples.get(), np * 8, cudaMemcpyDeviceToDevice, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int owec_set_pass_index(owec_ctx* ctx, uint64_t pass_index) {
    return guarded([&] {
        require(ctx != nullptr, "owec_set_pass_index: null context");
        require(pass_index < (1ull << 32), "owec_set_pass_index: the PCG32 stream index is 32 bits");
        ctx->passCount = pass_index;
    });
}

int owec_reset_film(owec_ctx* ctx) {
    return guarded([&] {
        require(ctx != nullptr, "owec_reset_film: null context");
        ctx->passCount = 0;
        ctx->dFilm.release();
        ctx->dComp.release();
        ctx->dSamples.release();
        ctx->dSplat.release();
        ctx->particles = 0;
        OWEC_CUDA(cudaMemsetAsync(ctx->dStats.get(), 0, sizeof(StatCounters), ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int owec_read_stats(owec_ctx* ctx, owec_stats* out) {
    return guarded([&] {
        require(ctx && out, "owec_read_stats: null argument");
        StatCounters h{};
        OWEC_CUDA(cudaMemcpyAsync(&h, ctx->dStats.get(), sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        out->paths = h.paths;
        out->segments = h.segments;
        out->inconsistencies = h.inconsistencies;
        out->leaks = h.leaks;
        out->shadow_rays = h.shadowRays;
        out->device_faults = h.faults;
    });
}

int owec_last_pass_timing(owec_ctx* ctx, double out[4]) {
    return guarded([&] {
        require(ctx && out, "owec_last_pass_timing: null argument");
        out[0] = ctx->lastPassSeconds;
        out[1] = ctx->lastIntersectSeconds;
        out[2] = ctx->lastShadowSeconds;
        out[3] = ctx->lastIntersectLaunches;
    });
}

int owec_cast_rays(owec_ctx* ctx, uint64_t n, const double* origins, const double* directions, uint32_t* boundary,
                   uint32_t* prim, double* t) {
    return guarded([&] {
        require(ctx && (n == 0 || (origins && directions && boundary && prim && t)), "owec_cast_rays: null argument");
        if (n == 0) return;
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureReady(*ctx);
        DBuf<double> o(3 * n), d(3 * n), tt(n);
        DBuf<uint32_t> b(n), p(n);
        OWEC_CUDA(cudaMemcpyAsync(o.get(), origins, 24 * n, cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(d.get(), directions, 24 * n, cudaMemcpyHostToDevice, ctx->stream));
        const int grid = ctx->numSMs * 8;
        switch (ctx->settings.precision) {
            case OWEC_PRECISION_MIXED:
                launchCastRays<OWEC_PRECISION_MIXED>(ctx->ds, n, o.get(), d.get(), b.get(), p.get(), tt.get(), grid, ctx->stream);
                break;
            case OWEC_PRECISION_FP32:
                launchCastRays<OWEC_PRECISION_FP32>(ctx->ds, n, o.get(), d.get(), b.get(), p.get(), tt.get(), grid, ctx->stream);
                break;
            default:
                launchCastRays<OWEC_PRECISION_FP64>(ctx->ds, n, o.get(), d.get(), b.get(), p.get(), tt.get(), grid, ctx->stream);
                break;
        }
        checkLaunch();
        OWEC_CUDA(cudaMemcpyAsync(boundary, b.get(), 4 * n, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(prim, p.get(), 4 * n, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(t, tt.get(), 8 * n, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int owec_cast_rays_device(owec_ctx* ctx, uint64_t n, const float* o, const float* d, uint32_t* b, uint32_t* p, float* t,
                          double* seconds) {
    return guarded([&] {
        require(ctx != nullptr, "owec_cast_rays_device: null context");
        if (n == 0) return;
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureReady(*ctx);
        OWEC_CUDA(cudaEventRecord(ctx->passStart, ctx->stream));
        launchCastRaysF(ctx->ds, n, o, d, b, p, t, ctx->numSMs * 8, ctx->stream);
        checkLaunch();
        OWEC_CUDA(cudaEventRecord(ctx->passStop, ctx->stream));
        if (seconds) {
            OWEC_CUDA(cudaEventSynchronize(ctx->passStop));
            float ms = 0;
            OWEC_CUDA(cudaEventElapsedTime(&ms, ctx->passStart, ctx->passStop));
            *seconds = ms * 1e-3;
        }
    });
}

int owec_trace_counters(owec_ctx* ctx, int enable, uint64_t out[6]) {
    return guarded([&] {
        require(ctx != nullptr, "owec_trace_counters: null context");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ctx->dTravCounters.reserve(6);
        if (out) {
            unsigned long long h[6];
            OWEC_CUDA(cudaMemcpyAsync(h, ctx->dTravCounters.get(), sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
            OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
            for (int k = 0; k < 6; ++k) out[k] = h[k];
        }
        if (enable) {
            OWEC_CUDA(cudaMemsetAsync(ctx->dTravCounters.get(), 0, 6 * sizeof(unsigned long long), ctx->stream));
            OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
            ctx->dLaunchQueries.reserve(owec_ctx::kLaunchLog);
            ctx->launchQueryCount = 0;
            ctx->ds.travCounters = ctx->dTravCounters.get();
        } else {
            ctx->ds.travCounters = nullptr;
        }
    });
}

int owec_trace_launch_queries(owec_ctx* ctx, uint64_t* out, int capacity, int* count) {
    return guarded([&] {
        require(ctx != nullptr && count != nullptr, "owec_trace_launch_queries: null argument");
        require(capacity >= 0 && (out != nullptr || capacity == 0), "owec_trace_launch_queries: no output array");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        const int n = std::min(capacity, ctx->launchQueryCount);
        *count = ctx->launchQueryCount;
        if (n == 0) return;
        std::vector<unsigned long long> h(static_cast<size_t>(n));
        OWEC_CUDA(cudaMemcpyAsync(h.data(), ctx->dLaunchQueries.get(), size_t(n) * sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int k = 0; k < n; ++k) out[k] = h[size_t(k)] - (k ? h[size_t(k - 1)] : 0ull);
    });
}

int owec_inconsistency_log(owec_ctx* ctx, int capacity) {
    return guarded([&] {
        require(ctx != nullptr, "owec_inconsistency_log: null context");
        require(capacity >= 0 && capacity <= (1 << 20), "owec_inconsistency_log: capacity out of range [0, 2^20]");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        if (capacity > 0) {
            ctx->dEventLog.reserve(size_t(capacity) * kEventRecord);
            ctx->dEventLogCount.reserve(1);
            OWEC_CUDA(cudaMemsetAsync(ctx->dEventLogCount.get(), 0, sizeof(uint32_t), ctx->stream));
            OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
            ctx->ds.eventLog = ctx->dEventLog.get();
            ctx->ds.eventLogCount = ctx->dEventLogCount.get();
        } else {
            ctx->ds.eventLog = nullptr;
            ctx->ds.eventLogCount = nullptr;
        }
        ctx->eventLogCap = uint32_t(capacity);
        ctx->ds.eventLogCap = uint32_t(capacity);
    });
}

int owec_read_inconsistency_log(owec_ctx* ctx, double* out, int capacity, int* count) {
    return guarded([&] {
        require(ctx != nullptr && count != nullptr, "owec_read_inconsistency_log: null argument");
        require(capacity >= 0 && (out != nullptr || capacity == 0), "owec_read_inconsistency_log: no output array");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        *count = 0;
        if (ctx->eventLogCap == 0) return;
        uint32_t n = 0;
        OWEC_CUDA(cudaMemcpyAsync(&n, ctx->dEventLogCount.get(), sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        *count = int(std::min<uint32_t>(n, uint32_t(INT32_MAX)));
        const size_t k = std::min<size_t>({size_t(capacity), size_t(n), size_t(ctx->eventLogCap)});
        if (k == 0) return;
        OWEC_CUDA(cudaMemcpyAsync(out, ctx->dEventLog.get(), k * kEventRecord * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

int owec_walk(owec_ctx* ctx, const owec_walk_desc* w, uint64_t first, uint64_t n) {
    return guarded([&] {
        require(ctx && w, "owec_walk: null argument");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureReady(*ctx);
        require(w->source_kind >= OWEC_SOURCE_POINT && w->source_kind <= OWEC_SOURCE_COLLIMATED_SQUARE, "unknown source kind");
        require(w->mode == OWEC_WALK_STOCHASTIC || w->mode == OWEC_WALK_PRIMARY_TRANSMISSION, "unknown walk mode");
        require(w->splat == OWEC_SPLAT_NEAREST || w->splat == OWEC_SPLAT_BILINEAR, "unknown splat");
        require(w->max_events > 0 && w->max_events <= 4096, "max_events out of range");
        require(w->target < ctx->ds.nBoundaries && w->region < ctx->ds.nRegions, "walk target or region out of range");
        require(w->width > 0 && w->height > 0 && uint64_t(w->width) * w->height <= (1ull << 26), "walk film size out of range");
        require(w->half_x > 0 && w->half_y > 0 && w->extent > 0, "walk film or source size out of range");
        require(w->lambda_min > 0 && w->lambda_max >= w->lambda_min, "bad wavelength range");
        const double al = std::sqrt(w->axis[0] * w->axis[0] + w->axis[1] * w->axis[1] + w->axis[2] * w->axis[2]);
        require(al > 0, "walk axis is zero");
        if (!ctx->hasWalk || std::memcmp(w, &ctx->walk, sizeof(owec_walk_desc)) != 0) {
            ctx->walk = *w;
            ctx->hasWalk = true;
            ctx->walks = 0;
            ctx->dWalkBins.resize(size_t(w->width) * w->height);
            ctx->dWalkStats.resize(5);
            OWEC_CUDA(cudaMemsetAsync(ctx->dWalkBins.get(), 0, ctx->dWalkBins.bytes(), ctx->stream));
            OWEC_CUDA(cudaMemsetAsync(ctx->dWalkStats.get(), 0, ctx->dWalkStats.bytes(), ctx->stream));
        }
        if (n == 0) return;
        OWEC_CUDA(cudaEventRecord(ctx->passStart, ctx->stream));
        launchWalk(ctx->settings.precision, ctx->ds, *w, ctx->boundaries[w->target].toLocal, first, n,
                   ctx->dWalkBins.get(), ctx->dWalkStats.get(), ctx->numSMs * 8, ctx->stream);
        checkLaunch();
        OWEC_CUDA(cudaEventRecord(ctx->passStop, ctx->stream));
        OWEC_CUDA(cudaEventSynchronize(ctx->passStop));
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, ctx->passStart, ctx->passStop));
        ctx->lastWalkSeconds = ms * 1e-3;
        ctx->walks += n;
    });
}

int owec_walk_resolve(owec_ctx* ctx, double* bins, owec_walk_stats* stats) {
    return guarded([&] {
        require(ctx != nullptr, "owec_walk_resolve: null context");
        require(ctx->hasWalk, "no walks run", OWEC_E_STATE);
        const owec_walk_desc& w = ctx->walk;
        const size_t nb = size_t(w.width) * w.height;
        std::vector<unsigned long long> fixed(nb), st(5);
        OWEC_CUDA(cudaMemcpyAsync(fixed.data(), ctx->dWalkBins.get(), nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(st.data(), ctx->dWalkStats.get(), 5 * 8, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        if (bins) {
            double measure;
            if (w.source_kind == OWEC_SOURCE_POINT) measure = 2 * kPi * (1 - std::cos(w.extent));
            else if (w.source_kind == OWEC_SOURCE_COLLIMATED) measure = kPi * w.extent * w.extent;
            else measure = 4 * w.extent * w.extent;
            const double binArea = (2 * w.half_x / w.width) * (2 * w.half_y / w.height);
            const double scale = ctx->walks ? measure / (double(ctx->walks) * binArea) / 4294967296.0 : 0.0;
            for (size_t i = 0; i < nb; ++i) bins[i] = double(fixed[i]) * scale;
        }
        if (stats) {
            stats->walks = st[0];
            stats->binned = st[1];
            stats->escaped = st[2];
            stats->events = st[3];
            stats->faults = st[4];
        }
    });
}

int owec_set_heightfield(owec_ctx* ctx, uint32_t boundary, uint64_t n_vertices, double base_z, const double* heights) {
    return guarded([&] {
        require(ctx && heights, "owec_set_heightfield: null argument");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        require(boundary < ctx->boundaries.size() && ctx->boundaries[boundary].shape == OWEC_SHAPE_MESH,
                "the heightfield must be a mesh boundary");
        const owec_ctx::MeshCopy& m = ctx->meshes[boundary];
        require(n_vertices == m.verts.size() / 3, "one height per vertex of the mesh");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        const DBoundary& bd = ctx->boundaries[boundary];
        auto asF = [](uint32_t v) { float f; std::memcpy(&f, &v, 4); return f; };
        const uint32_t base = ctx->triBase[boundary];
        const size_t nt = m.tris.size() / 3;
        for (size_t t = 0; t < nt; ++t) {
            double w[3][3];
            for (int k = 0; k < 3; ++k) {
                const uint32_t v = m.tris[3 * t + k];
                const double local[3] = {m.verts[3 * v], m.verts[3 * v + 1], base_z + heights[v]};
                xfPoint(bd.toWorld.m, local, w[k]);
            }
            const size_t p = base + t;
            const uint32_t ids[3] = {boundary, uint32_t(t), kPrimTriangle};
            double lo[3], hi[3];
            for (int k = 0; k < 3; ++k) {
                ctx->triRecs[3 * p + k] = make_float4(float(w[k][0]), float(w[k][1]), float(w[k][2]), asF(ids[k]));
                for (int a = 0; a < 3; ++a) ctx->tri64[9 * p + 3 * k + a] = w[k][a];
            }
            for (int a = 0; a < 3; ++a) {
                const float f0 = float(w[0][a]), f1 = float(w[1][a]), f2 = float(w[2][a]);
                lo[a] = std::min({double(f0), double(f1), double(f2), w[0][a], w[1][a], w[2][a]});
                hi[a] = std::max({double(f0), double(f1), double(f2), w[0][a], w[1][a], w[2][a]});
            }
            padPrimBox(lo, hi, ctx->primLo[p], ctx->primHi[p]);
        }
        OWEC_CUDA(cudaMemcpyAsync(ctx->dTri.get() + 3 * size_t(base), ctx->triRecs.data() + 3 * size_t(base),
                                  3 * nt * sizeof(float4), cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(ctx->dPrimLo.get() + base, ctx->primLo.data() + base, nt * sizeof(float4),
                                  cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(ctx->dPrimHi.get() + base, ctx->primHi.data() + base, nt * sizeof(float4),
                                  cudaMemcpyHostToDevice, ctx->stream));
        ctx->dHfTris.upload(m.tris.data(), m.tris.size(), ctx->stream);
        buildBvh(*ctx);
        ctx->hf.boundary = boundary;
        ctx->hf.tris = ctx->dHfTris.get();
        ctx->hfVertices = n_vertices;
        for (int k = 0; k < 3; ++k) ctx->hf.zdir[k] = bd.toWorld.m[4 * k + 2];
        ctx->hasWalk = false;  // the walk film of the old heights is stale
    });
}

int owec_walk_adjoint(owec_ctx* ctx, const owec_walk_desc* w, uint64_t first, uint64_t n, const double* g,
                      double* dheights) {
    return guarded([&] {
        require(ctx && w && g && dheights, "owec_walk_adjoint: null argument");
        require(ctx->hf.boundary != kNone, "no heightfield set (owec_set_heightfield)", OWEC_E_STATE);
        require(w->mode == OWEC_WALK_PRIMARY_TRANSMISSION && w->splat == OWEC_SPLAT_BILINEAR,
                "the adjoint needs primary-transmission walks and the bilinear splat");
        require(w->target < ctx->ds.nBoundaries && w->width > 0 && w->height > 0 && w->half_x > 0 && w->half_y > 0,
                "bad walk description");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureReady(*ctx);
        const size_t nb = size_t(w->width) * w->height, nh = ctx->hfVertices;
        DBuf<double> dG(nb), dDH(nh);
        DBuf<unsigned long long> st(5);
        OWEC_CUDA(cudaMemcpyAsync(dG.get(), g, nb * 8, cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemsetAsync(dDH.get(), 0, nh * 8, ctx->stream));
        OWEC_CUDA(cudaMemsetAsync(st.get(), 0, 5 * 8, ctx->stream));
        double measure;
        if (w->source_kind == OWEC_SOURCE_POINT) measure = 2 * kPi * (1 - std::cos(w->extent));
        else if (w->source_kind == OWEC_SOURCE_COLLIMATED) measure = kPi * w->extent * w->extent;
        else measure = 4 * w->extent * w->extent;
        const double binArea = (2 * w->half_x / w->width) * (2 * w->half_y / w->height);
        OWEC_CUDA(cudaEventRecord(ctx->passStart, ctx->stream));
        launchWalkAdjoint(ctx->settings.precision, ctx->ds, *w, ctx->boundaries[w->target].toLocal, ctx->hf, first, n,
                          measure / (double(n) * binArea), dG.get(), dDH.get(), st.get(), ctx->numSMs * 8, ctx->stream);
        checkLaunch();
        OWEC_CUDA(cudaEventRecord(ctx->passStop, ctx->stream));
        std::vector<double> h(nh);
        OWEC_CUDA(cudaMemcpyAsync(h.data(), dDH.get(), nh * 8, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, ctx->passStart, ctx->passStop));
        ctx->lastAdjointSeconds = ms * 1e-3;
        for (size_t i = 0; i < nh; ++i) dheights[i] += h[i];
    });
}

int owec_walk_adjoint_noalloc(owec_ctx* ctx, const owec_walk_desc* w, uint64_t first, uint64_t n, const double* g,
                              double* dheights) {
    return guarded([&] {
        require(ctx && w && g && dheights, "owec_walk_adjoint_noalloc: null argument");
        require(ctx->hf.boundary != kNone, "no heightfield set (owec_set_heightfield)", OWEC_E_STATE);
        require(w->mode == OWEC_WALK_PRIMARY_TRANSMISSION && w->splat == OWEC_SPLAT_BILINEAR,
                "the adjoint needs primary-transmission walks and the bilinear splat");
        require(w->target < ctx->ds.nBoundaries && w->width > 0 && w->height > 0 && w->half_x > 0 && w->half_y > 0,
                "bad walk description");
        const size_t nb = size_t(w->width) * w->height, nh = ctx->hfVertices;
        require(nb <= kNoAllocMaxBins, "owec_walk_adjoint_noalloc: the walk film has more than 512 x 512 = 262144 bins");
        require(nh <= kNoAllocMaxHeights,
                "owec_walk_adjoint_noalloc: the heightfield has more than 1048576 vertices");
        // building the BVH (or its FP64 primitives) would allocate: that belongs to set-up
        require(!ctx->bvhDirty, "owec_walk_adjoint_noalloc: build the BVH first (owec_build_bvh)", OWEC_E_STATE);
        require(ctx->settings.precision == OWEC_PRECISION_FP32 || ctx->prims64Ready,
                "owec_walk_adjoint_noalloc: build the BVH after setting the precision (owec_set_settings, then "
                "owec_build_bvh): that prepares the FP64 primitives",
                OWEC_E_STATE);
        OWEC_CUDA(cudaSetDevice(ctx->device));
        double* base = adjointScratch();
        double* dG = base;
        double* dDH = base + kNoAllocMaxBins;
        auto* st = reinterpret_cast<unsigned long long*>(base + kNoAllocMaxBins + kNoAllocMaxHeights);
        // the scratch keeps the previous call's contents: the accumulator starts from the caller's
        // dheights (so the kernel adds into it directly) and the counters from zero
        OWEC_CUDA(cudaMemcpyAsync(dG, g, nb * 8, cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(dDH, dheights, nh * 8, cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemsetAsync(st, 0, kNoAllocStatsWords * 8, ctx->stream));
        double measure;
        if (w->source_kind == OWEC_SOURCE_POINT) measure = 2 * kPi * (1 - std::cos(w->extent));
        else if (w->source_kind == OWEC_SOURCE_COLLIMATED) measure = kPi * w->extent * w->extent;
        else measure = 4 * w->extent * w->extent;
        const double binArea = (2 * w->half_x / w->width) * (2 * w->half_y / w->height);
        publishScene(*ctx);  // a copy into the context's own scene buffer: no allocation
        OWEC_CUDA(cudaEventRecord(ctx->passStart, ctx->stream));
        launchWalkAdjoint(ctx->settings.precision, ctx->ds, *w, ctx->boundaries[w->target].toLocal, ctx->hf, first, n,
                          measure / (double(n) * binArea), dG, dDH, st, ctx->numSMs * 8, ctx->stream);
        checkLaunch();
        OWEC_CUDA(cudaEventRecord(ctx->passStop, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(dheights, dDH, nh * 8, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, ctx->passStart, ctx->passStop));
        ctx->lastAdjointSeconds = ms * 1e-3;
    });
}

int owec_path_adjoint(owec_ctx* ctx, uint64_t first_pass, int spp, int flags, const double* g, double* dheights,
                      double* replay_xyz, owec_adjoint_stats* stats) {
    return guarded([&] {
        require(ctx && g && dheights, "owec_path_adjoint: null argument");
        require((flags & ~OWEC_ADJOINT_FIXED_DECISIONS) == 0, "owec_path_adjoint: unknown flags");
        require(spp > 0, "owec_path_adjoint: spp must be positive");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        require(ctx->hf.boundary != kNone, "no heightfield set (owec_set_heightfield)", OWEC_E_STATE);
        require(ctx->settings.integrator == OWEC_INTEGRATOR_PATH,
                "owec_path_adjoint differentiates the path integrator's film", OWEC_E_UNSUPPORTED);
        require(!ctx->hasNull, "owec_path_adjoint: scenes with null boundaries are not differentiated",
                OWEC_E_UNSUPPORTED);
        require(first_pass + uint64_t(spp) <= (1ull << 32), "owec_path_adjoint: the PCG32 stream index is 32 bits");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        ensureReady(*ctx);
        size_t freeBefore = 0, freeDuring = 0, total = 0;
        OWEC_CUDA(cudaMemGetInfo(&freeBefore, &total));
        const uint32_t nPix = uint32_t(ctx->ds.det.width) * uint32_t(ctx->ds.det.height);
        const size_t nh = ctx->hfVertices;
        DBuf<double> dG(3 * size_t(nPix)), dDH(nh), dRep(replay_xyz ? 3 * size_t(nPix) : 0);
        DBuf<unsigned long long> ctr(4);
        OWEC_CUDA(cudaMemcpyAsync(dG.get(), g, 3 * size_t(nPix) * 8, cudaMemcpyHostToDevice, ctx->stream));
        OWEC_CUDA(cudaMemsetAsync(dDH.get(), 0, nh * 8, ctx->stream));
        OWEC_CUDA(cudaMemsetAsync(ctr.get(), 0, 4 * 8, ctx->stream));
        if (replay_xyz) OWEC_CUDA(cudaMemsetAsync(dRep.get(), 0, dRep.bytes(), ctx->stream));
        PassParams pp{};
        pp.seed = ctx->settings.seed;
        pp.maxDepth = ctx->settings.max_depth;
        pp.rrDepth = ctx->settings.rr_depth;
        pp.wavelengthMode = ctx->settings.wavelength_mode;
        pp.lambdaMin = float(ctx->settings.lambda_min);
        pp.lambdaMax = float(ctx->settings.lambda_max);
        pp.fresnelFloor = float(std::min(0.49, std::max(0.0, ctx->settings.fresnel_floor)));
        pp.nPixels = nPix;
        pp.anyHitShadows = 1;
        PathAdjointTargets t{dG.get(), 1.0 / double(spp), dDH.get(), replay_xyz ? dRep.get() : nullptr, ctr.get()};
        const bool fixed = (flags & OWEC_ADJOINT_FIXED_DECISIONS) != 0;
        uint64_t cameraPaths = 0;  // the first phase's count (the replay kernel counts only what it walks)
        double replaySeconds = 0;
        OWEC_CUDA(cudaEventRecord(ctx->passStart, ctx->stream));
        if (replay_xyz) {
            // the replayed film needs every path: replay them all from the camera, up to 2^22 per
            // launch (whole samples of the film)
            const uint32_t perBatch = std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(spp), (1u << 22) / std::max(1u, nPix)));
            for (int done = 0; done < spp;) {
                const uint32_t S = std::min<uint32_t>(perBatch, uint32_t(spp - done));
                pp.nPaths = S * nPix;
                pp.streamBase = uint32_t(first_pass + uint64_t(done));
                launchPathAdjoint(ctx->settings.precision, ctx->ds, pp, ctx->hf, t, fixed, nullptr, nullptr,
                                  ctx->numSMs * 8, ctx->stream);
                checkLaunch();
                done += int(S);
            }
        } else if (ctx->settings.precision == OWEC_PRECISION_FP64) {
            cameraPaths = runAdjointCheckpointed<OWEC_PRECISION_FP64>(*ctx, pp, first_pass, spp, t, fixed, freeDuring,
                                                                      replaySeconds);
        } else if (ctx->settings.precision == OWEC_PRECISION_FP32) {
            cameraPaths = runAdjointCheckpointed<OWEC_PRECISION_FP32>(*ctx, pp, first_pass, spp, t, fixed, freeDuring,
                                                                      replaySeconds);
        } else {
            cameraPaths = runAdjointCheckpointed<OWEC_PRECISION_MIXED>(*ctx, pp, first_pass, spp, t, fixed, freeDuring,
                                                                      replaySeconds);
        }
        OWEC_CUDA(cudaEventRecord(ctx->passStop, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        if (replay_xyz) OWEC_CUDA(cudaMemGetInfo(&freeDuring, &total));  // the buffers and the kernel's stacks, held
        std::vector<double> h(nh);
        unsigned long long counts[4];
        OWEC_CUDA(cudaMemcpyAsync(h.data(), dDH.get(), nh * 8, cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaMemcpyAsync(counts, ctr.get(), sizeof(counts), cudaMemcpyDeviceToHost, ctx->stream));
        if (replay_xyz)
            OWEC_CUDA(cudaMemcpyAsync(replay_xyz, dRep.get(), dRep.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
        OWEC_CUDA(cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        OWEC_CUDA(cudaEventElapsedTime(&ms, ctx->passStart, ctx->passStop));
        ctx->lastPathAdjointSeconds = ms * 1e-3;
        for (size_t i = 0; i < nh; ++i) dheights[i] += h[i];
        if (stats) {
            stats->paths = replay_xyz ? counts[0] : cameraPaths;
            stats->heightfield = counts[1];
            stats->dropped = counts[2];
            stats->faults = counts[3];
            stats->seconds = ms * 1e-3;
            stats->device_bytes = freeBefore > freeDuring ? uint64_t(freeBefore - freeDuring) : 0;
            stats->replay_seconds = replay_xyz ? ms * 1e-3 : replaySeconds;
        }
    });
}

int owec_device_peaks(owec_ctx* ctx, double out[3]) {
    return guarded([&] {
        require(ctx && out, "owec_device_peaks: null argument");
        OWEC_CUDA(cudaSetDevice(ctx->device));
        int l2 = 0;
        OWEC_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->device));
        measurePeaks(ctx->numSMs, size_t(l2), ctx->stream, out);
    });
}

int owec_walk_timing(owec_ctx* ctx, double out[2]) {
    return guarded([&] {
        require(ctx && out, "owec_walk_timing: null argument");
        out[0] = ctx->lastWalkSeconds;
        out[1] = ctx->lastAdjointSeconds;
    });
}

int owec_walk_reset(owec_ctx* ctx) {
    return guarded([&] {
        require(ctx != nullptr, "owec_walk_reset: null context");
        ctx->hasWalk = false;
        ctx->walks = 0;
    });
}

int owec_scene_origin(owec_ctx* ctx, double origin[3]) {
    return guarded([&] {
        require(ctx && origin, "owec_scene_origin: null argument");
        require(ctx->hasScene, "no scene uploaded", OWEC_E_STATE);
        for (int k = 0; k < 3; ++k) origin[k] = ctx->ds.origin[k];
    });
}

}  // extern "C"
