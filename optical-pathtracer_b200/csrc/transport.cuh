// Device transport helpers shared by the wavefront kernels: hit geometry, next-event light
// sampling and emitter densities, medium coefficients, and the warp-aggregated queue push.
// Each follows the reference function it cites (src/owe/transport/transport.cpp,
// src/owe/scene/world.cpp, src/owe/scene/geometry.cpp).
#pragma once

#include "optics.cuh"
#include "path_state.cuh"
#include "textures.cuh"

namespace owec {

// ------------------------------------------------------------------ queues
// Appends item to a queue with one atomic per warp: the active lanes that push agree on a base
// with a ballot, the lowest of them reserves the block of slots.
__device__ __forceinline__ void warpPush(uint32_t* queue, uint32_t* count, bool pred, uint32_t item) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, pred);
    if (mask == 0) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, uint32_t(__popc(mask)));
    base = __shfl_sync(active, base, leader);
    if (pred) queue[base + __popc(mask & ((1u << lane) - 1u))] = item;
}
// A counter increment aggregated over the warp.
__device__ __forceinline__ void warpCount(unsigned long long* counter, bool pred) {
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, pred);
    if (mask == 0) return;
    if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(counter, (unsigned long long)__popc(mask));
}

// ------------------------------------------------------------------ media
// Medium flags: bit 0 absorbs, bit 1 scatters (Medium::absorbs / scatters, src/owe/core/medium.hpp:66-67).
__device__ __forceinline__ bool mediumAbsorbs(const owec_medium& m, const DeviceScene& sc) {
    if (m.absorption < 0) return false;
    const owec_spectrum s = sc.spectra[m.absorption];
    return !(s.kind == OWEC_SPEC_CONSTANT && s.a == 0.0);
}
__device__ __forceinline__ bool mediumScatters(const owec_medium& m, const DeviceScene& sc) {
    if (m.scattering < 0) return false;
    const owec_spectrum s = sc.spectra[m.scattering];
    return !(s.kind == OWEC_SPEC_CONSTANT && s.a == 0.0);
}

// ------------------------------------------------------------------ hit geometry
template <class R>
struct SurfacePoint {
    V3<double> p;   // camera-relative world point
    V3<R> n;        // unit geometric normal toward the front region
    V3<double> pLocal;
    V3<double> nLocal;
};

// The world point and normal of a hit. Triangles: the point on the ray at t and the plane normal
// from the two shorter edges (src/owe/scene/mesh.cpp:73-97). Analytic shapes: the crossing found
// again in the shape's frame, carried to the world by its transform (World::intersect,
// src/owe/scene/world.cpp:570-580).
// A triangle crossing's distance recomputed in FP64 from the triangle's FP64 vertices (leaf-order
// PrimRec64): the traversal finds the triangle in FP32, and the point a path continues from, built
// as origin + t d in FP64, then carries the FP64 vertices' precision instead of the FP32 ones'.
// Kept only when it lies near the FP32 distance (a degenerate triangle keeps the FP32 one).
__device__ __forceinline__ double refineTriangleT(const DeviceScene& sc, uint32_t slot, const V3<double>& od,
                                                  const V3<double>& d, double t32) {
    const PrimRec64& p = sc.prims64[slot];
    const V3<double> v0(p.v0[0], p.v0[1], p.v0[2]), v1(p.v1[0], p.v1[1], p.v1[2]), v2(p.v2[0], p.v2[1], p.v2[2]);
    const V3<double> n = triangleNormal(v0, v1, v2);
    const double t = dot(v0 - od, n) / dot(d, n);
    return (t > 0 && fabs(t - t32) <= 1e-3 * (1 + fabs(t32))) ? t : t32;
}

// Full: the scene may hold shapes beyond spheres, conic sags, plain apertures and cylinders
// (analyticCrossings).
template <class R, class Ro, class Rr, bool Full>
__device__ SurfacePoint<R> hitGeometry(const DeviceScene& sc, const PathRay<R>& ray, const HitRec& h) {
    SurfacePoint<R> sp;
    const DBoundary& bd = sc.boundaries[h.boundary];
    const V3<double> od(ray.o[0], ray.o[1], ray.o[2]);
    const V3<R> d(ray.d[0], ray.d[1], ray.d[2]);
    if (bd.shape == OWEC_SHAPE_MESH) {
        if (sizeof(Rr) == sizeof(double)) {
            // the FP64 vertices alone: the refined distance and the normal from them
            const PrimRec64& p = sc.prims64[h.slot];
            const V3<double> v0(p.v0[0], p.v0[1], p.v0[2]), v1(p.v1[0], p.v1[1], p.v1[2]),
                v2(p.v2[0], p.v2[1], p.v2[2]);
            const V3<double> n = triangleNormal(v0, v1, v2);
            const double t = dot(v0 - od, n) / dot(V3<double>(d), n);
            sp.p = od + V3<double>(d) * ((t > 0 && fabs(t - h.t) <= 1e-3 * (1 + fabs(h.t))) ? t : h.t);
            sp.n = V3<R>(normalize(n));
        } else {
            V3<R> v0, v1, v2;
            uint32_t b, prim, kind;
            TriFetch<R>::get(sc, h.slot, v0, v1, v2, b, prim, kind);
            sp.p = od + V3<double>(d) * h.t;
            sp.n = normalize(triangleNormal(v0, v1, v2));
        }
        sp.pLocal = bd.toLocal.point(sp.p);
        sp.nLocal = bd.toLocal.vector(V3<double>(sp.n));
        return sp;
    }
    if constexpr (Full && sizeof(Rr) == sizeof(double)) {
        // a hit on a sphere far larger than the ray's distance from it (a planet's surface): the
        // double-double solve, and the point on the ray in the world frame, where it keeps its digits
        if (nearSphere(bd, od)) {
            const double t = h.t, slack = 1e-6 * (1 + fabs(t));
            const AHits<double> hits = nearSphereCrossings(bd, od, V3<double>(d), 0.0, t + slack);
            const int n = hits.n;
            if (n > 0) {
                const AHit<double>& hb = (n == 2 && fabs(hits.h1.t - t) < fabs(hits.h0.t - t)) ? hits.h1 : hits.h0;
                sp.p = od + V3<double>(d) * hb.t;
                sp.pLocal = hb.p;
                sp.nLocal = hb.n;
                sp.n = V3<R>(normalize(bd.toWorld.vector(sp.nLocal)));
                return sp;
            }
        }
    }
    const V3<Rr> lo = bd.toLocal.point(V3<Rr>(od));
    const V3<Rr> ld = bd.toLocal.vector(V3<Rr>(d));
    const Rr t = Rr(h.t);
    const double* data = Full ? sc.shapeData + bd.dataOffset : nullptr;
    if (Full && numericShape(bd)) {
        // a bisected crossing is already as precise as its arithmetic: the point on the ray
        const V3<Rr> pl = lo + ld * t;
        sp.pLocal = V3<double>(pl);
        sp.nLocal = V3<double>(numericNormal(bd, data, pl));
        sp.p = bd.toWorld.point(sp.pLocal);
        sp.n = V3<R>(normalize(bd.toWorld.vector(sp.nLocal)));
        return sp;
    }
    AHits<Rr> hits;
    const Rr slack = Rr(1e-6) * (Rr(1) + fabs(t));
    const int n = analyticCrossings<Ro, Rr, Full>(bd, data, lo, ld, Rr(0), t + slack, ray.depB == h.boundary, hits);
    const AHit<Rr>& hb = (n == 2 && fabs(hits.h1.t - t) < fabs(hits.h0.t - t)) ? hits.h1 : hits.h0;
    if (n == 0) {  // not found again (rounding at a trim edge): the point on the ray
        sp.p = od + V3<double>(d) * h.t;
        sp.pLocal = bd.toLocal.point(sp.p);
        sp.nLocal = V3<double>(0, 0, 1);
        sp.n = V3<R>(normalize(bd.toWorld.vector(sp.nLocal)));
        return sp;
    }
    sp.pLocal = V3<double>(hb.p);
    sp.nLocal = V3<double>(hb.n);
    sp.p = bd.toWorld.point(sp.pLocal);
    sp.n = V3<R>(normalize(bd.toWorld.vector(sp.nLocal)));
    return sp;
}

// ------------------------------------------------------------------ sampling
// The concentric map of the unit square onto the unit disk (sampleUniformDiskConcentric,
// src/owe/core/shared/warps.hpp:45-60).
__device__ __forceinline__ void concentricDisk(double u1, double u2, double& x, double& y) {
    const double a = 2 * u1 - 1, b = 2 * u2 - 1;
    x = y = 0;
    if (a == 0 && b == 0) return;
    double r, phi;
    if (fabs(a) > fabs(b)) { r = a; phi = (kPi / 4) * (b / a); }
    else { r = b; phi = kPi / 2 - (kPi / 4) * (a / b); }
    x = r * cos(phi);
    y = r * sin(phi);
}

// The solid-angle density at p of directions toward a uniform point of the disk (centre, unit
// normal, radius). generatingDisk: the direction is known to come from that disk, which is then
// not tested again (diskAimPdf, src/owe/core/shared/optics.hpp:244-255).
__device__ __forceinline__ double diskAimPdf(const V3<double>& p, const V3<double>& wi, const V3<double>& center,
                                             const V3<double>& normal, double radius, bool generatingDisk) {
    if (!(radius > 0)) return 0;
    const double dn = dot(wi, normal);
    if (fabs(dn) < 1e-12) return 0;
    const double t = dot(center - p, normal) / dn;
    const V3<double> delta = p + wi * t - center;
    if (t <= 0 || (!generatingDisk && dot(delta, delta) > radius * radius)) return 0;
    return t * t / (fabs(dn) * kPi * radius * radius);
}

// A Lambertian surface's aim guide (sampleScatter and evalScatter's diffuse mixture,
// src/owe/transport/scattering.cpp:120-131, 173-174): in radiance transport met from the front, the
// uniform uc below the share draws the direction toward the guide's disk (the disk point from u1, u2
// by the concentric map) instead of from the cosine lobe (s, already drawn from u1, u2), and the pdf
// becomes the mixture. p: the camera-relative hit point; n: the normal toward the front.
template <class R>
__device__ __forceinline__ bool aimDiffuse(const owec_optics& o, const V3<double>& p, const V3<R>& n, R albedo, R uc,
                                           R u1, R u2, ScatterSample<R>& s) {
    const double share = o.aim_share;
    const V3<double> c(o.aim_center[0], o.aim_center[1], o.aim_center[2]);
    const V3<double> an(o.aim_normal[0], o.aim_normal[1], o.aim_normal[2]);
    const bool toDisk = double(uc) < share;
    V3<double> wi(s.wi);
    if (toDisk) {
        V3<double> a, b;
        basis(an, a, b);
        double dx, dy;
        concentricDisk(double(u1), double(u2), dx, dy);
        wi = normalize(c + (a * dx + b * dy) * o.aim_radius - p);
    }
    const double cs = dot(wi, V3<double>(n));
    if (cs <= 0) return false;
    const double pdf = (1 - share) * cs * kInvPi + share * diskAimPdf(p, wi, c, an, o.aim_radius, toDisk);
    s.wi = V3<R>(wi);
    s.pdf = R(pdf);
    s.weight = R(double(albedo) * cs * kInvPi / pdf);
    return pdf > 0;
}
// The mixture pdf of direction wi at a guided Lambertian surface, given its cosine-lobe pdf.
__device__ __forceinline__ double aimDiffusePdf(const owec_optics& o, const V3<double>& p, const V3<double>& wi,
                                                double cosinePdf) {
    const V3<double> c(o.aim_center[0], o.aim_center[1], o.aim_center[2]);
    const V3<double> an(o.aim_normal[0], o.aim_normal[1], o.aim_normal[2]);
    return (1 - o.aim_share) * cosinePdf + o.aim_share * diskAimPdf(p, wi, c, an, o.aim_radius, false);
}

// ------------------------------------------------------------------ sky
// The sky's radiance toward direction dir at wavelength lambda (Environment::sky,
// src/owe/scene/world.cpp:56-73): none, uniform, or the gradient from the ground through the
// horizon to the zenith.
template <class R>
__device__ __forceinline__ R skyRadiance(const DeviceScene& sc, const V3<double>& dir, R lambda) {
    if (sc.skyModel == OWEC_SKY_UNIFORM) return evalSpectrum(sc, sc.skySpectrum, lambda);
    if (sc.skyModel != OWEC_SKY_GRADIENT) return R(0);
    const double c = dir.x * sc.skyUp[0] + dir.y * sc.skyUp[1] + dir.z * sc.skyUp[2];
    if (c < 0) return evalSpectrum(sc, sc.skyGround, lambda);
    const R t = R(pow(c, 0.45));
    return evalSpectrum(sc, sc.skyHorizon, lambda) * (R(1) - t) + evalSpectrum(sc, sc.skySpectrum, lambda) * t;
}

// ------------------------------------------------------------------ emitters
// The solid-angle density at ref of a point p (normal n) drawn uniformly from an area
// (areaToSolidAngle, src/owe/core/shared/warps.hpp:103-113); 0 when seen edge-on.
__device__ __forceinline__ double areaToSolidAngle(const V3<double>& ref, const V3<double>& p, const V3<double>& n,
                                                   double area) {
    const V3<double> w = p - ref;
    const double d2 = dot(w, w);
    if (!(d2 > 0)) return 0;
    const double cosL = fabs(dot(n, w)) / sqrt(d2);
    if (cosL <= 1e-12) return 0;
    return d2 / (cosL * area);
}
// 1 - cos of the cone a sphere of radius R about the origin subtends at ref (0 inside it)
// (sphereConeSize, warps.hpp:117-123).
__device__ __forceinline__ double sphereConeSize(const V3<double>& ref, double R) {
    const double dc2 = dot(ref, ref);
    if (dc2 <= R * R * (1 + 1e-9)) return 0;
    const double sin2Max = R * R / dc2;
    return sin2Max / (1 + sqrt(fmax(0.0, 1 - sin2Max)));
}

// Shape::pdfFrom / SphereShape::pdfFrom (src/owe/scene/geometry.cpp:24-27, 477-480) for an emitter
// point seen from ref (both camera-relative world).
__device__ inline double shapePdfFrom(const DBoundary& bd, const V3<double>& ref, const V3<double>& p, const V3<double>& n) {
    if (bd.shape == OWEC_SHAPE_SPHERE) {
        const double omc = sphereConeSize(bd.toLocal.point(ref), bd.params[0]);
        if (omc > 0) return 1.0 / (2 * kPi * omc);
    }
    if (!(bd.area > 0)) return 0;
    return areaToSolidAngle(ref, p, n, bd.area);
}

// A point drawn on an emitting shape (Shape::sampleArea of the reference's shapes:
// geometry.cpp sphere / plane / flat sag / cylinder), in the shape's frame.
__device__ inline void sampleShapeArea(const DBoundary& bd, double u1, double u2, V3<double>& p, V3<double>& n) {
    const double* P = bd.params;
    n = V3<double>(0, 0, 1);
    switch (bd.shape) {
        case OWEC_SHAPE_SPHERE: {
            const double z = 1 - 2 * u1, r = sqrt(fmax(0.0, 1 - z * z)), phi = 2 * kPi * u2;
            n = V3<double>(r * cos(phi), r * sin(phi), z);
            p = n * P[0];
            return;
        }
        case OWEC_SHAPE_PLANE: {
            const int ap = int(P[0]);
            if (ap == OWEC_APERTURE_DISK) {
                const double r = sqrt(P[2] * P[2] + u1 * (P[1] * P[1] - P[2] * P[2])), phi = 2 * kPi * u2;
                p = V3<double>(r * cos(phi), r * sin(phi), 0);
            } else if (ap == OWEC_APERTURE_RECT) {
                p = V3<double>((2 * u1 - 1) * P[1], (2 * u2 - 1) * P[2], 0);
            } else {
                const double r = sqrt(u1), phi = 2 * kPi * u2;
                p = V3<double>(P[1] * r * cos(phi), P[2] * r * sin(phi), 0);
            }
            return;
        }
        case OWEC_SHAPE_SAG: {  // flat sag: an annulus rMin..rMax
            const double r = sqrt(P[3] * P[3] + u1 * (P[2] * P[2] - P[3] * P[3])), phi = 2 * kPi * u2;
            p = V3<double>(r * cos(phi), r * sin(phi), 0);
            return;
        }
        case OWEC_SHAPE_CYLINDER: {
            const double phi = 2 * kPi * u1;
            n = V3<double>(cos(phi), sin(phi), 0);
            p = V3<double>(P[0] * n.x, P[0] * n.y, P[1] + u2 * (P[2] - P[1]));
            return;
        }
        default: p = V3<double>(0, 0, 0); return;
    }
}

struct LightSampleD {
    V3<double> wi;
    double dist;          // Inf for the sun
    double pdf;           // solid angle, including selection
    uint32_t boundary;    // kNone for the sun
    uint32_t region;      // region on the emitting side (finite lights)
    V3<double> p, n;      // emitter point and normal (finite lights)
};

// World::pickLight and the light draw of sampleLightFrom (src/owe/transport/transport.cpp:35-70):
// one uniform selects the light, then u1, u2, u3 are drawn in that order.
template <class R>
__device__ bool sampleLight(const DeviceScene& sc, const V3<double>& ref, Pcg32& rng, LightSampleD& ls, int& li) {
    if (sc.nLights == 0) return false;
    const double u = rng.uniform();
    uint32_t lo = 0, hi = sc.nLights;  // first cdf > u (upper_bound)
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sc.lights[mid].cdf <= u) lo = mid + 1; else hi = mid;
    }
    li = int(lo < sc.nLights ? lo : sc.nLights - 1);
    const DLight L = sc.lights[li];
    const double u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
    (void)u3;
    if (L.kind == kLightSun) {
        // Environment::sampleSun: a uniform direction in the sun's cone (world.hpp:211-213)
        const double cosT = (1 - u1) + u1 * sc.sunCosMax;
        const double sinT = sqrt(fmax(0.0, 1 - cosT * cosT));
        const double phi = 2 * kPi * u2;
        const Frame<double> f(V3<double>(sc.sunDir[0], sc.sunDir[1], sc.sunDir[2]));
        ls.wi = f.toWorld(V3<double>(cos(phi) * sinT, sin(phi) * sinT, cosT));
        ls.dist = INFINITY;
        ls.pdf = L.pdf / sc.sunSolidAngle;
        ls.boundary = kNone;
        ls.region = 0;
        return true;
    }
    const DBoundary& bd = sc.boundaries[L.boundary];
    const V3<double> refL = bd.toLocal.point(ref);
    V3<double> pL, nL;
    double pdfW = 0;
    bool ok = true;
    const double omc = bd.shape == OWEC_SHAPE_SPHERE ? sphereConeSize(refL, bd.params[0]) : 0.0;
    if (omc > 0) {
        // SphereShape::sampleFrom: uniform in the cone the sphere subtends (geometry.cpp:463-475)
        const double Rad = bd.params[0];
        const V3<double> axis = -refL / sqrt(dot(refL, refL));
        V3<double> s, t;
        basis(axis, s, t);
        const double omcT = u1 * omc;
        const double cosT = 1 - omcT;
        const double sinT = sqrt(fmax(0.0, omcT * (2 - omcT)));
        const double phi = 2 * kPi * u2;
        const V3<double> w = s * (sinT * cos(phi)) + t * (sinT * sin(phi)) + axis * cosT;
        double t0, t1;
        bool hitS = false;
        if (sphereRoots(refL, w, Rad, t0, t1)) {
            for (double tt : {t0, t1}) {
                double tr;
                if (refinedRootIn<double, double>(kQuadSphere, Rad * Rad, 0.0, refL, w, tt, 0.0, INFINITY, tr)) {
                    pL = refL + w * tr;
                    hitS = true;
                    break;
                }
            }
        }
        if (!hitS) pL = normalize(refL + w * dot(-refL, w)) * Rad;  // grazing: the tangent point
        nL = normalize(pL);
        pdfW = 1 / (2 * kPi * omc);
    } else {
        sampleShapeArea(bd, u1, u2, pL, nL);
        const V3<double> pW = bd.toWorld.point(pL), nW = normalize(bd.toWorld.vector(nL));
        pdfW = areaToSolidAngle(ref, pW, nW, bd.area);
        ok = pdfW > 0 && bd.area > 0;
    }
    if (!ok) return false;
    ls.p = bd.toWorld.point(pL);
    ls.n = normalize(bd.toWorld.vector(nL));
    const V3<double> dv = ls.p - ref;
    ls.dist = length(dv);
    if (!(ls.dist > 0)) return false;
    ls.wi = dv / ls.dist;
    ls.pdf = L.pdf * pdfW;
    ls.boundary = L.boundary;
    const double cosL = dot(ls.n, -ls.wi);
    ls.region = cosL > 0 ? bd.front : bd.back;
    return true;
}

// The emitted radiance a light sample carries at wavelength lambda (sampleLightFrom's ls.Le).
template <class R>
__device__ R lightSampleLe(const DeviceScene& sc, const LightSampleD& ls, R lambda) {
    if (ls.boundary == kNone) return evalSpectrum(sc, sc.sunSpectrum, lambda);
    const DBoundary& bd = sc.boundaries[ls.boundary];
    const owec_emission e = sc.emissions[bd.emission];
    const double cosL = dot(ls.n, -ls.wi);
    return ((cosL > 0 && e.front) || (cosL < 0 && e.back)) ? evalSpectrum(sc, e.radiance, lambda) : R(0);
}

// ------------------------------------------------------------------ interfaces
// The interface of a boundary at one wavelength (Tracer::makeInterface, transport.cpp:168-185). tex:
// the hit's texture weights when its Lambertian albedo is textured (surfaceAlbedo,
// src/owe/transport/scattering.cpp:190-195), else null.
template <class R, bool Lambertian = false>
__device__ __forceinline__ Interface<R> makeInterface(const DeviceScene& sc, const DBoundary& bd, const V3<R>& n, R lambda,
                                                      R fresnelFloor, const V3<double>* tex = nullptr) {
    Interface<R> it;
    it.o = sc.optics[bd.optics];
    it.n = n;
    // a Lambertian interface as a compile-time fact (the lean surface kernel), so that the lobe
    // switches fold away
    if (Lambertian) it.o.type = OWEC_SURF_DIFFUSE;
    // only the dielectric and conductor lobes read the indices (a Lambertian surface, the most
    // common, skips two index evaluations per wavelength)
    if (it.o.type == OWEC_SURF_DIELECTRIC || it.o.type == OWEC_SURF_CONDUCTOR) {
        it.nFront = regionIndex(sc, bd.front, lambda);
        it.nBack = regionIndex(sc, bd.back, lambda);
    } else {
        it.nFront = it.nBack = R(1);
    }
    it.lambda = lambda;
    it.fresnelFloor = fresnelFloor;
    it.albedo = it.o.reflectance >= 0 ? evalSpectrum(sc, it.o.reflectance, lambda) : R(1);
    if (tex && it.o.type == OWEC_SURF_DIFFUSE) {
        R a = it.albedo * R(tex->x);
        if (tex->y != 0) a += R(tex->y) * evalSpectrum(sc, it.o.texture_b, lambda);
        if (tex->z != 0) a += R(tex->z) * evalSpectrum(sc, it.o.texture_c, lambda);
        it.albedo = a;
    }
    return it;
}

// The texture weights of a hit on boundary bd at local point pl with local normal nl, or null when
// its optics are not textured (or the kernel is the lean instantiation: Full false).
template <bool Full>
__device__ __forceinline__ const V3<double>* hitTexture(const DeviceScene& sc, const DBoundary& bd, const V3<double>& pl,
                                                        const V3<double>& nl, V3<double>& storage) {
    if constexpr (Full) {
        const owec_optics& o = sc.optics[bd.optics];
        if (o.texture == OWEC_TEXTURE_NONE || o.type != OWEC_SURF_DIFFUSE) return nullptr;
        storage = textureWeights(o.texture, o.texture_scale, o.texture_param, pl, nl);
        return &storage;
    } else {
        return nullptr;
    }
}

// Russian roulette against the throughput (CameraPath::survives, transport.cpp:369-374).
template <class R>
__device__ __forceinline__ bool survives(PathSpec<R>& sp, Pcg32& rng) {
    R m = sp.beta[0];
    for (int k = 1; k < NW; ++k) m = fmax(m, sp.beta[k]);
    const double q = fmin(1.0, double(m));
    if (rng.uniform() >= q) return false;
    for (int k = 0; k < NW; ++k) sp.beta[k] *= R(1.0 / q);
    return true;
}

// The anchor error of a point: a few hundred ulps of its magnitude in the precision of the
// arithmetic that produced it (float triangles, or FP64).
template <class R> __device__ __forceinline__ float anchorError(const V3<double>& p);
template <> __device__ __forceinline__ float anchorError<float>(const V3<double>& p) {
    return float(4e-6 * fmax(maxAbs(p), 1e-3));
}
template <> __device__ __forceinline__ float anchorError<double>(const V3<double>& p) {
    return float(1e-12 * fmax(maxAbs(p), 1e-3));
}

}  // namespace owec
