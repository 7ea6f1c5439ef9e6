// Particle tracing: the engine's "light" integrator (its GPU renderer's particle pass,
// src/owe/backends/gpu/shaders/particle.slang:356-427 and particle_kernel.slang, read as the
// specification of the estimator; the reference's CPU backend has no light integrator).
//
// A particle leaves an emitter with the flux it carries: a point of an area light with a cosine
// direction, or a point of a disc beyond the world for the sun and the sky. It walks through the
// world with the importance-transport form of the scattering lobes, and every non-specular vertex
// it makes (a surface with a non-delta lobe, a medium scattering event) is connected to the pinhole
// observer through a transmittance ray: the pixel the connection lands in receives
// beta * f * cos * Tr / (d^2 * pixel area * cos^3 at the eye). A surface sensor instead receives the
// particles that reach its front face: beta / pixel area. The area emitter's own point is connected
// too, which is how the emitters themselves appear. Divided by the number of particles, the film
// converges to the same image as the path integrator's wherever a pinhole can see a non-specular
// surface.
//
// One thread walks one particle at a time (grid-stride over the particle indices): a particle's walk
// is a few segments with one connection ray each, traced with the same wide-BVH traversal as the
// camera paths. Every particle draws from its own PCG32 stream keyed by (seed, particle index, pass),
// so a pass gives the same film however it is split into launches.
//
// Splats land in exact fixed-point sums: each pixel channel is a 192-bit integer of three 64-bit
// words, least significant first, whose lowest bit weighs 2^-80. A splat's FP64 significand is
// shifted to its binary exponent and added with 64-bit atomics, carries propagated word by word.
// Integer addition does not depend on order, so the particle film is bitwise reproducible even
// though many threads add to one pixel in no fixed order.
#include "particle.hpp"
#include "transport.cuh"
#include "wavefront.hpp"

namespace owec {

namespace {

template <int M>
using RT = typename Mode<M>::R;

// Keys a particle's stream apart from the camera paths' (hashCombine(seed, pixel)).
constexpr uint64_t kParticleKey = 0x5bd1e995ULL;

// Adds v to word w of a channel, carrying into the words above it.
__device__ __forceinline__ void addWord(unsigned long long* acc, int w, unsigned long long v) {
    const unsigned long long old = atomicAdd(acc + w, v);
    if (old + v >= old) return;  // no wrap-around
    for (int k = w + 1; k < kSplatWordsPerChannel; ++k)
        if (atomicAdd(acc + k, 1ull) != ~0ull) return;
}

// Adds v exactly to a channel's fixed-point sum. Zero, negative and NaN add nothing; bits below
// 2^-80 are dropped. False when v does not fit (infinite, or 2^112 and above).
__device__ bool addFixed(unsigned long long* acc, double v) {
    if (!(v > 0)) return true;
    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(v));
    const int e = int((bits >> 52) & 0x7FF);
    if (e == 0x7FF) return false;
    if (e == 0) return true;  // subnormal: far below the lowest bit
    unsigned long long mant = (bits & 0xFFFFFFFFFFFFFull) | (1ull << 52);  // v = mant * 2^(e - 1075)
    int p = e - 1075 - kSplatExp0;  // position of mant's lowest bit in the sum
    if (p < 0) {
        if (p <= -53) return true;
        mant >>= -p;
        p = 0;
    }
    const int w = p >> 6, r = p & 63;
    if (w >= kSplatWordsPerChannel) return false;
    const unsigned long long hi = r ? mant >> (64 - r) : 0ull;
    if (hi && w + 1 >= kSplatWordsPerChannel) return false;
    addWord(acc, w, mant << r);
    if (hi) addWord(acc, w + 1, hi);
    return true;
}

// A particle's wavelengths (Wavelengths::sample, src/owe/core/wavelengths.hpp:32-44: four hero
// strata from one uniform), or the one uniform wavelength of OWEC_WAVELENGTHS_UNIFORM1.
struct Spec {
    float lambda[NW], pdf[NW];  // pdf 0: a terminated secondary
};
__device__ Spec sampleWavelengths(const ParticleParams& P, double u) {
    Spec s;
    if (P.wavelengthMode == OWEC_WAVELENGTHS_UNIFORM1) {
        const double lam = double(P.lambdaMin) + (double(P.lambdaMax) - double(P.lambdaMin)) * u;
        for (int k = 0; k < NW; ++k) { s.lambda[k] = float(lam); s.pdf[k] = 0.f; }
        s.pdf[0] = float(1.0 / ((double(P.lambdaMax) - double(P.lambdaMin)) * NW));
    } else {
        for (int k = 0; k < NW; ++k) {
            double up = u + double(k) / NW;
            if (up >= 1) up -= 1;
            const double lam = sampleVisibleWavelength(up);
            s.lambda[k] = float(lam);
            s.pdf[k] = float(visibleWavelengthPdf(lam));
        }
    }
    return s;
}

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

// The Gaussian pixel response as an offset in pixels (Detector::filterOffset,
// src/owe/scene/detector.hpp:57-62); nothing is drawn without one.
__device__ __forceinline__ void filterOffset(const DDetector& det, Pcg32& rng, double& fx, double& fy) {
    if (!(det.sigma > 0)) return;
    const Draw2<double> g(rng);
    const double r = sqrt(-2 * log(1 - g.u1)), phi = 2 * kPi * g.u2;
    fx += r * cos(phi) * det.sigma;
    fy += r * sin(phi) * det.sigma;
}

// A connection of point x to the pinhole (IdealObserver::connect): the pixel, the direction and
// distance from x to the eye, and the factor 1 / (d^2 * pixel area * cos^3) of the observer's
// importance. False when x lies behind the eye or outside the field.
struct ObserverLink {
    V3<double> dir;
    double dist, factor;
    uint32_t pixel;
};
__device__ bool linkObserver(const DeviceScene& sc, const ParticleParams& P, const V3<double>& x, Pcg32& rng,
                             ObserverLink& k) {
    const DDetector& det = sc.det;
    const V3<double> eye(det.pos[0], det.pos[1], det.pos[2]);
    const V3<double> w = x - eye;
    const double d2 = dot(w, w);
    if (!(d2 > 0)) return false;
    const double dist = sqrt(d2);
    const V3<double> om = w / dist;
    const double c = dot(om, V3<double>(det.fwd[0], det.fwd[1], det.fwd[2]));
    if (c <= 1e-9) return false;
    const double sx = dot(om, V3<double>(det.right[0], det.right[1], det.right[2])) / c;
    const double sy = dot(om, V3<double>(det.up[0], det.up[1], det.up[2])) / c;
    double fx = (sx / det.tanX + 1) * 0.5 * det.width, fy = (1 - sy / det.tanY) * 0.5 * det.height;
    filterOffset(det, rng, fx, fy);
    if (!(fx >= 0 && fy >= 0 && fx < det.width && fy < det.height)) return false;
    const int px = min(int(fx), det.width - 1), py = min(int(fy), det.height - 1);
    k.pixel = uint32_t(py) * uint32_t(det.width) + uint32_t(px);
    k.factor = 1 / (d2 * P.pixelArea * c * c * c);
    k.dir = -om;
    k.dist = dist;
    return true;
}

// Adds a spectral contribution to a pixel as XYZ (Wavelengths::toXYZ, wavelengths.hpp:71-84).
template <class R>
__device__ void deposit(const DeviceScene& sc, unsigned long long* splat, uint32_t pixel, const Spec& s,
                        const R value[NW], uint32_t& faults) {
    const double inv = 1.0 / (NW * sc.cieYIntegral);
    double x = 0, y = 0, z = 0;
    for (int k = 0; k < NW; ++k) {
        if (s.pdf[k] == 0.f || value[k] == R(0)) continue;
        const double w = double(value[k]) / double(s.pdf[k]) * inv;
        const double l = double(s.lambda[k]);
        x += w * cieX(l);
        y += w * cieY(l);
        z += w * cieZ(l);
    }
    if (!isfinite(x + y + z)) return;
    unsigned long long* px = splat + size_t(pixel) * kSplatWordsPerPixel;
    bool ok = addFixed(px, x);
    ok = addFixed(px + kSplatWordsPerChannel, y) && ok;
    ok = addFixed(px + 2 * kSplatWordsPerChannel, z) && ok;
    faults += !ok;
}

template <int M>
__device__ __forceinline__ V3<double> plainPoint(const V3<double>& p) {
    return Mode<M>::plainOrigin ? V3<double>(V3<float>(p)) : p;
}

// The transmittance of the segment from o to a point `dist` along dir that must arrive in region
// endRegion (Tracer::connectionTransmittance, transport.cpp:237-321): null boundaries are crossed
// when met from the current region, any other matter blocks, media attenuate by Beer-Lambert.
template <int M, bool AnyHit>
__device__ bool connectTransmittance(const DeviceScene& sc, V3<double> o, uint32_t region, uint32_t depB, uint32_t depP,
                                     float errN, const V3<double>& dir, double dist, uint32_t endRegion,
                                     const Spec& s, RT<M> Tr[NW], StackEntry* stack, uint32_t& faults) {
    using R = RT<M>;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    for (int j = 0; j < NW; ++j) Tr[j] = R(1);
    const V3<R> d(dir);
    const float errN0 = errN;
    double remaining = dist;
    for (int guard = 0;; ++guard) {
        // stop short of the end point by its error (as the next-event rays do)
        const double tq = remaining - (4e-6 * remaining + double(errN0) + 1e-9);
        if (guard >= 256 || tq <= 0) break;
        RayQuery<R> rq;
        rq.od = o;
        rq.o = V3<R>(o);
        rq.d = d;
        rq.tmax = R(tq);
        rq.depB = depB;
        rq.depP = depP;
        rq.region = region;
        rq.errN = R(errN);
        HitRec h;
        h.boundary = kNone;
        h.t = INFINITY;
        const int st = traceRay<R, Ro, Rr, AnyHit>(sc, rq, stack, blockDim.x, h);
        if (st == kTraceOverflow) {
            ++faults;
            return false;
        }
        const bool found = st == kTraceHit;
        const double seg = found ? fmin(double(h.t), remaining) : remaining;
        const owec_medium& med = sc.media[sc.regionMedium[region]];
        if (mediumAbsorbs(med, sc) || mediumScatters(med, sc))
            for (int j = 0; j < NW; ++j) {
                const R lam = R(s.lambda[j]);
                Tr[j] *= exp(-(evalSpectrum(sc, med.absorption, lam) + evalSpectrum(sc, med.scattering, lam)) * R(seg));
            }
        if (!found) break;
        if (AnyHit) return false;
        const DBoundary& bd = sc.boundaries[h.boundary];
        if (sc.optics[bd.optics].type != OWEC_SURF_NULL) return false;
        PathRay<R> tmp;
        tmp.o[0] = o.x; tmp.o[1] = o.y; tmp.o[2] = o.z;
        tmp.d[0] = d.x; tmp.d[1] = d.y; tmp.d[2] = d.z;
        const SurfacePoint<R> gp = hitGeometry<R, Ro, Rr>(sc, tmp, h);
        const bool ff = dot(d, gp.n) < R(0);
        if ((ff ? bd.front : bd.back) != region) return false;
        region = ff ? bd.back : bd.front;
        o = plainPoint<M>(gp.p);
        depB = h.boundary;
        depP = h.prim;
        errN = anchorError<R>(gp.p);
        remaining -= double(h.t);
    }
    return region == endRegion;
}

// Counters a thread gathers over its particles, flushed once per warp at the end.
struct Tally {
    uint32_t paths = 0, segments = 0, inconsistencies = 0, leaks = 0, connections = 0, faults = 0;
};

// Connects a particle vertex at x to the observer: f holds the lobe (or phase function) per
// wavelength toward the eye, cosX the cosine at x.
template <int M, bool AnyHit>
__device__ void connectVertex(const DeviceScene& sc, const ParticleParams& P, const V3<double>& x, uint32_t region,
                              uint32_t depB, uint32_t depP, float errN, const ObserverLink& k, const Spec& s,
                              const RT<M> value[NW], unsigned long long* splat, StackEntry* stack, Tally& t) {
    using R = RT<M>;
    R Tr[NW];
    ++t.connections;
    if (!connectTransmittance<M, AnyHit>(sc, x, region, depB, depP, errN, k.dir, k.dist, sc.det.region, s, Tr, stack,
                                         t.faults))
        return;
    R v[NW];
    bool any = false;
    for (int j = 0; j < NW; ++j) {
        v[j] = value[j] * Tr[j];
        any = any || v[j] != R(0);
    }
    if (any) deposit(sc, splat, k.pixel, s, v, t.faults);
}

// One particle: Tracer::traceParticle's emission, walk, connections and sensor hits
// (particle.slang:356-427; the hybrid integrator's partition is not built).
template <int M, bool AnyHit>
__device__ void traceParticle(const DeviceScene& sc, const ParticleParams& P, uint64_t index, StackEntry* stack,
                              unsigned long long* splat, Tally& t) {
    using R = RT<M>;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    const DDetector& det = sc.det;
    const bool observer = det.kind == OWEC_DETECTOR_OBSERVER;
    Pcg32 rng = Pcg32::seeded(hashCombine(P.seed ^ kParticleKey, index), P.stream);
    const Spec s = sampleWavelengths(P, rng.uniform());
    ++t.paths;

    // ---- emission (emitParticle, particle.slang:310-338): the sky, or a light of the table
    const bool fromSky = rng.uniform() < P.pSky;
    uint32_t li = 0;
    if (!fromSky) {
        if (sc.nLights == 0) return;
        const double u = rng.uniform();
        uint32_t lo = 0, hi = sc.nLights;  // World::pickLight: the first cdf above u
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sc.lights[mid].cdf <= u) lo = mid + 1; else hi = mid;
        }
        li = lo < sc.nLights ? lo : sc.nLights - 1;
    }
    const bool distant = fromSky || sc.lights[li].kind == kLightSun;
    const double sel = fromSky ? P.pSky : (1 - P.pSky) * sc.lights[li].pdf;
    if (!(sel > 0)) return;
    V3<double> o, dir;
    uint32_t region, depB = kNone, depP = kNone;
    float errN = 0.f;
    R beta[NW];
    if (distant) {
        // emitDistant (particle.slang:223-262): a direction, then a point of a disc covering the
        // world, beyond it
        const Draw2<double> u(rng);
        V3<double> toward;
        double pdfDir;
        if (fromSky) {
            const double z = 1 - 2 * u.u1, r = sqrt(fmax(0.0, 1 - z * z)), phi = 2 * kPi * u.u2;
            toward = V3<double>(r * cos(phi), r * sin(phi), z);
            pdfDir = 1 / (4 * kPi);
        } else {
            // Environment::sampleSun: uniform in the sun's cone (src/owe/scene/world.hpp:211-213)
            const double cosT = (1 - u.u1) + u.u1 * sc.sunCosMax;
            const double sinT = sqrt(fmax(0.0, 1 - cosT * cosT)), phi = 2 * kPi * u.u2;
            const Frame<double> f(V3<double>(sc.sunDir[0], sc.sunDir[1], sc.sunDir[2]));
            toward = f.toWorld(V3<double>(cos(phi) * sinT, sin(phi) * sinT, cosT));
            pdfDir = 1 / sc.sunSolidAngle;
        }
        dir = -toward;
        V3<double> a1, a2;
        basis(dir, a1, a2);
        const Draw2<double> v(rng);
        double qx, qy;
        concentricDisk(v.u1, v.u2, qx, qy);
        const double Rd = P.discRadius;
        const V3<double> centre(P.discCentre[0], P.discCentre[1], P.discCentre[2]);
        o = centre - dir * (1.01 * Rd) + a1 * (qx * Rd) + a2 * (qy * Rd);
        region = 0;
        const double w = 1 / (sel * pdfDir / (kPi * Rd * Rd));
        for (int j = 0; j < NW; ++j) {
            const R lam = R(s.lambda[j]);
            const R Le = fromSky ? (sc.skyModel == OWEC_SKY_UNIFORM ? evalSpectrum(sc, sc.skySpectrum, lam) : R(0))
                                 : evalSpectrum(sc, sc.sunSpectrum, lam);
            beta[j] = Le * R(w);
        }
    } else {
        // emitFromArea (particle.slang:278-306): a point of the emitter, its own connection to the
        // eye, a side, then a cosine-distributed direction
        const DLight L = sc.lights[li];
        const DBoundary& bd = sc.boundaries[L.boundary];
        const owec_emission em = sc.emissions[bd.emission];
        const Draw2<double> u(rng);
        V3<double> pL, nL;
        sampleShapeArea(bd, u.u1, u.u2, pL, nL);
        const V3<double> p = bd.toWorld.point(pL), n = normalize(bd.toWorld.vector(nL));
        const double pdfA = 1 / bd.area;
        R Le[NW];
        for (int j = 0; j < NW; ++j) Le[j] = (j == 0 || s.pdf[j] != 0.f) ? evalSpectrum(sc, em.radiance, R(s.lambda[j])) : R(0);
        const float errP = anchorError<R>(p);
        ObserverLink k;
        if (observer && linkObserver(sc, P, p, rng, k)) {
            // the emitter's own point seen by the eye (areaEmitterToObserver)
            const double cosL = dot(n, k.dir);
            if ((cosL > 0 && em.front) || (cosL < 0 && em.back)) {
                R v[NW];
                const R f = R(fabs(cosL) * k.factor / (sel * pdfA));
                for (int j = 0; j < NW; ++j) v[j] = Le[j] * f;
                connectVertex<M, AnyHit>(sc, P, plainPoint<M>(p), cosL > 0 ? bd.front : bd.back, L.boundary, 0u, errP,
                                         k, s, v, splat, stack, t);
            }
        }
        bool front = em.front != 0;
        double sidePdf = 1;
        if (em.front && em.back) {
            front = rng.uniform() < 0.5;
            sidePdf = 0.5;
        }
        const Draw2<double> c(rng);
        double dx, dy;
        concentricDisk(c.u1, c.u2, dx, dy);
        dir = Frame<double>(front ? n : -n).toWorld(V3<double>(dx, dy, sqrt(fmax(0.0, 1 - dx * dx - dy * dy))));
        o = p;
        region = front ? bd.front : bd.back;
        depB = L.boundary;
        depP = 0;
        errN = errP;
        // beta = Le cos / (sel pdfA sidePdf cos / pi)
        const R w = R(kPi / (sel * pdfA * sidePdf));
        for (int j = 0; j < NW; ++j) beta[j] = Le[j] * w;
    }
    bool live = false;
    for (int j = 0; j < NW; ++j) {
        if (j > 0 && s.pdf[j] == 0.f) beta[j] = R(0);  // maskTerminated
        live = live || beta[j] != R(0);
    }
    if (!live) return;
    Spec sp = s;  // dispersion may terminate the secondaries on the way
    o = plainPoint<M>(o);
    V3<R> d(dir);

    // ---- the walk (traceParticle's loop, particle.slang:365-426)
    for (int depth = 0;; ++depth) {
        RayQuery<R> rq;
        rq.od = o;
        rq.o = V3<R>(o);
        rq.d = d;
        rq.tmax = R(INFINITY);
        rq.depB = depB;
        rq.depP = depP;
        rq.region = region;
        rq.errN = R(errN);
        HitRec h;
        h.boundary = kNone;
        h.t = INFINITY;
        const int st = traceRay<R, Ro, Rr, false>(sc, rq, stack, blockDim.x, h);
        ++t.segments;
        if (st == kTraceOverflow) {
            ++t.faults;
            return;
        }
        const bool found = st == kTraceHit;
        // sampleMedium (transport.cpp:95-113): hero-extinction distance sampling
        const owec_medium med = sc.media[sc.regionMedium[region]];
        const double seg = found ? double(h.t) : INFINITY;
        bool scatter = false;
        double tS = 0;
        if (mediumScatters(med, sc)) {
            R sT[NW];
            for (int j = 0; j < NW; ++j)
                sT[j] = evalSpectrum(sc, med.absorption, R(sp.lambda[j])) + evalSpectrum(sc, med.scattering, R(sp.lambda[j]));
            tS = -log(1 - rng.uniform()) / double(sT[0]);
            if (tS < seg) {
                const R pdf0 = sT[0] * exp(-sT[0] * R(tS));
                for (int j = 0; j < NW; ++j)
                    beta[j] *= evalSpectrum(sc, med.scattering, R(sp.lambda[j])) * exp(-sT[j] * R(tS)) / pdf0;
                scatter = true;
            } else if (isinf(seg)) {
                return;
            } else {
                const R pass0 = exp(-sT[0] * R(seg));
                for (int j = 0; j < NW; ++j) beta[j] *= exp(-sT[j] * R(seg)) / pass0;
            }
        } else if (mediumAbsorbs(med, sc)) {
            if (isinf(seg)) return;
            for (int j = 0; j < NW; ++j) beta[j] *= exp(-evalSpectrum(sc, med.absorption, R(sp.lambda[j])) * R(seg));
        }
        if (scatter) {
            const V3<double> x = plainPoint<M>(o + V3<double>(d) * tS);
            ObserverLink k;
            if (observer && linkObserver(sc, P, x, rng, k)) {
                const R ph = hgPhase(dot(-d, V3<R>(k.dir)), R(med.g));
                R v[NW];
                for (int j = 0; j < NW; ++j) v[j] = beta[j] * ph * R(k.factor);
                connectVertex<M, AnyHit>(sc, P, x, region, kNone, kNone, 0.f, k, sp, v, splat, stack, t);
            }
            if (depth >= P.maxDepth) return;
            const Draw2<R> u(rng);
            V3<R> wi;
            sampleHg(-d, R(med.g), u.u1, u.u2, wi);
            o = x;
            d = wi;
            depB = kNone;
            depP = kNone;
            errN = 0.f;
            if (depth >= P.rrDepth) {  // a fixed survival probability: any in (0, 1] is unbiased
                if (rng.uniform() >= 0.95) return;
                for (int j = 0; j < NW; ++j) beta[j] *= R(1 / 0.95);
            }
            continue;
        }
        if (!found) {
            t.leaks += region != 0;
            return;
        }
        // meetBoundary (transport.cpp:121-133)
        PathRay<R> ray;
        ray.o[0] = o.x; ray.o[1] = o.y; ray.o[2] = o.z;
        ray.d[0] = d.x; ray.d[1] = d.y; ray.d[2] = d.z;
        const DBoundary& bd = sc.boundaries[h.boundary];
        const SurfacePoint<R> g = hitGeometry<R, Ro, Rr>(sc, ray, h);
        const bool fromFront = dot(d, g.n) < R(0);
        const uint32_t inc = fromFront ? bd.front : bd.back, other = fromFront ? bd.back : bd.front;
        t.inconsistencies += inc != region;
        region = inc;
        const owec_optics& op = sc.optics[bd.optics];
        const V3<double> gp = plainPoint<M>(g.p);
        const float errG = anchorError<R>(g.p);
        if (op.type == OWEC_SURF_NULL) {
            region = other;
            o = gp;
            depB = h.boundary;
            depP = h.prim;
            errN = errG;
            if (depth >= 4 * P.maxDepth) return;
            continue;
        }
        // a surface sensor records the flux reaching its front face
        if (!observer && fromFront && h.boundary == det.boundary) {
            double fx = (g.pLocal.x / det.halfX + 1) * 0.5 * det.width, fy = (1 - g.pLocal.y / det.halfY) * 0.5 * det.height;
            filterOffset(det, rng, fx, fy);
            if (fx >= 0 && fy >= 0 && fx < det.width && fy < det.height) {
                const uint32_t pixel = uint32_t(min(int(fy), det.height - 1)) * uint32_t(det.width) +
                                       uint32_t(min(int(fx), det.width - 1));
                R v[NW];
                for (int j = 0; j < NW; ++j) v[j] = beta[j] * R(1 / P.pixelArea);
                deposit(sc, splat, pixel, sp, v, t.faults);
            }
        }
        if (op.type == OWEC_SURF_DETECTOR || op.type == OWEC_SURF_ABSORBER) return;
        const Interface<R> it = makeInterface(sc, bd, g.n, R(sp.lambda[0]), R(P.fresnelFloor));
        if (!isDeltaOptics<R>(op) && observer) {
            ObserverLink k;
            if (linkObserver(sc, P, gp, rng, k)) {
                const V3<R> wo(k.dir);
                R v[NW];
                bool any = false;
                for (int j = 0; j < NW; ++j) {
                    v[j] = R(0);
                    if (beta[j] == R(0)) continue;
                    R pdf;
                    const Interface<R> itj = j == 0 ? it : makeInterface(sc, bd, g.n, R(sp.lambda[j]), R(P.fresnelFloor));
                    v[j] = beta[j] * evalScatter(sc, itj, d, wo, false, pdf);
                    any = any || v[j] != R(0);
                }
                if (any) {
                    const R cosX = fabs(dot(wo, g.n));
                    for (int j = 0; j < NW; ++j) v[j] *= cosX * R(k.factor);
                    connectVertex<M, AnyHit>(sc, P, gp, dot(wo, g.n) > R(0) ? bd.front : bd.back, h.boundary, h.prim,
                                             errG, k, sp, v, splat, stack, t);
                }
            }
        }
        if (depth >= P.maxDepth) return;
        if (op.type == OWEC_SURF_DIELECTRIC) {  // terminateIfDispersive (transport.cpp:216-225)
            for (int j = 1; j < NW; ++j) {
                if (sp.pdf[j] == 0.f) continue;
                if (isDispersive(it, makeInterface(sc, bd, g.n, R(sp.lambda[j]), R(P.fresnelFloor)))) {
                    for (int m = 1; m < NW; ++m) { sp.pdf[m] = 0.f; beta[m] = R(0); }
                    sp.pdf[0] /= float(NW);
                    break;
                }
            }
        }
        // scatterAtSurface in importance transport (transport.cpp:437-471)
        const Draw3<R> u(rng);
        ScatterSample<R> ss;
        if (!sampleScatter(sc, it, d, u.u1, u.u2, u.u3, false, ss) || !(ss.weight > R(0))) return;
        beta[0] *= ss.weight;
        for (int j = 1; j < NW; ++j) {
            if (sp.pdf[j] == 0.f) continue;
            const Interface<R> itj = makeInterface(sc, bd, g.n, R(sp.lambda[j]), R(P.fresnelFloor));
            beta[j] *= secondaryScatterWeight(sc, itj, d, ss, false);
        }
        if (ss.transmitted) region = other;
        o = gp;
        d = ss.wi;
        depB = h.boundary;
        depP = h.prim;
        errN = errG;
        // particles carry flux: roulette against the event's own weight
        if (depth >= P.rrDepth && ss.weight < R(1)) {
            if (rng.uniform() >= double(ss.weight)) return;
            for (int j = 0; j < NW; ++j) beta[j] *= R(1) / ss.weight;
        }
    }
}

// Adds a per-lane count to a counter, one atomic per warp (all lanes of the warp present).
__device__ __forceinline__ void warpFlush(unsigned long long* counter, uint32_t v) {
    const uint32_t sum = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31u) == 0 && sum) atomicAdd(counter, (unsigned long long)sum);
}

template <int M, bool AnyHit>
__global__ void __launch_bounds__(128) kParticle(DeviceScene sc, ParticleParams P, unsigned long long* splat,
                                                 StatCounters* st) {
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    Tally t;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < P.n; k += uint64_t(gridDim.x) * blockDim.x)
        traceParticle<M, AnyHit>(sc, P, P.first + k, stack, splat, t);
    warpFlush(&st->paths, t.paths);
    warpFlush(&st->segments, t.segments);
    warpFlush(&st->inconsistencies, t.inconsistencies);
    warpFlush(&st->leaks, t.leaks);
    warpFlush(&st->shadowRays, t.connections);
    warpFlush(&st->faults, t.faults);
}

__global__ void __launch_bounds__(256) kResolveSplats(const unsigned long long* splat, uint32_t nPixels, double scale,
                                                      double* xyz) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nPixels) return;
    const unsigned long long* w = splat + size_t(i) * kSplatWordsPerChannel;
    // 2^-80, 2^-16, 2^48: the weights of the three words' lowest bits
    const double v = double(w[0]) * 8.271806125530277e-25 + double(w[1]) * 1.52587890625e-05 +
                     double(w[2]) * 281474976710656.0;
    xyz[i] = v * scale;
}

template <int M, bool AnyHit>
void launchOne(const DeviceScene& sc, const ParticleParams& P, unsigned long long* splat, StatCounters* st, int grid,
               cudaStream_t s) {
    kParticle<M, AnyHit><<<grid, 128, traversalSharedBytes(128), s>>>(sc, P, splat, st);
}

}  // namespace

void launchParticles(int mode, const DeviceScene& sc, const ParticleParams& P, unsigned long long* splat,
                     StatCounters* st, int grid, cudaStream_t s) {
    const bool any = P.anyHitShadows != 0;
    if (mode == OWEC_PRECISION_FP64) {
        if (any) launchOne<OWEC_PRECISION_FP64, true>(sc, P, splat, st, grid, s);
        else launchOne<OWEC_PRECISION_FP64, false>(sc, P, splat, st, grid, s);
    } else if (mode == OWEC_PRECISION_FP32) {
        if (any) launchOne<OWEC_PRECISION_FP32, true>(sc, P, splat, st, grid, s);
        else launchOne<OWEC_PRECISION_FP32, false>(sc, P, splat, st, grid, s);
    } else {
        if (any) launchOne<OWEC_PRECISION_MIXED, true>(sc, P, splat, st, grid, s);
        else launchOne<OWEC_PRECISION_MIXED, false>(sc, P, splat, st, grid, s);
    }
}

void launchResolveSplats(const unsigned long long* splat, uint32_t nPixels, double scale, double* xyz, cudaStream_t s) {
    kResolveSplats<<<(3 * nPixels + 255) / 256, 256, 0, s>>>(splat, nPixels, scale, xyz);
}

}  // namespace owec
