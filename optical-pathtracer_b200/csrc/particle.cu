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
// The particles run through the same wavefront as the camera paths, in the same path-state slots:
// kEmit starts a batch, then every bounce is kIntersect (the camera paths' closest-hit kernel),
// kParticleEvent (free flight, the boundary met, the connection, the scattering sample) and the
// connection kernels (the shadow rays' visibility kernels, splatting instead of adding radiance).
// Every particle draws from its own PCG32 stream keyed by (seed, particle index, pass), so a pass
// gives the same film however it is split into batches, and the splats are exact fixed-point sums
// (splat.cuh), so it does not depend on their order either.
#include "particle.hpp"
#include "transport.cuh"

namespace owec {

namespace {

template <int M>
using RT = typename Mode<M>::R;

// Keys a particle's stream apart from the camera paths' (hashCombine(seed, pixel)).
constexpr uint64_t kParticleKey = 0x5bd1e995ULL;

template <int M>
__device__ __forceinline__ V3<double> plainPoint(const V3<double>& p) {
    return Mode<M>::plainOrigin ? V3<double>(V3<float>(p)) : p;
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

// A connection of point x to the observer (IdealObserver::connect; particle.slang:48-84): a point q
// of the pupil (the eye itself for a pinhole), the pixel, the direction and distance from x to q,
// and the factor 1 / (d^2 * pixel area * cos^3) of the observer's importance (for a thin lens the
// pupil's area cancels against the density of q). False when x lies behind the eye or outside the
// field.
struct ObserverLink {
    V3<double> q, dir;
    double dist, factor;
    uint32_t pixel;
};
__device__ bool linkObserver(const DeviceScene& sc, const ParticleParams& P, const V3<double>& x, Pcg32& rng,
                             ObserverLink& k) {
    const DDetector& det = sc.det;
    const V3<double> eye(det.pos[0], det.pos[1], det.pos[2]);
    const V3<double> R3(det.right[0], det.right[1], det.right[2]), U3(det.up[0], det.up[1], det.up[2]);
    k.q = eye;
    if (det.pupil > 0) {
        const Draw2<double> u(rng);
        double dx, dy;
        concentricDisk(u.u1, u.u2, dx, dy);
        k.q = eye + (R3 * dx + U3 * dy) * det.pupil;
    }
    const V3<double> w = x - k.q;
    const double d2 = dot(w, w);
    if (!(d2 > 0)) return false;
    const double dist = sqrt(d2);
    const V3<double> om = w / dist;
    const double c = dot(om, V3<double>(det.fwd[0], det.fwd[1], det.fwd[2]));
    if (c <= 1e-9) return false;
    double sx, sy;
    if (det.pupil > 0 && isfinite(det.focus)) {
        // where the line from q through x meets the plane in focus, seen from the eye
        const V3<double> F = k.q + om * (det.focus / c) - eye;
        sx = dot(F, R3) / det.focus;
        sy = dot(F, U3) / det.focus;
    } else {
        sx = dot(om, R3) / c;
        sy = dot(om, U3) / c;
    }
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

// Queues the connection of a particle vertex at x to the eye with its contribution before
// transmittance (value per wavelength), one atomic per warp. Every lane of the warp that reaches
// this call takes part (push false: nothing queued).
template <int M>
__device__ void queueConnection(const DeviceScene& sc, PathBuffers<RT<M>>& pb, Queues& q, const SplatTarget& film,
                                uint32_t path, const float pdf[NW], const RT<M> value[NW], const ObserverLink& k,
                                const V3<double>& x, uint32_t region, uint32_t depB, uint32_t depP, float errN,
                                bool push) {
    using R = RT<M>;
    float c[NW];
    bool any = false;
    if (push) {
        const double inv = 1.0 / (NW * sc.cieYIntegral);
        for (int j = 0; j < NW; ++j) {
            c[j] = (pdf[j] != 0.f) ? float(double(value[j]) / double(pdf[j]) * inv) : 0.f;
            any = any || c[j] != 0.f;
        }
    }
    push = push && any;
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, push);
    if (mask == 0) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&q.counts[3], uint32_t(__popc(mask)));
    base = __shfl_sync(active, base, leader);
    if (!push) return;
    const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
    ShadowRay<R> sr;
    sr.o[0] = x.x; sr.o[1] = x.y; sr.o[2] = x.z;
    sr.d[0] = R(k.dir.x); sr.d[1] = R(k.dir.y); sr.d[2] = R(k.dir.z);
    sr.tmax = k.dist;
    sr.region = region;
    sr.endRegion = sc.det.region;
    sr.depB = depB;
    sr.depP = depP;
    sr.endB = kNone;
    sr.path = path;
    sr.errN = errN;
    for (int j = 0; j < NW; ++j) sr.contrib[j] = c[j];
    storeStream(pb.shadow + slot, sr);
    q.shadow[slot] = slot;
    film.pixel[slot] = k.pixel;
}

// ------------------------------------------------------------------ emission
// Particle P.first + i: its wavelengths, the emitter it leaves (emitParticle,
// particle.slang:310-338), the emitter point's own connection, and its first ray.
template <int M>
__global__ void __launch_bounds__(128) kEmit(DeviceScene sc, ParticleParams P, PathBuffers<RT<M>> pb, Queues q,
                                             StatCounters* st, SplatTarget film, uint32_t n) {
    using R = RT<M>;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DDetector& det = sc.det;
    const bool observer = det.kind == OWEC_DETECTOR_OBSERVER;
    Pcg32 rng = Pcg32::seeded(hashCombine(P.seed ^ kParticleKey, P.first + i), P.stream);
    // Wavelengths::sample (src/owe/core/wavelengths.hpp:32-44): four hero strata from one uniform
    PathSpec<R> sp;
    {
        const double u = rng.uniform();
        if (P.wavelengthMode == OWEC_WAVELENGTHS_UNIFORM1) {
            const double lam = double(P.lambdaMin) + (double(P.lambdaMax) - double(P.lambdaMin)) * u;
            for (int k = 0; k < NW; ++k) { sp.lambda[k] = float(lam); sp.pdf[k] = 0.f; }
            sp.pdf[0] = float(1.0 / ((double(P.lambdaMax) - double(P.lambdaMin)) * NW));
        } else {
            for (int k = 0; k < NW; ++k) {
                double up = u + double(k) / NW;
                if (up >= 1) up -= 1;
                const double lam = sampleVisibleWavelength(up);
                sp.lambda[k] = float(lam);
                sp.pdf[k] = float(visibleWavelengthPdf(lam));
            }
        }
        for (int k = 0; k < NW; ++k) sp.L[k] = 0.f;
    }
    // the sky, or a light of the table (World::pickLight: the first cdf above u)
    bool live = true;
    const bool fromSky = rng.uniform() < P.pSky;
    uint32_t li = 0;
    if (!fromSky) {
        if (sc.nLights == 0) {
            live = false;
        } else {
            const double u = rng.uniform();
            uint32_t lo = 0, hi = sc.nLights;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (sc.lights[mid].cdf <= u) lo = mid + 1; else hi = mid;
            }
            li = lo < sc.nLights ? lo : sc.nLights - 1;
        }
    }
    const bool distant = live && (fromSky || sc.lights[li].kind == kLightSun);
    const double sel = !live ? 0.0 : fromSky ? P.pSky : (1 - P.pSky) * sc.lights[li].pdf;
    live = live && sel > 0;
    PathRay<R> ray;
    ray.depB = kNone;
    ray.depP = kNone;
    ray.errN = 0.f;
    ray.region = 0;
    V3<double> o(0, 0, 0), dir(0, 0, 1);
    // the emitter point's own connection to the eye (areaEmitterToObserver)
    bool connect = false;
    ObserverLink k;
    R value[NW] = {R(0), R(0), R(0), R(0)};
    V3<double> cp;
    uint32_t cRegion = 0, cB = kNone;
    float cErr = 0.f;
    if (live && distant) {
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
        const double w = kPi * Rd * Rd / (sel * pdfDir);
        for (int j = 0; j < NW; ++j) {
            const R lam = R(sp.lambda[j]);
            const R Le = fromSky ? skyRadiance(sc, toward, lam) : evalSpectrum(sc, sc.sunSpectrum, lam);
            sp.beta[j] = Le * R(w);
        }
    } else if (live) {
        // emitFromArea (particle.slang:278-306): a point of the emitter, its own connection, a
        // side, then a cosine-distributed direction
        const DLight L = sc.lights[li];
        const DBoundary& bd = sc.boundaries[L.boundary];
        const owec_emission em = sc.emissions[bd.emission];
        const Draw2<double> u(rng);
        V3<double> pL, nL;
        sampleShapeArea(bd, u.u1, u.u2, pL, nL);
        const V3<double> p = bd.toWorld.point(pL), n = normalize(bd.toWorld.vector(nL));
        const double pdfA = 1 / bd.area;
        R Le[NW];
        for (int j = 0; j < NW; ++j)
            Le[j] = (j == 0 || sp.pdf[j] != 0.f) ? evalSpectrum(sc, em.radiance, R(sp.lambda[j])) : R(0);
        const float errP = anchorError<R>(p);
        if (observer && linkObserver(sc, P, p, rng, k)) {
            const double cosL = dot(n, k.dir);
            if ((cosL > 0 && em.front) || (cosL < 0 && em.back)) {
                const R f = R(fabs(cosL) * k.factor / (sel * pdfA));
                for (int j = 0; j < NW; ++j) value[j] = Le[j] * f;
                connect = true;
                cp = plainPoint<M>(p);
                cRegion = cosL > 0 ? bd.front : bd.back;
                cB = L.boundary;
                cErr = errP;
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
        ray.region = front ? bd.front : bd.back;
        ray.depB = L.boundary;
        ray.depP = 0;
        ray.errN = errP;
        // beta = Le cos / (sel pdfA sidePdf cos / pi)
        const R w = R(kPi / (sel * pdfA * sidePdf));
        for (int j = 0; j < NW; ++j) sp.beta[j] = Le[j] * w;
    }
    bool any = false;
    for (int j = 0; j < NW; ++j) {
        if (!live || (j > 0 && sp.pdf[j] == 0.f)) sp.beta[j] = R(0);  // maskTerminated
        any = any || sp.beta[j] != R(0);
    }
    live = live && any;
    const V3<double> op = plainPoint<M>(o);
    ray.o[0] = op.x; ray.o[1] = op.y; ray.o[2] = op.z;
    ray.d[0] = R(dir.x); ray.d[1] = R(dir.y); ray.d[2] = R(dir.z);
    PathAux aux;
    aux.stream = uint32_t(P.stream);
    aux.pixel = 0;
    aux.depth = 0;
    aux.flags = live ? kFlagAlive : 0u;
    aux.prevPdf = 0.f;
    aux.weight = 0.f;
    aux.prevP[0] = aux.prevP[1] = aux.prevP[2] = 0;
    aux.lastBoundary = kNone;
    aux.rngState = rng.state;
    pb.ray[i] = ray;
    pb.spec[i] = sp;
    pb.aux[i] = aux;
    queueConnection<M>(sc, pb, q, film, i, sp.pdf, value, k, cp, cRegion, cB, 0u, cErr, connect);
    warpCount(&st->paths, true);
    warpPush(q.active[0], &q.counts[0], live, i);
}

// ------------------------------------------------------------------ one event of every particle
// What a particle meets after its closest-hit query: free flight through the medium (with a
// connection at a scattering event), escape, the boundary (null crossing, sensor record,
// absorption), the connection of a non-delta surface vertex and the importance-transport
// scattering sample with roulette (traceParticle's loop body, particle.slang:365-426).
// Lean: the instantiation for scenes of Lambertian, absorbing and detecting boundaries in regions
// without participating media (DeviceScene::simpleOptics): the medium events, null boundaries and
// the other lobes fold away, and with them the registers they hold.
template <int M, bool Full, bool Lean>
__global__ void __launch_bounds__(128, Lean ? 4 : 3) kParticleEvent(DeviceScene sc, ParticleParams P, PathBuffers<RT<M>> pb,
                                                                   Queues q, int cur, StatCounters* st, SplatTarget film) {
    using R = RT<M>;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    const int nxt = cur ^ 1;
    const uint32_t n = q.counts[cur];
    const DDetector& det = sc.det;
    const bool observer = det.kind == OWEC_DETECTOR_OBSERVER;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t i = q.active[cur][e];
        const HitRec h = loadStream(pb.hit + i);
        PathRay<R> ray = loadStream(pb.ray + i);
        PathSpec<R> sp = loadStream(pb.spec + i);
        PathAux aux = loadStream(pb.aux + i);
        Pcg32 rng{aux.rngState, (uint64_t(aux.stream) << 1u) | 1u};
        const int depth = int(aux.depth);
        // a connection goes out with the spectrum it was made with, before a dispersive interface
        // ends the secondaries
        float pdfIn[NW];
        for (int j = 0; j < NW; ++j) pdfIn[j] = sp.pdf[j];
        const V3<double> o(ray.o[0], ray.o[1], ray.o[2]);
        const V3<R> d(ray.d[0], ray.d[1], ray.d[2]);
        const bool fault = h.boundary == kNone - 1u;
        const bool found = h.boundary < kNone - 1u;
        bool cont = false, leak = false, inconsistent = false, connect = false, lost = false;
        ObserverLink k;
        R value[NW] = {R(0), R(0), R(0), R(0)};
        V3<double> cp;
        uint32_t cRegion = 0, cB = kNone, cP = kNone;
        float cErr = 0.f;
        if (!fault) {
            // sampleMedium (transport.cpp:95-113): hero-extinction distance sampling
            const owec_medium med = sc.media[sc.regionMedium[ray.region]];
            const double seg = found ? h.t : INFINITY;
            int event = 0;  // 0 pass, 1 scatter, 2 end
            double tS = 0;
            if (Lean) {
            } else if (mediumScatters(med, sc)) {
                R sT[NW];
                for (int j = 0; j < NW; ++j)
                    sT[j] = evalSpectrum(sc, med.absorption, R(sp.lambda[j])) + evalSpectrum(sc, med.scattering, R(sp.lambda[j]));
                tS = -log(1 - rng.uniform()) / double(sT[0]);
                if (tS < seg) {
                    const R pdf0 = sT[0] * exp(-sT[0] * R(tS));
                    for (int j = 0; j < NW; ++j)
                        sp.beta[j] *= evalSpectrum(sc, med.scattering, R(sp.lambda[j])) * exp(-sT[j] * R(tS)) / pdf0;
                    event = 1;
                } else if (isinf(seg)) {
                    event = 2;
                } else {
                    const R pass0 = exp(-sT[0] * R(seg));
                    for (int j = 0; j < NW; ++j) sp.beta[j] *= exp(-sT[j] * R(seg)) / pass0;
                }
            } else if (mediumAbsorbs(med, sc)) {
                if (isinf(seg)) event = 2;
                else
                    for (int j = 0; j < NW; ++j)
                        sp.beta[j] *= exp(-evalSpectrum(sc, med.absorption, R(sp.lambda[j])) * R(seg));
            }
            if (!Lean && event == 1) {
                // a scattering event in the medium: its connection, then Henyey-Greenstein
                const V3<double> x = plainPoint<M>(o + V3<double>(d) * tS);
                if (observer && linkObserver(sc, P, x, rng, k)) {
                    const R ph = hgPhase(dot(-d, V3<R>(k.dir)), R(med.g));
                    for (int j = 0; j < NW; ++j) value[j] = sp.beta[j] * ph * R(k.factor);
                    connect = true;
                    cp = x;
                    cRegion = ray.region;
                }
                if (depth < P.maxDepth) {
                    const Draw2<R> u(rng);
                    V3<R> wi;
                    sampleHg(-d, R(med.g), u.u1, u.u2, wi);
                    ray.o[0] = x.x; ray.o[1] = x.y; ray.o[2] = x.z;
                    ray.d[0] = wi.x; ray.d[1] = wi.y; ray.d[2] = wi.z;
                    ray.depB = kNone;
                    ray.depP = kNone;
                    ray.errN = 0.f;
                    cont = true;
                    if (depth >= P.rrDepth) {  // a fixed survival probability: any in (0, 1] is unbiased
                        cont = rng.uniform() < 0.95;
                        for (int j = 0; j < NW; ++j) sp.beta[j] *= R(1 / 0.95);
                    }
                }
            } else if (event == 0 && !found) {
                leak = ray.region != 0;
            } else if (event == 0) {
                // meetBoundary (transport.cpp:121-133)
                const DBoundary& bd = sc.boundaries[h.boundary];
                const SurfacePoint<R> g = hitGeometry<R, Ro, Rr, Full>(sc, ray, h);
                const bool fromFront = dot(d, g.n) < R(0);
                const uint32_t inc = fromFront ? bd.front : bd.back, other = fromFront ? bd.back : bd.front;
                // an undecided contact counts as inconsistent and ends the particle
                const bool ambiguous = Full && (h.flags & kHitAmbiguous);
                inconsistent = inc != ray.region || ambiguous;
                ray.region = inc;
                const owec_optics& op = sc.optics[bd.optics];
                const V3<double> gp = plainPoint<M>(g.p);
                const float errG = anchorError<R>(g.p);
                if (ambiguous) {
                } else if (!Lean && op.type == OWEC_SURF_NULL) {
                    ray.region = other;
                    ray.o[0] = gp.x; ray.o[1] = gp.y; ray.o[2] = gp.z;
                    ray.depB = h.boundary;
                    ray.depP = h.prim;
                    ray.errN = errG;
                    cont = depth < 4 * P.maxDepth;
                } else {
                    // a surface sensor records the flux reaching its front face
                    if (!observer && fromFront && h.boundary == det.boundary) {
                        // SurfaceSensor::pixelOfHit (particle.slang:88-104)
                        double fx = (g.pLocal.x / det.halfX + 1) * 0.5 * det.width;
                        double fy = (1 - g.pLocal.y / det.halfY) * 0.5 * det.height;
                        if (det.flipX) fx = det.width - fx;
                        if (det.flipY) fy = det.height - fy;
                        filterOffset(det, rng, fx, fy);
                        if (fx >= 0 && fy >= 0 && fx < det.width && fy < det.height) {
                            const uint32_t pixel = uint32_t(min(int(fy), det.height - 1)) * uint32_t(det.width) +
                                                   uint32_t(min(int(fx), det.width - 1));
                            const double inv = 1.0 / (NW * sc.cieYIntegral * P.pixelArea);
                            float c[NW];
                            const R one[NW] = {R(1), R(1), R(1), R(1)};
                            for (int j = 0; j < NW; ++j)
                                c[j] = sp.pdf[j] != 0.f ? float(double(sp.beta[j]) / double(sp.pdf[j]) * inv) : 0.f;
                            lost = !splatXyz(film.words, pixel, sp.lambda, c, one);
                        }
                    }
                    if (op.type != OWEC_SURF_DETECTOR && op.type != OWEC_SURF_ABSORBER) {
                        V3<double> texW;
                        const V3<double>* tex = hitTexture<Full>(sc, bd, g.pLocal, g.nLocal, texW);
                        const Interface<R> it = makeInterface<R, Lean>(sc, bd, g.n, R(sp.lambda[0]), R(P.fresnelFloor), tex);
                        if (observer && (Lean || !isDeltaOptics<R>(op)) && linkObserver(sc, P, gp, rng, k)) {
                            const V3<R> wo(k.dir);
                            bool any = false;
                            for (int j = 0; j < NW; ++j) {
                                if (sp.beta[j] == R(0)) continue;
                                R pdf;
                                const Interface<R> itj =
                                    j == 0 ? it : makeInterface<R, Lean>(sc, bd, g.n, R(sp.lambda[j]), R(P.fresnelFloor), tex);
                                value[j] = sp.beta[j] * evalScatter(sc, itj, d, wo, false, pdf);
                                any = any || value[j] != R(0);
                            }
                            if (any) {
                                const R f = fabs(dot(wo, g.n)) * R(k.factor);
                                for (int j = 0; j < NW; ++j) value[j] *= f;
                                connect = true;
                                cp = gp;
                                cRegion = dot(wo, g.n) > R(0) ? bd.front : bd.back;
                                cB = h.boundary;
                                cP = h.prim;
                                cErr = errG;
                            }
                        }
                        if (depth < P.maxDepth) {
                            if (!Lean && op.type == OWEC_SURF_DIELECTRIC) {  // terminateIfDispersive (transport.cpp:216-225)
                                for (int j = 1; j < NW; ++j) {
                                    if (sp.pdf[j] == 0.f) continue;
                                    if (isDispersive(it, makeInterface(sc, bd, g.n, R(sp.lambda[j]), R(P.fresnelFloor), tex))) {
                                        for (int m = 1; m < NW; ++m) { sp.pdf[m] = 0.f; sp.beta[m] = R(0); }
                                        sp.pdf[0] /= float(NW);
                                        break;
                                    }
                                }
                            }
                            // scatterAtSurface in importance transport (transport.cpp:437-471)
                            const Draw3<R> u(rng);
                            ScatterSample<R> ss;
                            if (sampleScatter(sc, it, d, u.u1, u.u2, u.u3, false, ss) && ss.weight > R(0)) {
                                sp.beta[0] *= ss.weight;
                                for (int j = 1; j < NW; ++j) {
                                    if (sp.pdf[j] == 0.f) continue;
                                    const Interface<R> itj = makeInterface<R, Lean>(sc, bd, g.n, R(sp.lambda[j]), R(P.fresnelFloor), tex);
                                    sp.beta[j] *= secondaryScatterWeight(sc, itj, d, ss, false);
                                }
                                if (ss.transmitted) ray.region = other;
                                ray.o[0] = gp.x; ray.o[1] = gp.y; ray.o[2] = gp.z;
                                ray.d[0] = ss.wi.x; ray.d[1] = ss.wi.y; ray.d[2] = ss.wi.z;
                                ray.depB = h.boundary;
                                ray.depP = h.prim;
                                ray.errN = errG;
                                cont = true;
                                // particles carry flux: roulette against the event's own weight
                                if (depth >= P.rrDepth && ss.weight < R(1)) {
                                    cont = rng.uniform() < double(ss.weight);
                                    for (int j = 0; j < NW; ++j) sp.beta[j] *= R(1) / ss.weight;
                                }
                            }
                        }
                    }
                }
            }
        }
        queueConnection<M>(sc, pb, q, film, i, pdfIn, value, k, cp, cRegion, cB, cP, cErr, connect);
        if (cont) aux.depth += 1;
        else aux.flags &= ~kFlagAlive;
        aux.rngState = rng.state;
        storeStream(pb.ray + i, ray);
        storeStream(pb.spec + i, sp);
        storeStream(pb.aux + i, aux);
        warpCount(&st->leaks, leak);
        warpCount(&st->inconsistencies, inconsistent);
        warpCount(&st->faults, lost);
        warpPush(q.active[nxt], &q.counts[nxt], cont, i);
    }
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

}  // namespace

template <int M>
void launchEmit(const DeviceScene& sc, const ParticleParams& P, const PathBuffers<ModeR<M>>& pb, const Queues& q,
                StatCounters* st, const SplatTarget& film, uint32_t n, cudaStream_t s) {
    kEmit<M><<<(n + 127) / 128, 128, 0, s>>>(sc, P, pb, q, st, film, n);
}
template <int M>
void launchParticleEvent(const DeviceScene& sc, const ParticleParams& P, const PathBuffers<ModeR<M>>& pb,
                         const Queues& q, int cur, StatCounters* st, const SplatTarget& film, int grid, cudaStream_t s) {
    if (sc.fullFeatures) kParticleEvent<M, true, false><<<grid, 128, 0, s>>>(sc, P, pb, q, cur, st, film);
    else if (sc.simpleOptics) kParticleEvent<M, false, true><<<grid, 128, 0, s>>>(sc, P, pb, q, cur, st, film);
    else kParticleEvent<M, false, false><<<grid, 128, 0, s>>>(sc, P, pb, q, cur, st, film);
}
void launchResolveSplats(const unsigned long long* splat, uint32_t nPixels, double scale, double* xyz, cudaStream_t s) {
    kResolveSplats<<<(3 * nPixels + 255) / 256, 256, 0, s>>>(splat, nPixels, scale, xyz);
}

#define OWEC_INSTANTIATE_PARTICLES(M)                                                                              \
    template void launchEmit<M>(const DeviceScene&, const ParticleParams&, const PathBuffers<ModeR<M>>&,          \
                                const Queues&, StatCounters*, const SplatTarget&, uint32_t, cudaStream_t);         \
    template void launchParticleEvent<M>(const DeviceScene&, const ParticleParams&, const PathBuffers<ModeR<M>>&, \
                                         const Queues&, int, StatCounters*, const SplatTarget&, int, cudaStream_t);

OWEC_INSTANTIATE_PARTICLES(0)
OWEC_INSTANTIATE_PARTICLES(1)
OWEC_INSTANTIATE_PARTICLES(2)

}  // namespace owec
