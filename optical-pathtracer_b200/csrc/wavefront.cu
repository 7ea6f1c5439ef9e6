// The wavefront camera-path loop (the reference's Tracer::radiance, src/owe/transport/transport.cpp:
// 473-529, run over every pixel sample of a pass as CpuRenderer::pass does,
// src/owe/backends/cpu/cpu_backend.cpp:52-94).
//
// One bounce is four kernels joined by queues of path slots:
//   kIntersect  closest hit of every active path (the wide-BVH traversal);
//   kMedium     free flight through the current region's medium: Beer-Lambert, distance sampling
//               with sigma_a / sigma_s and Henyey-Greenstein scattering with next-event estimation,
//               escape to the sun and sky; surface hits go to the surface queue;
//   kSurface    the boundary met: region bookkeeping, emission with MIS, spectral interface optics
//               (index models at the hero wavelength, dispersion, Fresnel, GGX, conductors,
//               Lambertian, mirrors), next-event light sampling, the scattering sample, Russian
//               roulette; continuing paths go to the next active queue;
//   kShadow     the visibility of the next-event samples, adding their contributions.
// kGenerate starts a batch of samples; kFilm folds the batch's finished paths into the film in a
// fixed order, so the film does not depend on scheduling.
//
// Each path draws from its own PCG32 stream in the reference's order, so for a one-sample pass
// a device path makes the CPU path's decisions until rounding changes one of them.
#include "camera.cuh"
#include "splat.cuh"
#include "transport.cuh"
#include "wavefront.hpp"

namespace owec {

namespace {

template <int M>
using RT = typename Mode<M>::R;

// Adds one query's node visits and primitive tests to the counters (profiling passes only).
__device__ __forceinline__ void countTraversal(unsigned long long* c, uint32_t visits, uint32_t tests) {
    atomicAdd(c, 1ull);
    atomicAdd(c + 1, (unsigned long long)visits);
    atomicAdd(c + 2, (unsigned long long)tests);
}

// ------------------------------------------------------------------ generate
template <int M>
__global__ void __launch_bounds__(256) kGenerate(DeviceScene sc, PassParams pp, PathBuffers<RT<M>> pb, Queues q,
                                                 StatCounters* st) {
    using R = RT<M>;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pp.nPaths) return;
    PathRay<R> ray;
    PathSpec<R> sp;
    PathAux aux;
    Pcg32 rng;
    const bool live = generateCameraPath<M>(sc, pp, i, ray, sp, aux, rng);
    pb.ray[i] = ray;
    pb.spec[i] = sp;
    pb.aux[i] = aux;
    warpCount(&st->paths, live);
    warpPush(q.active[0], &q.counts[0], live, i);
}

// ------------------------------------------------------------------ intersect
// Visits a lane makes between two refills of its warp: small enough that a finished lane does not
// idle long, large enough to amortise the refill's vote, atomic and ray load.
#ifndef OWEC_REFILL_BUDGET
#define OWEC_REFILL_BUDGET 8
#endif
constexpr int kRefillBudget = OWEC_REFILL_BUDGET;
// Resident blocks per SM the traversal kernels are compiled for (a register cap of
// 65536 / (128 x blocks) per thread).
// Resident blocks per SM the medium and surface kernels are compiled for: they wait on their
// path-state loads, which more resident warps hide.
#ifndef OWEC_SHADING_MIN_BLOCKS
#define OWEC_SHADING_MIN_BLOCKS 3
#endif
#if defined(OWEC_TRAVERSAL_MAXNREG)
#define OWEC_TRAVERSAL_BOUNDS __maxnreg__(OWEC_TRAVERSAL_MAXNREG)
#else
#ifndef OWEC_TRAVERSAL_MIN_BLOCKS
#define OWEC_TRAVERSAL_MIN_BLOCKS 4
#endif
#define OWEC_TRAVERSAL_BOUNDS __launch_bounds__(128, OWEC_TRAVERSAL_MIN_BLOCKS)
#endif

// Hands the warp's idle lanes the next queries of a queue of n through the fetch counter, one
// atomic per warp. Returns this lane's query index (n or more: none). `exhausted` becomes true once
// the counter has passed n, so that a drained warp stops fetching.
__device__ __forceinline__ uint32_t refillLanes(bool idle, uint32_t* fetch, uint32_t n, bool& exhausted) {
    const uint32_t need = __ballot_sync(0xFFFFFFFFu, idle);
    if (need == 0 || exhausted) return n;
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(need) - 1;
    uint32_t base = 0;
    if (lane == uint32_t(leader)) base = atomicAdd(fetch, uint32_t(__popc(need)));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (base + uint32_t(__popc(need)) >= n) exhausted = true;
    return idle ? base + uint32_t(__popc(need & ((1u << lane) - 1u))) : n;
}

// Adds a per-lane count to a counter, one atomic per warp (all lanes of the warp present).
__device__ __forceinline__ void warpFlush(unsigned long long* counter, uint32_t v) {
    const uint32_t sum = __reduce_add_sync(0xFFFFFFFFu, v);
    if ((threadIdx.x & 31u) == 0 && sum) atomicAdd(counter, (unsigned long long)sum);
}

// Closest crossing of every active path's ray. Persistent: each lane advances its query a few
// visits at a time and, when it ends, takes the next query of the queue, so that lanes whose rays
// finish early do not idle until the warp's longest ray is done.
template <int M, bool Count, bool Full>
__global__ void OWEC_TRAVERSAL_BOUNDS kIntersect(DeviceScene sc, PathBuffers<RT<M>> pb, Queues q, int cur,
                                                  StatCounters* st, uint32_t* fetch) {
    using R = RT<M>;
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    const uint32_t n = q.counts[cur];
    Traversal<R, typename Mode<M>::Ro, typename Mode<M>::Rr, false, SharedStack, Count, Full> tr;
    uint32_t path = 0, segments = 0, faults = 0;
    bool alive = false, exhausted = false;
    for (;;) {
        const uint32_t k = refillLanes(!alive, fetch, n, exhausted);
        if (!alive && k < n) {
            path = q.active[cur][k];
            const PathRay<R> ray = loadStream(pb.ray + path);
            RayQuery<R> rq;
            rq.od = rayOrigin(ray.o);
            rq.o = V3<R>(rq.od);
            rq.d = rayDir(ray);
            rq.tmax = R(INFINITY);
            rq.depB = ray.depB;
            rq.depP = ray.depP;
            rq.region = ray.region;
            rq.errN = R(ray.errN);
            tr.begin(rq, stack, blockDim.x);
            alive = true;
        }
        if (__ballot_sync(0xFFFFFFFFu, alive) == 0) break;
        if (alive) {
            int s = tr.run(sc, kRefillBudget);
            if (s != kTraceRunning) {
                HitRec h = tr.hit;
                uint32_t nv = tr.nodeVisits, nt = tr.primTests;
                if (s == kTraceOverflow) {
                    h.boundary = kNone;
                    h.t = INFINITY;
                    const DeepResult d = traceRayDeep<R, typename Mode<M>::Ro, typename Mode<M>::Rr, false, Full>(sc.self, tr.q, h);
                    s = d.status;
                    h = d.hit;
                    nv += d.visits;
                    nt += d.tests;
                }
                if (s != kTraceHit) { h.boundary = kNone; h.t = INFINITY; }
                if (s == kTraceOverflow) h.boundary = kNone - 1u;  // a fault: the path ends
                storeStream(pb.hit + path, h);
                if (Count) countTraversal(sc.travCounters, nv, nt);
                ++segments;
                faults += s == kTraceOverflow;
                alive = false;
            }
        }
    }
    warpFlush(&st->segments, segments);
    warpFlush(&st->faults, faults);
}

// ------------------------------------------------------------------ next-event estimation
// Prepares the shadow ray of directLighting (transport.cpp:323-348) at a surface point (surface
// interface given) or a medium point (phase g), and queues it with its contribution.
template <int M>
__device__ void queueNee(const DeviceScene& sc, PathBuffers<RT<M>>& pb, Queues& q, uint32_t pathIdx,
                         const PathSpec<RT<M>>& sp, const RT<M> beta[NW], const LightSampleD& ls, const RT<M> f[NW],
                         RT<M> pdfScatter,
                         RT<M> cosFactor, const V3<double>& p, uint32_t startRegion, uint32_t depB, uint32_t depP,
                         float errN, bool valid) {
    using R = RT<M>;
    ShadowRay<R> sr;
    float contrib[NW] = {0.f, 0.f, 0.f, 0.f};
    bool any = false;
    if (valid) {
        const R w = powerHeuristic(R(ls.pdf), pdfScatter);
        for (int k = 0; k < NW; ++k) {
            if (sp.pdf[k] == 0.f && k > 0) continue;
            const R Le = lightSampleLe<R>(sc, ls, R(sp.lambda[k]));
            const R c = beta[k] * f[k] * Le * (cosFactor * w / R(ls.pdf));
            contrib[k] = float(c);
            any = any || (c != R(0));
        }
    }
    const bool push = valid && any;
    const unsigned active = __activemask();
    const unsigned mask = __ballot_sync(active, push);
    if (mask == 0) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&q.counts[3], uint32_t(__popc(mask)));
    base = __shfl_sync(active, base, leader);
    if (!push) return;
    const uint32_t slot = base + __popc(mask & ((1u << lane) - 1u));
    setOrigin<M>(sr.o, p);
    sr.d[0] = R(ls.wi.x);
    sr.d[1] = R(ls.wi.y);
    sr.d[2] = R(ls.wi.z);
    sr.tmax = ls.dist;
    sr.region = startRegion;
    sr.endRegion = ls.boundary == kNone ? 0u : ls.region;
    sr.depB = depB;
    sr.depP = depP;
    sr.endB = ls.boundary;
    sr.path = pathIdx;
    sr.errN = errN;
    for (int k = 0; k < NW; ++k) sr.contrib[k] = contrib[k];
    storeStream(pb.shadow + slot, sr);
    q.shadow[slot] = slot;
}

// ------------------------------------------------------------------ medium
// The adjoint's first phase: the path's state at its surface event on the checkpoint boundary, for
// the derivative replay to take over from; the path itself ends here.
template <int M>
__device__ __forceinline__ void checkpointPath(const PassParams& pp, const PathRay<RT<M>>& ray, const PathSpec<RT<M>>& sp,
                                               const PathAux& aux, const HitRec& h) {
    const uint32_t slot = atomicAdd(pp.ckptCount, 1u);
    storeStream(reinterpret_cast<PathCheckpoint<RT<M>>*>(pp.ckpt) + slot, PathCheckpoint<RT<M>>{ray, sp, aux, h});
}

template <int M>
__global__ void __launch_bounds__(128, OWEC_SHADING_MIN_BLOCKS) kMedium(DeviceScene sc, PassParams pp, PathBuffers<RT<M>> pb, Queues q,
                                               int cur, StatCounters* st) {
    using R = RT<M>;
    const int nxt = cur ^ 1;
    const uint32_t n = q.counts[cur];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = q.active[cur][k];
        const HitRec h = loadStream(pb.hit + i);
        {
            // A segment through a region without absorption or scattering that met a boundary has
            // no medium event (sampleMedium draws nothing and changes nothing): straight to the
            // surface queues, without reading or writing the rest of the path's state.
            const owec_medium& m0 = sc.media[sc.regionMedium[pb.ray[i].region]];
            if (h.boundary < kNone - 1u && !mediumAbsorbs(m0, sc) && !mediumScatters(m0, sc)) {
                if (h.boundary == pp.ckptBoundary) {
                    checkpointPath<M>(pp, loadStream(pb.ray + i), loadStream(pb.spec + i), loadStream(pb.aux + i), h);
                    continue;
                }
                const int32_t ot = sc.optics[sc.boundaries[h.boundary].optics].type;
                const bool simple = ot == OWEC_SURF_DIFFUSE || ot == OWEC_SURF_ABSORBER || ot == OWEC_SURF_DETECTOR;
                warpPush(q.surface, &q.counts[2], !simple, i);
                warpPush(q.surfaceSimple, &q.counts[6], simple, i);
                continue;
            }
        }
        PathRay<R> ray = loadStream(pb.ray + i);
        PathSpec<R> sp = loadStream(pb.spec + i);
        PathAux aux = loadStream(pb.aux + i);
        Pcg32 rng{aux.rngState, (uint64_t(aux.stream) << 1u) | 1u};
        const bool fault = h.boundary == kNone - 1u;
        const bool found = h.boundary < kNone - 1u;
        const owec_medium med = sc.media[sc.regionMedium[ray.region]];
        const V3<R> d = rayDir(ray);
        bool toSurface = false, cont = false, leak = false;
        bool neeValid = false;
        LightSampleD ls;
        R fN[NW] = {R(0), R(0), R(0), R(0)};
        R betaNee[NW] = {R(0), R(0), R(0), R(0)};
        R pdfS = R(0);
        V3<double> sp3;
        if (!fault) {
            // sampleMedium (transport.cpp:95-113)
            const double seg = found ? h.t : INFINITY;
            int event = 0;  // 0 pass, 1 scatter, 2 end
            double tS = 0;
            if (mediumScatters(med, sc)) {
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
            if (event == 1) {
                // scatterInMedium (transport.cpp:379-397)
                sp3 = rayOrigin(ray.o) + V3<double>(d) * tS;
                if (int(aux.depth) < pp.maxDepth) {
                    for (int j = 0; j < NW; ++j) betaNee[j] = sp.beta[j];  // directLighting sees beta before RR
                    int li;
                    if (sampleLight<R>(sc, sp3, rng, ls, li)) {
                        bool leZero = true;
                        for (int j = 0; j < NW; ++j)
                            if (lightSampleLe<R>(sc, ls, R(sp.lambda[j])) != R(0)) leZero = false;
                        if (!leZero && ls.pdf > 0) {
                            const R ph = hgPhase(dot(-d, V3<R>(ls.wi)), R(med.g));
                            pdfS = ph;
                            for (int j = 0; j < NW; ++j) fN[j] = ph;
                            neeValid = true;
                        }
                    }
                    const Draw2<R> u(rng);
                    V3<R> wi;
                    aux.prevPdf = float(sampleHg(-d, R(med.g), u.u1, u.u2, wi));
                    aux.flags &= ~kFlagSpecular;
                    aux.prevP[0] = sp3.x;
                    aux.prevP[1] = sp3.y;
                    aux.prevP[2] = sp3.z;
                    setOrigin<M>(ray.o, sp3);
                    ray.d[0] = wi.x;
                    ray.d[1] = wi.y;
                    ray.d[2] = wi.z;
                    ray.depB = kNone;
                    ray.depP = kNone;
                    ray.errN = 0.f;
                    cont = int(aux.depth) < pp.rrDepth || survives(sp, rng);
                }
            } else if (event == 0 && !found) {
                if (ray.region == 0) {
                    // skyMet (transport.cpp:401-417)
                    const bool spec = aux.flags & kFlagSpecular;
                    const V3<double> dd(d);
                    const bool inSun = sc.hasSun && dot(dd, V3<double>(sc.sunDir[0], sc.sunDir[1], sc.sunDir[2])) >= sc.sunCosMax;
                    R w = R(1);
                    if (!spec && inSun) w = powerHeuristic(R(aux.prevPdf), R(sc.sunSelectPdf / sc.sunSolidAngle));
                    for (int j = 0; j < NW; ++j) {
                        const R lam = R(sp.lambda[j]);
                        const R sky = skyRadiance(sc, dd, lam);
                        const R sun = inSun ? evalSpectrum(sc, sc.sunSpectrum, lam) : R(0);
                        sp.L[j] += float(sp.beta[j] * (sky + sun * w));
                    }
                } else {
                    leak = true;
                }
            } else if (event == 0) {
                toSurface = true;
            }
        }
        if (cont) aux.depth += 1;
        if (!toSurface && !cont) aux.flags &= ~kFlagAlive;
        aux.rngState = rng.state;
        storeStream(pb.ray + i, ray);
        storeStream(pb.spec + i, sp);
        storeStream(pb.aux + i, aux);
        queueNee<M>(sc, pb, q, i, sp, betaNee, ls, fN, pdfS, R(1), sp3, ray.region, kNone, kNone, 0.f, neeValid);
        warpCount(&st->leaks, leak);
        if (toSurface && h.boundary == pp.ckptBoundary) {
            checkpointPath<M>(pp, ray, sp, aux, h);
            toSurface = false;
        }
        // surface events on Lambertian, absorbing and detecting boundaries go to the lean kernel
        bool simple = false;
        if (toSurface) {
            const int32_t ot = sc.optics[sc.boundaries[h.boundary].optics].type;
            simple = ot == OWEC_SURF_DIFFUSE || ot == OWEC_SURF_ABSORBER || ot == OWEC_SURF_DETECTOR;
        }
        warpPush(q.surface, &q.counts[2], toSurface && !simple, i);
        warpPush(q.surfaceSimple, &q.counts[6], toSurface && simple, i);
        warpPush(q.active[nxt], &q.counts[nxt], cont, i);
    }
}

// ------------------------------------------------------------------ surface
// Simple: the lean instantiation for the simple surface queue (Lambertian, absorbing and detecting
// boundaries): the other lobes, dispersion and the index models compile out, and with them most of
// the registers.
#ifndef OWEC_SIMPLE_MIN_BLOCKS
#define OWEC_SIMPLE_MIN_BLOCKS 4
#endif
// One inconsistent crossing into the scene's event log: the boundary, triangle and hit flags, the
// ray's region and the region its crossing met, the boundary and triangle the ray left, the path's
// depth, the distance, the ray's camera-relative origin and direction, and its anchor error.
template <class R>
__device__ __noinline__ void logInconsistency(const DeviceScene& sc, const PathRay<R>& ray, const HitRec& h, uint32_t inc,
                                              uint32_t depth) {
    const uint32_t k = atomicAdd(sc.eventLogCount, 1u);
    if (k >= sc.eventLogCap) return;
    const double rec[kEventRecord] = {double(h.boundary), double(h.prim), double(h.flags), double(ray.region), double(inc),
                                      double(ray.depB), double(ray.depP), double(depth), h.t, ray.o[0], ray.o[1], ray.o[2],
                                      double(ray.d[0]), double(ray.d[1]), double(ray.d[2]), double(ray.errN)};
    for (int j = 0; j < kEventRecord; ++j) sc.eventLog[size_t(k) * kEventRecord + j] = rec[j];
}

template <int M, bool Simple, bool Full>
__global__ void __launch_bounds__(128, Simple ? OWEC_SIMPLE_MIN_BLOCKS : OWEC_SHADING_MIN_BLOCKS) kSurface(DeviceScene sc, PassParams pp, PathBuffers<RT<M>> pb, Queues q,
                                                int cur, StatCounters* st) {
    using R = RT<M>;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    const int nxt = cur ^ 1;
    const uint32_t n = Simple ? q.counts[6] : q.counts[2];
    const uint32_t* queue = Simple ? q.surfaceSimple : q.surface;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = queue[k];
        PathRay<R> ray = loadStream(pb.ray + i);
        PathSpec<R> sp = loadStream(pb.spec + i);
        PathAux aux = loadStream(pb.aux + i);
        const HitRec h = loadStream(pb.hit + i);
        Pcg32 rng{aux.rngState, (uint64_t(aux.stream) << 1u) | 1u};
        const DBoundary& bd = sc.boundaries[h.boundary];
        const SurfacePoint<R> g = hitGeometry<R, Ro, Rr, Full>(sc, ray, h);
        const V3<R> d = rayDir(ray);
        // meetBoundary (transport.cpp:121-133)
        const bool fromFront = dot(d, g.n) < R(0);
        const uint32_t inc = fromFront ? bd.front : bd.back;
        const uint32_t other = fromFront ? bd.back : bd.front;
        // an undecided contact counts as inconsistent and ends the path (transport.cpp:503)
        const bool ambiguous = Full && (h.flags & kHitAmbiguous);
        const bool inconsistent = inc != ray.region || ambiguous;
        if constexpr (Full) {
            if (inconsistent && sc.eventLog) logInconsistency(sc, ray, h, inc, aux.depth);
        }
        ray.region = inc;
        aux.lastBoundary = h.boundary;
        const bool specular = aux.flags & kFlagSpecular;
        // emissionMet (transport.cpp:420-433)
        if (bd.emission >= 0 && !ambiguous) {
            const owec_emission e = sc.emissions[bd.emission];
            if (fromFront ? e.front : e.back) {
                R w = R(1);
                if (!specular && bd.light >= 0) {
                    const V3<double> prev(aux.prevP[0], aux.prevP[1], aux.prevP[2]);
                    const double pl = sc.lights[bd.light].pdf * shapePdfFrom(bd, prev, g.p, V3<double>(g.n));
                    if (pl > 0) w = powerHeuristic(R(aux.prevPdf), R(pl));
                }
                for (int j = 0; j < NW; ++j)
                    sp.L[j] += float(sp.beta[j] * evalSpectrum(sc, e.radiance, R(sp.lambda[j])) * w);
            }
        }
        const owec_optics& o = sc.optics[bd.optics];
        const float errN = anchorError<R>(g.p);
        bool cont = false, neeValid = false;
        LightSampleD ls;
        R fN[NW] = {R(0), R(0), R(0), R(0)};
        R betaNee[NW] = {R(0), R(0), R(0), R(0)};
        R pdfS = R(0), cosF = R(0);
        uint32_t neeRegion = ray.region;
        if (ambiguous) {
        } else if (!Simple && o.type == OWEC_SURF_NULL) {
            ray.region = other;
            setOrigin<M>(ray.o, g.p);
            ray.depB = h.boundary;
            ray.depP = h.prim;
            ray.errN = errN;
            cont = int(aux.depth) < 4 * pp.maxDepth;
        } else if ((Simple ? o.type == OWEC_SURF_DIFFUSE : (o.type != OWEC_SURF_ABSORBER && o.type != OWEC_SURF_DETECTOR)) &&
                   int(aux.depth) < pp.maxDepth) {
            // scatterAtSurface (transport.cpp:437-471)
            const R hero = R(sp.lambda[0]);
            V3<double> texW;
            const V3<double>* tex = hitTexture<Full>(sc, bd, g.pLocal, g.nLocal, texW);
            const Interface<R> it = makeInterface<R, Simple>(sc, bd, g.n, hero, R(pp.fresnelFloor), tex);
            if (!Simple && o.type == OWEC_SURF_DIELECTRIC) {  // terminateIfDispersive
                bool alive2 = false;
                for (int j = 1; j < NW; ++j) alive2 = alive2 || sp.pdf[j] != 0.f;
                if (alive2) {
                    for (int j = 1; j < NW; ++j) {
                        if (sp.pdf[j] == 0.f) continue;
                        const Interface<R> it2 = makeInterface(sc, bd, g.n, R(sp.lambda[j]), R(pp.fresnelFloor), tex);
                        if (isDispersive(it, it2)) {
                            for (int m = 1; m < NW; ++m) sp.pdf[m] = 0.f;
                            sp.pdf[0] /= float(NW);
                            for (int m = 1; m < NW; ++m) sp.beta[m] = R(0);
                            break;
                        }
                    }
                }
            }
            for (int j = 0; j < NW; ++j) betaNee[j] = sp.beta[j];  // directLighting sees beta before the scatter
            if (Simple || !isDeltaOptics<R>(o)) {
                int li;
                if (sampleLight<R>(sc, g.p, rng, ls, li)) {
                    bool leZero = true;
                    for (int j = 0; j < NW; ++j)
                        if (lightSampleLe<R>(sc, ls, R(sp.lambda[j])) != R(0)) leZero = false;
                    if (!leZero && ls.pdf > 0) {
                        const V3<R> wi(ls.wi);
                        bool fZero = true;
                        for (int j = 0; j < NW; ++j) {
                            if (sp.pdf[j] == 0.f) continue;
                            R pdf;
                            const Interface<R> itj =
                                j == 0 ? it : makeInterface<R, Simple>(sc, bd, g.n, R(sp.lambda[j]), R(pp.fresnelFloor), tex);
                            fN[j] = evalScatter(sc, itj, d, wi, true, pdf);
                            if (j == 0) pdfS = pdf;
                            if (Full && j == 0 && pdf > R(0) && o.type == OWEC_SURF_DIFFUSE && fromFront && o.aim_share > 0)
                                pdfS = R(aimDiffusePdf(o, g.p, ls.wi, double(pdf)));
                            if (fN[j] != R(0)) fZero = false;
                        }
                        if (!fZero) {
                            cosF = fabs(dot(wi, g.n));
                            neeRegion = dot(wi, g.n) > R(0) ? bd.front : bd.back;
                            neeValid = true;
                        }
                    }
                }
            }
            const Draw3<R> u(rng);
            ScatterSample<R> s;
            bool ok = sampleScatter(sc, it, d, u.u1, u.u2, u.u3, true, s);
            if (Full && ok && o.type == OWEC_SURF_DIFFUSE && fromFront && o.aim_share > 0)
                ok = aimDiffuse(o, g.p, g.n, it.albedo, u.u1, u.u2, u.u3, s);
            if (ok && s.weight > R(0)) {
                // weighScatter (transport.cpp:227-233)
                sp.beta[0] *= s.weight;
                for (int j = 1; j < NW; ++j) {
                    if (sp.pdf[j] == 0.f) continue;
                    const Interface<R> itj = makeInterface<R, Simple>(sc, bd, g.n, R(sp.lambda[j]), R(pp.fresnelFloor), tex);
                    sp.beta[j] *= secondaryScatterWeight(sc, itj, d, s, true);
                }
                if (s.transmitted) ray.region = other;
                aux.flags = s.delta ? (aux.flags | kFlagSpecular) : (aux.flags & ~kFlagSpecular);
                aux.prevPdf = float(s.pdf);
                aux.prevP[0] = g.p.x;
                aux.prevP[1] = g.p.y;
                aux.prevP[2] = g.p.z;
                setOrigin<M>(ray.o, g.p);
                ray.d[0] = s.wi.x;
                ray.d[1] = s.wi.y;
                ray.d[2] = s.wi.z;
                ray.depB = h.boundary;
                ray.depP = h.prim;
                ray.errN = errN;
                cont = !(int(aux.depth) >= pp.rrDepth && !survives(sp, rng));
            }
        }
        if (cont) aux.depth += 1;
        else aux.flags &= ~kFlagAlive;
        aux.rngState = rng.state;
        storeStream(pb.ray + i, ray);
        storeStream(pb.spec + i, sp);
        storeStream(pb.aux + i, aux);
        queueNee<M>(sc, pb, q, i, sp, betaNee, ls, fN, pdfS, cosF, g.p, neeRegion, h.boundary, h.prim, errN, neeValid);
        warpCount(&st->inconsistencies, inconsistent);
        warpPush(q.active[nxt], &q.counts[nxt], cont, i);
    }
}

// ------------------------------------------------------------------ shadow rays
// The visibility of a next-event sample (Tracer::transmittance / connectionTransmittance,
// transport.cpp:237-308): blocked by any matter other than null boundaries, attenuated by the
// media it crosses, and it must arrive in the region on the light's emitting side (the ambient
// region for the sun). AnyHit: the scene has no null boundaries, so the first crossing blocks.
//
// Where a finite light lies: a scene without contacts has no other matter within the FP32 anchor
// error of a light's surface, so a segment that stops that far short of the light point (4e-6 of
// its length, plus the origin's error) passes its own face and misses nothing. With contacts (the
// Full instantiation) matter may lie that close: the segment is walked to the light point and a
// little past it, and a crossing clears it only when it is the light's own face there or lies
// beyond the light point, as the reference's visibility endpoint decides (Tracer::transmittance
// with an Endpoint, transport.cpp:237-284; an emitter is an analytic shape, one face).
//
// Persistent like kIntersect: a lane's job is one shadow ray, walked segment by segment through
// null boundaries; its traversal advances a few visits per round and a finished lane takes the
// next job. Splat: the rays are the light integrator's connections to the eye, whose
// contributions land in the film's pixels instead of the paths' radiance.
template <int M, bool AnyHit, bool Count, bool Splat, bool Full>
__global__ void OWEC_TRAVERSAL_BOUNDS kShadow(DeviceScene sc, PassParams pp, PathBuffers<RT<M>> pb, Queues q,
                                               StatCounters* st, uint32_t* fetch, SplatTarget film) {
    using R = RT<M>;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    const uint32_t n = q.counts[3];
    Traversal<R, Ro, Rr, AnyHit, SharedStack, Count, Full> tr;
    // the light point's identity decides (the Full instantiation's next-event rays)
    constexpr bool kEndpoint = Full && !Splat && !AnyHit;
    R Tr[NW];
    double remaining = 0;
    uint32_t job = 0, path = 0, region = 0, guard = 0, rays = 0, faults = 0, endB = kNone;
    float errN0 = 0.f;
    bool alive = false, exhausted = false;
    for (;;) {
        const uint32_t k = refillLanes(!alive, fetch, n, exhausted);
        bool begin = false;  // start a segment from rq
        RayQuery<R> rq;
        if (!alive && k < n) {
            const ShadowRay<R> sr = loadStream(pb.shadow + k);
            job = k;
            path = sr.path;
            for (int j = 0; j < NW; ++j) Tr[j] = R(1);
            region = sr.region;
            remaining = sr.tmax;
            guard = 0;
            errN0 = sr.errN;
            endB = sr.endB;
            rq.od = rayOrigin(sr.o);
            rq.o = V3<R>(rq.od);
            rq.d = V3<R>(sr.d[0], sr.d[1], sr.d[2]);
            rq.depB = sr.depB;
            rq.depP = sr.depP;
            rq.errN = R(sr.errN);
            alive = true;
            begin = true;
        }
        if (__ballot_sync(0xFFFFFFFFu, alive) == 0) break;
        if (!alive) continue;
        const bool finite = !isinf(remaining);
        int outcome = 0;  // 1 clear, 2 blocked, 3 fault
        if (!begin) {
            int s = tr.run(sc, kRefillBudget);
            if (s == kTraceRunning) continue;
            HitRec h = tr.hit;
            uint32_t nv = tr.nodeVisits, nt = tr.primTests;
            if (s == kTraceOverflow) {
                h.boundary = kNone;
                const DeepResult d = traceRayDeep<R, Ro, Rr, AnyHit, Full>(sc.self, tr.q, h);
                s = d.status;
                h = d.hit;
                nv += d.visits;
                nt += d.tests;
            }
            if (Count) countTraversal(sc.travCounters + 3, nv, nt);
            ++guard;
            if (s == kTraceOverflow) {
                outcome = 3;
            } else {
                const bool found = s == kTraceHit;
                const double seg = found ? fmin(h.t, remaining) : remaining;
                const owec_medium med = sc.media[sc.regionMedium[region]];
                if (mediumAbsorbs(med, sc) || mediumScatters(med, sc)) {
                    if (isinf(seg)) {
                        outcome = 2;
                    } else {
                        for (int j = 0; j < NW; ++j) {
                            const R lam = R(pb.spec[path].lambda[j]);
                            Tr[j] *= exp(-(evalSpectrum(sc, med.absorption, lam) + evalSpectrum(sc, med.scattering, lam)) *
                                         R(seg));
                        }
                    }
                }
                if (outcome == 0) {
                    if (!found) {
                        outcome = (!finite && region != 0) ? 2 : 1;
                    } else if (AnyHit) {
                        outcome = 2;
                    } else if (kEndpoint && finite &&
                               (h.t > remaining ||
                                (h.boundary == endB && !(h.flags & kHitAmbiguous) &&
                                 fabs(h.t - remaining) <= 4e-6 * remaining + double(errN0) + 1e-9))) {
                        outcome = 1;  // the light's own face at the light point, or matter beyond it
                    } else {
                        const DBoundary& bd = sc.boundaries[h.boundary];
                        if (sc.optics[bd.optics].type != OWEC_SURF_NULL || (Full && (h.flags & kHitAmbiguous))) {
                            outcome = 2;
                        } else {
                            // pass the null boundary, if met from this region
                            PathRay<R> tmp;
                            tmp.o[0] = tr.q.od.x; tmp.o[1] = tr.q.od.y; tmp.o[2] = tr.q.od.z;
                            tmp.d[0] = tr.q.d.x; tmp.d[1] = tr.q.d.y; tmp.d[2] = tr.q.d.z;
                            const SurfacePoint<R> gp = hitGeometry<R, Ro, Rr, Full>(sc, tmp, h);
                            const bool ff = dot(tr.q.d, gp.n) < R(0);
                            if ((ff ? bd.front : bd.back) != region) {
                                outcome = 2;
                            } else {
                                region = ff ? bd.back : bd.front;
                                rq = tr.q;
                                rq.od = gp.p;
                                if (Mode<M>::plainOrigin) rq.od = V3<double>(V3<float>(gp.p));
                                rq.o = V3<R>(rq.od);
                                rq.depB = h.boundary;
                                rq.depP = h.prim;
                                rq.errN = R(anchorError<R>(gp.p));
                                if (finite) remaining -= h.t;
                                begin = true;
                            }
                        }
                    }
                }
            }
        }
        if (begin) {
            // the next segment: short of the light's own surface, or with the light point's identity
            // a little past it
            const double w = 4e-6 * remaining + double(errN0) + 1e-9;
            const double tq = finite ? (kEndpoint ? remaining + w : remaining - w) : INFINITY;
            if (guard >= 256) {
                outcome = 2;  // an exhausted walk is no evidence that the rest is clear (transport.cpp:283)
            } else if (finite && tq <= 0) {
                outcome = 1;
            } else {
                rq.tmax = R(tq);
                rq.region = region;
                tr.begin(rq, stack, blockDim.x);
            }
        }
        if (outcome != 0) {
            bool clear = outcome == 1;
            const ShadowRay<R>& sr = pb.shadow[job];
            if (clear && finite && region != sr.endRegion) clear = false;
            if (clear && Splat) {
                faults += !splatXyz(film.words, film.pixel[job], pb.spec[path].lambda, sr.contrib, Tr);
            } else if (clear) {
                float* L = pb.spec[path].L;
                for (int j = 0; j < NW; ++j) L[j] += float(R(sr.contrib[j]) * Tr[j]);
            }
            ++rays;
            faults += outcome == 3;
            alive = false;
        }
    }
    warpFlush(&st->shadowRays, rays);
    warpFlush(&st->faults, faults);
}

// Without null boundaries a shadow ray is one any-hit query, and its bookkeeping (the medium's
// transmittance, the arrival region, the contribution) needs nothing of the traversal. kShadowVis
// runs the queries alone, persistent like kIntersect, and records one visibility byte per shadow ray
// (0 blocked, 1 clear, 2 fault); kShadowApply then adds the contributions in one coalesced pass,
// so the bookkeeping does not run divergently inside the traversal loop.
template <int M, bool Count, bool Full>
__global__ void OWEC_TRAVERSAL_BOUNDS kShadowVis(DeviceScene sc, PathBuffers<RT<M>> pb, Queues q, uint8_t* vis,
                                                  uint32_t* fetch) {
    using R = RT<M>;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    const uint32_t n = q.counts[3];
    Traversal<R, Ro, Rr, true, SharedStack, Count, Full> tr;
    uint32_t job = 0;
    bool alive = false, exhausted = false;
    for (;;) {
        const uint32_t k = refillLanes(!alive, fetch, n, exhausted);
        if (!alive && k < n) {
            const ShadowRay<R>& sr = pb.shadow[k];
            job = k;
            const double tmax = sr.tmax;
            const bool finite = !isinf(tmax);
            // stop short of the light's own surface
            const double tq = finite ? tmax - (4e-6 * tmax + double(sr.errN) + 1e-9) : INFINITY;
            if (finite && tq <= 0) {
                vis[k] = 1;
            } else {
                RayQuery<R> rq;
                rq.od = rayOrigin(sr.o);
                rq.o = V3<R>(rq.od);
                rq.d = V3<R>(sr.d[0], sr.d[1], sr.d[2]);
                rq.depB = sr.depB;
                rq.depP = sr.depP;
                rq.errN = R(sr.errN);
                rq.tmax = R(tq);
                rq.region = sr.region;
                tr.begin(rq, stack, blockDim.x);
                alive = true;
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, alive) == 0 && exhausted) break;
        if (!alive) continue;
        int s = tr.run(sc, kRefillBudget);
        if (s == kTraceRunning) continue;
        uint32_t nv = tr.nodeVisits, nt = tr.primTests;
        if (s == kTraceOverflow) {
            HitRec h = tr.hit;
            h.boundary = kNone;
            const DeepResult d = traceRayDeep<R, Ro, Rr, true, Full>(sc.self, tr.q, h);
            s = d.status;
            nv += d.visits;
            nt += d.tests;
        }
        if (Count) countTraversal(sc.travCounters + 3, nv, nt);
        vis[job] = s == kTraceOverflow ? uint8_t(2) : (s == kTraceHit ? uint8_t(0) : uint8_t(1));
        alive = false;
    }
}

template <int M, bool Splat = false>
__global__ void __launch_bounds__(256) kShadowApply(DeviceScene sc, PathBuffers<RT<M>> pb, Queues q, const uint8_t* vis,
                                                    StatCounters* st, SplatTarget film) {
    using R = RT<M>;
    const uint32_t n = q.counts[3];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint8_t v = vis[k];
        bool clear = v == 1;
        if (clear) {
            const ShadowRay<R> sr = loadStream(pb.shadow + k);
            const bool finite = !isinf(sr.tmax);
            // Tracer::transmittance's one segment (transport.cpp:237-308): the medium it crosses
            R Tr[NW] = {R(1), R(1), R(1), R(1)};
            const owec_medium& med = sc.media[sc.regionMedium[sr.region]];
            if (mediumAbsorbs(med, sc) || mediumScatters(med, sc)) {
                if (!finite) {
                    clear = false;
                } else {
                    const PathSpec<R>& spc = pb.spec[sr.path];
                    for (int j = 0; j < NW; ++j) {
                        const R lam = R(spc.lambda[j]);
                        Tr[j] = exp(-(evalSpectrum(sc, med.absorption, lam) + evalSpectrum(sc, med.scattering, lam)) *
                                    R(sr.tmax));
                    }
                }
            }
            if (!finite && sr.region != 0) clear = false;
            if (finite && sr.region != sr.endRegion) clear = false;
            if (clear && Splat) {
                if (!splatXyz(film.words, film.pixel[k], pb.spec[sr.path].lambda, sr.contrib, Tr)) v = 2;
            } else if (clear) {
                float* L = pb.spec[sr.path].L;
                for (int j = 0; j < NW; ++j) L[j] += float(R(sr.contrib[j]) * Tr[j]);
            }
        }
        warpCount(&st->shadowRays, true);
        warpCount(&st->faults, v == 2);
    }
}

// ------------------------------------------------------------------ film
// XYZ of one path (Wavelengths::toXYZ of L * weight, wavelengths.hpp:71-84); false for a path that
// adds nothing: no estimate, or a non-finite one, which CpuRenderer::pass skips.
template <int M>
__device__ __forceinline__ bool pathXYZ(const DeviceScene& sc, const PathBuffers<RT<M>>& pb, uint32_t i, double v[3]) {
    using R = RT<M>;
    const PathAux aux = pb.aux[i];
    if (!(aux.weight > 0.f)) return false;
    const PathSpec<R> sp = pb.spec[i];
    const double inv = 1.0 / (NW * sc.cieYIntegral);
    double x = 0, y = 0, z = 0;
    for (int k = 0; k < NW; ++k) {
        const double Lk = double(sp.L[k]) * double(aux.weight);
        if (sp.pdf[k] == 0.f || Lk == 0) continue;
        const double w = Lk / double(sp.pdf[k]) * inv;
        const double l = double(sp.lambda[k]);
        x += w * cieX(l);
        y += w * cieY(l);
        z += w * cieZ(l);
    }
    if (!isfinite(x + y + z)) return false;
    v[0] = x;
    v[1] = y;
    v[2] = z;
    return true;
}

// One compensated (Kahan) addition.
__device__ __forceinline__ void kahanAdd(double& s, double& c, double v) {
    const double yv = v - c;
    const double t = s + yv;
    c = (t - s) - yv;
    s = t;
}

// Folds the batch's samples of every pixel into the film in sample order, with compensated FP64
// sums as CpuRenderer::pass keeps them; one thread per pixel (films with many pixels).
template <int M>
__global__ void __launch_bounds__(256) kFilm(DeviceScene sc, PassParams pp, PathBuffers<RT<M>> pb, double* film,
                                             double* comp, double* samples, uint32_t samplesPerPixel) {
    const uint32_t pixel = blockIdx.x * blockDim.x + threadIdx.x;
    if (pixel >= pp.nPixels) return;
    double s[3], c[3];
    for (int ch = 0; ch < 3; ++ch) { s[ch] = film[3 * pixel + ch]; c[ch] = comp[3 * pixel + ch]; }
    for (uint32_t sub = 0; sub < samplesPerPixel; ++sub) {
        double v[3];
        if (!pathXYZ<M>(sc, pb, sub * pp.nPixels + pixel, v)) continue;
        for (int ch = 0; ch < 3; ++ch) kahanAdd(s[ch], c[ch], v[ch]);
    }
    for (int ch = 0; ch < 3; ++ch) { film[3 * pixel + ch] = s[ch]; comp[3 * pixel + ch] = c[ch]; }
    samples[pixel] += samplesPerPixel;
}

// The same fold for films of few pixels and many samples per pixel: one block per pixel. Its
// threads turn 256 consecutive samples into XYZ at a time; three lanes, one per channel, then add
// them to the compensated sums in sample order, so the film is kFilm's to the bit.
constexpr int kFilmChunk = 256;

template <int M>
__global__ void __launch_bounds__(kFilmChunk) kFilmPerPixel(DeviceScene sc, PassParams pp, PathBuffers<RT<M>> pb,
                                                            double* film, double* comp, double* samples,
                                                            uint32_t samplesPerPixel) {
    __shared__ double xyz[3][kFilmChunk];
    __shared__ uint8_t keep[kFilmChunk];
    const uint32_t pixel = blockIdx.x;
    const int ch = threadIdx.x;  // the folding lanes
    double s = 0, c = 0;
    if (ch < 3) { s = film[3 * pixel + ch]; c = comp[3 * pixel + ch]; }
    for (uint32_t base = 0; base < samplesPerPixel; base += kFilmChunk) {
        const uint32_t sub = base + threadIdx.x;
        double v[3];
        const bool ok = sub < samplesPerPixel && pathXYZ<M>(sc, pb, sub * pp.nPixels + pixel, v);
        keep[threadIdx.x] = ok;
        if (ok)
            for (int k = 0; k < 3; ++k) xyz[k][threadIdx.x] = v[k];
        __syncthreads();
        if (ch < 3) {
            const int n = int(umin(uint32_t(kFilmChunk), samplesPerPixel - base));
            for (int j = 0; j < n; ++j)
                if (keep[j]) kahanAdd(s, c, xyz[ch][j]);
        }
        __syncthreads();
    }
    if (ch < 3) { film[3 * pixel + ch] = s; comp[3 * pixel + ch] = c; }
    if (threadIdx.x == 0) samples[pixel] += samplesPerPixel;
}

// The film's compensated sums as plain sums (sum - compensation), for a device-side reduction.
__global__ void __launch_bounds__(256) kFoldFilm(const double* film, const double* comp, double* out, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = film[i] - comp[i];
}

// ------------------------------------------------------------------ ray casts
template <int M, bool Full>
__global__ void __launch_bounds__(128) kCastRays(DeviceScene sc, uint64_t n, const double* o, const double* d,
                                                 uint32_t* boundary, uint32_t* prim, double* t) {
    using R = RT<M>;
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        RayQuery<R> rq;
        rq.od = V3<double>(o[3 * i] - sc.origin[0], o[3 * i + 1] - sc.origin[1], o[3 * i + 2] - sc.origin[2]);
        if (Mode<M>::plainOrigin) rq.od = V3<double>(V3<float>(rq.od));
        rq.o = V3<R>(rq.od);
        rq.d = V3<R>(R(d[3 * i]), R(d[3 * i + 1]), R(d[3 * i + 2]));
        rq.tmax = R(INFINITY);
        rq.depB = rq.depP = kNone;
        rq.region = kNone;
        rq.errN = R(0);
        HitRec h;
        const int s = traceRay<R, typename Mode<M>::Ro, typename Mode<M>::Rr, false, Full>(sc, rq, stack, blockDim.x, h);
        if (s == kTraceHit) {
            boundary[i] = h.boundary;
            prim[i] = h.prim;
            const bool refine = sizeof(typename Mode<M>::Rr) == sizeof(double) && sc.boundaries[h.boundary].shape == OWEC_SHAPE_MESH;
            t[i] = refine ? refineTriangleT(sc, h.slot, rq.od, V3<double>(d[3 * i], d[3 * i + 1], d[3 * i + 2]), h.t) : h.t;
        } else {
            boundary[i] = s == kTraceOverflow ? kNone - 1u : kNone;
            prim[i] = 0;
            t[i] = INFINITY;
        }
    }
}

// Device-resident FP32 camera-relative rays (the benchmark's ray-cast workload).
template <bool Full>
__global__ void __launch_bounds__(128) kCastRaysF(DeviceScene sc, uint64_t n, const float* o, const float* d,
                                                  uint32_t* boundary, uint32_t* prim, float* t) {
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        RayQuery<float> rq;
        rq.o = V3<float>(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
        rq.od = V3<double>(rq.o);
        rq.d = V3<float>(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
        rq.tmax = INFINITY;
        rq.depB = rq.depP = kNone;
        rq.region = kNone;
        rq.errN = 0.f;
        HitRec h;
        const int s = traceRay<float, float, double, false, Full>(sc, rq, stack, blockDim.x, h);
        boundary[i] = s == kTraceHit ? h.boundary : (s == kTraceOverflow ? kNone - 1u : kNone);
        prim[i] = s == kTraceHit ? h.prim : 0u;
        t[i] = s == kTraceHit ? float(h.t) : INFINITY;
    }
}

// Primitive records in leaf order (the triangles' camera-relative vertices and identities).
__global__ void kMaterialize(const uint32_t* leafOrder, uint32_t n, const float4* tri, const double* tri64,
                             PrimRec* prims, PrimRec64* prims64) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t p = leafOrder[s];
    const float4 a = tri[3 * p], b = tri[3 * p + 1], c = tri[3 * p + 2];
    PrimRec r;
    r.ax = a.x; r.ay = a.y; r.az = a.z; r.aw = a.w;
    r.bx = b.x; r.by = b.y; r.bz = b.z; r.bw = b.w;
    r.cx = c.x; r.cy = c.y; r.cz = c.z; r.cw = c.w;
    prims[s] = r;
    if (prims64) {
        PrimRec64 q;
        for (int k = 0; k < 3; ++k) {
            q.v0[k] = tri64[9 * size_t(p) + k];
            q.v1[k] = tri64[9 * size_t(p) + 3 + k];
            q.v2[k] = tri64[9 * size_t(p) + 6 + k];
        }
        q.boundary = __float_as_uint(a.w);
        q.prim = __float_as_uint(b.w);
        q.kind = __float_as_uint(c.w);
        q.pad = 0;
        prims64[s] = q;
    }
}

// Per-pixel mean XYZ of the film (Renderer::resolve): the compensated sums over the sample count.
__global__ void __launch_bounds__(256) kResolve(const double* film, const double* comp, const double* samples, uint32_t nPixels,
                                                double* xyz) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nPixels) return;
    const double n = samples[i / 3];
    xyz[i] = n > 0 ? (film[i] - comp[i]) * (1.0 / n) : 0.0;
}

}  // namespace

// ------------------------------------------------------------------ launchers
size_t traversalSharedBytes(int block) { return size_t(block) * kStackDepth * sizeof(StackEntry); }

template <int M>
void launchGenerate(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q,
                    StatCounters* st, cudaStream_t s) {
    kGenerate<M><<<(pp.nPaths + 255) / 256, 256, 0, s>>>(sc, pp, pb, q, st);
}
template <int M>
void launchIntersect(const DeviceScene& sc, const PathBuffers<RT<M>>& pb, const Queues& q, int cur, StatCounters* st,
                     uint32_t* fetch, int grid, cudaStream_t s) {
    const size_t smem = traversalSharedBytes(128);
    if (sc.fullFeatures) {
        if (sc.travCounters) kIntersect<M, true, true><<<grid, 128, smem, s>>>(sc, pb, q, cur, st, fetch);
        else kIntersect<M, false, true><<<grid, 128, smem, s>>>(sc, pb, q, cur, st, fetch);
    } else {
        if (sc.travCounters) kIntersect<M, true, false><<<grid, 128, smem, s>>>(sc, pb, q, cur, st, fetch);
        else kIntersect<M, false, false><<<grid, 128, smem, s>>>(sc, pb, q, cur, st, fetch);
    }
}
template <int M>
void launchMedium(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q, int cur,
                  StatCounters* st, int grid, cudaStream_t s) {
    kMedium<M><<<grid, 128, 0, s>>>(sc, pp, pb, q, cur, st);
}
template <int M>
void launchSurface(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q, int cur,
                   StatCounters* st, int grid, cudaStream_t s) {
    if (sc.fullFeatures) {
        kSurface<M, true, true><<<grid, 128, 0, s>>>(sc, pp, pb, q, cur, st);
        kSurface<M, false, true><<<grid, 128, 0, s>>>(sc, pp, pb, q, cur, st);
    } else {
        kSurface<M, true, false><<<grid, 128, 0, s>>>(sc, pp, pb, q, cur, st);
        kSurface<M, false, false><<<grid, 128, 0, s>>>(sc, pp, pb, q, cur, st);
    }
}
// The shadow-ray kernels of a bounce: visibility then contributions without null boundaries, the
// ordered walk with them; instantiated for the counting passes and for the scene's shapes.
template <int M, bool Splat, bool Count, bool Full>
void shadowKernelsOf(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q,
                     StatCounters* st, uint32_t* fetch, uint8_t* vis, const SplatTarget& film, int grid, cudaStream_t s) {
    const size_t smem = traversalSharedBytes(128);
    // next-event rays of a scene with contacts take the ordered walk, where the light point's
    // identity decides what lies at its end
    if (pp.anyHitShadows && !(Full && !Splat)) {
        kShadowVis<M, Count, Full><<<grid, 128, smem, s>>>(sc, pb, q, vis, fetch);
        kShadowApply<M, Splat><<<grid, 256, 0, s>>>(sc, pb, q, vis, st, film);
    } else {
        kShadow<M, false, Count, Splat, Full><<<grid, 128, smem, s>>>(sc, pp, pb, q, st, fetch, film);
    }
}
template <int M, bool Splat>
void shadowKernels(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q,
                   StatCounters* st, uint32_t* fetch, uint8_t* vis, const SplatTarget& film, int grid, cudaStream_t s) {
    if (sc.fullFeatures) {
        if (sc.travCounters) shadowKernelsOf<M, Splat, true, true>(sc, pp, pb, q, st, fetch, vis, film, grid, s);
        else shadowKernelsOf<M, Splat, false, true>(sc, pp, pb, q, st, fetch, vis, film, grid, s);
    } else {
        if (sc.travCounters) shadowKernelsOf<M, Splat, true, false>(sc, pp, pb, q, st, fetch, vis, film, grid, s);
        else shadowKernelsOf<M, Splat, false, false>(sc, pp, pb, q, st, fetch, vis, film, grid, s);
    }
}

template <int M>
void launchShadow(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q,
                  StatCounters* st, uint32_t* fetch, uint8_t* vis, int grid, cudaStream_t s) {
    shadowKernels<M, false>(sc, pp, pb, q, st, fetch, vis, SplatTarget{}, grid, s);
}
template <int M>
void launchConnect(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, const Queues& q,
                   StatCounters* st, uint32_t* fetch, uint8_t* vis, const SplatTarget& film, int grid, cudaStream_t s) {
    shadowKernels<M, true>(sc, pp, pb, q, st, fetch, vis, film, grid, s);
}
void launchFoldFilm(const double* film, const double* comp, double* out, size_t n, cudaStream_t s) {
    kFoldFilm<<<int(std::min<size_t>((n + 255) / 256, 4096)), 256, 0, s>>>(film, comp, out, n);
}

template <int M>
void launchFilm(const DeviceScene& sc, const PassParams& pp, const PathBuffers<RT<M>>& pb, double* film, double* comp,
                double* samples, uint32_t spp, cudaStream_t s) {
    // a thread per pixel fills the GPU from 148 x 256 pixels on; below that, with many samples per
    // pixel, the serial loop over a pixel's samples is the kernel's length
    if (pp.nPixels < 148u * 256u && spp >= 64)
        kFilmPerPixel<M><<<pp.nPixels, kFilmChunk, 0, s>>>(sc, pp, pb, film, comp, samples, spp);
    else
        kFilm<M><<<(pp.nPixels + 255) / 256, 256, 0, s>>>(sc, pp, pb, film, comp, samples, spp);
}
template <int M>
void launchCastRays(const DeviceScene& sc, uint64_t n, const double* o, const double* d, uint32_t* b, uint32_t* p,
                    double* t, int grid, cudaStream_t s) {
    if (sc.fullFeatures) kCastRays<M, true><<<grid, 128, traversalSharedBytes(128), s>>>(sc, n, o, d, b, p, t);
    else kCastRays<M, false><<<grid, 128, traversalSharedBytes(128), s>>>(sc, n, o, d, b, p, t);
}
void launchCastRaysF(const DeviceScene& sc, uint64_t n, const float* o, const float* d, uint32_t* b, uint32_t* p,
                     float* t, int grid, cudaStream_t s) {
    if (sc.fullFeatures) kCastRaysF<true><<<grid, 128, traversalSharedBytes(128), s>>>(sc, n, o, d, b, p, t);
    else kCastRaysF<false><<<grid, 128, traversalSharedBytes(128), s>>>(sc, n, o, d, b, p, t);
}
void launchResolve(const double* film, const double* comp, const double* samples, uint32_t nPixels, double* xyz,
                   cudaStream_t s) {
    kResolve<<<(3 * nPixels + 255) / 256, 256, 0, s>>>(film, comp, samples, nPixels, xyz);
}
void launchMaterialize(const uint32_t* leafOrder, uint32_t n, const float4* tri, const double* tri64, PrimRec* prims,
                       PrimRec64* prims64, cudaStream_t s) {
    kMaterialize<<<(n + 255) / 256, 256, 0, s>>>(leafOrder, n, tri, tri64, prims, prims64);
}
void configureKernels() {
    const int smem = int(traversalSharedBytes(128));
    cudaFuncSetAttribute(kIntersect<0, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(kIntersect<1, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(kIntersect<2, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(kIntersect<0, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(kIntersect<1, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(kIntersect<2, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

#define OWEC_INSTANTIATE(M)                                                                                         \
    template void launchGenerate<M>(const DeviceScene&, const PassParams&, const PathBuffers<RT<M>>&, const Queues&, \
                                    StatCounters*, cudaStream_t);                                                   \
    template void launchIntersect<M>(const DeviceScene&, const PathBuffers<RT<M>>&, const Queues&, int,             \
                                     StatCounters*, uint32_t*, int, cudaStream_t);                                             \
    template void launchMedium<M>(const DeviceScene&, const PassParams&, const PathBuffers<RT<M>>&, const Queues&,   \
                                  int, StatCounters*, int, cudaStream_t);                                           \
    template void launchSurface<M>(const DeviceScene&, const PassParams&, const PathBuffers<RT<M>>&, const Queues&,  \
                                   int, StatCounters*, int, cudaStream_t);                                          \
    template void launchShadow<M>(const DeviceScene&, const PassParams&, const PathBuffers<RT<M>>&, const Queues&,   \
                                  StatCounters*, uint32_t*, uint8_t*, int, cudaStream_t);                                                \
    template void launchConnect<M>(const DeviceScene&, const PassParams&, const PathBuffers<RT<M>>&, const Queues&,  \
                                   StatCounters*, uint32_t*, uint8_t*, const SplatTarget&, int, cudaStream_t);      \
    template void launchFilm<M>(const DeviceScene&, const PassParams&, const PathBuffers<RT<M>>&, double*, double*,  \
                                double*, uint32_t, cudaStream_t);                                                   \
    template void launchCastRays<M>(const DeviceScene&, uint64_t, const double*, const double*, uint32_t*,          \
                                    uint32_t*, double*, int, cudaStream_t);

OWEC_INSTANTIATE(0)
OWEC_INSTANTIATE(1)
OWEC_INSTANTIATE(2)

}  // namespace owec
