// The path-replay adjoint of the camera film (Tracer::radiance, src/owe/transport/transport.cpp:
// 473-529, over the pixel samples of CpuRenderer::pass, src/owe/backends/cpu/cpu_backend.cpp:52-94)
// with respect to the heights of a refractive heightfield.
//
// Every camera path of the replayed samples is regenerated from its PCG32 stream (seed, pixel,
// sample) and walked again in one thread, bounce by bounce, with the wavefront kernels' own
// arithmetic and draws in the same order (kGenerate, kIntersect, kMedium, kSurface, the shadow
// rays), so it makes the forward pass's decisions. Nothing of the forward pass is stored.
//
// Derivatives are carried forward, sparsely: a path depends on the heights only after it crosses
// the heightfield, and then only on the heights of the triangles it crossed. At such a crossing the
// path opens a slot for each new vertex of the triangle, and from there on carries, in FP64, the
// derivatives of its vertex position, direction, hero throughput and last scattering pdf with
// respect to each slot's height. The sampling follows the detached convention:
//   - distances, Lambertian and Henyey-Greenstein directions are drawn in world space and held
//     fixed, and a phase function's value at the moved incident direction enters as the weight
//     phase(moved) / phase(drawn) (value 1, derivative dphase / phase);
//   - the Fresnel branch and roulette probabilities are held fixed: the branch weight R / pR or
//     (1 - R) (ni/nt)^2 / (1 - pR) moves with R, the roulette's 1 / q does not;
//   - refraction and reflection at the moved normal are differentiated (attached), and every hit
//     point moves within its surface (implicit differentiation of the crossing).
// With fixed decisions the branch and roulette probabilities and the Henyey-Greenstein frame move
// with the path instead (attached): the result is then the derivative of the estimator at fixed
// random numbers, which is what central differences with common random numbers measure, but it
// leaves out the branches' boundary terms (a path switching from refraction to reflection as R
// moves) and so is not the gradient of the expected film.
// Each contribution (next-event estimates, emission and sky with MIS) is differentiated with respect
// to the vertex's position, incident direction and pdf through dual numbers, and the derivative of
// the path's hero radiance is summed per slot. At the end of the path the slots are weighted as the
// film weighs the radiance (detector importance, CIE matching, the hero pdf, 1 / samples, and the
// loss gradient of the pixel) and added to the vertices' gradients.
//
// What the derivative does not follow (the path is dropped from the gradient and counted): more than
// kSlots heights, a rough or conductor lobe, a textured or aimed Lambertian, an analytic shape
// other than planes and spheres, sphere or cylinder lights met after the heightfield, a gradient sky,
// secondaries still alive past the crossing (a non-dispersive heightfield), and scenes with null
// boundaries (refused on the host). Visibility changes (edges and shadows sweeping over a point)
// are not differentiated, as in path-replay adjoints generally.
#include "camera.cuh"
#include "path_adjoint.hpp"
#include "tangents.cuh"

namespace owec {

namespace {

constexpr int kSlots = 12;  // heights one path may depend on: four crossings' triangles

struct PathTangents {
    int n;
    bool valid;
    int vert[kSlots];
    double dO[kSlots][3];  // the current vertex (the ray's origin, or the hit point being shaded)
    double dD[kSlots][3];  // the current direction
    double dB[kSlots];     // the hero throughput
    double dPdf[kSlots];   // the last scattering vertex's pdf of the current direction (MIS)
    double acc[kSlots];    // the hero radiance gathered
};

__device__ __forceinline__ V3<double> ld3(const double a[3]) { return V3<double>(a[0], a[1], a[2]); }
__device__ __forceinline__ void st3(double a[3], const V3<double>& v) { a[0] = v.x; a[1] = v.y; a[2] = v.z; }

// Russian roulette (survives) that also reports its continuation probability.
template <class R>
__device__ __forceinline__ bool survivesQ(PathSpec<R>& sp, Pcg32& rng, double& q) {
    R m = sp.beta[0];
    for (int k = 1; k < NW; ++k) m = fmax(m, sp.beta[k]);
    q = fmin(1.0, double(m));
    if (rng.uniform() >= q) return false;
    for (int k = 0; k < NW; ++k) sp.beta[k] *= R(1.0 / q);
    return true;
}

// The roulette's effect on the throughput derivatives: beta / q with q held fixed (the detached
// convention), or with q = min(1, max beta) moving with the hero throughput b0 it was taken from
// (the derivative of the estimator at fixed random numbers; the secondaries are dead whenever a path
// carries derivatives, so the maximum is the hero's).
__device__ __forceinline__ void rouletteTangents(double* dB, int n, double q, double b0, bool fixedDecisions) {
    const bool moves = fixedDecisions && q < 1 && b0 > 0;
    for (int k = 0; k < n; ++k) dB[k] = moves ? dB[k] / q - b0 * dB[k] / (q * q) : dB[k] / q;
}

// The derivative of a Henyey-Greenstein direction drawn about wo = -d (sampleHg's frame, the Duff et al.
// basis of wo) when wo moves by dwo with the drawn angles held: the direction attached to the incident
// one.
__device__ V3<double> hgDirectionTangent(const V3<double>& wo, const V3<double>& wi, const V3<double>& dwo) {
    const double sgn = copysign(1.0, wo.z);
    const double a = -1 / (sgn + wo.z), da = a * a * dwo.z;
    const double b = wo.x * wo.y * a, db = (dwo.x * wo.y + wo.x * dwo.y) * a + wo.x * wo.y * da;
    const V3<double> b1(1 + sgn * wo.x * wo.x * a, sgn * b, -sgn * wo.x), b2(b, sgn + wo.y * wo.y * a, -wo.y);
    const V3<double> db1(sgn * (2 * wo.x * dwo.x * a + wo.x * wo.x * da), sgn * db, -sgn * dwo.x);
    const V3<double> db2(db, 2 * wo.y * dwo.y * a + wo.y * wo.y * da, -dwo.y);
    return db1 * dot(wi, b1) + db2 * dot(wi, b2) + dwo * dot(wi, wo);
}

// The next-event estimate toward a point light sample y (normal nL, emitter area, selection pdf)
// from a vertex at x, divided by the throughput: f * Le * cosF * w / pdfL * Tr as a dual in x (and in
// the incident direction d for a medium vertex, through the phase function). Surface vertices:
// Lambertian f = albedo / pi with pdf |cos| / pi about the fixed normal n. Medium vertices: the
// Henyey-Greenstein phase of -d . wi as f and pdf, cosF = 1.
template <int N>
__device__ Dual<N> neeToArea(const DV3<N>& x, const DV3<N>* d, double g, const V3<double>& n, double albedoOverPi,
                             const V3<double>& y, const V3<double>& nL, double area, double sel, double Le,
                             double sigmaT) {
    const DV3<N> v = y - x;
    const Dual<N> d2 = ddot(v, v);
    const Dual<N> dist = dsqrt(d2);
    const DV3<N> wi = v / dist;
    const Dual<N> cosL = dabs(ddot(wi, nL));
    const Dual<N> pdfL = sel * d2 / (cosL * area);
    Dual<N> f, pdfS, cosF;
    if (d) {
        const Dual<N> c = -ddot(*d, wi);
        f = dhgPhase(c, g);
        pdfS = f;
        cosF = Dual<N>(1.0);
    } else {
        cosF = dabs(ddot(wi, n));
        f = Dual<N>(albedoOverPi);
        pdfS = cosF * kInvPi;
    }
    Dual<N> c = f * Le * cosF * dpowerHeuristic(pdfL, pdfS) / pdfL;
    if (sigmaT > 0) c = c * dexp(-sigmaT * dist);
    return c;
}

struct AdjointParams {
    PassParams pp;
    HeightfieldParams hf;
    PathAdjointTargets t;
    bool fixedDecisions;
};

// Adds slot k's derivative of a contribution c = beta * c', c' a dual in the vertex position (vars
// 0-2, tangents pos), the incident direction (vars 3-5) and the last pdf (var 6), whichever are used.
template <int N>
__device__ __forceinline__ void gather(PathTangents& tg, double beta, const Dual<N>& cb, const double (*pos)[3],
                                       bool useDir, bool usePdf) {
    for (int k = 0; k < tg.n; ++k) {
        double s = 0;
        if (pos) s += cb.d[0] * pos[k][0] + cb.d[1] * pos[k][1] + cb.d[2] * pos[k][2];
        if constexpr (N >= 6) {
            if (useDir) s += cb.d[3] * tg.dD[k][0] + cb.d[4] * tg.dD[k][1] + cb.d[5] * tg.dD[k][2];
        }
        if constexpr (N >= 7) {
            if (usePdf) s += cb.d[6] * tg.dPdf[k];
        }
        tg.acc[k] += cb.v * tg.dB[k] + beta * s;
    }
}

// The visibility and transmittance of a next-event sample (kShadowVis and kShadowApply: any-hit
// visibility short of the light, the medium's Beer-Lambert factor, the arrival regions; in the Full
// instantiation kShadow's decision at a finite light: the closest crossing up to a little past the
// light point, which clears the segment when it is the light's own face there or lies beyond it).
// Returns whether the segment is clear; Tr receives the transmittance per wavelength.
template <int M, bool Full>
__device__ bool neeClear(const DeviceScene& sc, const LightSampleD& ls, const V3<double>& p, uint32_t region,
                         uint32_t depB, uint32_t depP, float errN, const float lambda[NW], typename Mode<M>::R Tr[NW],
                         StackEntry* stack, int stride, bool& fault) {
    using R = typename Mode<M>::R;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    const bool finite = !isinf(ls.dist);
    bool clear = true;
    const double w = 4e-6 * ls.dist + double(errN) + 1e-9;
    constexpr bool kEndpoint = Full;  // the light point's identity decides, as in the forward pass
    const double tq = finite ? (kEndpoint ? ls.dist + w : ls.dist - w) : INFINITY;
    if (!(finite && tq <= 0)) {
        RayQuery<R> sq;
        V3<double> so = p;
        if (Mode<M>::plainOrigin) so = V3<double>(V3<float>(so));
        sq.od = so;
        sq.o = V3<R>(so);
        sq.d = V3<R>(R(ls.wi.x), R(ls.wi.y), R(ls.wi.z));
        sq.depB = depB;
        sq.depP = depP;
        sq.errN = R(errN);
        sq.tmax = R(tq);
        sq.region = region;
        HitRec sh;
        sh.boundary = kNone;
        sh.t = INFINITY;
        sh.flags = 0;
        if (kEndpoint && finite) {
            const int vs = traceRay<R, Ro, Rr, false, Full>(sc, sq, stack, stride, sh);
            if (vs == kTraceOverflow) {
                fault = true;
                return false;
            }
            clear = vs != kTraceHit || sh.t > ls.dist ||
                    (sh.boundary == ls.boundary && !(sh.flags & kHitAmbiguous) && fabs(sh.t - ls.dist) <= w);
        } else {
            const int vs = traceRay<R, Ro, Rr, true, Full>(sc, sq, stack, stride, sh);
            if (vs == kTraceOverflow) {
                fault = true;
                return false;
            }
            clear = vs != kTraceHit;
        }
    }
    for (int j = 0; j < NW; ++j) Tr[j] = R(1);
    const owec_medium& nm = sc.media[sc.regionMedium[region]];
    if (clear && (mediumAbsorbs(nm, sc) || mediumScatters(nm, sc))) {
        if (!finite) return false;
        for (int j = 0; j < NW; ++j) {
            const R lam = R(lambda[j]);
            Tr[j] = exp(-(evalSpectrum(sc, nm.absorption, lam) + evalSpectrum(sc, nm.scattering, lam)) * R(ls.dist));
        }
    }
    const uint32_t endRegion = ls.boundary == kNone ? 0u : ls.region;
    if (!finite && region != 0) return false;
    if (finite && region != endRegion) return false;
    return clear;
}

// One camera path from `ray`, `sp`, `aux`, `rng` on: from its camera ray (resume null), or from a
// checkpoint at its first heightfield surface event (resume: that event's hit, whose segment's free
// flight the forward pass has already taken).
template <int M, bool Full>
__device__ void adjointPath(const DeviceScene& sc, const AdjointParams& P, PathRay<typename Mode<M>::R> ray,
                            PathSpec<typename Mode<M>::R> sp, PathAux aux, Pcg32 rng, const HitRec* resume,
                            StackEntry* stack, int stride) {
    using R = typename Mode<M>::R;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    const PassParams& pp = P.pp;
    unsigned long long* ctr = P.t.counters;
    PathTangents tg;
    tg.n = 0;
    tg.valid = true;
    bool metHeightfield = false, fault = false;
    for (;;) {
        const V3<R> d = rayDir(ray);
        const V3<double> dd(d);
        const owec_medium med = sc.media[sc.regionMedium[ray.region]];
        const bool absorbs = mediumAbsorbs(med, sc), scatters = mediumScatters(med, sc);
        HitRec h;
        bool found;
        int event = 0;  // 0 pass, 1 scatter, 2 end
        double tS = 0;
        R beforeAbs = sp.beta[0], sigmaA0 = R(0);
        bool cont = false;
        // The next-event estimate of a vertex is resolved at once (its shadow ray draws nothing, and
        // the forward pass adds it to the radiance right after the vertex's own emission, too).
        LightSampleD ls;
        R contrib[NW] = {R(0), R(0), R(0), R(0)};
        R Tr[NW];
        if (resume) {
            // the checkpointed surface event: its segment's Beer-Lambert factor is already applied
            h = *resume;
            resume = nullptr;
            found = true;
            if (absorbs && !scatters) {
                sigmaA0 = evalSpectrum(sc, med.absorption, R(sp.lambda[0]));
                const R att = exp(-sigmaA0 * R(h.t));
                beforeAbs = att > R(0) ? sp.beta[0] / att : R(0);
            }
        } else {
            // ------------------------------------------------------------ closest hit (kIntersect)
            RayQuery<R> rq;
            rq.od = rayOrigin(ray.o);
            rq.o = V3<R>(rq.od);
            rq.d = d;
            rq.tmax = R(INFINITY);
            rq.depB = ray.depB;
            rq.depP = ray.depP;
            rq.region = ray.region;
            rq.errN = R(ray.errN);
            h.boundary = kNone;
            h.t = INFINITY;
            h.flags = 0;
            const int s = traceRay<R, Ro, Rr, false, Full>(sc, rq, stack, stride, h);
            if (s != kTraceHit) { h.boundary = kNone; h.t = INFINITY; }
            if (s == kTraceOverflow) { fault = true; break; }
            found = h.boundary < kNone - 1u;
            // ------------------------------------------------------------ free flight (kMedium)
            if (!(found && !absorbs && !scatters)) {
                const double seg = found ? h.t : INFINITY;
                if (scatters) {
                    R sT[NW];
                    for (int j = 0; j < NW; ++j)
                        sT[j] = evalSpectrum(sc, med.absorption, R(sp.lambda[j])) + evalSpectrum(sc, med.scattering, R(sp.lambda[j]));
                    tS = -log(1 - rng.uniform()) / double(sT[0]);
                    if (tS < seg) {
                        const R pdf0 = sT[0] * exp(-sT[0] * R(tS));
                        const R b0 = sp.beta[0];
                        for (int j = 0; j < NW; ++j)
                            sp.beta[j] *= evalSpectrum(sc, med.scattering, R(sp.lambda[j])) * exp(-sT[j] * R(tS)) / pdf0;
                        // the hero's weight sigma_s / sigma_t does not move with the heights
                        const double w0 = b0 != R(0) ? double(sp.beta[0]) / double(b0) : 0.0;
                        for (int k = 0; k < tg.n; ++k) tg.dB[k] *= w0;
                        event = 1;
                    } else if (isinf(seg)) {
                        event = 2;
                    } else {
                        const R pass0 = exp(-sT[0] * R(seg));
                        for (int j = 0; j < NW; ++j) sp.beta[j] *= exp(-sT[j] * R(seg)) / pass0;
                    }
                } else if (absorbs) {
                    if (isinf(seg)) {
                        event = 2;
                    } else {
                        beforeAbs = sp.beta[0];
                        sigmaA0 = evalSpectrum(sc, med.absorption, R(sp.lambda[0]));
                        for (int j = 0; j < NW; ++j)
                            sp.beta[j] *= exp(-evalSpectrum(sc, med.absorption, R(sp.lambda[j])) * R(seg));
                    }
                }
            }
        }
        if (event == 1) {
            // ------------------------------------------------------------ scatterInMedium
            const V3<double> sp3 = rayOrigin(ray.o) + dd * tS;
            for (int k = 0; k < tg.n; ++k)
                for (int a = 0; a < 3; ++a) tg.dO[k][a] += tS * tg.dD[k][a];
            if (int(aux.depth) >= pp.maxDepth) break;
            R betaNee[NW];
            for (int j = 0; j < NW; ++j) betaNee[j] = sp.beta[j];
            int li;
            if (sampleLight<R>(sc, sp3, rng, ls, li)) {
                bool leZero = true;
                for (int j = 0; j < NW; ++j)
                    if (lightSampleLe<R>(sc, ls, R(sp.lambda[j])) != R(0)) leZero = false;
                if (!leZero && ls.pdf > 0) {
                    const R ph = hgPhase(dot(-d, V3<R>(ls.wi)), R(med.g));
                    const R w = powerHeuristic(R(ls.pdf), ph);
                    bool any = false;
                    for (int k = 0; k < NW; ++k) {
                        if (sp.pdf[k] == 0.f && k > 0) continue;
                        contrib[k] = R(float(betaNee[k] * ph * lightSampleLe<R>(sc, ls, R(sp.lambda[k])) * (R(1) * w / R(ls.pdf))));
                        any = any || contrib[k] != R(0);
                    }
                    if (any && neeClear<M, Full>(sc, ls, sp3, ray.region, kNone, kNone, 0.f, sp.lambda, Tr, stack, stride, fault)) {
                        for (int j = 0; j < NW; ++j) sp.L[j] += float(R(float(contrib[j])) * Tr[j]);
                        if (tg.n > 0 && tg.valid && ls.boundary != kNone) {
                            // (the sun is never clear from inside a medium)
                            if (sc.boundaries[ls.boundary].shape != OWEC_SHAPE_PLANE) {
                                tg.valid = false;
                            } else {
                                const DBoundary& lb = sc.boundaries[ls.boundary];
                                const double sigmaT = double(evalSpectrum(sc, med.absorption, R(sp.lambda[0])) +
                                                             evalSpectrum(sc, med.scattering, R(sp.lambda[0])));
                                const DV3<6> x = dvar3<6>(sp3, 0), dv = dvar3<6>(dd, 3);
                                const Dual<6> cb = neeToArea<6>(x, &dv, med.g, V3<double>(), 0.0, ls.p, ls.n, lb.area,
                                                                sc.lights[li].pdf,
                                                                double(lightSampleLe<R>(sc, ls, R(sp.lambda[0]))), sigmaT);
                                gather<6>(tg, double(betaNee[0]), cb, tg.dO, true, false);
                            }
                        }
                    }
                }
            }
            const Draw2<R> u(rng);
            V3<R> wi;
            aux.prevPdf = float(sampleHg(-d, R(med.g), u.u1, u.u2, wi));
            if (tg.n > 0 && P.fixedDecisions) {
                // the drawn angles stay: the direction turns with the incident one, weight 1
                const V3<double> wo = -dd, w(wi);
                for (int k = 0; k < tg.n; ++k) {
                    st3(tg.dD[k], hgDirectionTangent(wo, w, -ld3(tg.dD[k])));
                    tg.dPdf[k] = 0;
                }
            } else if (tg.n > 0) {
                // the drawn direction stays; the phase at the moved incident direction weighs it
                const V3<double> w(wi);
                const double g = med.g, c = dot(-dd, w);
                const double denom = 1 + g * g + 2 * g * c;
                const double ph = (1 - g * g) / (4 * kPi * denom * sqrt(denom));
                const double dphdc = ph * (-1.5) * (2 * g) / denom;
                for (int k = 0; k < tg.n; ++k) {
                    const double dc = -(tg.dD[k][0] * w.x + tg.dD[k][1] * w.y + tg.dD[k][2] * w.z);
                    tg.dB[k] += double(sp.beta[0]) * dphdc * dc / ph;
                    tg.dPdf[k] = dphdc * dc;
                    tg.dD[k][0] = tg.dD[k][1] = tg.dD[k][2] = 0;
                }
            }
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
            double q = 1;
            const double b0 = double(sp.beta[0]);
            cont = int(aux.depth) < pp.rrDepth || survivesQ(sp, rng, q);
            rouletteTangents(tg.dB, tg.n, q, b0, P.fixedDecisions);
        } else if (event == 0 && !found) {
            if (ray.region == 0) {
                // skyMet (transport.cpp:401-417)
                const bool spec = aux.flags & kFlagSpecular;
                const bool inSun = sc.hasSun && dot(dd, V3<double>(sc.sunDir[0], sc.sunDir[1], sc.sunDir[2])) >= sc.sunCosMax;
                R w = R(1);
                const double sunPdf = sc.sunSelectPdf / sc.sunSolidAngle;
                if (!spec && inSun) w = powerHeuristic(R(aux.prevPdf), R(sunPdf));
                for (int j = 0; j < NW; ++j) {
                    const R lam = R(sp.lambda[j]);
                    const R sky = skyRadiance(sc, dd, lam);
                    const R sun = inSun ? evalSpectrum(sc, sc.sunSpectrum, lam) : R(0);
                    sp.L[j] += float(sp.beta[j] * (sky + sun * w));
                }
                if (tg.n > 0 && tg.valid) {
                    if (sc.skyModel == OWEC_SKY_GRADIENT) {
                        tg.valid = false;
                    } else {
                        const R lam = R(sp.lambda[0]);
                        const double sky = double(skyRadiance(sc, dd, lam));
                        const double sun = inSun ? double(evalSpectrum(sc, sc.sunSpectrum, lam)) : 0.0;
                        Dual<7> a = Dual<7>::var(double(aux.prevPdf), 6);
                        const Dual<7> wd = (!spec && inSun) ? dpowerHeuristic(a, Dual<7>(sunPdf)) : Dual<7>(1.0);
                        const Dual<7> cb = sky + sun * wd;
                        gather<7>(tg, double(sp.beta[0]), cb, nullptr, false, !spec && inSun);
                    }
                }
            }
            break;
        } else if (event == 2) {
            break;
        } else {
            // ------------------------------------------------------------ the boundary met (kSurface)
            const DBoundary& bd = sc.boundaries[h.boundary];
            const SurfacePoint<R> gp = hitGeometry<R, Ro, Rr, Full>(sc, ray, h);
            const V3<double> n(gp.n);
            // the tangents of the hit point and its normal
            double dP[kSlots][3], dN[kSlots][3];
            const bool hfHit = bd.shape == OWEC_SHAPE_MESH && h.boundary == P.hf.boundary;
            if (hfHit) metHeightfield = true;
            if (tg.valid && (tg.n > 0 || hfHit)) {
                V3<double> v0, v1, v2;
                int vid[3] = {-1, -1, -1};
                V3<double> nu = n;  // the plane the point solves (unnormalised for a triangle)
                const V3<double> zdir(P.hf.zdir[0], P.hf.zdir[1], P.hf.zdir[2]);
                if (bd.shape == OWEC_SHAPE_MESH) {
                    if (sizeof(Rr) == sizeof(double)) {
                        const PrimRec64& pr = sc.prims64[h.slot];
                        v0 = V3<double>(pr.v0[0], pr.v0[1], pr.v0[2]);
                        v1 = V3<double>(pr.v1[0], pr.v1[1], pr.v1[2]);
                        v2 = V3<double>(pr.v2[0], pr.v2[1], pr.v2[2]);
                    } else {
                        V3<R> a, b, c;
                        uint32_t bb, pr, kind;
                        TriFetch<R>::get(sc, h.slot, a, b, c, bb, pr, kind);
                        v0 = V3<double>(a);
                        v1 = V3<double>(b);
                        v2 = V3<double>(c);
                    }
                    nu = cross(v1 - v0, v2 - v0);
                    if (hfHit) {
                        for (int a = 0; a < 3; ++a) vid[a] = int(P.hf.tris[3 * size_t(h.prim) + a]);
                        for (int a = 0; a < 3 && tg.valid; ++a) {
                            bool present = false;
                            for (int k = 0; k < tg.n; ++k) present = present || tg.vert[k] == vid[a];
                            if (present) continue;
                            if (tg.n == kSlots) { tg.valid = false; break; }
                            const int k = tg.n++;
                            tg.vert[k] = vid[a];
                            for (int c = 0; c < 3; ++c) tg.dO[k][c] = tg.dD[k][c] = 0;
                            tg.dB[k] = tg.dPdf[k] = tg.acc[k] = 0;
                        }
                    }
                } else if (bd.shape != OWEC_SHAPE_PLANE && bd.shape != OWEC_SHAPE_SPHERE) {
                    tg.valid = false;
                }
                if (tg.valid) {
                    const double nlen = length(nu);
                    const double sgn = dot(nu, n) >= 0 ? 1.0 : -1.0;  // nu's side against the front normal
                    const double dnu = dot(dd, nu);
                    const double t = dot(gp.p - rayOrigin(ray.o), dd);  // the refined distance
                    V3<double> center;
                    if (bd.shape == OWEC_SHAPE_SPHERE) center = bd.toWorld.point(V3<double>(0, 0, 0));
                    for (int k = 0; k < tg.n; ++k) {
                        V3<double> dv0, dv1, dv2, dnuk;
                        if (hfHit) {
                            if (tg.vert[k] == vid[0]) dv0 = zdir;
                            if (tg.vert[k] == vid[1]) dv1 = zdir;
                            if (tg.vert[k] == vid[2]) dv2 = zdir;
                            dnuk = cross(dv1 - dv0, v2 - v0) + cross(v1 - v0, dv2 - dv0);
                        }
                        const V3<double> q = ld3(tg.dO[k]) + ld3(tg.dD[k]) * t - dv0;
                        const double dt = -(dot(q, nu) + (hfHit ? dot(gp.p - v0, dnuk) : 0.0)) / dnu;
                        const V3<double> dPk = ld3(tg.dO[k]) + ld3(tg.dD[k]) * t + dd * dt;
                        V3<double> dNk;
                        if (hfHit) dNk = (dnuk - (nu / nlen) * dot(nu / nlen, dnuk)) * (sgn / nlen);
                        else if (bd.shape == OWEC_SHAPE_SPHERE)
                            dNk = (dPk - n * dot(n, dPk)) * ((dot(n, gp.p - center) >= 0 ? 1.0 : -1.0) / bd.params[0]);
                        st3(dP[k], dPk);
                        st3(dN[k], dNk);
                        // Beer-Lambert over the segment in a purely absorbing medium
                        if (sigmaA0 != R(0) && beforeAbs != R(0))
                            tg.dB[k] = double(sp.beta[0]) / double(beforeAbs) * (tg.dB[k] - double(beforeAbs) * double(sigmaA0) * dt);
                    }
                }
            }
            const bool fromFront = dot(d, gp.n) < R(0);
            const uint32_t inc = fromFront ? bd.front : bd.back;
            const uint32_t other = fromFront ? bd.back : bd.front;
            const bool ambiguous = Full && (h.flags & kHitAmbiguous);
            ray.region = inc;
            aux.lastBoundary = h.boundary;
            const bool specular = aux.flags & kFlagSpecular;
            // emissionMet (transport.cpp:420-433)
            if (bd.emission >= 0 && !ambiguous) {
                const owec_emission e = sc.emissions[bd.emission];
                if (fromFront ? e.front : e.back) {
                    R w = R(1);
                    const bool mis = !specular && bd.light >= 0;
                    double pl = 0;
                    const V3<double> prev(aux.prevP[0], aux.prevP[1], aux.prevP[2]);
                    if (mis) {
                        pl = sc.lights[bd.light].pdf * shapePdfFrom(bd, prev, gp.p, n);
                        if (pl > 0) w = powerHeuristic(R(aux.prevPdf), R(pl));
                    }
                    for (int j = 0; j < NW; ++j)
                        sp.L[j] += float(sp.beta[j] * evalSpectrum(sc, e.radiance, R(sp.lambda[j])) * w);
                    if (tg.n > 0 && tg.valid) {
                        const double Le = double(evalSpectrum(sc, e.radiance, R(sp.lambda[0])));
                        if (!mis || pl <= 0) {
                            gather<7>(tg, double(sp.beta[0]), Dual<7>(Le * double(w)), nullptr, false, false);
                        } else if (bd.shape != OWEC_SHAPE_PLANE) {
                            tg.valid = false;
                        } else {
                            // w = power(prevPdf, sel * |p - prevP|^2 / (cosL area)) as a dual in the
                            // previous vertex (vars 0-2), the hit point (3-5) and the pdf (6)
                            const DV3<7> a = dvar3<7>(prev, 0), b = dvar3<7>(gp.p, 3);
                            const DV3<7> v = b - a;
                            const Dual<7> d2 = ddot(v, v);
                            const Dual<7> cosL = dabs(ddot(v, n)) / dsqrt(d2);
                            const Dual<7> plD = sc.lights[bd.light].pdf * d2 / (cosL * bd.area);
                            const Dual<7> cb = Le * dpowerHeuristic(Dual<7>::var(double(aux.prevPdf), 6), plD);
                            for (int k = 0; k < tg.n; ++k) {
                                double dc = cb.v * tg.dB[k];
                                double s3 = 0;
                                for (int c = 0; c < 3; ++c) s3 += cb.d[c] * tg.dO[k][c] + cb.d[3 + c] * dP[k][c];
                                s3 += cb.d[6] * tg.dPdf[k];
                                tg.acc[k] += dc + double(sp.beta[0]) * s3;
                            }
                        }
                    }
                }
            }
            const owec_optics& o = sc.optics[bd.optics];
            const float errN = anchorError<R>(gp.p);
            bool scattered = false;
            if (ambiguous) {
            } else if (o.type == OWEC_SURF_NULL) {
                ray.region = other;
                setOrigin<M>(ray.o, gp.p);
                ray.depB = h.boundary;
                ray.depP = h.prim;
                ray.errN = errN;
                cont = int(aux.depth) < 4 * pp.maxDepth;
                if (tg.valid)
                    for (int k = 0; k < tg.n; ++k)
                        for (int c = 0; c < 3; ++c) tg.dO[k][c] = dP[k][c];
            } else if (o.type != OWEC_SURF_ABSORBER && o.type != OWEC_SURF_DETECTOR && int(aux.depth) < pp.maxDepth) {
                // scatterAtSurface (transport.cpp:437-471)
                const R hero = R(sp.lambda[0]);
                V3<double> texW;
                const V3<double>* tex = hitTexture<Full>(sc, bd, gp.pLocal, gp.nLocal, texW);
                const Interface<R> it = makeInterface<R, false>(sc, bd, gp.n, hero, R(pp.fresnelFloor), tex);
                if (o.type == OWEC_SURF_DIELECTRIC) {  // terminateIfDispersive
                    bool alive2 = false;
                    for (int j = 1; j < NW; ++j) alive2 = alive2 || sp.pdf[j] != 0.f;
                    if (alive2) {
                        for (int j = 1; j < NW; ++j) {
                            if (sp.pdf[j] == 0.f) continue;
                            const Interface<R> it2 = makeInterface(sc, bd, gp.n, R(sp.lambda[j]), R(pp.fresnelFloor), tex);
                            if (isDispersive(it, it2)) {
                                for (int m = 1; m < NW; ++m) sp.pdf[m] = 0.f;
                                sp.pdf[0] /= float(NW);
                                for (int m = 1; m < NW; ++m) sp.beta[m] = R(0);
                                break;
                            }
                        }
                    }
                }
                if (tg.n > 0 && tg.valid) {
                    // the derivative follows the hero wavelength alone
                    for (int j = 1; j < NW; ++j)
                        if (sp.pdf[j] != 0.f) tg.valid = false;
                    const bool plainDiffuse = o.type == OWEC_SURF_DIFFUSE && !tex && !(Full && o.aim_share > 0);
                    const bool smoothDielectric = o.type == OWEC_SURF_DIELECTRIC && o.roughness < kSmoothRoughness;
                    if (!plainDiffuse && !smoothDielectric && o.type != OWEC_SURF_MIRROR) tg.valid = false;
                }
                R betaNee[NW];
                for (int j = 0; j < NW; ++j) betaNee[j] = sp.beta[j];
                if (!isDeltaOptics<R>(o)) {
                    int li;
                    if (sampleLight<R>(sc, gp.p, rng, ls, li)) {
                        bool leZero = true;
                        for (int j = 0; j < NW; ++j)
                            if (lightSampleLe<R>(sc, ls, R(sp.lambda[j])) != R(0)) leZero = false;
                        if (!leZero && ls.pdf > 0) {
                            const V3<R> wi(ls.wi);
                            bool fZero = true;
                            R fN[NW] = {R(0), R(0), R(0), R(0)};
                            R pdfS = R(0);
                            for (int j = 0; j < NW; ++j) {
                                if (sp.pdf[j] == 0.f) continue;
                                R pdf;
                                const Interface<R> itj =
                                    j == 0 ? it : makeInterface<R, false>(sc, bd, gp.n, R(sp.lambda[j]), R(pp.fresnelFloor), tex);
                                fN[j] = evalScatter(sc, itj, d, wi, true, pdf);
                                if (j == 0) pdfS = pdf;
                                if (Full && j == 0 && pdf > R(0) && o.type == OWEC_SURF_DIFFUSE && fromFront && o.aim_share > 0)
                                    pdfS = R(aimDiffusePdf(o, gp.p, ls.wi, double(pdf)));
                                if (fN[j] != R(0)) fZero = false;
                            }
                            if (!fZero) {
                                const R cosF = fabs(dot(wi, gp.n));
                                const uint32_t neeRegion = dot(wi, gp.n) > R(0) ? bd.front : bd.back;
                                const R w = powerHeuristic(R(ls.pdf), pdfS);
                                bool any = false;
                                for (int k = 0; k < NW; ++k) {
                                    if (sp.pdf[k] == 0.f && k > 0) continue;
                                    const R Le = lightSampleLe<R>(sc, ls, R(sp.lambda[k]));
                                    contrib[k] = R(float(betaNee[k] * fN[k] * Le * (cosF * w / R(ls.pdf))));
                                    any = any || contrib[k] != R(0);
                                }
                                if (any && neeClear<M, Full>(sc, ls, gp.p, neeRegion, h.boundary, h.prim, errN, sp.lambda, Tr,
                                                             stack, stride, fault)) {
                                    for (int j = 0; j < NW; ++j) sp.L[j] += float(R(float(contrib[j])) * Tr[j]);
                                    if (tg.n > 0 && tg.valid) {
                                        const double b0 = double(betaNee[0]);
                                        if (ls.boundary == kNone) {
                                            // the sun: a fixed direction, a constant pdf, the fixed normal
                                            if (b0 != 0)
                                                gather<6>(tg, b0, Dual<6>(double(R(float(contrib[0])) * Tr[0]) / b0), nullptr,
                                                          false, false);
                                        } else if (sc.boundaries[ls.boundary].shape != OWEC_SHAPE_PLANE) {
                                            tg.valid = false;
                                        } else {
                                            const owec_medium& nm = sc.media[sc.regionMedium[neeRegion]];
                                            const double sigmaT =
                                                (mediumAbsorbs(nm, sc) || mediumScatters(nm, sc))
                                                    ? double(evalSpectrum(sc, nm.absorption, R(sp.lambda[0])) +
                                                             evalSpectrum(sc, nm.scattering, R(sp.lambda[0])))
                                                    : 0.0;
                                            const DV3<6> x = dvar3<6>(gp.p, 0);
                                            const Dual<6> cb = neeToArea<6>(
                                                x, nullptr, 0.0, n, double(it.albedo) * kInvPi, ls.p, ls.n,
                                                sc.boundaries[ls.boundary].area, sc.lights[li].pdf,
                                                double(lightSampleLe<R>(sc, ls, R(sp.lambda[0]))), sigmaT);
                                            gather<6>(tg, b0, cb, dP, false, false);
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
                const Draw3<R> u(rng);
                ScatterSample<R> ss;
                bool ok = sampleScatter(sc, it, d, u.u1, u.u2, u.u3, true, ss);
                if (Full && ok && o.type == OWEC_SURF_DIFFUSE && fromFront && o.aim_share > 0)
                    ok = aimDiffuse(o, gp.p, gp.n, it.albedo, u.u1, u.u2, u.u3, ss);
                if (ok && ss.weight > R(0)) {
                    if (tg.n > 0 && tg.valid) {
                        const double beta0 = double(sp.beta[0]);
                        if (o.type == OWEC_SURF_DIELECTRIC) {
                            const double eta = double(it.nBack) / double(it.nFront);
                            double Rf, dRdc;
                            fresnelWithDerivative(-dot(dd, n), eta, Rf, dRdc);
                            const double pR = double(fresnelBranchProbability(R(Rf), it.fresnelFloor));
                            // dpR/dR: held (detached), or moving with R unless the floor clamps it
                            const double fl = double(it.fresnelFloor);
                            const double dpR = !P.fixedDecisions ? 0.0
                                               : ((fl > 0 && Rf < 1 && (Rf < fl || Rf > 1 - fl)) ? 0.0 : 1.0);
                            const bool fr = dot(dd, n) < 0;
                            const double ni = fr ? double(it.nFront) : double(it.nBack);
                            const double nt = fr ? double(it.nBack) : double(it.nFront);
                            for (int k = 0; k < tg.n; ++k) {
                                const V3<double> dnk = ld3(dN[k]), dDk = ld3(tg.dD[k]);
                                const double dc = -(dot(dDk, n) + dot(dd, dnk));  // d cos(incidence) against n
                                V3<double> dOut;
                                if (ss.transmitted) {
                                    const double radiance = sqr(ni / nt);
                                    tg.dB[k] = tg.dB[k] * double(ss.weight) -
                                               beta0 * dRdc * dc * ((1 - pR) - (1 - Rf) * dpR) / ((1 - pR) * (1 - pR)) * radiance;
                                    dOut = refractTangent(dd, n, ni, nt, dDk, dnk);
                                } else {
                                    tg.dB[k] = tg.dB[k] * double(ss.weight) + beta0 * dRdc * dc * (pR - Rf * dpR) / (pR * pR);
                                    dOut = reflectTangent(dd, n, dDk, dnk);
                                }
                                st3(tg.dD[k], dOut);
                                tg.dPdf[k] = 0;
                            }
                        } else if (o.type == OWEC_SURF_MIRROR) {
                            for (int k = 0; k < tg.n; ++k) {
                                tg.dB[k] *= double(ss.weight);
                                st3(tg.dD[k], reflectTangent(dd, n, ld3(tg.dD[k]), ld3(dN[k])));
                                tg.dPdf[k] = 0;
                            }
                        } else {
                            // Lambertian: the direction drawn about the fixed normal stays; its
                            // weight (the albedo) and pdf do not move
                            for (int k = 0; k < tg.n; ++k) {
                                tg.dB[k] *= double(ss.weight);
                                tg.dD[k][0] = tg.dD[k][1] = tg.dD[k][2] = 0;
                                tg.dPdf[k] = 0;
                            }
                        }
                        for (int k = 0; k < tg.n; ++k)
                            for (int c = 0; c < 3; ++c) tg.dO[k][c] = dP[k][c];
                    }
                    // weighScatter (transport.cpp:227-233)
                    sp.beta[0] *= ss.weight;
                    for (int j = 1; j < NW; ++j) {
                        if (sp.pdf[j] == 0.f) continue;
                        const Interface<R> itj = makeInterface<R, false>(sc, bd, gp.n, R(sp.lambda[j]), R(pp.fresnelFloor), tex);
                        sp.beta[j] *= secondaryScatterWeight(sc, itj, d, ss, true);
                    }
                    if (ss.transmitted) ray.region = other;
                    aux.flags = ss.delta ? (aux.flags | kFlagSpecular) : (aux.flags & ~kFlagSpecular);
                    aux.prevPdf = float(ss.pdf);
                    aux.prevP[0] = gp.p.x;
                    aux.prevP[1] = gp.p.y;
                    aux.prevP[2] = gp.p.z;
                    setOrigin<M>(ray.o, gp.p);
                    ray.d[0] = ss.wi.x;
                    ray.d[1] = ss.wi.y;
                    ray.d[2] = ss.wi.z;
                    ray.depB = h.boundary;
                    ray.depP = h.prim;
                    ray.errN = errN;
                    scattered = true;
                    double q = 1;
                    const double b0 = double(sp.beta[0]);
                    cont = !(int(aux.depth) >= pp.rrDepth && !survivesQ(sp, rng, q));
                    rouletteTangents(tg.dB, tg.n, q, b0, P.fixedDecisions);
                }
            }
            (void)scattered;
        }
        if (!cont) break;
        aux.depth += 1;
    }
    // ---------------------------------------------------------------- the film's weighting (kFilm)
    const uint32_t pixel = aux.pixel;
    const double inv = 1.0 / (NW * sc.cieYIntegral);
    double xyz[3] = {0, 0, 0};
    for (int k = 0; k < NW; ++k) {
        const double Lk = double(sp.L[k]) * double(aux.weight);
        if (sp.pdf[k] == 0.f || Lk == 0) continue;
        const double w = Lk / double(sp.pdf[k]) * inv;
        const double l = double(sp.lambda[k]);
        xyz[0] += w * cieX(l);
        xyz[1] += w * cieY(l);
        xyz[2] += w * cieZ(l);
    }
    const bool finite = isfinite(xyz[0] + xyz[1] + xyz[2]);
    if (P.t.replay && finite)
        for (int c = 0; c < 3; ++c) atomicAdd(P.t.replay + 3 * size_t(pixel) + c, xyz[c] * P.t.invSamples);
    warpCount(ctr + 0, true);
    warpCount(ctr + 3, fault);
    warpCount(ctr + 1, metHeightfield);
    const bool dropped = metHeightfield && (!tg.valid || !finite);
    warpCount(ctr + 2, dropped);
    if (!metHeightfield || dropped || tg.n == 0 || sp.pdf[0] == 0.f) return;
    const double l0 = double(sp.lambda[0]);
    const double* g = P.t.g + 3 * size_t(pixel);
    const double gam = double(aux.weight) * inv / double(sp.pdf[0]) * (g[0] * cieX(l0) + g[1] * cieY(l0) + g[2] * cieZ(l0)) *
                       P.t.invSamples;
    if (gam == 0) return;
    for (int k = 0; k < tg.n; ++k)
        if (tg.acc[k] != 0) atomicAdd(P.t.dH + tg.vert[k], tg.acc[k] * gam);
}

// Full replay: every camera path of the batch from its camera ray.
template <int M, bool Full>
__global__ void __launch_bounds__(128) kPathAdjoint(DeviceScene sc, AdjointParams P) {
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.pp.nPaths; i += gridDim.x * blockDim.x) {
        PathRay<typename Mode<M>::R> ray;
        PathSpec<typename Mode<M>::R> sp;
        PathAux aux;
        Pcg32 rng;
        if (generateCameraPath<M>(sc, P.pp, i, ray, sp, aux, rng))
            adjointPath<M, Full>(sc, P, ray, sp, aux, rng, nullptr, stack, blockDim.x);
    }
}

// From the checkpoints the wavefront left at the paths' first heightfield surface events.
template <int M, bool Full>
__global__ void __launch_bounds__(128) kPathAdjointResume(DeviceScene sc, AdjointParams P,
                                                          const PathCheckpoint<typename Mode<M>::R>* ckpt,
                                                          const uint32_t* count) {
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const PathCheckpoint<typename Mode<M>::R> c = loadStream(ckpt + i);
        const Pcg32 rng{c.aux.rngState, (uint64_t(c.aux.stream) << 1u) | 1u};
        adjointPath<M, Full>(sc, P, c.ray, c.spec, c.aux, rng, &c.hit, stack, blockDim.x);
    }
}

template <int M>
void launchMode(const DeviceScene& sc, const AdjointParams& P, const void* ckpt, const uint32_t* count, int grid,
                cudaStream_t s) {
    using C = PathCheckpoint<typename Mode<M>::R>;
    const size_t smem = traversalSharedBytes(128);
    if (ckpt) {
        if (sc.fullFeatures) kPathAdjointResume<M, true><<<grid, 128, smem, s>>>(sc, P, static_cast<const C*>(ckpt), count);
        else kPathAdjointResume<M, false><<<grid, 128, smem, s>>>(sc, P, static_cast<const C*>(ckpt), count);
    } else {
        if (sc.fullFeatures) kPathAdjoint<M, true><<<grid, 128, smem, s>>>(sc, P);
        else kPathAdjoint<M, false><<<grid, 128, smem, s>>>(sc, P);
    }
}

}  // namespace

size_t pathCheckpointBytes(int mode) {
    return mode == OWEC_PRECISION_FP64 ? sizeof(PathCheckpoint<double>) : sizeof(PathCheckpoint<float>);
}

void launchPathAdjoint(int mode, const DeviceScene& sc, const PassParams& pp, const HeightfieldParams& hf,
                       const PathAdjointTargets& t, bool fixedDecisions, const void* ckpt, const uint32_t* ckptCount,
                       int grid, cudaStream_t s) {
    AdjointParams P{pp, hf, t, fixedDecisions};
    if (mode == OWEC_PRECISION_FP64) launchMode<OWEC_PRECISION_FP64>(sc, P, ckpt, ckptCount, grid, s);
    else if (mode == OWEC_PRECISION_FP32) launchMode<OWEC_PRECISION_FP32>(sc, P, ckpt, ckptCount, grid, s);
    else launchMode<OWEC_PRECISION_MIXED>(sc, P, ckpt, ckptCount, grid, s);
}

}  // namespace owec
