// Forward light walks (the reference's Tracer::walk, src/owe/transport/transport.cpp:531-595),
// one thread per walk, binned where they end on a target boundary; and their path-replay adjoint
// with respect to the heights of a refractive heightfield.
//
// A walk is short (a lens: a handful of crossings and the odd ghost; a slab: three), so each thread
// loops over its own events with the same wide-BVH traversal as the camera paths. Bins accumulate
// in 64-bit fixed point (2^-32 per unit throughput), so the film is the same whatever order the
// walks finish in.
//
// The adjoint replays every walk from its seed with the forward's own arithmetic (the same
// decisions) and carries, in FP64, the derivatives of the ray and the throughput with respect to
// the heights of the heightfield triangles it crossed: implicit differentiation of each crossing
// (the hit point moves within its surface), of refraction and reflection, of the Fresnel weight,
// of Beer-Lambert attenuation, and finally of the bilinear splat on the target. Nothing of the
// forward pass is stored.
#include "tangents.cuh"
#include "transport.cuh"
#include "walk.hpp"

namespace owec {

namespace {

constexpr double kFixedScale = 4294967296.0;  // 2^32
constexpr int kSlots = 6;                      // heights a walk's derivative can depend on (two crossings)

struct WalkParams {
    owec_walk_desc w;
    double srcFrame[9];   // s, t, axis of the emitter
    double cosMax;
    Xform targetToLocal;
    uint64_t first, n;
    double scale;         // bins per unit throughput: measure / (walks * bin area)
    HeightfieldParams hf;
};

// The bins a landing point (x, y) in the target's frame contributes to, their weights, and the
// weights' derivatives with respect to x and y.
__device__ int splatBins(const WalkParams& P, double x, double y, int idx[4], double wgt[4], double dwx[4],
                         double dwy[4]) {
    const owec_walk_desc& w = P.w;
    const double fx = (x / w.half_x + 1) * 0.5 * w.width, fy = (1 - y / w.half_y) * 0.5 * w.height;
    const double kx = 0.5 * w.width / w.half_x, ky = -0.5 * w.height / w.half_y;  // d fx / dx, d fy / dy
    if (w.splat == OWEC_SPLAT_NEAREST) {
        if (!(fx >= 0 && fy >= 0 && fx < w.width && fy < w.height)) return 0;
        idx[0] = int(fy) * w.width + int(fx);
        wgt[0] = 1;
        dwx[0] = dwy[0] = 0;
        return 1;
    }
    // a tent one bin wide centred on the landing point, over the bin centres
    const double gx = fx - 0.5, gy = fy - 0.5;
    const double fx0 = floor(gx), fy0 = floor(gy);
    const int x0 = int(fx0), y0 = int(fy0);
    const double ax = gx - fx0, ay = gy - fy0;
    int n = 0;
    for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
            const int xi = x0 + i, yj = y0 + j;
            if (xi < 0 || yj < 0 || xi >= w.width || yj >= w.height) continue;
            idx[n] = yj * w.width + xi;
            const double wx = i ? ax : 1 - ax, wy = j ? ay : 1 - ay;
            wgt[n] = wx * wy;
            dwx[n] = (i ? 1.0 : -1.0) * wy * kx;
            dwy[n] = wx * (j ? 1.0 : -1.0) * ky;
            ++n;
        }
    return n;
}

// Derivatives of a walk's state with respect to the heights it has met so far.
struct Tangents {
    int n;
    int vert[kSlots];
    V3<double> dO[kSlots], dD[kSlots];
    double dB[kSlots];
    bool valid;
};

template <int M, bool ADJ, bool Full>
__device__ void walkOne(const DeviceScene& sc, const WalkParams& P, uint64_t walkIndex, StackEntry* stack, int stride,
                        unsigned long long* bins, unsigned long long* stats, const double* g, double* dH) {
    using R = typename Mode<M>::R;
    using Ro = typename Mode<M>::Ro;
    using Rr = typename Mode<M>::Rr;
    const owec_walk_desc& w = P.w;
    Pcg32 rng = Pcg32::seeded(hashCombine(w.seed, walkIndex), w.stream);
    const double lambda = w.lambda_min + (w.lambda_max - w.lambda_min) * rng.uniform();
    // emission
    const Draw2<double> e(rng);
    const V3<double> S(P.srcFrame[0], P.srcFrame[1], P.srcFrame[2]), T(P.srcFrame[3], P.srcFrame[4], P.srcFrame[5]),
        Ax(P.srcFrame[6], P.srcFrame[7], P.srcFrame[8]);
    V3<double> o(w.position[0] - sc.origin[0], w.position[1] - sc.origin[1], w.position[2] - sc.origin[2]);
    V3<double> dir;
    if (w.source_kind == OWEC_SOURCE_POINT) {
        const double cosT = (1 - e.u1) + e.u1 * P.cosMax;
        const double sinT = sqrt(fmax(0.0, 1 - cosT * cosT)), phi = 2 * kPi * e.u2;
        dir = S * (cos(phi) * sinT) + T * (sin(phi) * sinT) + Ax * cosT;
    } else if (w.source_kind == OWEC_SOURCE_COLLIMATED) {
        const double a = 2 * e.u1 - 1, b = 2 * e.u2 - 1;
        double dx = 0, dy = 0;
        if (!(a == 0 && b == 0)) {
            double r, phi;
            if (fabs(a) > fabs(b)) { r = a; phi = (kPi / 4) * (b / a); }
            else { r = b; phi = kPi / 2 - (kPi / 4) * (a / b); }
            dx = r * cos(phi);
            dy = r * sin(phi);
        }
        o = o + (S * dx + T * dy) * w.extent;
        dir = Ax;
    } else {
        o = o + (S * (2 * e.u1 - 1) + T * (2 * e.u2 - 1)) * w.extent;
        dir = Ax;
    }
    PathRay<R> ray;
    ray.o[0] = o.x; ray.o[1] = o.y; ray.o[2] = o.z;
    ray.d[0] = R(dir.x); ray.d[1] = R(dir.y); ray.d[2] = R(dir.z);
    ray.region = w.region;
    ray.depB = kNone;
    ray.depP = kNone;
    ray.errN = 0.f;
    R beta = R(1);
    Tangents tg;
    tg.n = 0;
    tg.valid = ADJ;
    bool binned = false, escaped = false, fault = false;
    int events = 0;
    for (int ev = 0; ev < w.max_events; ++ev) {
        ++events;
        RayQuery<R> rq;
        rq.od = V3<double>(ray.o[0], ray.o[1], ray.o[2]);
        rq.o = V3<R>(rq.od);
        rq.d = V3<R>(ray.d[0], ray.d[1], ray.d[2]);
        rq.tmax = R(INFINITY);
        rq.depB = ray.depB;
        rq.depP = ray.depP;
        rq.region = ray.region;
        rq.errN = R(ray.errN);
        HitRec h;
        const int s = traceRay<R, Ro, Rr, false, Full>(sc, rq, stack, stride, h);
        if (s == kTraceOverflow) { fault = true; break; }
        if (s != kTraceHit) { escaped = true; break; }
        const owec_medium med = sc.media[sc.regionMedium[ray.region]];
        const DBoundary bd = sc.boundaries[h.boundary];
        const SurfacePoint<R> gp = hitGeometry<R, Ro, Rr, Full>(sc, ray, h);
        const V3<R> d(ray.d[0], ray.d[1], ray.d[2]);
        const R betaBefore = beta;
        R atten = R(1);
        R sigmaA = R(0);
        if (mediumAbsorbs(med, sc)) {
            sigmaA = evalSpectrum(sc, med.absorption, R(lambda));
            atten = exp(-sigmaA * R(h.t));
            beta *= atten;
        }
        V3<double> dn_u[kSlots];  // derivatives of the unit normal at this crossing
        if (ADJ && tg.valid) {
            // The hit point stays on its surface as the heights move: implicit differentiation of
            // the crossing's distance, then of the point and the normal.
            const V3<double> dd(d), p = gp.p, n(gp.n);
            const double t = h.t;
            V3<double> nu = n;  // the (unnormalised) normal whose plane the point solves
            double nlen = 1;
            const bool hfHit = bd.shape == OWEC_SHAPE_MESH && h.boundary == P.hf.boundary;
            const bool sphere = bd.shape == OWEC_SHAPE_SPHERE;
            V3<double> v0, v1, v2;
            int vid[3] = {-1, -1, -1};
            if (hfHit) {
                V3<R> a, b, c;
                uint32_t bb, pr, kind;
                TriFetch<R>::get(sc, h.slot, a, b, c, bb, pr, kind);
                v0 = V3<double>(a);
                v1 = V3<double>(b);
                v2 = V3<double>(c);
                for (int a3 = 0; a3 < 3; ++a3) vid[a3] = int(P.hf.tris[3 * size_t(h.prim) + a3]);
                for (int a3 = 0; a3 < 3 && tg.valid; ++a3) {  // a slot for every vertex of the triangle
                    bool present = false;
                    for (int k = 0; k < tg.n; ++k) present = present || tg.vert[k] == vid[a3];
                    if (present) continue;
                    if (tg.n == kSlots) { tg.valid = false; break; }
                    tg.vert[tg.n] = vid[a3];
                    tg.dO[tg.n] = V3<double>();
                    tg.dD[tg.n] = V3<double>();
                    tg.dB[tg.n] = 0;
                    ++tg.n;
                }
                nu = cross(v1 - v0, v2 - v0);
                nlen = length(nu);
            } else if (tg.n > 0 && bd.shape != OWEC_SHAPE_MESH && bd.shape != OWEC_SHAPE_PLANE && !sphere) {
                tg.valid = false;  // sags and cylinders after a height dependence are not differentiated
            }
            if (tg.valid) {
                const V3<double> zdir(P.hf.zdir[0], P.hf.zdir[1], P.hf.zdir[2]);
                const double dnu = dot(dd, nu);
                for (int k = 0; k < tg.n; ++k) {
                    V3<double> dv0, dv1, dv2, dnk;
                    if (hfHit) {
                        if (tg.vert[k] == vid[0]) dv0 = zdir;
                        if (tg.vert[k] == vid[1]) dv1 = zdir;
                        if (tg.vert[k] == vid[2]) dv2 = zdir;
                        dnk = cross(dv1 - dv0, v2 - v0) + cross(v1 - v0, dv2 - dv0);
                    }
                    const V3<double> q = tg.dO[k] + tg.dD[k] * t - dv0;
                    const double dt = -(dot(q, nu) + (hfHit ? dot(p - v0, dnk) : 0.0)) / dnu;
                    const V3<double> dP = tg.dO[k] + tg.dD[k] * t + dd * dt;
                    if (hfHit) dn_u[k] = (dnk - n * dot(n, dnk)) / nlen;
                    else if (sphere) dn_u[k] = (dP - n * dot(n, dP)) / bd.params[0];
                    else dn_u[k] = V3<double>();
                    if (atten != R(1))  // Beer-Lambert over the segment
                        tg.dB[k] = double(atten) * (tg.dB[k] - double(betaBefore) * double(sigmaA) * dt);
                    tg.dO[k] = dP;  // the next segment starts at the hit point
                }
            }
        }
        const bool fromFront = dot(d, gp.n) < R(0);
        const uint32_t inc = fromFront ? bd.front : bd.back, other = fromFront ? bd.back : bd.front;
        ray.region = inc;
        const owec_optics op = sc.optics[bd.optics];
        const float errN = anchorError<R>(gp.p);
        if (op.type == OWEC_SURF_NULL) {
            ray.region = other;
            ray.o[0] = gp.p.x; ray.o[1] = gp.p.y; ray.o[2] = gp.p.z;
            ray.depB = h.boundary; ray.depP = h.prim; ray.errN = errN;
            continue;
        }
        if (op.type == OWEC_SURF_ABSORBER || op.type == OWEC_SURF_DETECTOR ||
            (w.mode == OWEC_WALK_PRIMARY_TRANSMISSION && op.type == OWEC_SURF_DIFFUSE)) {
            if (h.boundary == w.target) {
                const V3<double> pl = P.targetToLocal.point(gp.p);
                int idx[4];
                double wg[4], dwx[4], dwy[4];
                const int nb = splatBins(P, pl.x, pl.y, idx, wg, dwx, dwy);
                if (!ADJ) {
                    for (int b = 0; b < nb; ++b) {
                        const double v = double(beta) * wg[b] * kFixedScale;
                        if (v > 0) atomicAdd(bins + idx[b], (unsigned long long)(v + 0.5));
                    }
                } else if (tg.valid) {
                    // d(sum_b g_b beta w_b) = sum_b g_b (dbeta w_b + beta (dw_b/dx dx + dw_b/dy dy))
                    for (int k = 0; k < tg.n; ++k) {
                        const V3<double> dpl = P.targetToLocal.vector(tg.dO[k]);
                        double acc = 0;
                        for (int b = 0; b < nb; ++b)
                            acc += g[idx[b]] * (tg.dB[k] * wg[b] + double(beta) * (dwx[b] * dpl.x + dwy[b] * dpl.y));
                        atomicAdd(dH + tg.vert[k], acc * P.scale);
                    }
                }
                binned = nb > 0;
            }
            break;
        }
        Interface<R> it;
        it.o = op;
        it.n = gp.n;
        it.nFront = regionIndex(sc, bd.front, R(lambda));
        it.nBack = regionIndex(sc, bd.back, R(lambda));
        it.lambda = R(lambda);
        it.fresnelFloor = R(0);
        it.albedo = op.reflectance >= 0 ? evalSpectrum(sc, op.reflectance, R(lambda)) : R(1);
        {
            V3<double> texW;
            const V3<double>* tex = hitTexture<Full>(sc, bd, gp.pLocal, gp.nLocal, texW);
            if (tex) {
                R a = it.albedo * R(tex->x);
                if (tex->y != 0) a += R(tex->y) * evalSpectrum(sc, op.texture_b, R(lambda));
                if (tex->z != 0) a += R(tex->z) * evalSpectrum(sc, op.texture_c, R(lambda));
                it.albedo = a;
            }
        }
        ScatterSample<R> ss;
        bool ok;
        if (w.mode == OWEC_WALK_PRIMARY_TRANSMISSION && op.type == OWEC_SURF_DIELECTRIC) {
            const Draw2<R> u(rng);
            ok = sampleScatter(sc, it, d, R(1), u.u1, u.u2, false, ss);
            if (!ok) {
                const Draw2<R> v(rng);
                ok = sampleScatter(sc, it, d, R(0), v.u1, v.u2, false, ss);
            }
            if (ok && ss.delta) ss.weight = ss.transmitted ? ss.Tt : ss.R;
        } else {
            const Draw3<R> u(rng);
            ok = sampleScatter(sc, it, d, u.u1, u.u2, u.u3, false, ss);
        }
        if (!ok) break;
        if (ADJ && tg.valid && tg.n > 0) {
            const V3<double> dd(d), n(gp.n);
            if (op.type == OWEC_SURF_DIELECTRIC && ss.delta && w.mode == OWEC_WALK_PRIMARY_TRANSMISSION) {
                // Fresnel weight and Snell refraction (or the mirror reflection) differentiated
                const double eta = double(it.nBack) / double(it.nFront);
                double Rf, dRdc;
                fresnelWithDerivative(-dot(dd, n), eta, Rf, dRdc);
                const bool fr = dot(dd, n) < 0;
                const V3<double> nn = fr ? n : -n;
                const double ni = fr ? double(it.nFront) : double(it.nBack);
                const double nt = fr ? double(it.nBack) : double(it.nFront);
                for (int k = 0; k < tg.n; ++k) {
                    const V3<double> dn = dn_u[k];
                    const double dc = -(dot(tg.dD[k], n) + dot(dd, dn));  // d cos(incidence) against n
                    if (ss.transmitted) {
                        tg.dB[k] = tg.dB[k] * (1 - Rf) - double(beta) * dRdc * dc;
                        const V3<double> dnn = fr ? dn : -dn;
                        const double eta2 = ni / nt, cosi = -dot(dd, nn);
                        const double dcosi = -(dot(tg.dD[k], nn) + dot(dd, dnn));
                        const double kk = 1 - eta2 * eta2 * (1 - cosi * cosi), sq = sqrt(fmax(kk, 1e-300));
                        const V3<double> u = dd * eta2 + nn * (eta2 * cosi - sq);
                        const double ds = eta2 * eta2 * cosi * dcosi / sq;
                        const V3<double> du = tg.dD[k] * eta2 + dnn * (eta2 * cosi - sq) + nn * (eta2 * dcosi - ds);
                        const double ul = length(u);
                        const V3<double> out = u / ul;
                        tg.dD[k] = (du - out * dot(out, du)) / ul;
                    } else {
                        tg.dB[k] = tg.dB[k] * Rf + double(beta) * dRdc * dc;
                        const double dn0 = dot(dd, n);
                        tg.dD[k] = tg.dD[k] - n * (2 * (dot(tg.dD[k], n) + dot(dd, dn))) - dn * (2 * dn0);
                    }
                }
            } else if (op.type == OWEC_SURF_MIRROR) {
                const double dn0 = dot(dd, n);
                for (int k = 0; k < tg.n; ++k) {
                    tg.dB[k] *= double(ss.weight);
                    tg.dD[k] = tg.dD[k] - n * (2 * (dot(tg.dD[k], n) + dot(dd, dn_u[k]))) - dn_u[k] * (2 * dn0);
                }
            } else {
                tg.valid = false;  // a stochastic or rough event after a height dependence
            }
        }
        beta *= ss.weight;
        if (ss.transmitted) ray.region = other;
        ray.o[0] = gp.p.x; ray.o[1] = gp.p.y; ray.o[2] = gp.p.z;
        ray.d[0] = ss.wi.x; ray.d[1] = ss.wi.y; ray.d[2] = ss.wi.z;
        ray.depB = h.boundary;
        ray.depP = h.prim;
        ray.errN = errN;
    }
    if (!ADJ) {
        atomicAdd(stats + 0, 1ull);
        if (binned) atomicAdd(stats + 1, 1ull);
        if (escaped) atomicAdd(stats + 2, 1ull);
        atomicAdd(stats + 3, (unsigned long long)events);
        if (fault) atomicAdd(stats + 4, 1ull);
    } else if (fault || (!tg.valid && tg.n > 0)) {
        atomicAdd(stats + 4, 1ull);
    }
}

template <int M, bool ADJ, bool Full>
__global__ void __launch_bounds__(128) kWalk(DeviceScene sc, WalkParams P, unsigned long long* bins,
                                             unsigned long long* stats, const double* g, double* dH) {
    extern __shared__ StackEntry stackMem[];
    StackEntry* stack = stackMem + threadIdx.x;
    for (uint64_t k = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; k < P.n; k += uint64_t(gridDim.x) * blockDim.x)
        walkOne<M, ADJ, Full>(sc, P, P.first + k, stack, blockDim.x, bins, stats, g, dH);
}

// kWalk for the scene's shapes (the lean traversal unless the scene needs the full set).
template <int M, bool ADJ>
void walkKernel(const DeviceScene& sc, const WalkParams& P, unsigned long long* bins, unsigned long long* stats,
                const double* g, double* dH, int grid, cudaStream_t s) {
    const size_t smem = traversalSharedBytes(128);
    if (sc.fullFeatures) kWalk<M, ADJ, true><<<grid, 128, smem, s>>>(sc, P, bins, stats, g, dH);
    else kWalk<M, ADJ, false><<<grid, 128, smem, s>>>(sc, P, bins, stats, g, dH);
}

WalkParams makeParams(const owec_walk_desc& w, const Xform& targetToLocal, uint64_t first, uint64_t n, double scale,
                      const HeightfieldParams& hf) {
    WalkParams P{};
    P.w = w;
    V3<double> ax(w.axis[0], w.axis[1], w.axis[2]);
    ax = normalize(ax);
    V3<double> a, b;
    basis(ax, a, b);
    const double f[9] = {a.x, a.y, a.z, b.x, b.y, b.z, ax.x, ax.y, ax.z};
    for (int k = 0; k < 9; ++k) P.srcFrame[k] = f[k];
    P.cosMax = cos(w.extent);
    P.targetToLocal = targetToLocal;
    P.first = first;
    P.n = n;
    P.scale = scale;
    P.hf = hf;
    return P;
}

}  // namespace

void launchWalk(int mode, const DeviceScene& sc, const owec_walk_desc& w, const Xform& targetToLocal, uint64_t first,
                uint64_t n, unsigned long long* bins, unsigned long long* stats, int grid, cudaStream_t s) {
    HeightfieldParams hf{};
    hf.boundary = kNone;
    const WalkParams P = makeParams(w, targetToLocal, first, n, 1.0, hf);
    if (mode == OWEC_PRECISION_FP64) walkKernel<OWEC_PRECISION_FP64, false>(sc, P, bins, stats, nullptr, nullptr, grid, s);
    else if (mode == OWEC_PRECISION_FP32) walkKernel<OWEC_PRECISION_FP32, false>(sc, P, bins, stats, nullptr, nullptr, grid, s);
    else walkKernel<OWEC_PRECISION_MIXED, false>(sc, P, bins, stats, nullptr, nullptr, grid, s);
}

void launchWalkAdjoint(int mode, const DeviceScene& sc, const owec_walk_desc& w, const Xform& targetToLocal,
                       const HeightfieldParams& hf, uint64_t first, uint64_t n, double scale, const double* g,
                       double* dH, unsigned long long* stats, int grid, cudaStream_t s) {
    const WalkParams P = makeParams(w, targetToLocal, first, n, scale, hf);
    if (mode == OWEC_PRECISION_FP64) walkKernel<OWEC_PRECISION_FP64, true>(sc, P, nullptr, stats, g, dH, grid, s);
    else if (mode == OWEC_PRECISION_FP32) walkKernel<OWEC_PRECISION_FP32, true>(sc, P, nullptr, stats, g, dH, grid, s);
    else walkKernel<OWEC_PRECISION_MIXED, true>(sc, P, nullptr, stats, g, dH, grid, s);
}

}  // namespace owec
