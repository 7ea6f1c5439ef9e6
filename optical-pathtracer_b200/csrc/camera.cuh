// Camera-path generation shared by the wavefront's kGenerate and the path-replay adjoint: both must
// draw a pixel sample's numbers in the same order (IdealObserver::generate / SurfaceSensor::generate
// and the hero strata of CpuRenderer::pass).
#pragma once

#include "transport.cuh"

namespace owec {

template <class R>
__device__ __forceinline__ V3<R> rayDir(const PathRay<R>& r) { return V3<R>(r.d[0], r.d[1], r.d[2]); }
__device__ __forceinline__ V3<double> rayOrigin(const double o[3]) { return V3<double>(o[0], o[1], o[2]); }

template <int M>
__device__ __forceinline__ void setOrigin(double o[3], const V3<double>& p) {
    if (Mode<M>::plainOrigin) {
        o[0] = double(float(p.x));
        o[1] = double(float(p.y));
        o[2] = double(float(p.z));
    } else {
        o[0] = p.x;
        o[1] = p.y;
        o[2] = p.z;
    }
}

// The camera ray of path slot i of a batch (kGenerate's work, also replayed by the adjoint): the
// pixel sample's PCG32 stream, its wavelengths, the detector's ray and importance. Fills the path's
// ray, spectral state and bookkeeping, rng left after the generation's draws; returns whether the
// path carries weight.
template <int M>
__device__ __forceinline__ bool generateCameraPath(const DeviceScene& sc, const PassParams& pp, uint32_t i,
                                                  PathRay<typename Mode<M>::R>& ray, PathSpec<typename Mode<M>::R>& sp,
                                                  PathAux& aux, Pcg32& rngOut) {
    using R = typename Mode<M>::R;
    const uint32_t pixel = i % pp.nPixels;
    const uint32_t sub = i / pp.nPixels;
    const DDetector& det = sc.det;
    const int x = int(pixel % uint32_t(det.width)), y = int(pixel / uint32_t(det.width));
    Pcg32 rng = Pcg32::seeded(hashCombine(pp.seed, pixel), pp.streamBase + sub);
    // Hero strata of a one-sample pass: u = (0 + xi) / 1 + rot (cpu_backend.cpp:68-73)
    const double rot = rng.uniform();
    double u = rng.uniform() + rot;
    u -= floor(u);
    if (pp.wavelengthMode == OWEC_WAVELENGTHS_UNIFORM1) {
        const double lam = double(pp.lambdaMin) + (double(pp.lambdaMax) - double(pp.lambdaMin)) * u;
        for (int k = 0; k < NW; ++k) { sp.lambda[k] = float(lam); sp.pdf[k] = 0.f; }
        sp.pdf[0] = float(1.0 / ((double(pp.lambdaMax) - double(pp.lambdaMin)) * NW));
    } else {
        for (int k = 0; k < NW; ++k) {
            double up = u + double(k) / NW;
            if (up >= 1) up -= 1;
            const double lam = sampleVisibleWavelength(up);
            sp.lambda[k] = float(lam);
            sp.pdf[k] = float(visibleWavelengthPdf(lam));
        }
    }
    double px = x + rng.uniform(), py = y + rng.uniform();
    if (det.sigma > 0) {  // Detector::filterOffset: a Gaussian displacement (detector.hpp:57-62)
        const Draw2<double> g(rng);
        const double r = sqrt(-2 * log(1 - g.u1)), phi = 2 * kPi * g.u2;
        px += r * cos(phi) * det.sigma;
        py += r * sin(phi) * det.sigma;
    }
    double weight = 0;
    V3<double> o, dir;
    if (det.kind == OWEC_DETECTOR_OBSERVER) {
        // IdealObserver::generate (detector.cpp:61-91): a pinhole, or a thin lens whose pupil point
        // is drawn uniformly or, when a guide is set, from the guide's disk with its share
        const double sx = (2 * px / det.width - 1) * det.tanX;
        const double sy = (1 - 2 * py / det.height) * det.tanY;
        const V3<double> R3(det.right[0], det.right[1], det.right[2]), U3(det.up[0], det.up[1], det.up[2]),
            F3(det.fwd[0], det.fwd[1], det.fwd[2]);
        const V3<double> eye(det.pos[0], det.pos[1], det.pos[2]);
        dir = normalize(R3 * sx + U3 * sy + F3);
        o = eye;
        weight = 1;
        if (det.pupil > 0) {
            V3<double> c;
            bool guided = false;
            if (det.guideR > 0) {  // IdealObserver::guideCenter (detector.cpp:29-34)
                const double dn = dot(dir, F3);
                if (dn > 0) {
                    const V3<double> gc(det.guideC[0], det.guideC[1], det.guideC[2]);
                    c = gc - dir * (dot(gc - eye, F3) / dn);
                    guided = dot(c - eye, c - eye) < sqr(det.pupil + det.guideR);
                }
            }
            const bool fromGuide = guided && rng.uniform() < det.guideShare;
            const Draw2<double> u(rng);
            double dx, dy;
            concentricDisk(u.u1, u.u2, dx, dy);
            o = fromGuide ? c + (R3 * dx + U3 * dy) * det.guideR : eye + (R3 * dx + U3 * dy) * det.pupil;
            if (guided) {
                // radiance averaged over the eye's pupil: (1 / A_eye) / p(q), nothing outside the eye
                if (fromGuide && dot(o - eye, o - eye) > sqr(det.pupil)) {
                    weight = 0;
                } else {
                    const double pEye = 1 / (kPi * sqr(det.pupil));
                    const bool inGuide = fromGuide || dot(o - c, o - c) <= sqr(det.guideR);
                    const double pGuide = inGuide ? 1 / (kPi * sqr(det.guideR)) : 0;
                    weight = pEye / ((1 - det.guideShare) * pEye + det.guideShare * pGuide);
                }
            }
            if (isfinite(det.focus)) dir = normalize(eye + (R3 * sx + U3 * sy + F3) * det.focus - o);
        }
        ray.region = det.region;
        ray.depB = kNone;
        ray.depP = kNone;
        ray.errN = 0.f;
    } else if (!(px < 0 || py < 0 || px >= det.width || py >= det.height)) {
        // SurfaceSensor::generate (detector.cpp:113-148): hemispherical, or aimed at a disk (and a
        // focus disk) with cosine support kept by the remaining share
        if (det.flipX) px = det.width - px;
        if (det.flipY) py = det.height - py;
        const DBoundary& bd = sc.boundaries[det.boundary];
        const V3<double> pl((2 * px / det.width - 1) * det.halfX, (1 - 2 * py / det.height) * det.halfY, 0);
        o = bd.toWorld.point(pl);
        const V3<double> nrm(det.normal[0], det.normal[1], det.normal[2]);
        weight = kPi;
        if (det.aimR > 0) {
            const V3<double> aN(det.aimN[0], det.aimN[1], det.aimN[2]), aC(det.aimC[0], det.aimC[1], det.aimC[2]);
            const V3<double> fC(det.focusC[0], det.focusC[1], det.focusC[2]);
            V3<double> a1, a2;
            basis(aN, a1, a2);
            const bool useAim = det.aimShare >= 1 || rng.uniform() < det.aimShare;
            const bool useFocus = det.focusShare > 0 && rng.uniform() < det.focusShare;
            const Draw2<double> u(rng);
            double dx, dy;
            concentricDisk(u.u1, u.u2, dx, dy);
            const V3<double> w = (useFocus ? fC : aC) + (a1 * dx + a2 * dy) * (useFocus ? det.focusR : det.aimR) - o;
            dir = w / length(w);
            if (!useAim) {
                double hx, hy;
                concentricDisk(u.u1, u.u2, hx, hy);
                dir = Frame<double>(nrm).toWorld(V3<double>(hx, hy, sqrt(fmax(0.0, 1 - hx * hx - hy * hy))));
            }
            const double cosS = dot(dir, nrm);
            double pdfW = 0;
            if (cosS > 0) {
                pdfW = (1 - det.focusShare) * diskAimPdf(o, dir, aC, aN, det.aimR, useAim && !useFocus);
                if (det.focusShare > 0) pdfW += det.focusShare * diskAimPdf(o, dir, fC, aN, det.focusR, useAim && useFocus);
                pdfW = det.aimShare * pdfW + (1 - det.aimShare) * cosS * kInvPi;
            }
            weight = cosS > 0 && pdfW > 0 ? cosS / pdfW : 0.0;
        } else {
            const Draw2<double> g(rng);
            double dx, dy;
            concentricDisk(g.u1, g.u2, dx, dy);
            dir = Frame<double>(nrm).toWorld(V3<double>(dx, dy, sqrt(fmax(0.0, 1 - dx * dx - dy * dy))));
        }
        ray.region = det.region;
        ray.depB = det.boundary;
        ray.depP = 0;
        ray.errN = anchorError<R>(o);
    }
    aux.flags = 0;
    aux.weight = float(weight);
    aux.pixel = pixel;
    aux.stream = pp.streamBase + sub;
    aux.depth = 0;
    aux.prevPdf = 0.f;
    aux.lastBoundary = kNone;
    for (int k = 0; k < NW; ++k) {
        sp.beta[k] = (k == 0 || sp.pdf[k] != 0.f) ? R(1) : R(0);  // maskTerminated
        sp.L[k] = 0.f;
    }
    const bool live = weight > 0;
    if (live) {
        setOrigin<M>(ray.o, o);
        ray.d[0] = R(dir.x);
        ray.d[1] = R(dir.y);
        ray.d[2] = R(dir.z);
        aux.flags = kFlagSpecular | kFlagAlive;
        aux.prevP[0] = o.x;
        aux.prevP[1] = o.y;
        aux.prevP[2] = o.z;
    }
    aux.rngState = rng.state;
    rngOut = rng;
    return live;
}

}  // namespace owec
