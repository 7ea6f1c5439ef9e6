// Interface optics on the device: Snell refraction, Fresnel for dielectrics and conductors, GGX
// microfacet lobes with visible-normal sampling, and the per-surface scattering sample and
// evaluation of the reference (src/owe/core/shared/optics.hpp:14-246,
// src/owe/transport/scattering.cpp:65-222). Local lobes work in a frame whose +z is the normal;
// wo points back along the incident ray, wi along the scattered one.
#pragma once

#include "spectral.cuh"

namespace owec {

template <class T> struct C2 { T re, im; };
template <class T> OWEC_HD C2<T> cmul(C2<T> a, C2<T> b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
template <class T> OWEC_HD C2<T> cdiv(C2<T> a, C2<T> b) {
    const T d = b.re * b.re + b.im * b.im;
    return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
template <class T> OWEC_HD C2<T> csqrtp(C2<T> z) {
    const T r = sqrt(z.re * z.re + z.im * z.im);
    return {sqrt(fmax(T(0), (r + z.re) / T(2))), copysign(sqrt(fmax(T(0), (r - z.re) / T(2))), z.im)};
}

// Snell refraction of propagation direction d (optics.hpp:14-24). False on total internal reflection.
template <class T>
OWEC_HD bool refractDirection(const V3<T>& d, const V3<T>& n, T ni, T nt, V3<T>& out) {
    const V3<T> nn = dot(d, n) < T(0) ? n : -n;
    const T cosi = -dot(d, nn);
    const T eta = ni / nt;
    const T k = T(1) - eta * eta * (T(1) - cosi * cosi);
    out = d;
    if (k < T(0)) return false;
    out = normalize(d * eta + nn * (eta * cosi - sqrt(k)));
    return true;
}

// Unpolarised dielectric reflectance, eta = n_back / n_front, cosThetaI signed (optics.hpp:42-54).
template <class T>
OWEC_HD T fresnelDielectric(T cosThetaI, T eta) {
    cosThetaI = clampv(cosThetaI, T(-1), T(1));
    if (cosThetaI < T(0)) {
        eta = T(1) / eta;
        cosThetaI = -cosThetaI;
    }
    const T sin2T = (T(1) - cosThetaI * cosThetaI) / (eta * eta);
    if (sin2T >= T(1)) return T(1);
    const T cosT = safeSqrt(T(1) - sin2T);
    const T rParl = (eta * cosThetaI - cosT) / (eta * cosThetaI + cosT);
    const T rPerp = (cosThetaI - eta * cosT) / (cosThetaI + eta * cosT);
    return (rParl * rParl + rPerp * rPerp) / T(2);
}

// Reflectance of a conductor of complex relative index eta (optics.hpp:69-79).
template <class T>
OWEC_HD T fresnelConductor(T cosThetaI, C2<T> eta) {
    cosThetaI = clampv(cosThetaI, T(0), T(1));
    const C2<T> c{cosThetaI, T(0)};
    const C2<T> sin2T = cdiv(C2<T>{T(1) - cosThetaI * cosThetaI, T(0)}, cmul(eta, eta));
    const C2<T> cosT = csqrtp(C2<T>{T(1) - sin2T.re, -sin2T.im});
    const C2<T> ec{eta.re * cosThetaI, eta.im * cosThetaI}, ect = cmul(eta, cosT);
    const C2<T> rParl = cdiv(C2<T>{ec.re - cosT.re, ec.im - cosT.im}, C2<T>{ec.re + cosT.re, ec.im + cosT.im});
    const C2<T> rPerp = cdiv(C2<T>{c.re - ect.re, c.im - ect.im}, C2<T>{c.re + ect.re, c.im + ect.im});
    return (rParl.re * rParl.re + rParl.im * rParl.im + rPerp.re * rPerp.re + rPerp.im * rPerp.im) / T(2);
}

template <class T> OWEC_HD bool sameHemisphere(const V3<T>& a, const V3<T>& b) { return a.z * b.z > T(0); }

// pbrt-v4 style refraction of wi about n, eta = n_t/n_i relative to n's hemisphere (optics.hpp:83-98).
template <class T>
OWEC_HD bool refractLocal(V3<T> wi, V3<T> n, T eta, T& etap, V3<T>& wt) {
    T cosI = dot(n, wi);
    etap = T(1);
    wt = wi;
    if (cosI < T(0)) {
        eta = T(1) / eta;
        cosI = -cosI;
        n = -n;
    }
    const T sin2T = fmax(T(0), T(1) - cosI * cosI) / (eta * eta);
    if (sin2T >= T(1)) return false;
    const T cosT = safeSqrt(T(1) - sin2T);
    wt = -wi / eta + n * (cosI / eta - cosT);
    etap = eta;
    return true;
}

template <class T>
OWEC_HD T fresnelBranchProbability(T R, T floorP) {
    return floorP > T(0) && R < T(1) ? clampv(R, floorP, T(1) - floorP) : R;
}

// ------------------------------------------------------------------ GGX (Trowbridge-Reitz)
constexpr double kSmoothRoughness = 1e-3;
template <class T> OWEC_HD T ggxAlpha(T roughness) { return fmax(roughness, T(1e-4)); }
template <class T>
OWEC_HD T ggxD(T a, const V3<T>& wm) {
    const T c2 = wm.z * wm.z;
    if (c2 <= T(0)) return T(0);
    const T c4 = c2 * c2;
    if (c4 < T(1e-16)) return T(0);
    const T e = (T(1) - c2) / c2 / (a * a);
    return T(1) / (T(kPi) * a * a * c4 * sqr(T(1) + e));
}
template <class T>
OWEC_HD T ggxLambda(T a, const V3<T>& w) {
    const T c2 = w.z * w.z;
    if (c2 <= T(0)) return T(0);
    return (sqrt(T(1) + a * a * ((T(1) - c2) / c2)) - T(1)) / T(2);
}
template <class T> OWEC_HD T ggxG1(T a, const V3<T>& w) { return T(1) / (T(1) + ggxLambda(a, w)); }
template <class T> OWEC_HD T ggxG(T a, const V3<T>& wo, const V3<T>& wi) {
    return T(1) / (T(1) + ggxLambda(a, wo) + ggxLambda(a, wi));
}
template <class T>
OWEC_HD T ggxPdf(T a, const V3<T>& w, const V3<T>& wm) {
    if (w.z == T(0)) return T(0);
    return ggxG1(a, w) / fabs(w.z) * ggxD(a, wm) * fabs(dot(w, wm));
}
// Visible-normal sampling (Heitz 2018), as optics.hpp:137-151.
template <class T>
OWEC_HD V3<T> ggxSampleWm(T a, const V3<T>& w, T u1, T u2) {
    V3<T> wh = normalize(V3<T>(a * w.x, a * w.y, w.z));
    if (wh.z < T(0)) wh = -wh;
    const V3<T> T1 = wh.z < T(0.99999) ? normalize(cross(V3<T>(0, 0, 1), wh)) : V3<T>(1, 0, 0);
    const V3<T> T2 = cross(wh, T1);
    const T r = sqrt(u1), phi = T(2 * kPi) * u2;
    const T px = r * cos(phi);
    T py = r * sin(phi);
    const T h = sqrt(fmax(T(0), T(1) - px * px));
    const T s = (T(1) + wh.z) / T(2);
    py = (T(1) - s) * h + s * py;
    const T pz = safeSqrt(T(1) - px * px - py * py);
    const V3<T> nh = T1 * px + T2 * py + wh * pz;
    return normalize(V3<T>(a * nh.x, a * nh.y, fmax(T(1e-6), nh.z)));
}

template <class T>
struct LobeSample {
    V3<T> wi;
    T weight, pdf;
    bool transmitted;
    T R, T_;
};

// Rough dielectric (Walter et al. 2007, pbrt-v4 formulation), eta = n_back / n_front (optics.hpp:165-196).
template <class T>
OWEC_HD bool sampleRoughDielectric(T a, const V3<T>& wo, T eta, T uc, T u1, T u2, bool radiance, LobeSample<T>& s) {
    const V3<T> wm = ggxSampleWm(a, wo, u1, u2);
    const T R = fresnelDielectric(dot(wo, wm), eta), Tr = T(1) - R;
    s.wi = wo;
    s.weight = T(0);
    s.pdf = T(0);
    s.transmitted = false;
    s.R = R;
    s.T_ = Tr;
    if (uc < R / (R + Tr)) {
        s.wi = reflect(-wo, wm);
        if (!sameHemisphere(wo, s.wi)) return false;
        s.pdf = ggxPdf(a, wo, wm) / (T(4) * fabs(dot(wo, wm))) * R / (R + Tr);
        const T f = ggxD(a, wm) * ggxG(a, wo, s.wi) * R / (T(4) * fabs(s.wi.z) * fabs(wo.z));
        s.weight = f * fabs(s.wi.z) / s.pdf;
    } else {
        T etap;
        V3<T> wi;
        if (!refractLocal(wo, wm, eta, etap, wi)) return false;
        if (sameHemisphere(wo, wi) || wi.z == T(0)) return false;
        s.wi = wi;
        s.transmitted = true;
        const T denom = sqr(dot(wi, wm) + dot(wo, wm) / etap);
        s.pdf = ggxPdf(a, wo, wm) * (fabs(dot(wi, wm)) / denom) * Tr / (R + Tr);
        T ft = Tr * ggxD(a, wm) * ggxG(a, wo, wi) * fabs(dot(wi, wm) * dot(wo, wm) / (wi.z * wo.z * denom));
        if (radiance) ft /= sqr(etap);
        s.weight = ft * fabs(wi.z) / s.pdf;
    }
    return isfinite(s.weight) && s.pdf > T(0);
}

template <class T>
OWEC_HD T evalRoughDielectric(T a, const V3<T>& wo, const V3<T>& wi, T eta, bool radiance, T& pdf) {
    pdf = T(0);
    const T co = wo.z, ci = wi.z;
    if (co == T(0) || ci == T(0)) return T(0);
    const bool refl = co * ci > T(0);
    T etap = T(1);
    if (!refl) etap = co > T(0) ? eta : T(1) / eta;
    V3<T> wm = wi * etap + wo;
    if (dot(wm, wm) == T(0)) return T(0);
    wm = normalize(wm);
    if (wm.z < T(0)) wm = -wm;
    if (dot(wm, wi) * ci < T(0) || dot(wm, wo) * co < T(0)) return T(0);
    const T R = fresnelDielectric(dot(wo, wm), eta), Tr = T(1) - R;
    if (refl) {
        pdf = ggxPdf(a, wo, wm) / (T(4) * fabs(dot(wo, wm))) * R / (R + Tr);
        return ggxD(a, wm) * ggxG(a, wo, wi) * R / fabs(T(4) * ci * co);
    }
    const T denom = sqr(dot(wi, wm) + dot(wo, wm) / etap);
    pdf = ggxPdf(a, wo, wm) * fabs(dot(wi, wm)) / denom * Tr / (R + Tr);
    T ft = ggxD(a, wm) * Tr * ggxG(a, wo, wi) * fabs(dot(wi, wm) * dot(wo, wm) / (denom * ci * co));
    if (radiance) ft /= sqr(etap);
    return ft;
}

// Rough conductor seen from the upper hemisphere (optics.hpp:220-246).
template <class T>
OWEC_HD bool sampleRoughConductor(T a, const V3<T>& w, C2<T> eta, T tint, T u1, T u2, LobeSample<T>& s) {
    const V3<T> wm = ggxSampleWm(a, w, u1, u2);
    s.wi = reflect(-w, wm);
    s.weight = T(0);
    s.pdf = T(0);
    s.transmitted = false;
    s.T_ = T(0);
    s.R = fresnelConductor(fabs(dot(w, wm)), eta) * tint;
    if (s.wi.z <= T(0)) return false;
    s.pdf = ggxPdf(a, w, wm) / (T(4) * fabs(dot(w, wm)));
    if (!(s.pdf > T(0))) return false;
    const T f = ggxD(a, wm) * s.R * ggxG(a, w, s.wi) / (T(4) * s.wi.z * w.z);
    s.weight = f * s.wi.z / s.pdf;
    return isfinite(s.weight);
}
template <class T>
OWEC_HD T evalRoughConductor(T a, const V3<T>& wo, const V3<T>& wi, C2<T> eta, T tint, T& pdf) {
    pdf = T(0);
    V3<T> wm = wo + wi;
    if (dot(wm, wm) == T(0)) return T(0);
    wm = normalize(wm);
    const T F = fresnelConductor(fabs(dot(wo, wm)), eta) * tint;
    pdf = ggxPdf(a, wo, wm) / (T(4) * fabs(dot(wo, wm)));
    return ggxD(a, wm) * F * ggxG(a, wo, wi) / (T(4) * wi.z * wo.z);
}

// ------------------------------------------------------------------ the interface of a hit
template <class T>
struct Interface {
    owec_optics o;
    V3<T> n;           // world normal toward the front region
    T nFront, nBack;   // indices at the interface's wavelength
    T lambda;
    T fresnelFloor;
    T albedo;          // reflectance spectrum at lambda
};

enum EventKind : uint8_t { kEvNone, kEvReflect, kEvRefract, kEvTIR, kEvGlossy, kEvGlossyT, kEvDiffuse };

template <class T>
struct ScatterSample {
    V3<T> wi;
    T weight = T(0), pdf = T(0);
    bool delta = false, transmitted = false;
    T R = T(0), Tt = T(0), cosI = T(0);
    uint8_t event = kEvNone;
};

template <class T>
OWEC_HD C2<T> conductorEta(const DeviceScene& s, const owec_optics& o, T lambda, T nMedium) {
    return {evalSpectrum(s, o.conductor_n, lambda) / nMedium, evalSpectrum(s, o.conductor_k, lambda) / nMedium};
}

template <class T>
OWEC_HD bool isDeltaOptics(const owec_optics& o) {
    if (o.type == OWEC_SURF_DIELECTRIC || o.type == OWEC_SURF_CONDUCTOR) return o.roughness < kSmoothRoughness;
    return o.type == OWEC_SURF_MIRROR;
}

// sampleScatter (scattering.cpp:65-145), radiance or importance transport.
template <class T>
OWEC_HD bool sampleScatter(const DeviceScene& sc, const Interface<T>& it, const V3<T>& d, T uc, T u1, T u2,
                           bool radiance, ScatterSample<T>& s) {
    const Frame<T> frame(it.n);
    const V3<T> wo = frame.toLocal(-d);
    const bool fromFront = wo.z > T(0);
    s = ScatterSample<T>{};
    s.cosI = fabs(wo.z);
    const owec_optics& o = it.o;
    switch (o.type) {
        case OWEC_SURF_DIELECTRIC: {
            const T eta = it.nBack / it.nFront;
            if (o.roughness >= kSmoothRoughness && eta != T(1)) {
                LobeSample<T> l;
                if (!sampleRoughDielectric(ggxAlpha(T(o.roughness)), wo, eta, uc, u1, u2, radiance, l)) return false;
                s.wi = frame.toWorld(l.wi);
                s.weight = l.weight;
                s.pdf = l.pdf;
                s.transmitted = l.transmitted;
                s.event = l.transmitted ? kEvGlossyT : kEvGlossy;
                s.R = l.R;
                s.Tt = l.T_;
                return true;
            }
            const T ni = fromFront ? it.nFront : it.nBack;
            const T nt = fromFront ? it.nBack : it.nFront;
            const T R = fresnelDielectric(wo.z, eta);
            const T pR = fresnelBranchProbability(R, it.fresnelFloor);
            s.R = R;
            s.Tt = T(1) - R;
            s.delta = true;
            if (uc < pR) {
                s.wi = frame.toWorld(V3<T>(-wo.x, -wo.y, wo.z));
                s.weight = R / pR;
                s.event = R >= T(1) ? kEvTIR : kEvReflect;
                return s.weight > T(0);
            }
            if (!refractDirection(d, it.n, ni, nt, s.wi)) return false;
            s.weight = (T(1) - R) / (T(1) - pR) * (radiance ? sqr(ni / nt) : T(1));
            s.event = kEvRefract;
            s.transmitted = true;
            return true;
        }
        case OWEC_SURF_DIFFUSE: {
            if (!fromFront && o.back_absorbs) return false;
            const T albedo = it.albedo;
            if (albedo <= T(0)) return false;
            // sampleCosineHemisphere over the concentric disk (warps.hpp:45-70)
            const T a = T(2) * u1 - T(1), b = T(2) * u2 - T(1);
            T dx = T(0), dy = T(0);
            if (!(a == T(0) && b == T(0))) {
                T r, phi;
                if (fabs(a) > fabs(b)) { r = a; phi = T(kPi / 4) * (b / a); }
                else { r = b; phi = T(kPi / 2) - T(kPi / 4) * (a / b); }
                dx = r * cos(phi);
                dy = r * sin(phi);
            }
            V3<T> w(dx, dy, safeSqrt(T(1) - dx * dx - dy * dy));
            if (!fromFront) w.z = -w.z;
            s.wi = frame.toWorld(w);
            s.pdf = fabs(w.z) * T(kInvPi);
            s.weight = albedo;
            s.event = kEvDiffuse;
            s.R = albedo;
            return s.pdf > T(0);
        }
        case OWEC_SURF_MIRROR:
            if (!fromFront && o.back_absorbs) return false;
            s.wi = frame.toWorld(V3<T>(-wo.x, -wo.y, wo.z));
            s.weight = it.albedo;
            s.delta = true;
            s.event = kEvReflect;
            s.R = s.weight;
            return s.weight > T(0);
        case OWEC_SURF_CONDUCTOR: {
            if (!fromFront && o.back_absorbs) return false;
            const C2<T> eta = conductorEta(sc, o, it.lambda, fromFront ? it.nFront : it.nBack);
            const T tint = it.albedo;
            const V3<T> w = fromFront ? wo : V3<T>(wo.x, wo.y, -wo.z);
            if (o.roughness < kSmoothRoughness) {
                s.wi = frame.toWorld(V3<T>(-wo.x, -wo.y, wo.z));
                s.weight = fresnelConductor(w.z, eta) * tint;
                s.delta = true;
                s.event = kEvReflect;
                s.R = s.weight;
                return s.weight > T(0);
            }
            LobeSample<T> l;
            if (!sampleRoughConductor(ggxAlpha(T(o.roughness)), w, eta, tint, u1, u2, l)) return false;
            if (!fromFront) l.wi.z = -l.wi.z;
            s.wi = frame.toWorld(l.wi);
            s.weight = l.weight;
            s.pdf = l.pdf;
            s.event = kEvGlossy;
            s.R = l.R;
            return true;
        }
        default: return false;
    }
}

// evalScatter (scattering.cpp:147-172): f(wo = -d, wi) without the cosine, and the pdf of wi.
template <class T>
OWEC_HD T evalScatter(const DeviceScene& sc, const Interface<T>& it, const V3<T>& d, const V3<T>& wiW, bool radiance,
                      T& pdf) {
    pdf = T(0);
    const owec_optics& o = it.o;
    if (isDeltaOptics<T>(o)) return T(0);
    const Frame<T> frame(it.n);
    V3<T> wo = frame.toLocal(-d);
    V3<T> wi = frame.toLocal(wiW);
    const bool fromFront = wo.z > T(0);
    switch (o.type) {
        case OWEC_SURF_DIFFUSE:
            if (!fromFront && o.back_absorbs) return T(0);
            if (!sameHemisphere(wo, wi)) return T(0);
            pdf = fabs(wi.z) * T(kInvPi);
            return it.albedo * T(kInvPi);
        case OWEC_SURF_CONDUCTOR: {
            if (!fromFront && o.back_absorbs) return T(0);
            if (!sameHemisphere(wo, wi)) return T(0);
            if (!fromFront) { wo.z = -wo.z; wi.z = -wi.z; }
            const C2<T> eta = conductorEta(sc, o, it.lambda, fromFront ? it.nFront : it.nBack);
            return evalRoughConductor(ggxAlpha(T(o.roughness)), wo, wi, eta, it.albedo, pdf);
        }
        case OWEC_SURF_DIELECTRIC:
            return evalRoughDielectric(ggxAlpha(T(o.roughness)), wo, wi, it.nBack / it.nFront, radiance, pdf);
        default: return T(0);
    }
}

template <class T>
OWEC_HD bool isDispersive(const Interface<T>& hero, const Interface<T>& other) {
    const T a = hero.nBack / hero.nFront, b = other.nBack / other.nFront;
    return fabs(a - b) > T(1e-12) * fabs(a);
}

// Throughput multiplier at another wavelength for the hero's sample (scattering.cpp:202-222).
template <class T>
OWEC_HD T secondaryScatterWeight(const DeviceScene& sc, const Interface<T>& it, const V3<T>& d,
                                 const ScatterSample<T>& s, bool radiance) {
    if (!s.delta) {
        T pdf;
        const T f = evalScatter(sc, it, d, s.wi, radiance, pdf);
        return s.pdf > T(0) ? f * fabs(dot(s.wi, it.n)) / s.pdf : T(0);
    }
    const T cosI = fabs(dot(d, it.n));
    switch (it.o.type) {
        case OWEC_SURF_DIELECTRIC: return s.weight;
        case OWEC_SURF_MIRROR: return it.albedo;
        case OWEC_SURF_CONDUCTOR: {
            const bool fromFront = dot(d, it.n) < T(0);
            const T nMed = fromFront ? it.nFront : it.nBack;
            return fresnelConductor(cosI, conductorEta(sc, it.o, it.lambda, nMed)) * it.albedo;
        }
        default: return T(0);
    }
}

// Henyey-Greenstein phase function and its sampling (warps.hpp:145-162).
template <class T>
OWEC_HD T hgPhase(T cosTheta, T g) {
    const T denom = T(1) + g * g + T(2) * g * cosTheta;
    return (T(1) - g * g) / (T(4 * kPi) * denom * sqrt(fmax(denom, T(1e-30))));
}
template <class T>
OWEC_HD T sampleHg(const V3<T>& wo, T g, T u1, T u2, V3<T>& wi) {
    T cosTheta;
    if (fabs(g) < T(1e-3)) cosTheta = T(1) - T(2) * u1;
    else cosTheta = T(-1) / (T(2) * g) * (T(1) + g * g - sqr((T(1) - g * g) / (T(1) + g - T(2) * g * u1)));
    const T sinTheta = safeSqrt(T(1) - cosTheta * cosTheta);
    const T phi = T(2 * kPi) * u2;
    V3<T> s, t;
    basis(wo, s, t);
    wi = s * (sinTheta * cos(phi)) + t * (sinTheta * sin(phi)) + wo * cosTheta;
    return hgPhase(dot(wo, wi), g);
}

template <class T>
OWEC_HD T powerHeuristic(T fPdf, T gPdf) {
    const T f = fPdf * fPdf, g = gPdf * gPdf;
    if (isinf(f)) return T(1);
    if (f + g == T(0)) return T(0);
    return f / (f + g);
}

}  // namespace owec
