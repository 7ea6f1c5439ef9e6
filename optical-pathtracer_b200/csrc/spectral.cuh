// Spectral quantities on the device: spectra, refractive-index models, hero-wavelength sampling
// and the CIE colour-matching fit. Formulas follow src/owe/core/shared/spectra.hpp:10-61,
// src/owe/core/spectrum.cpp:131-148, src/owe/core/medium.cpp:45-60 and
// src/owe/core/wavelengths.hpp:32-84.
#pragma once

#include "device_scene.cuh"

namespace owec {

constexpr double kLambdaMin = 360.0, kLambdaMax = 830.0;
constexpr int NW = 4;  // hero wavelengths per path

// Planck spectral radiance for lambda in nm, evaluated in micrometres (spectra.hpp:38-44).
template <class T>
OWEC_HD T planck(T lambdaNm, T kelvin) {
    const T c1 = T(1.191042972e8), c2 = T(1.438776877e4);
    const T l = lambdaNm * T(1e-3);
    const T l2 = l * l;
    return T(1e6) * c1 / (l2 * l2 * l * (exp(c2 / (l * kelvin)) - T(1)));
}

// Spectrum::eval (spectrum.cpp:131-148) for the kinds a scene description carries.
template <class T>
OWEC_HD T evalSpectrum(const DeviceScene& s, int32_t idx, T lambda) {
    if (idx < 0) return T(0);
    const owec_spectrum sp = s.spectra[idx];
    if (sp.kind == OWEC_SPEC_CONSTANT) return T(sp.a);
    if (sp.kind == OWEC_SPEC_BLACKBODY) return T(sp.scale) * planck(lambda, T(sp.a));
    const double* t = s.table + 2 * sp.table_offset;
    const int n = sp.table_count;
    if (lambda <= T(t[0])) return T(sp.scale * t[1]);
    if (lambda >= T(t[2 * (n - 1)])) return T(sp.scale * t[2 * (n - 1) + 1]);
    int lo = 0, hi = n - 1;  // the first entry above lambda (upper_bound), by bisection
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (T(t[2 * mid]) <= lambda) lo = mid; else hi = mid;
    }
    const T l0 = T(t[2 * lo]), l1 = T(t[2 * hi]);
    const T u = (lambda - l0) / (l1 - l0);
    return T(sp.scale) * (T(t[2 * lo + 1]) * (T(1) - u) + T(t[2 * hi + 1]) * u);
}

// Standard dry air, Ciddor (1996) two-term form, l2 in um^2 (spectra.hpp:55-58).
template <class T>
OWEC_HD T ciddorAir(T l2) {
    const T s2 = T(1) / l2;
    return T(1) + T(0.05792105) / (T(238.0185) - s2) + T(0.00167917) / (T(57.362) - s2);
}

// IndexModel::n (medium.cpp:45-60).
template <class T>
OWEC_HD T mediumIndex(const DeviceScene& s, const owec_medium& m, T lambdaNm) {
    const T l = lambdaNm * T(1e-3);
    const T l2 = l * l;
    T v;
    switch (m.index_kind) {
        case OWEC_INDEX_CONSTANT: v = T(m.coef_a[0]); break;
        case OWEC_INDEX_CAUCHY: v = T(m.coef_a[0]) + T(m.coef_a[1]) / l2 + T(m.coef_a[2]) / (l2 * l2); break;
        case OWEC_INDEX_SELLMEIER: {
            T acc = T(1);
            for (int i = 0; i < m.n_terms; ++i) acc += T(m.coef_a[i]) * l2 / (l2 - T(m.coef_b[i]));
            v = sqrt(acc);
            break;
        }
        case OWEC_INDEX_CIDDOR: v = ciddorAir(l2); break;
        default: v = evalSpectrum(s, m.index_table, lambdaNm); break;
    }
    return m.rel_air ? v * ciddorAir(l2) : v;
}

template <class T>
OWEC_HD T regionIndex(const DeviceScene& s, uint32_t region, T lambdaNm) {
    return mediumIndex(s, s.media[s.regionMedium[region]], lambdaNm);
}

// CIE 1931 2-degree colour matching functions, Wyman-Sloan-Shirley multi-lobe fit (spectra.hpp:13-24).
template <class T>
OWEC_HD T cieLobe(T x, T mu, T s1, T s2) {
    const T t = (x - mu) / (x < mu ? s1 : s2);
    return exp(T(-0.5) * t * t);
}
template <class T>
OWEC_HD T cieX(T l) {
    return T(1.056) * cieLobe(l, T(599.8), T(37.9), T(31.0)) + T(0.362) * cieLobe(l, T(442.0), T(16.0), T(26.7)) -
           T(0.065) * cieLobe(l, T(501.1), T(20.4), T(26.2));
}
template <class T>
OWEC_HD T cieY(T l) {
    return T(0.821) * cieLobe(l, T(568.8), T(46.9), T(40.5)) + T(0.286) * cieLobe(l, T(530.9), T(16.3), T(31.1));
}
template <class T>
OWEC_HD T cieZ(T l) {
    return T(1.217) * cieLobe(l, T(437.0), T(11.8), T(36.0)) + T(0.681) * cieLobe(l, T(459.0), T(26.0), T(13.8));
}

// Importance sampling of visible wavelengths, pdf proportional to 1/cosh^2(0.0072 (l - 538))
// (spectra.hpp:28-35).
template <class T>
OWEC_HD T sampleVisibleWavelength(T u) {
    return clampv(T(538) - T(138.888889) * atanh(T(0.85691062) - T(1.82750197) * u), T(kLambdaMin), T(kLambdaMax));
}
template <class T>
OWEC_HD T visibleWavelengthPdf(T l) {
    if (l < T(kLambdaMin) || l > T(kLambdaMax)) return T(0);
    return T(0.0039398042) / sqr(cosh(T(0.0072) * (l - T(538))));
}

// A path's wavelengths: the hero first; pdf 0 marks a terminated secondary (wavelengths.hpp:26-84).
template <class T>
struct Wavelengths {
    T lambda[NW];
    T pdf[NW];
    OWEC_HD bool secondaryTerminated() const {
        for (int i = 1; i < NW; ++i)
            if (pdf[i] != T(0)) return false;
        return true;
    }
    OWEC_HD void terminateSecondary() {
        if (secondaryTerminated()) return;
        for (int i = 1; i < NW; ++i) pdf[i] = T(0);
        pdf[0] /= T(NW);
    }
};

template <class T>
OWEC_HD Wavelengths<T> sampleHero(T u) {
    Wavelengths<T> w;
    for (int i = 0; i < NW; ++i) {
        T up = u + T(i) / T(NW);
        if (up >= T(1)) up -= T(1);
        w.lambda[i] = sampleVisibleWavelength(up);
        w.pdf[i] = visibleWavelengthPdf(w.lambda[i]);
    }
    return w;
}

// One wavelength uniform in [lo, hi]; the others share it with pdf 0 (already terminated). The
// hero's pdf carries the 1/NW that Wavelengths::toXYZ's average over NW undoes.
template <class T>
OWEC_HD Wavelengths<T> sampleUniformSingle(T u, T lo, T hi) {
    Wavelengths<T> w;
    const T l = lo + (hi - lo) * u;
    for (int i = 0; i < NW; ++i) { w.lambda[i] = l; w.pdf[i] = T(0); }
    w.pdf[0] = T(1) / ((hi - lo) * T(NW));
    return w;
}

}  // namespace owec
