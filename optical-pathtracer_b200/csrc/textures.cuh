// Procedural textures of Lambertian albedos: the mixing weights of a texture's three spectra at a
// boundary-local point and normal (the reference's solid textures, src/owe/core/shared/textures.hpp:
// value noise on a 64-bit hashed lattice, its fractal sum, and the checker, noise, rings, terrain,
// bands, radial and marble patterns). The lattice hash and the 53-bit lattice values are the
// reference CPU's, in FP64, so a device path reads the same albedo as the CPU path at the same point.
#pragma once

#include "rng.cuh"

namespace owec {

// The value in [0, 1) of lattice key k: its top 53 bits.
__device__ __forceinline__ double latticeValue(uint64_t k) { return double(k >> 11) * (1.0 / 9007199254740992.0); }

// Value noise in [0, 1) with a smoothstep fade, at p (textures.hpp:20-49): the eight corners of
// p's cell hashed as hashCombine(hashCombine(x, y), z), the y and z mixes shared between corners.
__device__ inline double valueNoise3(const V3<double>& p) {
    const double fx = floor(p.x), fy = floor(p.y), fz = floor(p.z);
    const int ix = int(fx), iy = int(fy), iz = int(fz);
    const double ux = p.x - fx, uy = p.y - fy, uz = p.z - fz;
    const double tx = ux * ux * (3 - 2 * ux), ty = uy * uy * (3 - 2 * uy), tz = uz * uz * (3 - 2 * uz);
    constexpr uint64_t C = 0x9e3779b97f4a7c15ULL;
    const uint64_t my0 = mixBits(uint64_t(uint32_t(iy))) + C, my1 = mixBits(uint64_t(uint32_t(iy + 1))) + C;
    const uint64_t mz0 = mixBits(uint64_t(uint32_t(iz))) + C, mz1 = mixBits(uint64_t(uint32_t(iz + 1))) + C;
    double r = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        const bool dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
        const uint64_t kxy = mixBits(uint64_t(uint32_t(ix + (dx ? 1 : 0))) ^ (dy ? my1 : my0));
        const double v = latticeValue(mixBits(kxy ^ (dz ? mz1 : mz0)));
        r += (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz) * v;
    }
    return r;
}

// Fractal sum of value noise over `octaves`, normalised to [0, 1) (textures.hpp:55-66).
__device__ inline double fbm3(V3<double> q, int octaves) {
    double sum = 0, amp = 0.5, norm = 0;
    for (int i = 0; i < octaves; ++i) {
        sum += amp * valueNoise3(q);
        norm += amp;
        amp *= 0.5;
        q = q * 2.03 + V3<double>(17.1, 5.3, 9.7);
    }
    return sum / norm;
}

__device__ __forceinline__ double saturate01(double x) { return fmin(1.0, fmax(0.0, x)); }

// The weights of the spectra a, b, c of texture `kind` at local point p with normal n (wavelength
// independent; textures.hpp:93-138). scale: the cell or feature size; param: the snow line or the
// turbulence.
__device__ inline V3<double> textureWeights(int kind, double scale, double param, const V3<double>& p,
                                            const V3<double>& n) {
    constexpr double relTol = 1e-9;
    switch (kind) {
        case OWEC_TEXTURE_CHECKER: {
            const V3<double> q = p / scale;
            const int s = int(floor(q.x + relTol)) + int(floor(q.y + relTol)) + int(floor(q.z + relTol));
            return (s & 1) ? V3<double>(0, 1, 0) : V3<double>(1, 0, 0);
        }
        case OWEC_TEXTURE_NOISE: {
            const double t = saturate01((fbm3(p / scale, 6) - 0.25) * 2);
            return V3<double>(1 - t, t, 0);
        }
        case OWEC_TEXTURE_RINGS: {
            const double r = sqrt(p.x * p.x + p.z * p.z) / scale + param * fbm3(p / scale, 4);
            double t = 0.5 + 0.5 * sin(2 * kPi * r);
            t = t * t;
            return V3<double>(1 - t, t, 0);
        }
        case OWEC_TEXTURE_BANDS: {
            const double z = p.z / scale + param * (fbm3(V3<double>(p.x, p.y, p.z * 4) / scale, 5) - 0.5);
            const double t = 0.5 + 0.5 * sin(2 * kPi * z) * (0.6 + 0.4 * sin(2 * kPi * z * 0.37 + 1.3));
            const double mix = saturate01(fbm3(V3<double>(0, 0, z * 3.1), 3) * 1.4 - 0.2);
            return V3<double>((1 - t) * (1 - 0.35 * mix), t * (1 - 0.35 * mix), 0.35 * mix);
        }
        case OWEC_TEXTURE_RADIAL: {
            const double r = sqrt(p.x * p.x + p.y * p.y) / scale;
            const double t = saturate01(fbm3(V3<double>(r * 3, 0.5, 0.5), 6) * 1.6 - 0.3);
            return V3<double>(1 - t, t, 0);
        }
        case OWEC_TEXTURE_MARBLE: {
            const V3<double> q = p / scale;
            const double v = fabs(sin(q.x * 0.9 + q.y * 0.5 + q.z * 0.3 + param * 6 * fbm3(q * 0.7, 6)));
            const double t = pow(1 - v, 6.0);  // thin dark veins
            const double base = 0.94 + 0.06 * fbm3(q * 3.0, 4);
            return V3<double>(base * (1 - t), t, 0);
        }
        case OWEC_TEXTURE_TERRAIN: {
            // grass on gentle slopes, rock on steep ones, snow above the snow line
            const double jitter = fbm3(p / scale, 5) - 0.5;
            const double slope = 1 - fabs(n.z);
            const double rock = saturate01((slope + 0.3 * jitter - 0.25) * 6);
            double snow = 0;
            if (param > 0) snow = saturate01((p.z - param + 40 * jitter) / 30) * saturate01(1 - slope * 1.6);
            return V3<double>((1 - rock) * (1 - snow), rock * (1 - snow), snow);
        }
        default: return V3<double>(1, 0, 0);
    }
}

}  // namespace owec
