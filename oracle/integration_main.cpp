// Drop-in check (test infrastructure): the reference engine, compiled from its own sources, renders
// through the `cuda` backend adapter (optical-pathtracer_b200/owe_adapter/cuda_backend.cpp) exactly
// as its front ends would after the registry lists it, and the result is compared with the
// reference's own `cpu` backend on scenes built with the reference's builders.
//
// Prints one line per check and exits non-zero on the first failure. Built by oracle/Makefile into
// oracle/_ref/owe_cuda_integration; run by tests/test_gpu_integration.py on a GPU machine.
#include <cmath>
#include <cstdio>
#include <memory>
#include <string>

#include "owe/backends/cpu/cpu_backend.hpp"
#include "owe/backends/compare.hpp"
#include "owe/scene/builders.hpp"

namespace owe {
const Backend& cudaBackend();
}

using namespace owe;

namespace {

int failures = 0;

void check(bool ok, const char* what, double got, double expected) {
    std::printf("%s %s: %.6g (expected %.6g)\n", ok ? "ok  " : "FAIL", what, got, expected);
    if (!ok) ++failures;
}

Image render(const Backend& b, const Scene& sc, int spp, uint64_t seed, const char* integrator = "path") {
    RenderSettings rs;
    rs.backend = b.name();
    rs.seed = seed;
    rs.spp = spp;
    rs.integrator = integrator;
    auto r = b.createRenderer(sc, 0, rs);
    r->runPass(spp);
    std::printf("     %s: %lld spp in %.3f s, %llu paths, %llu leaks\n", r->backend().c_str(), r->samplesPerPixel(),
                r->seconds(), (unsigned long long)r->stats().paths, (unsigned long long)r->stats().leaks);
    return r->resolve();
}

// tests/test_backends.cpp:349-378 and :540-574: a closed diffuse sphere emitting Le = 1 inward,
// L = 1 / (1 - rho), with the path integrator and with the light integrator (particles).
void whiteFurnace(double rho, const char* integrator) {
    Scene sc;
    SurfaceOptics o;
    o.type = SurfaceType::Diffuse;
    o.reflectance = Spectrum::constant(rho);
    const uint32_t optics = sc.world.addOptics(o);
    Emission e;
    e.radiance = Spectrum::constant(1.0);
    e.front = false;
    e.back = true;
    const int emission = sc.world.addEmission(e);
    const int b = sc.world.addBody("shell", "sphere", -1, Transform{});
    const uint32_t inside = sc.world.addRegion("shell.inside", sc.world.medium("air"), b);
    sc.world.addBoundary(b, "surface", std::make_shared<SphereShape>(1.0), Transform{}, kOutside, inside, optics, emission);
    auto obs = std::make_unique<IdealObserver>();
    obs->width = obs->height = 16;
    obs->position = {0.2, 0.1, -0.3};
    obs->lookAt = {1, 0.3, 0};
    obs->fovY = radians(70);
    sc.detectors.push_back(std::move(obs));
    sc.build();
    const bool light = std::string(integrator) == "light";
    const double y = render(cudaBackend(), sc, light ? 4096 : 1024, 1, integrator).meanY();
    check(std::fabs(y - 1 / (1 - rho)) < (light ? 0.02 : 0.01) / (1 - rho),
          light ? "white furnace, light integrator" : "white furnace", y, 1 / (1 - rho));
}

// A glass ball over a floor under the sun, through compareRenderers (compare.cpp:66-119).
void agreesWithReference() {
    Scene sc;
    sc.world.env.hasSun = true;
    sc.world.env.sunDir = normalize(Vec3(0.3, -0.5, 0.8));
    sc.world.env.sunRadiance = Spectrum::constant(2e4);
    sc.world.env.skyModel = Environment::Sky::Uniform;
    sc.world.env.zenith = Spectrum::constant(0.3);
    SurfaceOptics floor;
    floor.type = SurfaceType::Diffuse;
    floor.reflectance = Spectrum::constant(0.7);
    buildSheet(sc.world, "floor", 4, 4, sc.world.addOptics(floor), -1, -1, Transform{}, true);
    BodyMaterial glass;
    glass.transparent = true;
    glass.medium = "N-BK7";
    glass.optics = sc.world.dielectricOptics();
    buildSphere(sc.world, "ball", 0.4, glass, -1, Transform::translate({0, 0, 0.4}));
    auto eye = std::make_unique<IdealObserver>();
    eye->position = {0, -2.5, 1.2};
    eye->lookAt = {0, 0, 0.3};
    eye->fovY = radians(40);
    eye->width = 36;
    eye->height = 24;
    sc.detectors.push_back(std::move(eye));
    sc.build();
    RenderSettings a, b;
    a.backend = "cpu";
    b.backend = "cuda";
    // compareRenderers goes through the registry; run its statistics on the two backends directly
    const int runs = 8, spp = 128;
    std::vector<Image> ra, rb;
    for (int k = 0; k < runs; ++k) {
        ra.push_back(render(cpuBackend(), sc, spp, 1000 + uint64_t(k)));
        rb.push_back(render(cudaBackend(), sc, spp, 2000 + uint64_t(k)));
    }
    double ma = 0, mb = 0, va = 0, vb = 0;
    for (int k = 0; k < runs; ++k) { ma += ra[size_t(k)].meanY() / runs; mb += rb[size_t(k)].meanY() / runs; }
    for (int k = 0; k < runs; ++k) {
        va += sqr(ra[size_t(k)].meanY() - ma) / (runs - 1);
        vb += sqr(rb[size_t(k)].meanY() - mb) / (runs - 1);
    }
    const double z = (mb - ma) / std::sqrt(va / runs + vb / runs);
    check(std::fabs(z) < 4, "glass ball image mean, z against the cpu backend", z, 0);
}

}  // namespace

int main() {
    std::string why;
    if (!cudaBackend().available(&why)) {
        std::printf("FAIL cuda backend unavailable: %s\n", why.c_str());
        return 2;
    }
    std::printf("cuda backend: %s\n", cudaBackend().summary().c_str());
    for (double rho : {0.0, 0.5, 0.8}) whiteFurnace(rho, "path");
    for (double rho : {0.0, 0.5}) whiteFurnace(rho, "light");
    agreesWithReference();
    return failures ? 1 : 0;
}
