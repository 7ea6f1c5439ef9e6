// Scene suite (test infrastructure): every scene file given on the command line, loaded by the
// reference engine's own loader (src/owe/loader/scene_loader.hpp, built from its sources), rendered
// on its `cpu` backend and on the `cuda` backend (the registry with cudaBackend() added, as in the
// conformance build), and compared by the reference's own statistics (compareRenderers,
// src/owe/backends/compare.cpp) at a reduced film size. The scenes are the reference's `scenes/`
// and `benchmarks/` (the `owe bench` suites, benchmarks/suites.json).
//
// One line per scene and detector:
//   LOAD-FAILED <file>: <why>            the reference itself cannot load it here (missing assets)
//   REFUSED <file> <detector>: <why>     the cuda backend refuses a feature of the scene
//   ok|FAIL <file> <detector>: <report>  the comparison (consistent() of ComparisonReport)
// Exits 1 when any comparison fails, 0 otherwise.
//
// With --same-streams N, each scene and detector is rendered instead on both backends from the same
// seed, N one-sample passes, and the pixels whose images differ beyond 1e-4 relative are listed
// (one-sample paths that make different decisions): for locating a difference the statistics find.
//
// --pixel-sigma S sets every detector's pixel filter width, --pinhole closes every observer's pupil:
// for telling which part of the camera a same-streams difference comes from; --dump PREFIX writes the
// two images of each same-streams comparison (width, height as ints, then XYZ doubles).
//
// Usage: owe_scene_suite [--width W] [--spp S] [--runs R] [--all-detectors] [--same-streams N]
//                        [--pixel-sigma S] [--pinhole] FILE...
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>
#include <vector>

#include "owe/backends/compare.hpp"
#include "owe/backends/registry.hpp"
#include "owe/loader/scene_loader.hpp"
#include "owe/scene/detector.hpp"

using namespace owe;

namespace {

Image renderOn(const std::string& name, const Scene& sc, int di, RenderSettings rs, int passes) {
    rs.backend = name;
    auto r = backend(name).createRenderer(sc, di, rs);
    for (int k = 0; k < passes; ++k) r->runPass(1);
    return r->resolve();
}

std::string dumpPrefix;  // --dump PREFIX: the two images of a same-streams comparison, raw XYZ doubles

void dump(const std::string& path, const Image& im) {
    if (FILE* f = std::fopen(path.c_str(), "wb")) {
        const int wh[2] = {im.width, im.height};
        std::fwrite(wh, sizeof(int), 2, f);
        std::fwrite(im.xyz.data(), sizeof(double), im.xyz.size(), f);
        std::fclose(f);
    }
}

void sameStreams(const std::string& file, const Scene& sc, int di, const RenderSettings& rs, int passes) {
    const Image a = renderOn("cpu", sc, di, rs, passes), b = renderOn("cuda", sc, di, rs, passes);
    if (!dumpPrefix.empty()) {
        std::string name = file;
        for (char& ch : name)
            if (ch == '/' || ch == '.') ch = '_';
        dump(dumpPrefix + name + "_" + std::to_string(di) + "_cpu.bin", a);
        dump(dumpPrefix + name + "_" + std::to_string(di) + "_cuda.bin", b);
    }
    int differ = 0, listed = 0;
    int hist[7] = {0, 0, 0, 0, 0, 0, 0};  // |relative difference| < 1e-6, 1e-5, ..., 1e-1, >= 1e-1
    const int n = a.width * a.height;
    for (int i = 0; i < n; ++i) {
        const double ya = a.xyz[3 * size_t(i) + 1], yb = b.xyz[3 * size_t(i) + 1];
        const double rel = std::fabs(ya - yb) / std::max(std::max(std::fabs(ya), std::fabs(yb)), 1e-30);
        int bin = 0;
        for (double lim = 1e-6; bin < 6 && rel >= lim; lim *= 10) ++bin;
        ++hist[bin];
        if (std::fabs(ya - yb) <= 1e-4 * std::max(std::fabs(ya), 1e-3)) continue;
        ++differ;
        if (listed++ < 12) std::printf("  pixel (%d, %d): cpu %.6g cuda %.6g\n", i % a.width, i / a.width, ya, yb);
    }
    std::printf("SAME-STREAMS %s %s: %d passes, %d of %d pixels differ, mean Y cpu %.6g cuda %.6g; relative "
                "differences <1e-6 %d, <1e-5 %d, <1e-4 %d, <1e-3 %d, <1e-2 %d, <1e-1 %d, larger %d\n",
                file.c_str(), sc.detectors[size_t(di)]->name.c_str(), passes, differ, n, a.meanY(), b.meanY(), hist[0],
                hist[1], hist[2], hist[3], hist[4], hist[5], hist[6]);
}

}  // namespace

int main(int argc, char** argv) {
    int width = 64, spp = 8, runs = 6;
    bool allDetectors = false;
    int sameStreamPasses = 0;
    double pixelSigma = -1;
    bool pinhole = false;
    std::vector<std::string> files;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--width" && i + 1 < argc) width = std::atoi(argv[++i]);
        else if (a == "--spp" && i + 1 < argc) spp = std::atoi(argv[++i]);
        else if (a == "--runs" && i + 1 < argc) runs = std::atoi(argv[++i]);
        else if (a == "--all-detectors") allDetectors = true;
        else if (a == "--same-streams" && i + 1 < argc) sameStreamPasses = std::atoi(argv[++i]);
        else if (a == "--pixel-sigma" && i + 1 < argc) pixelSigma = std::atof(argv[++i]);
        else if (a == "--pinhole") pinhole = true;
        else if (a == "--dump" && i + 1 < argc) dumpPrefix = argv[++i];
        else files.push_back(a);
    }
    int failures = 0;
    for (const std::string& file : files) {
        Scene sc;
        try {
            sc = loadScene(file);
        } catch (const std::exception& e) {
            std::printf("LOAD-FAILED %s: %s\n", file.c_str(), e.what());
            std::fflush(stdout);
            continue;
        }
        const int nd = allDetectors ? int(sc.detectors.size()) : std::min<int>(1, int(sc.detectors.size()));
        if (nd == 0) {
            std::printf("LOAD-FAILED %s: no detector\n", file.c_str());
            continue;
        }
        for (int di = 0; di < nd; ++di) {
            Detector& det = *sc.detectors[size_t(di)];
            // the same measurement on a coarser film: the detector's aspect kept
            if (pixelSigma >= 0) det.pixelSigma = pixelSigma;
            if (auto* eye = dynamic_cast<IdealObserver*>(&det); eye && pinhole) eye->pupilRadius = 0;
            const int w0 = det.width, h0 = det.height;
            det.width = std::min(width, w0);
            det.height = std::max(1, int(std::lround(double(h0) * det.width / std::max(1, w0))));
            // the detector's derived quantities (an observer's field of view across, its frame) follow
            // the new film, as when the scene was built
            det.prepare(sc.world);
            RenderSettings a = sc.settingsFor(di), b = a;
            a.backend = "cpu";
            b.backend = "cuda";
            adaptToBackend(a);
            adaptToBackend(b);
            b.integrator = a.integrator;  // the one both implement: the comparison is like for like
            if (sameStreamPasses > 0) {
                try {
                    sameStreams(file, sc, di, a, sameStreamPasses);
                } catch (const std::exception& e) {
                    std::printf("REFUSED %s %s: %s\n", file.c_str(), det.name.c_str(), e.what());
                }
                std::fflush(stdout);
                continue;
            }
            try {
                const ComparisonReport r = compareRenderers(sc, di, a, b, spp, runs, 4);
                const bool ok = r.consistent();
                if (!ok) ++failures;
                std::printf("%s %s %s (%dx%d, %s): zImage %.2f, blocks over 4 sigma %d of %d, chi2/test %.2f, "
                            "mean Y cpu %.6g cuda %.6g, %.2f s / %.2f s\n",
                            ok ? "ok  " : "FAIL", file.c_str(), det.name.c_str(), det.width, det.height,
                            a.integrator.c_str(), r.zImage, r.over4, r.tests, r.chi2PerTest, r.meanA, r.meanB,
                            r.secondsA, r.secondsB);
            } catch (const std::exception& e) {
                std::printf("REFUSED %s %s: %s\n", file.c_str(), det.name.c_str(), e.what());
            }
            std::fflush(stdout);
        }
    }
    return failures ? 1 : 0;
}
