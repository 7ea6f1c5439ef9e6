// The scene as the kernels see it: flat arrays in HBM, camera-relative. Positions are stored
// relative to `origin` (the detector's position), so FP32 keeps its precision where the detector
// looks; shape frames stay FP64 for root refinement.
#pragma once

#include "common.cuh"
#include "owec.h"

namespace owec {

// A primitive in BVH leaf order: a triangle (three camera-relative float vertices) or an analytic
// boundary. a.w = boundary (bit pattern), b.w = triangle index within its mesh, c.w = kind.
struct alignas(16) PrimRec {
    float ax, ay, az, aw;
    float bx, by, bz, bw;
    float cx, cy, cz, cw;
};
constexpr uint32_t kPrimTriangle = 0u, kPrimAnalytic = 1u;

// The same triangle in FP64 for the all-FP64 instantiation (leaf order).
struct alignas(16) PrimRec64 {
    double v0[3], v1[3], v2[3];
    uint32_t boundary, prim;
    uint32_t kind, pad;
};

// One boundary with its frame relative to the camera origin.
struct DBoundary {
    int32_t shape;
    int32_t emission;
    uint32_t front, back;
    uint32_t optics;
    int32_t light;        // index in the light table, -1 when next-event estimation never samples it
    Xform toWorld;        // shape -> camera-relative world
    Xform toLocal;
    double params[4];
    double area;          // emitter area (planes, spheres, flat sags, cylinders)
    double scale;         // size of the frame (error model of anchors)
    // what the numeric crossings need beyond params: an asphere's z slab (zMin, zMax); a torus
    // patch's rMax, zMin, zMax and its arc's end a1
    double ext[4];
    uint32_t dataOffset;  // the shape's data in DeviceScene::shapeData (asphere terms, openings, ...)
    uint32_t dataCount;
};

struct DLight {
    int32_t kind;         // 0 boundary, 1 sun
    uint32_t boundary;
    double pdf;           // selection probability
    double cdf;           // running sum (the last one is 1)
};
constexpr int32_t kLightBoundary = 0, kLightSun = 1;

struct DDetector {
    int32_t kind;
    int32_t width, height;
    uint32_t region;
    double pos[3];        // camera-relative (zero for an observer)
    double fwd[3], right[3], up[3];
    double tanX, tanY;
    double sigma;
    uint32_t boundary;    // sensor
    double halfX, halfY;
    double normal[3];
    // observer: thin lens (pupil 0: a pinhole; focus INFINITY: at infinity) and its pupil guide
    double pupil, focus;
    double guideC[3];     // camera-relative
    double guideR, guideShare;
    // sensor: readout flips and the aimed direction mixture (aimR 0: hemispherical)
    int32_t flipX, flipY;
    double aimC[3], aimN[3];  // camera-relative centre, unit normal
    double aimR, aimShare;
    double focusC[3];
    double focusR, focusShare;
};

// An 8-wide BVH node with children quantised to 8 bits against the node's box (80 bytes, five
// 16-byte loads). Slot i of an inner child has meta[i] = 8 | k and points to node child_base + k;
// slot i of a leaf holds meta[i] >> 5 primitives (1..3) from prim_base + (meta[i] & 31). Empty slots
// have meta 0.
struct alignas(16) WideNode {
    float ox, oy, oz;
    uint8_t ex, ey, ez, imask;
    uint32_t child_base;
    uint32_t prim_base;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(WideNode) == 80, "wide node must stay 80 bytes");

struct DeviceScene {
    // This description's own copy in device memory: the out-of-line traversal functions read the
    // scene through it, so that a kernel need not copy its by-value scene parameter to local memory
    // to pass its address.
    const DeviceScene* self;
    const owec_spectrum* spectra;
    const double* table;
    const owec_medium* media;
    const uint32_t* regionMedium;
    const owec_optics* optics;
    const owec_emission* emissions;
    const DBoundary* boundaries;
    const DLight* lights;
    const double* shapeData;  // the shapes' data, addressed by DBoundary::dataOffset
    int32_t simpleOptics;     // 1: every boundary Lambertian, absorbing or detecting, no null boundary,
                              // no region's medium absorbs or scatters (the particles' lean event kernel)
    int32_t fullFeatures;     // 1: shapes beyond spheres, conic sags, plain apertures and cylinders, a
                              // planet-sized sphere, contacts or textured materials (the kernels' Full
                              // instantiations)
    uint32_t nRegions, nBoundaries, nLights, nMedia;
    const WideNode* nodes;
    const PrimRec* prims;
    const PrimRec64* prims64;
    uint32_t nNodes, nPrims;
    // environment
    int32_t skyModel, skySpectrum;      // skySpectrum: the uniform sky, or the gradient's zenith
    int32_t skyHorizon, skyGround;      // the gradient's horizon and ground spectra
    double skyUp[3];
    int32_t hasSun, sunSpectrum;
    double sunDir[3];
    double sunCosMax, sunSolidAngle;
    double sunSelectPdf;  // the sun's light-selection probability (0 without a sun)
    double sceneRadius;
    double sceneCenter[3];  // camera-relative
    double origin[3];       // world position of the camera-relative origin
    DDetector det;
    double cieYIntegral;
    double contactScale;    // size of the scene (anchor error model)
    // When set: [0] closest-hit queries, [1] wide nodes visited, [2] primitives tested, [3] shadow
    // queries, [4] their nodes, [5] their primitives (the algorithmic traffic of a pass).
    unsigned long long* travCounters;
    // When set (owec_inconsistency_log): the contact-resolving surface kernel records up to
    // eventLogCap crossings that met a region other than the ray's, kEventRecord doubles each.
    double* eventLog;
    uint32_t* eventLogCount;
    uint32_t eventLogCap;
};
constexpr int kEventRecord = 16;

}  // namespace owec
