// Closest-hit and any-hit traversal of the 8-wide quantised BVH.
//
// One thread follows one ray. Node records (80 B) are read with five 128-bit read-only loads; the
// eight child boxes are decoded from 8-bit offsets against the node's origin and power-of-two
// scales and slab-tested together. The hits are not sorted: the builder placed each child in the
// slot of the octant it lies towards, so visiting the hit slots in the order slot ^ (ray octant
// ^ 7) meets them roughly near to far (Ylitie, Karras and Laine, HPG 2017). A visited node leaves
// two groups behind: its hit leaf primitives (a 24-bit mask over the node's primitive range),
// tested first, and its hit inner children (an 8-bit mask in visiting order), of which one is
// entered and the rest go on the stack as one 8-byte entry. The stack therefore grows by at most
// one entry per level. Crossings beyond the closest found so far are cut by the box tests, as
// the reference's Bvh::traverseSlots cuts them (src/owe/scene/bvh.hpp:39-78).
//
// Which crossings count near a ray's departure follows the reference's contact rule
// (src/owe/scene/world.cpp:451-513): the face the ray left never does, and within the anchor's
// error only a crossing met from the ray's own region does.
#pragma once

#include "shapes.cuh"

namespace owec {

constexpr int kStackDepth = 32;      // group entries per thread in shared memory: one per level
constexpr int kDeepStackDepth = 96;  // the rare query of a deeper tree is traversed again with a stack
                                     // of this depth in local memory; beyond it the query ends and is
                                     // counted as a fault
constexpr uint32_t kMaxTraversalSteps = 1u << 20;  // a bound on visits: a malformed tree cannot hang

// A deferred node group: the inner children of one node still to be visited.
struct StackEntry {
    uint32_t base;  // node index of the node's first inner child (child_base)
    uint32_t bits;  // bits 0-7: hit children left, by visiting position; bits 8-15: the node's inner-slot mask
};

// The short traversal stack: this thread's column of the block's shared-memory stack (stride =
// block size), so that a warp's entries of one level are consecutive words.
struct SharedStack {
    static constexpr int kDepth = kStackDepth;
    StackEntry* sh;
    int stride;
    __device__ __forceinline__ void init(StackEntry* stack, int s) { sh = stack; stride = s; }
    __device__ __forceinline__ StackEntry get(int i) const { return sh[i * stride]; }
    __device__ __forceinline__ void set(int i, const StackEntry& e) { sh[i * stride] = e; }
};
// The deep stack, in local memory, for the queries that overflow the short one.
struct LocalStack {
    static constexpr int kDepth = kDeepStackDepth;
    StackEntry e[kDeepStackDepth];
    __device__ __forceinline__ void init(StackEntry*, int) {}
    __device__ __forceinline__ StackEntry get(int i) const { return e[i]; }
    __device__ __forceinline__ void set(int i, const StackEntry& x) { e[i] = x; }
};

template <class T>
struct RayQuery {
    V3<T> o, d;           // camera-relative
    V3<double> od;        // the origin in FP64 (analytic shapes are refined there)
    T tmax;
    uint32_t depB, depP;  // the boundary and primitive the ray left (kNone: none)
    uint32_t region;      // the region it travels in (kNone: no region test)
    T errN;               // the anchor's error normal to a surface
};

struct HitRec {
    double t;
    uint32_t boundary;
    uint32_t prim;        // triangle index within its mesh; 0 for analytic shapes
    uint32_t slot;        // leaf-order primitive slot
    uint32_t flags;       // kHitFront, kHitAmbiguous (kept by the contact-resolving traversal only)
};
// The crossing was met from its boundary's front side; it tied with another boundary's crossing that
// the ray's region matches as well, which leaves their order undecided (NearestCrossing::offer,
// src/owe/scene/world.cpp:515-550): the reference ends such a path.
constexpr uint32_t kHitFront = 1u, kHitAmbiguous = 2u;
// Crossings of two boundaries closer than this relative distance are the same contact: coincident
// faces' FP32 distances, computed from different vertices, differ by a few ulps of the coordinates.
// The contact-resolving traversal culls nodes with the closest distance widened by it.
template <class T> __device__ __forceinline__ T tieWindow();
template <> __device__ __forceinline__ float tieWindow<float>() { return 4e-6f; }
template <> __device__ __forceinline__ double tieWindow<double>() { return 3e-16; }
// How far behind its origin a crossing of another boundary through the anchor may fall by the
// rounding of the origin and of its distance: a few ulps of the origin's magnitude. (The reference
// searches from minus the anchor's error for every boundary but a departed mesh, world.cpp:473-476.)
template <class T>
__device__ __forceinline__ T behindWindow(const V3<T>& o) {
    return T(sizeof(T) == 4 ? 5e-7 : 1e-15) * fmax(fmax(fabs(o.x), fabs(o.y)), fmax(fabs(o.z), T(1e-3)));
}

// The acceptance rule of a candidate crossing at distance t with (unnormalised) normal n. Near the
// anchor a departed analytic boundary is excluded, and a crossing counts only if it is met from the
// ray's region. Of a departed mesh only the departed triangle is excluded (World::intersect's mesh
// departure, src/owe/scene/world.cpp:463-471, and MeshShape::intersect's same-face test,
// src/owe/scene/mesh.cpp:85): another of its triangles near the anchor counts when it is met from
// the ray's region (the neighbour across a concave edge, which excluded let the ray into the body)
// and not otherwise (a coplanar neighbour, met from behind: the root excludedRoot skips,
// world.cpp:497-503); the far face of a plate thinner than the anchor's error is met the same way.
template <class T>
__device__ __forceinline__ bool acceptCrossing(const DeviceScene& sc, const RayQuery<T>& q, uint32_t b, uint32_t prim, bool mesh, T t,
                            const V3<T>& n) {
    if (mesh && b == q.depB && prim == q.depP) return false;
    const T dn = dot(q.d, n);
    const T nl = sqrt(dot(n, n));
    const bool near = fabs(t * dn) <= q.errN * nl;
    if (!near) return true;
    if (b == q.depB && !mesh) return false;
    if (q.region == kNone) return true;
    const DBoundary& bd = sc.boundaries[b];
    const uint32_t incident = dn < T(0) ? bd.front : bd.back;
    return incident == q.region;
}

// Relative widening of far planes against the rounding of the slab distances (a few ulps).
template <class T> __device__ __forceinline__ T farWiden();
template <> __device__ __forceinline__ float farWiden<float>() { return 4e-7f; }
template <> __device__ __forceinline__ double farWiden<double>() { return 4e-16; }

// The analytic boundary b's first acceptable crossing in (0, best); FP64 refinement when Rr = double.
template <class R, class Rr, class T, bool Full>
__device__ __forceinline__ bool analyticCandidate(const DeviceScene& sc, const RayQuery<T>& q, uint32_t b, T best, Rr& tOut,
                                                  bool& frontOut, float& cosOut) {
    const DBoundary& bd = sc.boundaries[b];
    const V3<Rr> lo = bd.toLocal.point(V3<Rr>(q.od));
    const V3<Rr> ld = bd.toLocal.vector(V3<Rr>(q.d));
    // Leaving this boundary, the anchor lies on it to the precision of the refinement, not of FP32:
    // with the FP32 window a grazing ray's far crossing of the same sphere (at t = 2 R cos) fell
    // inside it and was rejected as the departure, and the path leaked.
    RayQuery<T> qs = q;
    if (b == q.depB && sizeof(Rr) > sizeof(R)) qs.errN = q.errN * T(2.5e-7);
    AHits<Rr> hits;
    int n;
    // contacts: another surface through the anchor may lie just behind it (world.cpp:473-476); such
    // roots must lie within the rounding of the origin along the surface normal (checked below)
    const Rr tLow = Full ? -Rr(64) * Rr(q.errN) : Rr(0);
    bool solved = false;
    if constexpr (Full && sizeof(Rr) == sizeof(double)) {
        // a ray near a planet-sized sphere: the double-double solve
        if (nearSphere(bd, q.od)) {
            hits = nearSphereCrossings(bd, q.od, V3<double>(q.d), tLow, double(best));
            n = hits.n;
            solved = true;
        }
    }
    if (solved) {
    } else if constexpr (Full)
        n = analyticCrossings<R, Rr, true>(bd, sc.shapeData + bd.dataOffset, lo, ld, tLow, Rr(best), b == q.depB, hits,
                                           Rr(qs.errN), Rr(q.errN));
    else n = analyticCrossings<R, Rr, false>(bd, nullptr, lo, ld, Rr(0), Rr(best), false, hits);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        if (i >= n) break;
        const AHit<Rr>& h = hits.get(i);
        const V3<T> nw = V3<T>(bd.toWorld.vector(h.n));
        if (Full && !(h.t > Rr(0)) && (b == q.depB || !(fabs(T(h.t) * dot(q.d, nw)) <= behindWindow(q.o)))) continue;
        if (!acceptCrossing<T>(sc, qs, b, 0u, false, T(h.t), nw)) continue;
        tOut = h.t;
        frontOut = dot(q.d, nw) < T(0);
        cosOut = float(fabs(dot(q.d, nw)));
        return true;
    }
    return false;
}

// analyticCandidate out of line: the FP64 refinement of every analytic shape needs many registers,
// and inlined it would set the register count of the whole traversal loop. Arguments and result go
// by value, so that nothing of the caller's has to live in memory for the call.
template <class Rr>
struct AnalyticResult {
    Rr t;
    bool ok;
    bool front;  // met from the boundary's front side
    float cosAbs;  // |cos| between the ray and the surface normal there
};
template <class T, class R, class Rr, bool Full>
__device__ __noinline__ AnalyticResult<Rr> analyticHit(const DeviceScene* scp, uint32_t b, V3<double> od, V3<T> d, T best,
                                                        uint32_t depB, uint32_t region, T errN) {
    RayQuery<T> q;
    q.od = od;
    q.o = V3<T>(od);
    q.d = d;
    q.tmax = best;
    q.depB = depB;
    q.depP = kNone;
    q.region = region;
    q.errN = errN;
    AnalyticResult<Rr> r;
    r.t = Rr(0);
    r.front = false;
    r.cosAbs = 1.f;
    r.ok = analyticCandidate<R, Rr, T, Full>(*scp, q, b, best, r.t, r.front, r.cosAbs);
    return r;
}

// A wide node as the five 128-bit words it is loaded in (the WideNode layout of device_scene.cuh):
//   a = (ox, oy, oz, ex | ey << 8 | ez << 16 | imask << 24)
//   b = (child_base, prim_base, meta[0..3], meta[4..7])
//   c = (qlox[0..3], qlox[4..7], qloy[0..3], qloy[4..7])
//   d = (qloz[0..3], qloz[4..7], qhix[0..3], qhix[4..7])
//   e = (qhiy[0..3], qhiy[4..7], qhiz[0..3], qhiz[4..7])
struct NodeWords {
    uint4 a, b, c, d, e;
};

// Read-only 16-byte load of a BVH word with the L2 eviction priority evict-last (a createpolicy cache
// hint): every traversal rereads the nodes and primitives, while the path state that streams past
// them is evict-first.
#ifndef OWEC_BVH_KEEP
#define OWEC_BVH_KEEP 1
#endif
__device__ __forceinline__ uint4 ldgKeep(const uint4* p) {
#if defined(__CUDA_ARCH__) && OWEC_BVH_KEEP
    uint64_t policy;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(policy));
    uint4 v;
    asm("ld.global.nc.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(policy));
    return v;
#elif defined(__CUDA_ARCH__)
    return __ldg(p);
#else
    return *p;
#endif
}

__device__ __forceinline__ void loadNode(const WideNode* nodes, uint32_t i, NodeWords& nd) {
#if defined(__CUDA_ARCH__)
    const uint4* src = reinterpret_cast<const uint4*>(nodes + i);
    nd.a = ldgKeep(src + 0);
    nd.b = ldgKeep(src + 1);
    nd.c = ldgKeep(src + 2);
    nd.d = ldgKeep(src + 3);
    nd.e = ldgKeep(src + 4);
#else
    const uint4* src = reinterpret_cast<const uint4*>(nodes + i);
    nd.a = src[0]; nd.b = src[1]; nd.c = src[2]; nd.d = src[3]; nd.e = src[4];
#endif
}


// Decoded child boxes of a node, slab-tested against the ray. Returns the hit mask (slot order).
template <class T>
__device__ __forceinline__ uint32_t intersectChildren(const NodeWords& nd, const V3<T>& inv, const V3<T>& oinv, T tmin, T tmax) {
    const T sx = T(__uint_as_float((nd.a.w & 0xFFu) << 23));
    const T sy = T(__uint_as_float(((nd.a.w >> 8) & 0xFFu) << 23));
    const T sz = T(__uint_as_float(((nd.a.w >> 16) & 0xFFu) << 23));
    // t = (origin + q * s - o) * inv = q * (s * inv) + (origin * inv - o * inv). A plane byte q enters
    // as the float f = 2^23 + 256 q (one byte permute places it in the second mantissa byte), so
    // t = f * (a / 256) + (b - 2^15 a) with a = s * inv: one FMA per plane and no conversion. a / 256
    // and 2^15 a are exact; the one rounding of b - 2^15 a is below 2^-9 a + half an ulp of b, taken
    // off the near planes and added to the far ones (with their widening against the FMA's own
    // rounding), so the boxes stay conservative and grow by well under a percent of a quantum.
    const T ax = sx * inv.x, ay = sy * inv.y, az = sz * inv.z;
    const T ax8 = ax * T(0.00390625), ay8 = ay * T(0.00390625), az8 = az * T(0.00390625);
    const T b0x = T(__uint_as_float(nd.a.x)) * inv.x - oinv.x;
    const T b0y = T(__uint_as_float(nd.a.y)) * inv.y - oinv.y;
    const T b0z = T(__uint_as_float(nd.a.z)) * inv.z - oinv.z;
    const T bx = b0x - T(32768) * ax, by = b0y - T(32768) * ay, bz = b0z - T(32768) * az;
    const T mx = T(0.00390625) * fabs(ax) + T(2.4e-7) * fabs(bx);
    const T my = T(0.00390625) * fabs(ay) + T(2.4e-7) * fabs(by);
    const T mz = T(0.00390625) * fabs(az) + T(2.4e-7) * fabs(bz);
    const T nbx = bx - mx, nby = by - my, nbz = bz - mz;
    const T fbx = bx + mx + (fabs(b0x) + T(255) * fabs(ax)) * farWiden<T>();
    const T fby = by + my + (fabs(b0y) + T(255) * fabs(ay)) * farWiden<T>();
    const T fbz = bz + mz + (fabs(b0z) + T(255) * fabs(az)) * farWiden<T>();
    const bool nx = inv.x < T(0), ny = inv.y < T(0), nz = inv.z < T(0);
    // near and far planes per axis, chosen by the ray's direction on whole words
    const uint32_t nxl0 = nx ? nd.d.z : nd.c.x, nxl1 = nx ? nd.d.w : nd.c.y;
    const uint32_t fxl0 = nx ? nd.c.x : nd.d.z, fxl1 = nx ? nd.c.y : nd.d.w;
    const uint32_t nyl0 = ny ? nd.e.x : nd.c.z, nyl1 = ny ? nd.e.y : nd.c.w;
    const uint32_t fyl0 = ny ? nd.c.z : nd.e.x, fyl1 = ny ? nd.c.w : nd.e.y;
    const uint32_t nzl0 = nz ? nd.e.z : nd.d.x, nzl1 = nz ? nd.e.w : nd.d.y;
    const uint32_t fzl0 = nz ? nd.d.x : nd.e.z, fzl1 = nz ? nd.d.y : nd.e.w;
    uint32_t mask = 0;
    // an empty slot's box is stored inverted (low planes 255, high planes 0), so it never passes
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t sel = 0x7504u | (uint32_t(i & 3) << 4);
        const T lx = T(__uint_as_float(__byte_perm(i < 4 ? nxl0 : nxl1, 0x4B000000u, sel)));
        const T hx = T(__uint_as_float(__byte_perm(i < 4 ? fxl0 : fxl1, 0x4B000000u, sel)));
        const T ly = T(__uint_as_float(__byte_perm(i < 4 ? nyl0 : nyl1, 0x4B000000u, sel)));
        const T hy = T(__uint_as_float(__byte_perm(i < 4 ? fyl0 : fyl1, 0x4B000000u, sel)));
        const T lz = T(__uint_as_float(__byte_perm(i < 4 ? nzl0 : nzl1, 0x4B000000u, sel)));
        const T hz = T(__uint_as_float(__byte_perm(i < 4 ? fzl0 : fzl1, 0x4B000000u, sel)));
        const T t0x = fma(lx, ax8, nbx), t1x = fma(hx, ax8, fbx);
        const T t0y = fma(ly, ay8, nby), t1y = fma(hy, ay8, fby);
        const T t0z = fma(lz, az8, nbz), t1z = fma(hz, az8, fbz);
        const T te = fmax(fmax(t0x, t0y), fmax(t0z, tmin));
        const T tx = fmin(fmin(t1x, t1y), t1z);
        const T tl = fmin(tx, tmax);
        if (te <= tl) mask |= 1u << i;
    }
    return mask;
}

__device__ __forceinline__ void loadPrim(const PrimRec* prims, uint32_t i, PrimRec& p) {
#if defined(__CUDA_ARCH__)
    const uint4* src = reinterpret_cast<const uint4*>(prims + i);
    uint4 w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) w[k] = ldgKeep(src + k);
    memcpy(&p, w, sizeof(PrimRec));
#else
    p = prims[i];
#endif
}

// Triangle of slot i in the traversal's precision.
template <class T> struct TriFetch;
template <> struct TriFetch<float> {
    __device__ __forceinline__ static void get(const DeviceScene& sc, uint32_t i, V3<float>& a, V3<float>& b, V3<float>& c, uint32_t& bnd,
                            uint32_t& prim, uint32_t& kind) {
        PrimRec p;
        loadPrim(sc.prims, i, p);
        a = {p.ax, p.ay, p.az};
        b = {p.bx, p.by, p.bz};
        c = {p.cx, p.cy, p.cz};
        bnd = __float_as_uint(p.aw);
        prim = __float_as_uint(p.bw);
        kind = __float_as_uint(p.cw);
    }
};
template <> struct TriFetch<double> {
    __device__ __forceinline__ static void get(const DeviceScene& sc, uint32_t i, V3<double>& a, V3<double>& b, V3<double>& c,
                            uint32_t& bnd, uint32_t& prim, uint32_t& kind) {
        const PrimRec64& p = sc.prims64[i];
        a = {p.v0[0], p.v0[1], p.v0[2]};
        b = {p.v1[0], p.v1[1], p.v1[2]};
        c = {p.v2[0], p.v2[1], p.v2[2]};
        bnd = p.boundary;
        prim = p.prim;
        kind = p.kind;
    }
};

enum TraceStatus : int { kTraceMiss = 0, kTraceHit = 1, kTraceOverflow = 2 };

constexpr int kTraceRunning = 3;  // Traversal::run: the query is not finished yet

// 1 / d for the slab tests, with a zero component taken as a tiny one of its sign: an infinite
// inverse makes the affine slab distances inf - inf = NaN, which the min / max ignore, and a ray
// parallel to an axis (a collimated beam, normal incidence) would then pass every box's slab on
// that axis and visit the whole tree. 1e-18 keeps every product finite in FP32.
template <class T>
__device__ __forceinline__ T safeInverse(T d) {
    return T(1) / (fabs(d) > T(1e-18) ? d : copysign(T(1e-18), d));
}

// Moves bit s of an 8-bit mask to bit s ^ x: slot order to visiting order and back.
__device__ __forceinline__ uint32_t permuteSlots(uint32_t m, uint32_t x) {
    m = (x & 1u) ? (((m & 0x55u) << 1) | ((m >> 1) & 0x55u)) : m;
    m = (x & 2u) ? (((m & 0x33u) << 2) | ((m >> 2) & 0x33u)) : m;
    m = (x & 4u) ? (((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu)) : m;
    return m;
}

// Closest (AnyHit = false) or first (AnyHit = true) acceptable crossing in (0, q.tmax), as a state
// machine that a persistent kernel can advance a few visits at a time and then hand the thread a
// new query when this one ends. R / Rr: precision of analytic roots and of their refinement.
// Count: keep the per-query visit and test counts (the counting pass; the timed kernels leave them out).
// Full: the scene has shapes beyond spheres, conic sags, plain apertures and cylinders
// (analyticCrossings).
template <class T, class R, class Rr, bool AnyHit, class Stack = SharedStack, bool Count = true, bool Full = false>
struct Traversal {
    RayQuery<T> q;
    V3<T> inv, oinv;
    ShearedRay<T> sh;
    T best;
    T bestCos;            // contact-resolving instantiation: |cos| of the closest crossing's incidence
    double bestD;         // and its distance in the refinement's precision
    HitRec hit;           // written when a crossing is accepted
    Stack st;
    uint32_t nodeBase, nodeBits;  // the current node group (as a stack entry)
    uint32_t primBase, primBits;  // the current primitive group: primBase + bit, 24 bits
    uint32_t first;               // the slot visited first: the octant opposite the ray's
    uint32_t steps, nodeVisits, primTests;
    int sp;
    bool found;

    // `stack` is this thread's column of the block's shared-memory stack (stride = block size).
    __device__ __forceinline__ void begin(const RayQuery<T>& query, StackEntry* stack, int stride) {
        q = query;
        inv = V3<T>(safeInverse(q.d.x), safeInverse(q.d.y), safeInverse(q.d.z));
        oinv = V3<T>(q.o.x * inv.x, q.o.y * inv.y, q.o.z * inv.z);
        sh = shearRay(q.d);
        best = q.tmax;
        bestCos = T(1);
        bestD = double(q.tmax);
        found = false;
        sp = 0;
        st.init(stack, stride);
        nodeVisits = primTests = 0;
        steps = 0;
        // bit k set: the ray runs towards +k, so it meets the children on the negative side first
        first = ((q.d.x < T(0)) ? 0u : 1u) | ((q.d.y < T(0)) ? 0u : 2u) | ((q.d.z < T(0)) ? 0u : 4u);
        // the root as a group of one: position 0, an inner slot of rank 0
        nodeBase = 0;
        nodeBits = 1u | (1u << (8 + first));
        primBase = 0;
        primBits = 0;
    }

    // Advances by at most `budget` node or primitive visits: kTraceRunning, or the query's TraceStatus.
    __device__ __forceinline__ int run(const DeviceScene& sc, int budget) {
        if (sc.nNodes == 0) return kTraceMiss;
        for (int it = 0; it < budget; ++it) {
            if (++steps > kMaxTraversalSteps) return kTraceOverflow;
            if (primBits) {
                const uint32_t b = uint32_t(__ffs(primBits) - 1);
                primBits &= primBits - 1u;
                if (Count) ++primTests;
                if (testPrim(sc, primBase + b) && AnyHit) return kTraceHit;
                continue;
            }
            if ((nodeBits & 0xFFu) == 0) {
                if (sp == 0) return found ? kTraceHit : kTraceMiss;
                --sp;
                const StackEntry e = st.get(sp);
                nodeBase = e.base;
                nodeBits = e.bits;
            }
            // the group's next child in visiting order; the rest of the group waits on the stack
            const uint32_t pos = uint32_t(__ffs(nodeBits & 0xFFu) - 1);
            nodeBits &= ~(1u << pos);
            const uint32_t slot = pos ^ first;
            const uint32_t node = nodeBase + uint32_t(__popc((nodeBits >> 8) & ((1u << slot) - 1u)));
            if (nodeBits & 0xFFu) {
                if (sp >= Stack::kDepth) return kTraceOverflow;
                st.set(sp, {nodeBase, nodeBits});
                ++sp;
            }
            NodeWords nd;
            loadNode(sc.nodes, node, nd);
            if (Count) ++nodeVisits;
            const uint32_t mask = intersectChildren(nd, inv, oinv, T(0), (Full && !AnyHit) ? tieLimit() : best);
            const uint32_t inner = nd.a.w >> 24;
            nodeBase = nd.b.x;
            nodeBits = permuteSlots(mask & inner, first) | (inner << 8);
            primBase = nd.b.y;
            uint32_t pb = 0;
            // the hit leaf slots' primitive ranges (meta: count << 5 | offset), one leaf at a time
            for (uint32_t leaves = mask & ~inner; leaves; leaves &= leaves - 1u) {
                const uint32_t i = uint32_t(__ffs(leaves) - 1);
                const uint32_t meta = ((i < 4 ? nd.b.z : nd.b.w) >> (8 * (i & 3))) & 0xFFu;
                pb |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);
            }
            primBits = pb;
        }
        return kTraceRunning;
    }

    // Contact decisions compare FP64 distances where the instantiation has them: the FP64 one, and
    // FP32 traversal with FP64 refinement (triangles' distances from their FP64 vertices and the FP64
    // origin, analytic roots refined in FP64). Plain FP32 compares its own distances.
    static constexpr bool kExactTies = sizeof(T) == sizeof(double) || sizeof(Rr) == sizeof(double);

    // The magnitude of the coordinates a crossing's distance is computed from (origin and hit point).
    __device__ __forceinline__ double coordScale() const {
        return fmax(fmax(fabs(q.od.x), fabs(q.od.y)), fabs(q.od.z)) + fmin(fabs(bestD), 1e30);
    }

    // The tie window of two crossings' distances: coincident faces' distances differ by the rounding
    // of their offsets over the cosine of incidence. With FP64 distances, the reference's contact
    // error, 64 ulps of the coordinates' magnitude (contactError, src/owe/core/math.hpp:15,
    // NearestCrossing::offer, src/owe/scene/world.cpp:526); plain FP32 keeps a relative window.
    __device__ __forceinline__ double tieSpanD(T c) const {
        if constexpr (kExactTies) return 64 * 2.220446049250313e-16 * fmax(coordScale(), 1e-3) / fmax(double(c), 1e-3);
        else return fabs(bestD) * double(tieWindow<T>()) / fmax(double(c), 1e-3);
    }

    // How far beyond the closest crossing the contact-resolving traversal still looks (node culling
    // and the crossings it admits): the tie window in the traversal's precision, and with FP64
    // decisions at least the FP64 window plus, for FP32 traversal, its distances' own rounding (a few
    // ulps of the coordinates' magnitude), so that every near tie reaches the FP64 test.
    __device__ __forceinline__ T tieSpan(T c) const {
        // |best|: a crossing just behind the anchor (a contact through it) may be the closest
        T s = fabs(best) * tieWindow<T>();
        if constexpr (kExactTies) {
            const T scale = T(fmax(coordScale(), 1e-3));
            s += T(64 * 2.220446049250313e-16) * scale;
            if constexpr (sizeof(T) == sizeof(float)) s += T(1e-6) * scale;
        }
        return s / fmax(c, T(1e-3));
    }
    __device__ __forceinline__ T tieLimit() const { return best + tieSpan(bestCos); }

    // Whether boundary b's crossing at t, met from its front side when `front` at incidence |cos| c,
    // replaces the current closest (the contact-resolving instantiation; NearestCrossing::offer,
    // src/owe/scene/world.cpp:515-550). Crossings of different boundaries within the tie span are
    // one contact: the one met from the ray's region wins, matter wins over a zero-thickness
    // readout, then the lower boundary index; two that both match leave the order undecided
    // (kHitAmbiguous). `flags` receives the winner's flags.
    __device__ __forceinline__ bool winsContact(const DeviceScene& sc, uint32_t b, double tD, bool front, T c,
                                                uint32_t& flags) {
        const uint32_t frontFlag = front ? kHitFront : 0u;
        // outside the tie window, or two crossings of one boundary: the nearer one
        if (!found || b == hit.boundary || !(fabs(tD - bestD) <= tieSpanD(fmin(c, bestCos)))) {
            flags = frontFlag;
            return !found || tD < bestD;
        }
        const bool hinted = q.region != kNone;
        auto incident = [&](uint32_t bb, bool fr) {
            const DBoundary& bd = sc.boundaries[bb];
            return fr ? bd.front : bd.back;
        };
        auto readout = [&](uint32_t bb) {
            const DBoundary& bd = sc.boundaries[bb];
            return sc.optics[bd.optics].type == OWEC_SURF_DETECTOR && bd.front == bd.back;
        };
        const bool mNew = !hinted || incident(b, front) == q.region;
        const bool mOld = !hinted || incident(hit.boundary, hit.flags & kHitFront) == q.region;
        const bool rNew = readout(b), rOld = readout(hit.boundary);
        bool ambiguous = hit.flags & kHitAmbiguous;
        if (mNew && mOld && rNew != rOld) {
            if (rNew) return false;  // physical matter precedes a coincident readout
            ambiguous = false;
        } else if (hinted && mNew && mOld) {
            ambiguous = true;
        }
        const bool replace = mNew != mOld ? mNew : (rNew != rOld ? rOld : b < hit.boundary);
        if (!replace) {
            hit.flags = (hit.flags & ~kHitAmbiguous) | (ambiguous ? kHitAmbiguous : 0u);
            return false;
        }
        flags = frontFlag | (ambiguous ? kHitAmbiguous : 0u);
        return true;
    }

    // The distance of triangle slot i's crossing from its FP64 vertices and the FP64 origin when the
    // traversal runs in FP32 and refines in FP64 (the value the closest hit is later refined to); t
    // itself otherwise, or when the two disagree beyond the refinement's reach.
    __device__ __forceinline__ double refinedTriangleT(const DeviceScene& sc, uint32_t i, T t) const {
        if constexpr (sizeof(T) == sizeof(float) && sizeof(Rr) == sizeof(double)) {
            const PrimRec64& p = sc.prims64[i];
            const V3<double> v0(p.v0[0], p.v0[1], p.v0[2]), v1(p.v1[0], p.v1[1], p.v1[2]), v2(p.v2[0], p.v2[1], p.v2[2]);
            const V3<double> n = triangleNormal(v0, v1, v2);
            const double tD = dot(v0 - q.od, n) / dot(V3<double>(q.d), n);
            return fabs(tD - double(t)) <= 1e-3 * (1 + fabs(double(t))) ? tD : double(t);
        } else {
            return double(t);
        }
    }

    // Tests primitive slot i; true when its crossing was accepted as the new closest.
    __device__ __forceinline__ bool testPrim(const DeviceScene& sc, uint32_t i) {
        V3<T> v0, v1, v2;
        uint32_t b, prim, kind;
        TriFetch<T>::get(sc, i, v0, v1, v2, b, prim, kind);
        // the contact-resolving instantiation looks a tie window beyond the closest so far; a query for
        // any crossing asks only about (0, tmax): the window there reached the light's own surface
        // past the end of a shadow ray (4e-6 of its length short of it) whenever it was wider
        const T limit = (Full && !AnyHit) ? tieLimit() : best;
        uint32_t flags = 0;
        if (kind == kPrimTriangle) {
            const V3<T> a = v0 - q.o, bb = v1 - q.o, c = v2 - q.o;
            if (!lineCrossesTriangle(sh, a, bb, c)) return false;
            const V3<T> n = triangleNormal(v0, v1, v2);
            const T dn = dot(q.d, n);
            const T t = -dot(q.o - v0, n) / dn;
            // contacts: another boundary's face through the anchor may fall just behind it
            if (!((Full ? t > T(0) || (b != q.depB && fabs(t * dn) <= behindWindow(q.o) * sqrt(dot(n, n))) : t > T(0)) &&
                  t < limit))
                return false;
            if (!acceptCrossing<T>(sc, q, b, prim, true, t, n)) return false;
            if constexpr (Full) {
                const T c = fabs(dn) / sqrt(dot(n, n));
                const double tD = refinedTriangleT(sc, i, t);
                if (!winsContact(sc, b, tD, dn < T(0), c, flags)) return false;
                bestCos = c;
                bestD = tD;
            }
            best = t;
            hit.t = double(t);
            hit.prim = prim;
        } else {
            const AnalyticResult<Rr> ar = analyticHit<T, R, Rr, Full>(sc.self, b, q.od, q.d, limit, q.depB, q.region, q.errN);
            if (!ar.ok) return false;
            if constexpr (Full) {
                if (!winsContact(sc, b, double(ar.t), ar.front, T(ar.cosAbs), flags)) return false;
                bestCos = T(ar.cosAbs);
                bestD = double(ar.t);
            }
            best = T(ar.t);
            hit.t = double(ar.t);
            hit.prim = 0;
        }
        if constexpr (Full) hit.flags = flags;
        hit.boundary = b;
        hit.slot = i;
        found = true;
        return true;
    }
};

// A query that overflowed the short stack, from the start with the deep one. Out of line: its
// stack lives in local memory and only these rare queries touch it. By value in and out, so that
// the caller's query need not live in memory.
struct DeepResult {
    HitRec hit;
    int status;
    uint32_t visits, tests;
};
template <class T, class R, class Rr, bool AnyHit, bool Full = false>
__device__ __noinline__ DeepResult traceRayDeep(const DeviceScene* scp, RayQuery<T> q, HitRec hitIn) {
    const DeviceScene& sc = *scp;
    Traversal<T, R, Rr, AnyHit, LocalStack, true, Full> tr;
    tr.begin(q, nullptr, 0);
    tr.hit = hitIn;
    int s;
    do {
        s = tr.run(sc, 1 << 30);
    } while (s == kTraceRunning);
    DeepResult r;
    r.hit = tr.hit;
    r.status = s;
    r.visits = tr.nodeVisits;
    r.tests = tr.primTests;
    return r;
}

// The whole query in one call (cast rays, forward walks and the adjoint's replay).
template <class T, class R, class Rr, bool AnyHit, bool Full = false>
__device__ __forceinline__ int traceRay(const DeviceScene& sc, const RayQuery<T>& q, StackEntry* stack, int stride, HitRec& hit,
                                        uint32_t* visits = nullptr, uint32_t* tests = nullptr) {
    Traversal<T, R, Rr, AnyHit, SharedStack, true, Full> tr;
    tr.begin(q, stack, stride);
    tr.hit = hit;
    int s;
    do {
        s = tr.run(sc, 1 << 30);
    } while (s == kTraceRunning);
    uint32_t nv = tr.nodeVisits, nt = tr.primTests;
    if (s == kTraceOverflow) {
        const DeepResult d = traceRayDeep<T, R, Rr, AnyHit, Full>(sc.self, q, hit);
        s = d.status;
        hit = d.hit;
        nv += d.visits;
        nt += d.tests;
    } else {
        hit = tr.hit;
    }
    if (visits) *visits += nv;
    if (tests) *tests += nt;
    return s;
}

}  // namespace owec
