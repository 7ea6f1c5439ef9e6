// Closest-hit and any-hit traversal of the 8-wide quantised BVH.
//
// One thread follows one ray. Node records (80 B) are read with five 128-bit read-only loads;
// the eight child boxes are decoded from 8-bit offsets against the node's origin and power-of-two
// scales and slab-tested together; the hits are ordered near-first and pushed on a short per-thread
// stack staged in shared memory (transposed so that a warp's entries of one level are consecutive
// words). Deferred entries whose entry distance lies beyond the closest hit found since are culled
// on pop, as the reference's Bvh::traverseSlots does (src/owe/scene/bvh.hpp:39-78).
//
// Which crossings count near a ray's departure follows the reference's contact rule
// (src/owe/scene/world.cpp:451-513): the face the ray left never does, and within the anchor's
// error only a crossing met from the ray's own region does.
#pragma once

#include "shapes.cuh"

namespace owec {

constexpr int kStackDepth = 32;  // entries per thread; an overflow ends the query and is counted
constexpr uint32_t kMaxTraversalSteps = 1u << 20;  // a bound on stack pops: a malformed tree cannot hang

struct StackEntry {
    uint32_t ref;   // bit 31: leaf; leaf: prim start << 2 | (count - 1); inner: node index
    float tEnter;
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
    uint32_t pad;
};

// The acceptance rule of a candidate crossing at distance t with (unnormalised) normal n.
template <class T>
__device__ __forceinline__ bool acceptCrossing(const DeviceScene& sc, const RayQuery<T>& q, uint32_t b, uint32_t prim, bool mesh, T t,
                            const V3<T>& n) {
    if (mesh && b == q.depB && prim == q.depP) return false;
    const T dn = dot(q.d, n);
    const T nl = sqrt(dot(n, n));
    const bool near = fabs(t * dn) <= q.errN * nl;
    if (!near) return true;
    if (b == q.depB) return false;
    if (q.region == kNone) return true;
    const DBoundary& bd = sc.boundaries[b];
    const uint32_t incident = dn < T(0) ? bd.front : bd.back;
    return incident == q.region;
}

template <class T> __device__ __forceinline__ T farWiden();
template <> __device__ __forceinline__ float farWiden<float>() { return 1.0000004f; }
template <> __device__ __forceinline__ double farWiden<double>() { return 1.0 + 4e-16; }

// Entry distances on the stack are FP32: rounded down when stored, compared with the closest hit
// rounded up, so an FP64 query never culls an entry it must visit.
__device__ __forceinline__ float toFloatDown(float x) { return x; }
__device__ __forceinline__ float toFloatDown(double x) { return __double2float_rd(x); }
__device__ __forceinline__ float toFloatUp(float x) { return x; }
__device__ __forceinline__ float toFloatUp(double x) { return __double2float_ru(x); }

// The analytic boundary b's first acceptable crossing in (0, best); FP64 refinement when Rr = double.
template <class R, class Rr, class T>
__device__ __forceinline__ bool analyticCandidate(const DeviceScene& sc, const RayQuery<T>& q, uint32_t b, T best, Rr& tOut) {
    const DBoundary& bd = sc.boundaries[b];
    const V3<Rr> lo = bd.toLocal.point(V3<Rr>(q.od));
    const V3<Rr> ld = bd.toLocal.vector(V3<Rr>(q.d));
    AHit<Rr> hits[2];
    const int n = analyticCrossings<R, Rr>(bd, lo, ld, Rr(0), Rr(best), hits);
    for (int i = 0; i < n; ++i) {
        const V3<T> nw = V3<T>(bd.toWorld.vector(hits[i].n));
        if (!acceptCrossing(sc, q, b, 0u, false, T(hits[i].t), nw)) continue;
        tOut = hits[i].t;
        return true;
    }
    return false;
}

// Decoded child boxes of a node, slab-tested against the ray. Returns the hit mask and fills tEnter.
template <class T>
__device__ __forceinline__ uint32_t intersectChildren(const WideNode& nd, const V3<T>& inv, const V3<T>& oinv, T tmin, T tmax,
                                   T tEnter[8]) {
    const T sx = T(__uint_as_float(uint32_t(nd.ex) << 23));
    const T sy = T(__uint_as_float(uint32_t(nd.ey) << 23));
    const T sz = T(__uint_as_float(uint32_t(nd.ez) << 23));
    // t = (origin + q * s - o) * inv = q * (s * inv) + (origin * inv - o * inv)
    const T ax = sx * inv.x, ay = sy * inv.y, az = sz * inv.z;
    const T bx = T(nd.ox) * inv.x - oinv.x, by = T(nd.oy) * inv.y - oinv.y, bz = T(nd.oz) * inv.z - oinv.z;
    const bool nx = inv.x < T(0), ny = inv.y < T(0), nz = inv.z < T(0);
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (nd.meta[i] == 0) continue;  // empty slot (inner slots carry bit 3, leaves a count)
        const T lx = T(nx ? nd.qhix[i] : nd.qlox[i]), hx = T(nx ? nd.qlox[i] : nd.qhix[i]);
        const T ly = T(ny ? nd.qhiy[i] : nd.qloy[i]), hy = T(ny ? nd.qloy[i] : nd.qhiy[i]);
        const T lz = T(nz ? nd.qhiz[i] : nd.qloz[i]), hz = T(nz ? nd.qloz[i] : nd.qhiz[i]);
        const T t0x = fma(lx, ax, bx), t1x = fma(hx, ax, bx);
        const T t0y = fma(ly, ay, by), t1y = fma(hy, ay, by);
        const T t0z = fma(lz, az, bz), t1z = fma(hz, az, bz);
        const T te = fmax(fmax(t0x, t0y), fmax(t0z, tmin));
        const T tx = fmin(fmin(t1x, t1y), t1z) * farWiden<T>();
        const T tl = fmin(tx, tmax);
        if (te <= tl) {
            mask |= 1u << i;
            tEnter[i] = te;
        }
    }
    return mask;
}

__device__ __forceinline__ void loadNode(const WideNode* nodes, uint32_t i, WideNode& nd) {
#if defined(__CUDA_ARCH__)
    const uint4* src = reinterpret_cast<const uint4*>(nodes + i);
    uint4* dst = reinterpret_cast<uint4*>(&nd);
#pragma unroll
    for (int k = 0; k < 5; ++k) dst[k] = __ldg(src + k);
#else
    nd = nodes[i];
#endif
}

__device__ __forceinline__ void loadPrim(const PrimRec* prims, uint32_t i, PrimRec& p) {
#if defined(__CUDA_ARCH__)
    const float4* src = reinterpret_cast<const float4*>(prims + i);
    float4* dst = reinterpret_cast<float4*>(&p);
#pragma unroll
    for (int k = 0; k < 3; ++k) dst[k] = __ldg(src + k);
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

// Closest (AnyHit = false) or first (AnyHit = true) acceptable crossing in (0, q.tmax).
// R / Rr: precision of analytic roots and of their refinement. `stack` is this thread's column of
// the block's shared-memory stack (stride = block size).
template <class T, class R, class Rr, bool AnyHit>
__device__ int traceRay(const DeviceScene& sc, const RayQuery<T>& q, StackEntry* stack, int stride, HitRec& hit,
                        uint32_t* visits = nullptr, uint32_t* tests = nullptr) {
    const V3<T> inv(T(1) / q.d.x, T(1) / q.d.y, T(1) / q.d.z);
    const V3<T> oinv(q.o.x * inv.x, q.o.y * inv.y, q.o.z * inv.z);
    const ShearedRay<T> sh = shearRay(q.d);
    T best = q.tmax;
    bool found = false;
    int sp = 0;
    uint32_t nodeVisits = 0, primTests = 0;
    stack[0] = {0u, 0.0f};
    sp = 1;
    uint32_t steps = 0;
    while (sp > 0) {
        if (++steps > kMaxTraversalSteps) return kTraceOverflow;
        const StackEntry e = stack[(sp - 1) * stride];
        --sp;
        if (e.tEnter > toFloatUp(best)) continue;
        if ((e.ref & 0x80000000u) == 0) {
            WideNode nd;
            loadNode(sc.nodes, e.ref, nd);
            ++nodeVisits;
            T tEnter[8];
            uint32_t mask = intersectChildren(nd, inv, oinv, T(0), best, tEnter);
            // Push in far-to-near order: repeatedly take the farthest remaining hit.
            const int nHits = __popc(mask);
            if (sp + nHits > kStackDepth) return kTraceOverflow;
            while (mask) {
                int far = -1;
                T tf = T(-1);
                uint32_t m = mask;
                while (m) {
                    const int i = __ffs(m) - 1;
                    m &= m - 1;
                    if (tEnter[i] >= tf) { tf = tEnter[i]; far = i; }
                }
                mask &= ~(1u << far);
                const uint8_t meta = nd.meta[far];
                uint32_t ref;
                if (nd.imask & (1u << far)) {
                    ref = nd.child_base + (meta & 7u);
                } else {
                    const uint32_t cnt = meta >> 5;
                    ref = 0x80000000u | ((nd.prim_base + (meta & 31u)) << 2) | (cnt - 1u);
                }
                stack[sp * stride] = {ref, toFloatDown(tf)};
                ++sp;
            }
        } else {
            const uint32_t start = (e.ref & 0x7FFFFFFFu) >> 2, cnt = (e.ref & 3u) + 1u;
            primTests += cnt;
            for (uint32_t k = 0; k < cnt; ++k) {
                V3<T> v0, v1, v2;
                uint32_t b, prim, kind;
                TriFetch<T>::get(sc, start + k, v0, v1, v2, b, prim, kind);
                if (kind == kPrimTriangle) {
                    const V3<T> a = v0 - q.o, bb = v1 - q.o, c = v2 - q.o;
                    if (!lineCrossesTriangle(sh, a, bb, c)) continue;
                    const V3<T> n = triangleNormal(v0, v1, v2);
                    const T t = -dot(q.o - v0, n) / dot(q.d, n);
                    if (!(t > T(0) && t < best)) continue;
                    if (!acceptCrossing(sc, q, b, prim, true, t, n)) continue;
                    best = t;
                    hit.t = double(t);
                    hit.boundary = b;
                    hit.prim = prim;
                    hit.slot = start + k;
                    found = true;
                } else {
                    Rr tr;
                    if (!analyticCandidate<R, Rr, T>(sc, q, b, best, tr)) continue;
                    best = T(tr);
                    hit.t = double(tr);
                    hit.boundary = b;
                    hit.prim = 0;
                    hit.slot = start + k;
                    found = true;
                }
                if (AnyHit) {
                    if (visits) *visits += nodeVisits;
                    if (tests) *tests += primTests;
                    return kTraceHit;
                }
            }
        }
        // cull deferred entries beyond the closest hit
        while (sp > 0 && stack[(sp - 1) * stride].tEnter > toFloatUp(best)) --sp;
    }
    if (visits) *visits += nodeVisits;
    if (tests) *tests += primTests;
    return found ? kTraceHit : kTraceMiss;
}

}  // namespace owec
