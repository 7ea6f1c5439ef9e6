// Device construction of the 8-wide quantised BVH.
//
//  1. 63-bit Morton codes of the primitives' box centres (21 bits per axis in the centres' bounds),
//     the 64th bit set for a primitive larger than an eighth of the scene;
//  2. a radix sort of (code, primitive) pairs (CUB);
//  3. the binary radix tree over the sorted codes, one thread per inner node (Karras 2012), every
//     node covering a contiguous range of sorted primitives;
//  4. boxes and primitive counts bottom-up, the second child to finish computing its parent;
//  5. a top-down collapse into 8-wide nodes, level by level: each wide node opens the binary
//     subtree below it greedily by surface area until it has eight children; a child with at most
//     kLeafMax (two) primitives becomes a leaf slot, the others new wide nodes; children boxes are stored
//     as 8-bit offsets against the node's origin and per-axis power-of-two scales, rounded outward.
//     Children take the node's eight slots by direction: slot s (bit k set: negative along axis k)
//     goes to the child whose centre lies farthest along that octant's diagonal from the node's
//     centre (a greedy auction), so that a ray of octant o meets the children roughly in the order
//     of slot ^ o ^ 7, and the traversal orders its hits without a sort (Ylitie, Karras and Laine,
//     "Efficient incoherent ray traversal on GPUs through compressed wide BVHs", HPG 2017).
//
// This replaces the reference's host-side binned SAH builds (src/owe/scene/bvh.cpp:100-337) of the
// world hierarchy and of every mesh's own hierarchy with one hierarchy over all primitives.
#include <cub/device/device_radix_sort.cuh>

#include <vector>

#include "bvh_build.hpp"

namespace owec {

namespace {

// Primitives a leaf slot may hold (at most 3: eight slots of three fill the traversal's 24-bit mask).
// Two: a ray tests fewer primitives per leaf it enters (2.98 instead of 5.43 per query on the
// 2^20-triangle room, with 3.94 node visits instead of 4.09), and the pass runs 8 % faster.
#ifndef OWEC_LEAF_MAX
#define OWEC_LEAF_MAX 2
#endif
constexpr uint32_t kLeafMax = OWEC_LEAF_MAX;
static_assert(kLeafMax >= 1 && kLeafMax <= 3, "a leaf slot holds one to three primitives");
// The size, against the scene's, from which a primitive counts as large (sorted after the others).
#ifndef OWEC_LARGE_PRIMITIVE
#define OWEC_LARGE_PRIMITIVE 0.125f
#endif
constexpr uint32_t kNoParent = 0xFFFFFFFFu;

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
    v &= 0x1FFFFFull;
    v = (v | v << 32) & 0x1F00000000FFFFull;
    v = (v | v << 16) & 0x1F0000FF0000FFull;
    v = (v | v << 8) & 0x100F00F00F00F00Full;
    v = (v | v << 4) & 0x10C30C30C30C30C3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
}

// Order-preserving integer image of a float (and back), so integer atomics give float min / max.
__device__ __forceinline__ int floatToOrdered(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}

__global__ void kCentroidBounds(const float4* lo, const float4* hi, uint32_t n, int* bounds) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 a = lo[i], b = hi[i];
        const float c[3] = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)};
        for (int k = 0; k < 3; ++k) { mn[k] = fminf(mn[k], c[k]); mx[k] = fmaxf(mx[k], c[k]); }
    }
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(0xFFFFFFFFu, mn[k], off));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xFFFFFFFFu, mx[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) {
            atomicMin(bounds + k, floatToOrdered(mn[k]));
            atomicMax(bounds + 3 + k, floatToOrdered(mx[k]));
        }
    }
}

__device__ __forceinline__ float orderedToFloat(int v) { return __int_as_float(v >= 0 ? v : v ^ 0x7FFFFFFF); }

__global__ void kMorton(const float4* lo, const float4* hi, uint32_t n, const int* bounds, uint64_t* keys,
                        uint32_t* vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int* bi = bounds;
    const float mn[3] = {orderedToFloat(bi[0]), orderedToFloat(bi[1]), orderedToFloat(bi[2])};
    const float mx[3] = {orderedToFloat(bi[3]), orderedToFloat(bi[4]), orderedToFloat(bi[5])};
    const float4 a = lo[i], b = hi[i];
    const float c[3] = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)};
    const float size[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
    uint64_t code = 0;
    float sceneExt = 0.f, primExt = 0.f;
    for (int k = 0; k < 3; ++k) {
        const float ext = mx[k] - mn[k];
        float u = ext > 0.f ? (c[k] - mn[k]) / ext : 0.5f;
        u = fminf(fmaxf(u, 0.f), 1.f);
        const uint64_t q = uint64_t(fminf(u * 2097152.0f, 2097151.0f));
        code |= spread21(q) << (2 - k);
        sceneExt = fmaxf(sceneExt, ext);
        primExt = fmaxf(primExt, size[k]);
    }
    // A primitive larger than an eighth of the scene (a wall, a floor, a lamp beside a finely
    // tessellated body) sorts after all the others: the tree's root split separates the two sets,
    // so no subtree of small primitives takes a wall's box.
    if (primExt > OWEC_LARGE_PRIMITIVE * sceneExt) code |= 1ull << 63;
    keys[i] = code;
    vals[i] = i;
}

__device__ __forceinline__ int commonPrefix(const uint64_t* k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a == b) return 64 + __clz(uint32_t(i ^ j));
    return __clzll(a ^ b);
}

// Inner node i of the radix tree: children (combined index: inner 0..n-2, leaf k at n-1+k) and range.
__global__ void kRadixTree(const uint64_t* keys, int n, int2* children, int2* ranges, uint32_t* parents) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = commonPrefix(keys, n, i, i + 1) - commonPrefix(keys, n, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = commonPrefix(keys, n, i, i - d);
    int lmax = 2;
    while (commonPrefix(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (commonPrefix(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = commonPrefix(keys, n, i, j);
    int s = 0;
    for (int div = 2;; div *= 2) {
        const int t = (l + div - 1) / div;
        if (commonPrefix(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const int left = lo == gamma ? (n - 1 + gamma) : gamma;
    const int right = hi == gamma + 1 ? (n - 1 + gamma + 1) : gamma + 1;
    children[i] = make_int2(left, right);
    ranges[i] = make_int2(lo, hi);
    parents[left] = uint32_t(i);
    parents[right] = uint32_t(i);
}

__global__ void kBottomUp(const float4* primLo, const float4* primHi, const uint32_t* vals, int n,
                          const int2* children, const uint32_t* parents, float4* boxLo, float4* boxHi,
                          uint32_t* counts, uint32_t* flags) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int leaf = n - 1 + k;
    boxLo[leaf] = primLo[vals[k]];
    boxHi[leaf] = primHi[vals[k]];
    counts[leaf] = 1;
    __threadfence();
    uint32_t p = parents[leaf];
    for (int level = 0; p != kNoParent; ++level) {
        if (level > 4096 || p >= uint32_t(n - 1)) {  // a malformed tree: stop and report
            atomicAdd(&flags[n - 1 > 0 ? n - 1 : 0], 0x10000u);
            return;
        }
        if (atomicAdd(&flags[p], 1u) == 0) return;  // the sibling finishes this parent
        __threadfence();
        const int2 c = children[p];
        const float4 la = __ldcg(boxLo + c.x), lb = __ldcg(boxLo + c.y);
        const float4 ha = __ldcg(boxHi + c.x), hb = __ldcg(boxHi + c.y);
        boxLo[p] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
        boxHi[p] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
        counts[p] = __ldcg(counts + c.x) + __ldcg(counts + c.y);
        __threadfence();
        p = parents[p];
    }
}

__device__ __forceinline__ float halfArea(float4 lo, float4 hi) {
    const float x = hi.x - lo.x, y = hi.y - lo.y, z = hi.z - lo.z;
    return x * y + y * z + z * x;
}

// Smallest power-of-two scale (as a biased exponent byte) whose 254 steps cover ext (one step of
// slack for the rounding of ext / 254).
__device__ __forceinline__ uint32_t scaleExponent(float ext) {
    const float s = ext / 254.0f;
    if (!(s > 0.f)) return 1u;
    int e;
    const float m = frexpf(s, &e);  // s = m * 2^e, m in [0.5, 1)
    int biased = (m == 0.5f ? e - 1 : e) + 127;
    if (biased < 1) biased = 1;
    if (biased > 254) biased = 254;
    return uint32_t(biased);
}

struct CollapseArgs {
    const int2* children;
    const int2* ranges;
    const float4* boxLo;
    const float4* boxHi;
    const uint32_t* counts;
    const uint32_t* vals;
    int n;
    WideNode* nodes;
    uint32_t* leafOrder;
    uint32_t* counters;  // [0] nodes allocated, [1] primitives placed, [2] next work count
    uint2* work;         // (binary node, wide node)
    uint2* next;
};

__global__ void kCollapse(CollapseArgs a, uint32_t nWork) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nWork) return;
    const uint2 item = a.work[w];
    const int n = a.n;
    int c[8];
    int nc;
    if (int(item.x) >= n - 1) {  // a single-leaf root
        c[0] = int(item.x);
        nc = 1;
    } else {
        const int2 ch = a.children[item.x];
        c[0] = ch.x;
        c[1] = ch.y;
        nc = 2;
        while (nc < 8) {
            int best = -1;
            float bestArea = -1.f;
            for (int i = 0; i < nc; ++i) {
                if (c[i] >= n - 1 || a.counts[c[i]] <= kLeafMax) continue;
                const float ar = halfArea(a.boxLo[c[i]], a.boxHi[c[i]]);
                if (ar > bestArea) { bestArea = ar; best = i; }
            }
            if (best < 0) break;
            const int2 ch2 = a.children[c[best]];
            c[best] = ch2.x;
            c[nc++] = ch2.y;
        }
    }
    float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
    uint32_t nInner = 0, nLeafPrims = 0;
    for (int i = 0; i < nc; ++i) {
        const float4 l = a.boxLo[c[i]], h = a.boxHi[c[i]];
        lo = make_float4(fminf(lo.x, l.x), fminf(lo.y, l.y), fminf(lo.z, l.z), 0.f);
        hi = make_float4(fmaxf(hi.x, h.x), fmaxf(hi.y, h.y), fmaxf(hi.z, h.z), 0.f);
        const uint32_t cnt = a.counts[c[i]];
        if (cnt > kLeafMax) ++nInner; else nLeafPrims += cnt;
    }
    // slot auction: repeatedly give the free slot and unplaced child with the largest projection of
    // the child's centre (relative to the node's) on the slot's octant diagonal to each other
    int childAt[8];
    for (int k = 0; k < 8; ++k) childAt[k] = -1;
    {
        float cost[8][8];
        const float px = 0.5f * (lo.x + hi.x), py = 0.5f * (lo.y + hi.y), pz = 0.5f * (lo.z + hi.z);
        for (int i = 0; i < nc; ++i) {
            const float4 l = a.boxLo[c[i]], h = a.boxHi[c[i]];
            const float cx = 0.5f * (l.x + h.x) - px, cy = 0.5f * (l.y + h.y) - py, cz = 0.5f * (l.z + h.z) - pz;
            for (int k = 0; k < 8; ++k)
                cost[i][k] = ((k & 1) ? -cx : cx) + ((k & 2) ? -cy : cy) + ((k & 4) ? -cz : cz);
        }
        uint32_t placed = 0;
        for (int round = 0; round < nc; ++round) {
            int bi = -1, bk = -1;
            float bc = -INFINITY;
            for (int i = 0; i < nc; ++i) {
                if (placed & (1u << i)) continue;
                for (int k = 0; k < 8; ++k)
                    if (childAt[k] < 0 && (bi < 0 || cost[i][k] > bc)) { bc = cost[i][k]; bi = i; bk = k; }
            }
            childAt[bk] = bi;
            placed |= 1u << bi;
        }
    }
    const uint32_t childBase = nInner ? atomicAdd(&a.counters[0], nInner) : 0u;
    const uint32_t primBase = nLeafPrims ? atomicAdd(&a.counters[1], nLeafPrims) : 0u;
    WideNode nd;
    nd.ox = lo.x;
    nd.oy = lo.y;
    nd.oz = lo.z;
    const uint32_t ex = scaleExponent(hi.x - lo.x), ey = scaleExponent(hi.y - lo.y), ez = scaleExponent(hi.z - lo.z);
    nd.ex = uint8_t(ex);
    nd.ey = uint8_t(ey);
    nd.ez = uint8_t(ez);
    const float sx = __uint_as_float(ex << 23), sy = __uint_as_float(ey << 23), sz = __uint_as_float(ez << 23);
    nd.imask = 0;
    nd.child_base = childBase;
    nd.prim_base = primBase;
    // inner children are stored in slot order, so that the k-th inner slot's node is child_base + k
    uint32_t innerK = 0, leafOff = 0;
    for (int i = 0; i < 8; ++i) {
        if (childAt[i] < 0) {
            nd.meta[i] = 0;
            nd.qlox[i] = nd.qloy[i] = nd.qloz[i] = 255;
            nd.qhix[i] = nd.qhiy[i] = nd.qhiz[i] = 0;
            continue;
        }
        const int ci = c[childAt[i]];
        const float4 l = a.boxLo[ci], h = a.boxHi[ci];
        auto qlo = [](float v, float o, float s) {
            return uint8_t(fminf(fmaxf(floorf(__fsub_rd(v, o) / s), 0.f), 255.f));
        };
        auto qhi = [](float v, float o, float s) {
            return uint8_t(fminf(fmaxf(ceilf(__fsub_ru(v, o) / s), 0.f), 255.f));
        };
        nd.qlox[i] = qlo(l.x, lo.x, sx);
        nd.qloy[i] = qlo(l.y, lo.y, sy);
        nd.qloz[i] = qlo(l.z, lo.z, sz);
        nd.qhix[i] = qhi(h.x, lo.x, sx);
        nd.qhiy[i] = qhi(h.y, lo.y, sy);
        nd.qhiz[i] = qhi(h.z, lo.z, sz);
        const uint32_t cnt = a.counts[ci];
        if (cnt > kLeafMax) {
            nd.imask |= uint8_t(1u << i);
            nd.meta[i] = uint8_t(8u | innerK);
            const uint32_t slot = atomicAdd(&a.counters[2], 1u);
            a.next[slot] = make_uint2(uint32_t(ci), childBase + innerK);
            ++innerK;
        } else {
            nd.meta[i] = uint8_t((cnt << 5) | leafOff);
            const int first = ci >= n - 1 ? ci - (n - 1) : a.ranges[ci].x;
            for (uint32_t k = 0; k < cnt; ++k) a.leafOrder[primBase + leafOff + k] = a.vals[first + k];
            leafOff += cnt;
        }
    }
    a.nodes[item.y] = nd;
}

}  // namespace

uint32_t buildWideBvh(const float4* primLo, const float4* primHi, uint32_t n, BvhScratch& s, DBuf<WideNode>& nodes,
                      DBuf<uint32_t>& leafOrder, cudaStream_t stream) {
    if (n == 0) return 0;
    const uint32_t nAll = 2 * n - 1;
    s.keys.reserve(n);
    s.keysAlt.reserve(n);
    s.vals.reserve(n);
    s.valsAlt.reserve(n);
    s.children.reserve(n);
    s.ranges.reserve(n);
    s.parents.reserve(nAll);
    s.boxLo.reserve(nAll);
    s.boxHi.reserve(nAll);
    s.counts.reserve(nAll);
    s.flags.reserve(n);
    s.work.reserve(n);
    s.next.reserve(n);
    s.counters.reserve(8);
    s.bounds.reserve(8);
    nodes.reserve(std::max<uint32_t>(1, n));
    leafOrder.reserve(n);

    // +inf and -inf in the ordered integer image
    const int init[6] = {0x7F800000, 0x7F800000, 0x7F800000, int(0x807FFFFFu), int(0x807FFFFFu), int(0x807FFFFFu)};
    OWEC_CUDA(cudaMemcpyAsync(s.bounds.get(), init, sizeof(init), cudaMemcpyHostToDevice, stream));
    const int T = 256;
    kCentroidBounds<<<std::min<uint32_t>((n + T - 1) / T, 1184), T, 0, stream>>>(primLo, primHi, n, s.bounds.get());
    kMorton<<<(n + T - 1) / T, T, 0, stream>>>(primLo, primHi, n, s.bounds.get(), s.keys.get(), s.vals.get());
    size_t tempBytes = 0;
    cub::DoubleBuffer<uint64_t> dk(s.keys.get(), s.keysAlt.get());
    cub::DoubleBuffer<uint32_t> dv(s.vals.get(), s.valsAlt.get());
    OWEC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, dk, dv, int(n), 0, 64, stream));
    s.cubTemp.reserve(tempBytes);
    OWEC_CUDA(cub::DeviceRadixSort::SortPairs(s.cubTemp.get(), tempBytes, dk, dv, int(n), 0, 64, stream));
    const uint64_t* keys = dk.Current();
    const uint32_t* vals = dv.Current();

    OWEC_CUDA(cudaMemsetAsync(s.parents.get(), 0xFF, nAll * sizeof(uint32_t), stream));
    OWEC_CUDA(cudaMemsetAsync(s.flags.get(), 0, n * sizeof(uint32_t), stream));
    if (n > 1)
        kRadixTree<<<(n - 1 + T - 1) / T, T, 0, stream>>>(keys, int(n), s.children.get(), s.ranges.get(),
                                                           s.parents.get());
    kBottomUp<<<(n + T - 1) / T, T, 0, stream>>>(primLo, primHi, vals, int(n), s.children.get(), s.parents.get(),
                                                  s.boxLo.get(), s.boxHi.get(), s.counts.get(), s.flags.get());

    {
        uint32_t err = 0;  // flags[n - 1] is no inner node's: it collects malformed-tree reports
        OWEC_CUDA(cudaMemcpyAsync(&err, s.flags.get() + (n - 1), sizeof(err), cudaMemcpyDeviceToHost, stream));
        OWEC_CUDA(cudaStreamSynchronize(stream));
        if (err >= 0x10000u) throw std::runtime_error("BVH build: malformed radix tree");
    }
    const uint32_t counters[4] = {1u, 0u, 0u, 0u};  // the root is wide node 0
    OWEC_CUDA(cudaMemcpyAsync(s.counters.get(), counters, sizeof(counters), cudaMemcpyHostToDevice, stream));
    // the binary root: inner node 0, or with one primitive its leaf (combined index n - 1 = 0)
    const uint2 root = make_uint2(0u, 0u);
    OWEC_CUDA(cudaMemcpyAsync(s.work.get(), &root, sizeof(root), cudaMemcpyHostToDevice, stream));
    CollapseArgs a{s.children.get(), s.ranges.get(), s.boxLo.get(), s.boxHi.get(), s.counts.get(), vals, int(n),
                   nodes.get(), leafOrder.get(), s.counters.get(), s.work.get(), s.next.get()};
    uint32_t nWork = 1;
    for (int level = 0; nWork > 0; ++level) {
        if (level > 4096) throw std::runtime_error("BVH collapse did not terminate");
        kCollapse<<<(nWork + 127) / 128, 128, 0, stream>>>(a, nWork);
        uint32_t h[4];
        OWEC_CUDA(cudaMemcpyAsync(h, s.counters.get(), sizeof(h), cudaMemcpyDeviceToHost, stream));
        OWEC_CUDA(cudaStreamSynchronize(stream));
        nWork = h[2];
        const uint32_t zero = 0;
        OWEC_CUDA(cudaMemcpyAsync(s.counters.get() + 2, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream));
        std::swap(a.work, a.next);
        s.nodeCount = h[0];
        s.placedPrims = h[1];
    }
    OWEC_CUDA(cudaStreamSynchronize(stream));
    if (s.placedPrims != n) throw std::runtime_error("BVH collapse placed " + std::to_string(s.placedPrims) +
                                                     " of " + std::to_string(n) + " primitives");
    return s.nodeCount;
}

}  // namespace owec
