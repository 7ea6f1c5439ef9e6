// Device construction of the 8-wide quantised BVH (bvh_build.cu).
#pragma once

#include "dbuf.hpp"
#include "device_scene.cuh"

namespace owec {

// Working memory of a build, kept by the context between builds (a refit of a deformed heightfield
// rebuilds with the same sizes and allocates nothing).
struct BvhScratch {
    DBuf<uint64_t> keys, keysAlt;
    DBuf<uint32_t> vals, valsAlt;
    DBuf<uint8_t> cubTemp;
    DBuf<int2> children, ranges;
    DBuf<uint32_t> parents, counts, flags, counters;
    DBuf<float4> boxLo, boxHi;
    DBuf<uint2> work, next;
    DBuf<int> bounds;
    uint32_t nodeCount = 0, placedPrims = 0;
};

// Builds the wide BVH over n primitive boxes (camera-relative, padded outward). Fills `nodes`
// (wide node 0 is the root) and `leafOrder` (the primitive of every leaf slot). Returns the node
// count. Synchronises `stream`.
uint32_t buildWideBvh(const float4* primLo, const float4* primHi, uint32_t n, BvhScratch& s, DBuf<WideNode>& nodes,
                      DBuf<uint32_t>& leafOrder, cudaStream_t stream);

}  // namespace owec
