// hk_resort.h -- the per-node re-sampling SAH builder (HK_BUILD_SAH_RESORT).
#pragma once
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/hulkcuda.h"

namespace hk {

struct ResortParams {
    float ct, ci;         // traversal / intersection cost
    uint32_t max_depth;   // a node at this depth is a leaf
    uint32_t leaf_size;   // a node of at most this many references is a leaf
    uint32_t sample;      // every sample-th reference of a node makes candidates
};

// growable device array owned by the builder
template <class T>
struct RBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n);
    void release();
};

struct ResortState {
    // per node of the current / next level
    RBuf<float4> lo[2], hi[2];
    RBuf<float> surf[2];
    RBuf<uint32_t> off[2], cnt[2], ropes[2];
    // per reference of the current / next level
    RBuf<uint32_t> refs[2], ref_node[2];
    // per node scratch
    RBuf<uint32_t> nkeys, koff, jflag, jrank, leafcnt, loff, efirst, decision;
    RBuf<float> plane, surf_lo, surf_hi;
    RBuf<unsigned long long> best;
    // keys, sort and sweep scratch
    RBuf<unsigned long long> keys[2], kscan_a, kscan_b, rscan, rflag;
    RBuf<uint32_t> hist, gfirst, scan_part;
    RBuf<unsigned long long> scan_part64;
    RBuf<uint32_t> dev_u32;   // small device scalars read back per level
    // output tree (compact layout, see hk_api.cu)
    RBuf<uint2> nodes;
    RBuf<uint32_t> out_refs, out_ropes;
    RBuf<float4> out_cbox;
    uint32_t nn = 0, nr = 0, depth = 0;
    void release();
};

// Builds the tree of the scene (verts, tris) in its box (host copy hbox[8])
// on stream st; on success S.nodes / out_refs / out_ropes / out_cbox hold
// S.nn compact nodes and S.nr leaf references.
hk_status resort_build(ResortState &S, const ResortParams &p, const float4 *verts, const uint4 *tris, uint32_t nt,
                       const float *hbox, cudaStream_t st, std::string *err);

}  // namespace hk
