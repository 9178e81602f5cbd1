// hk_stream.h -- out-of-core leaf geometry: leaves paged into a device pool on
// demand (HulkEngine/src/GPUTrace_stackless.cl:6-120 and
// GLVisitorGPUTrace::launchTraceIterations, GLVisitorGPUTrace.cpp:412-502).
#pragma once
#include <cstdint>
#include <deque>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/hulkcuda.h"
#include "hk_common.cuh"

namespace hk {

// a resident leaf: compact cell, pool offset, records
struct StreamEntry {
    uint32_t cell, off, size;
};

struct StreamState {
    // host: every leaf's triangle records in the tree's reference order
    // (pinned, mapped: the device reads them directly when it pages a leaf in)
    TriRec *h_recs = nullptr;
    const TriRec *d_hrecs = nullptr;
    size_t nrecs = 0;
    std::vector<uint2> nodes;   // the tree's compact nodes (leaf start / count)
    uint32_t nn = 0;
    uint64_t tree_epoch = 0, rec_epoch = 0;
    // the pool ring (records), leaves in load order
    uint32_t cap = 0, head = 0, tail = 0;
    bool wrapped = false;
    std::deque<StreamEntry> fifo;
    // device
    TriRec *pool = nullptr;
    uint32_t *res = nullptr;        // per cell: 0 absent, 1 requested, 2 resident
    uint32_t *pool_off = nullptr;   // per cell: pool offset of a resident leaf
    uint32_t *req = nullptr;        // requested cells of one launch (nn), then the count
    uint4 *loads = nullptr;         // (cell, pool offset, record start, count)
    uint32_t *evicts = nullptr;     // cells
    // per ray: the kd-restart resume state (ThreadContext) and completion
    float *tmin = nullptr, *tmax = nullptr;
    uint32_t *rnode = nullptr, *done = nullptr;
    size_t cap_rays = 0;
    bool ready = false;
    void release();
};

struct StreamTraceArgs {
    const uint2 *nodes;
    const uint32_t *refs;
    const float4 *rays;      // n x (o, d)
    hk_hit *hits;            // n
    uint32_t n;
    const float *box;        // device scene box
    uint32_t max_steps;
    uint32_t *err;
};

// Copies the current tree's leaf records to pinned host memory and sets up an
// empty pool of cap records.
hk_status stream_setup(StreamState &S, const uint2 *d_nodes, uint32_t nn, const uint32_t *d_refs, uint32_t nr,
                       const TriRec *d_recs, uint32_t cap, cudaStream_t st, std::string *err);
// kd-restart with paging: launch, page the requested leaves in, relaunch
// until no ray waits for a leaf.
hk_status stream_trace(StreamState &S, const StreamTraceArgs &a, cudaStream_t st, hk_stream_stats *stats,
                       std::string *err);

}  // namespace hk
