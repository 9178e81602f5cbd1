// hk_build.h -- GPU KD-tree builder state (binned SAH and the learned
// split proposer). Every launch reads its work size from device memory, so a
// whole build is a fixed sequence of kernels that a CUDA graph can capture.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/hulkcuda.h"
#include "hk_mlp.h"

namespace hk {

struct BuildParams {
    float ct = 1.0f, ci = 1.5f;
    uint32_t max_depth = 24;
    uint32_t leaf_size = 4;
    uint32_t max_refs = 0;      // reference arena (also the leaf list) capacity
    int mode = 0;               // hk_build_mode
    uint32_t topk = 4;
    float fallback_ratio = 1.02f;
    int record = 0;             // binned mode with exact_max >= 33: append (features, label) rows of
                                // the exactly searched nodes of 33..1024 references
    uint32_t exact_max = 0;     // nodes with at most this many refs (0, or 32..1024) take the exact SAH
    int prop_log = 0;           // learned mode: log every proposer row's proposed bins by compact node
    uint32_t spin_limit = 0;    // polls before a bounded wait gives up (0: the default, 4M)
    uint32_t debug_flags = 0;   // test aid, bit 0: plan tile 0 of level 1 withholds its done flag
    uint32_t defer = 32;        // nodes of 2..defer references: subtrees built after the levels (0: none)
    uint32_t defer_margin = 8;  // ... when within defer_margin levels of max_depth (0: any level)
    uint32_t level_streams = 1; // binned: 1 = k_decide per level, 2 = k_hist on a second stream beside k_small
};

// learned-proposer buffers owned by the context (device pointers)
struct LearnBuffers {
    MlpDevice mlp{};
    bool have_mlp = false;
    float *rec_X = nullptr;      // recorded features [cap][200]
    int32_t *rec_y = nullptr;    // recorded labels (axis * 32 + plane index)
    uint32_t *rec_rows = nullptr;
    uint32_t rec_cap = 0;
};

constexpr int kMaxLevels = 52;  // max_depth <= 48, plus the level after the last

// the binned SAH's decision for a proposer row (axis -1: leaf, or no plane
// when cost is infinite)
struct LearnBin {
    float cost, plane;
    int32_t axis;
    uint32_t nb, na, pad[3];
};

// counters of one tree level; level L's kernels read lvl[L] and the plan
// scan that emits its children writes lvl[L + 1], so no bookkeeping launch
// is needed
struct LevelCounters {
    uint32_t nodes;             // active nodes of the level
    uint32_t refs;              // their references
    uint32_t nodes_total;       // compact nodes written before this level
    uint32_t leafrefs_total;    // leaf references written before this level
    uint32_t defer_refs_total;  // references of the deferred subtree roots recorded before this level
    uint32_t defer_nodes_total; // deferred subtree roots recorded before this level
    uint32_t stop;              // the level stops splitting (capacity)
    uint32_t n_large;           // large nodes (chunked histograms)
    uint32_t n_chunks;          // histogram chunks
    uint32_t n_medium;          // exact-SAH nodes of 33..exact_max refs (one CTA each)
    uint32_t n_learn;           // learned mode: proposer rows of the level (nodes of 33..1024 refs)
    // tallies of the level's decisions (the capacity guard's inputs)
    uint32_t t_leafrefs, t_leafnodes, t_splits, t_next, t_childrefs, t_deferrefs, t_defernodes;
    // tile tickets of the single-pass scans; level 0's sub_ticket: the
    // subtree tickets of the deferred roots
    uint32_t plan_ticket, ref_ticket, sub_ticket;
};

// device scalars of one build (one struct in device memory)
struct BuildCounters {
    uint32_t depth;             // deepest level reached
    uint32_t leaves;            // leaves written (empty cells excluded)
    uint32_t capacity_hit;
    uint32_t learned_nodes;
    uint32_t fallback_nodes;
    // deferred subtrees (built after the levels, one warp each)
    uint32_t sub_leaves;        // leaves of the subtrees (empty cells excluded)
    uint32_t sub_depth;         // deepest subtree node
    uint32_t sub_overflow;      // a scratch arena ran out (the roots then stay leaves)
    uint32_t sc_node_ctr, sc_ref_ctr;   // scratch slots handed out (in chunks)
    uint32_t sub_ticket;        // tile tickets of the subtree-size scan
    uint32_t sub_fits;          // 1: the subtrees are placed; 0: the roots stay leaves
    uint32_t sub_n0, sub_r0;    // nodes / leaf references of the levels (where the subtrees start)
    uint32_t sub_nodes, sub_refs;   // the subtrees' nodes and leaf references
    uint32_t pad[3];
    LevelCounters lvl[kMaxLevels];
};

struct BuildOutputs {
    uint2 *nodes;
    uint32_t *refs;
};

struct BuildState {
    BuildParams p{};
    uint32_t nt = 0, cap_refs = 0, cap_nodes = 0, cap_level = 0, cap_large = 0, cap_chunks = 0, cap_medium = 0;
    uint32_t alloc_depth = 0;   // max_depth the subtree scratch was sized for

    int sm_count = 148;
    bool active = false;        // a built tree is the current tree
    uint32_t last_level = 0;    // lvl[] index holding the final totals
    uint32_t last_err = 0;      // error bits of the last build: 2 arena capacity, 4 scan wait ran
                                // out, 8 partition / decision count mismatch, 16 plan bounds
    // per-triangle bounds
    float4 *tb_lo = nullptr, *tb_hi = nullptr;
    // level nodes (ping-pong)
    float4 *n_lo[2] = {nullptr, nullptr}, *n_hi[2] = {nullptr, nullptr};
    uint4 *n_info[2] = {nullptr, nullptr};      // start, count, cidx, -
    // decision per node
    int32_t *d_axis = nullptr;
    float *d_plane = nullptr;
    uint2 *d_cnt = nullptr;                      // below, above
    float4 *d_split = nullptr;                   // axis bits, plane, node min / max on the axis
    uint4 *d_scat = nullptr;                     // reference destinations (plan scan)
    uint2 *chunks = nullptr;                     // (large rank, chunk index); tail: large_slot
    uint32_t *hist = nullptr;                    // per large node 3 x 96
    uint32_t *done = nullptr;                    // per large node: chunks finished
    uint32_t *medium_slot = nullptr;             // exact-SAH medium nodes of the level
    // references (ping-pong)
    uint32_t *refs[2] = {nullptr, nullptr};
    uint32_t *ref_node[2] = {nullptr, nullptr};
    // single-pass scan tile states (flags, aggregates, inclusive prefixes)
    uint32_t *plan_flags = nullptr, *ref_flags = nullptr;
    uint32_t *plan_done = nullptr;               // per plan tile: emitted (tag of the level)
    void *plan_agg = nullptr, *plan_incl = nullptr;
    uint2 *ref_agg = nullptr, *ref_incl = nullptr;
    uint32_t plan_tiles = 0, ref_tiles = 0;
    uint32_t *epoch = nullptr;                   // build counter (scan flag tags)
    // second stream: large-node histograms run beside the small-node work;
    // third stream: the proposer's warp-costed rows beside its CTA-costed ones
    cudaStream_t aux = nullptr, aux2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_learn = nullptr, ev_join2 = nullptr;

    BuildCounters *ctr = nullptr;
    uint32_t *err = nullptr;
    // output
    uint2 *out_nodes = nullptr;
    uint32_t *out_refs = nullptr;
    uint32_t *out_ropes = nullptr;               // 6 per node: -x,+x,-y,+y,-z,+z (0xffffffff = none)
    float4 *out_cbox = nullptr;                  // 2 per node: cell min, max
    // deferred subtree roots (nodes of at most 32 references): their records
    // (compact index, reference offset, count, depth), cells and references
    uint32_t cap_defer = 0;
    uint4 *d_root = nullptr;
    float4 *d_lo = nullptr, *d_hi = nullptr;
    uint32_t *defer_refs = nullptr;
    // subtree scratch: node slots (subtree, local index), their entries, cells
    // and ropes; reference slots (subtree, local index, triangle); per subtree
    // its sizes, root entry and place
    uint32_t cap_sc_nodes = 0, cap_sc_refs = 0;
    uint2 *sc_key = nullptr, *sc_node = nullptr;
    float4 *sc_cbox = nullptr;
    uint32_t *sc_rope = nullptr;
    uint4 *sc_ref = nullptr;
    uint2 *st_cnt = nullptr, *st_root = nullptr, *st_base = nullptr;
    uint32_t sub_tiles = 0;
    uint32_t *sub_flags = nullptr;
    uint2 *sub_agg = nullptr, *sub_incl = nullptr;
    // learned proposer: per-level rows (nodes of 33..1024 references), their
    // node slots, binned decisions and features
    uint32_t cap_learn = 0;
    uint32_t *learn_slot = nullptr;              // row -> node slot
    LearnBin *learn_bin = nullptr;               // row -> the binned SAH's decision
    uint2 *learn_prop = nullptr;                 // row -> proposed bins (bytes, 0xff: none)
    float *feat = nullptr;                       // [cap_learn][200]
    int32_t *prop_log = nullptr;                 // [cap_nodes][8] proposed bins (axis * 32 + bin, -1: none)
    LearnBuffers *learn = nullptr;               // context-owned (weights, recording)
};

hk_status build_prepare(BuildState &S, const BuildParams &p, uint32_t nt, int sm_count);
hk_status build_ensure_outputs(BuildState &S, BuildOutputs *o);
cudaError_t build_launch(BuildState &S, const float4 *verts, const uint4 *tris, uint32_t nt, const float *box,
                         cudaStream_t s);
hk_status build_read_stats(BuildState &S, cudaStream_t s, hk_tree_stats *st);
// the learned level kernel's shared-memory opt-in on the current device
// (done once per device; call before capturing a graph that builds)
cudaError_t build_learn_setup();
// device address of the built tree's node count (valid once build_launch ran)
const uint32_t *build_nodes_total_ptr(const BuildState &S);
void build_release(BuildState &S);

}  // namespace hk
