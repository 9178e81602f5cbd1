// hk_trace.cu -- KD-tree traversal kernels (sm_100a).
//
// One persistent kernel per traversal variant. Each warp takes 32 rays at a
// time from a global counter (atomicAdd by lane 0, broadcast with
// __shfl_sync), so the grid is sized to the SM count rather than the ray
// count and uneven ray batches balance themselves. Traversal semantics follow
// the reference kernels exactly (comparison operators, near/far rule, the
// "child 0" sentinel, strict < between hits in leaf order); see the comments
// at each variant. Closest-hit single-scene launches test the leaves of a
// whole warp together (coop_leaf), which keeps the same hits bit for bit.
#include "hk_common.cuh"
#include "hk_internal.h"

namespace hk {

struct TraceArgs {
    const uint2 *nodes;       // compact nodes
    const uint32_t *refs;     // leaf references (triangle indices)
    const TriRec *tris;       // per-triangle records
    const float4 *rays;       // n x (o, d)
    hk_hit *hits;             // n
    uint32_t n;
    const uint32_t *n_dev;    // device-side ray count (overrides n when set)
    uint32_t ntris;
    const float *box;         // scene box, device memory (min4, max4)
    uint32_t *fetch;          // ray-batch counter (zeroed before launch)
    unsigned long long *counters;  // node visits, refs, tests (when counting)
    uint32_t *err;            // error word (bounded loops)
    uint32_t stack_depth;     // ring depth for the short-stack variants
    uint32_t max_steps;       // per-ray iteration bound
    const uint32_t *ropes;    // ropes variant: 6 per node
    const float4 *cbox;       // ropes variant: cell min, max per node
    uint32_t rope_nn;         // compact node count (legs bound 4 n + 8) ...
    const uint32_t *rope_nn_dev;  // ... or its device copy
    // batch mode: many scenes in one launch
    uint32_t *leaf_out;            // ropes: per ray, the leaf its traversal ended in (or nullptr)
    const SceneDesc *scenes;
    const uint32_t *ray_offsets;   // nscenes + 1, ascending
    uint32_t nscenes;
    uint32_t *remaining;           // rays left per scene
    unsigned long long *done_ns;   // globaltimer when a scene's last ray finished
    unsigned long long *start_ns;  // globaltimer at launch start (min over CTAs)
};

// per-scene arrays a traversal reads
struct SceneView {
    const uint2 *nodes;
    const uint32_t *refs;
    const TriRec *tris;
    const uint32_t *ropes;
    const float4 *cbox;
};

// ---------------------------------------------------------------------------
// leaf test: KDTreeCPU::testNodePolygons (KDTreeCPU.cpp:255-283): triangles
// in leaf order, a hit replaces the best only when strictly closer. ANY
// (occlusion rays) returns at the first hit closer than lim.
// ---------------------------------------------------------------------------
template <bool COUNT, bool ANY = false>
__device__ __forceinline__ void test_leaf(const SceneView &A, uint2 leaf, float3 o, float3 d,
                                          float &best, int32_t &best_id, uint32_t &c_refs, float lim = 0.0f) {
    uint32_t start = leaf.x >> 2, cnt = leaf.y;
    // the next reference index is loaded while the current triangle is tested
    uint32_t tri = cnt ? __ldg(&A.refs[start]) : 0u;
    for (uint32_t i = 0; i < cnt; i++) {
        const uint32_t next = i + 1 < cnt ? __ldg(&A.refs[start + i + 1]) : 0u;
        float t = isect_tri(&A.tris[tri], o, d, best);
        if (t < best) {
            best = t;
            best_id = (int32_t)tri;
            if (ANY && best < lim) {
                if (COUNT) c_refs += i + 1;
                return;
            }
        }
        tri = next;
    }
    if (COUNT) c_refs += cnt;
}

__device__ __forceinline__ float comp(float3 v, uint32_t a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// child selection result: node index (0 = the reference's "no child", i.e.
// the root) and the node itself
__device__ __forceinline__ void pick_child(const uint2 *nodes, uint32_t pair, bool take_below,
                                           uint32_t &idx, uint2 &node, uint2 root) {
    uint32_t c = take_below ? pair : pair + 1;
    uint2 n = nodes[c];
    if (is_leaf(n) && n.y == 0) {
        idx = 0;
        node = root;
    } else {
        idx = c;
        node = n;
    }
}

__device__ __forceinline__ uint32_t sentinel_to_root(const uint2 *nodes, uint32_t c) {
    uint2 n = nodes[c];
    return (is_leaf(n) && n.y == 0) ? 0u : c;
}

// ---------------------------------------------------------------------------
// persistent driver with per-lane refill
//
// Every lane keeps its ray's traversal state across iterations of the warp
// loop. One iteration runs one "leg" per active lane: pop (or restart at the
// root), descend to a leaf, test it. A lane whose ray is finished writes its
// hit and takes a new ray at the next iteration: the warp counts its idle
// lanes with __ballot_sync, lane 0 takes that many rays with one atomicAdd
// and each idle lane picks its own by rank. Rays of different cost therefore
// no longer hold a warp hostage until the slowest of 32 finishes.
// ---------------------------------------------------------------------------
struct LaneState {
    float3 o, d, inv;
    float te, tmin, tmax, best;
    float lim;         // occlusion rays: the light distance
    int32_t best_id;
    uint32_t cur;
    uint2 node;
    int size, idx;     // ring (short stack) / todo count (full stack)
    uint32_t ray;
};

// A leg run with DEFER leaves its leaf test to the warp (coop_leaf): it
// records the leaf's reference run and what follows the test -- kDoneIfCloser:
// finished when the closest hit precedes tmax; kGoOn: not finished; kDone:
// finished.
enum : int { kNoTest = 0, kDoneIfCloser = 2, kGoOn = 3, kDone = 4 };
struct Defer {
    uint32_t start, cnt;
    int after;
};

// one leg of the ring short stack (KDTreeCPU::searchKDTreeStackless,
// KDTreeCPU.cpp:363-447; GPUTrace_shortStack.cl:6-105; GPUTrace_LDSshortStack.cl:
// 7-105 with the ring in shared memory, one column per thread); true = finished
template <bool SMEM, bool COUNT, bool ANY, bool DEFER = false>
__device__ __forceinline__ bool leg_shortstack(const TraceArgs &A, const SceneView &V, LaneState &L, uint2 root, float *s_s, float *s_e,
                                               uint32_t *s_n, float *l_s, float *l_e, uint32_t *l_n,
                                               uint32_t &c_nodes, uint32_t &c_refs, uint32_t &steps, Defer *df = nullptr) {
    const uint32_t D = A.stack_depth, stride = blockDim.x, tid = threadIdx.x;
    if (!(L.tmax < L.te)) return true;
    if (L.size == 0) {
        L.cur = 0;
        L.node = root;
        L.tmin = L.tmax;
        L.tmax = L.te;
    } else {
        --L.size;
        --L.idx;
        if (L.idx == -1) L.idx += (int)D;
        if (SMEM) {
            L.tmin = s_s[L.idx * stride + tid];
            L.tmax = s_e[L.idx * stride + tid];
            L.cur = s_n[L.idx * stride + tid];
        } else {
            L.tmin = l_s[L.idx];
            L.tmax = l_e[L.idx];
            L.cur = l_n[L.idx];
        }
        L.node = V.nodes[L.cur];
    }
    while (!is_leaf(L.node)) {
        if (COUNT) c_nodes++;
        if (++steps > A.max_steps) {
            atomicOr(A.err, 1u);
            return true;
        }
        uint32_t axis = L.node.x & 3u, pair = L.node.x >> 2;
        float pl = __int_as_float(L.node.y);
        float rs = comp(L.o, axis), dc = comp(L.d, axis);
        float split = __fmul_rn(__fsub_rn(pl, rs), comp(L.inv, axis));
        bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
        if (split >= L.tmax || split <= 0.0f) {
            pick_child(V.nodes, pair, below_first, L.cur, L.node, root);
        } else if (split <= L.tmin) {
            pick_child(V.nodes, pair, !below_first, L.cur, L.node, root);
        } else {
            uint32_t second = sentinel_to_root(V.nodes, below_first ? pair + 1 : pair);
            if (SMEM) {
                s_s[L.idx * stride + tid] = split;
                s_e[L.idx * stride + tid] = L.tmax;
                s_n[L.idx * stride + tid] = second;
            } else {
                l_s[L.idx] = split;
                l_e[L.idx] = L.tmax;
                l_n[L.idx] = second;
            }
            L.idx = (L.idx + 1) % (int)D;
            L.size++;
            L.size = L.size > (int)D ? (int)D : L.size;
            pick_child(V.nodes, pair, below_first, L.cur, L.node, root);
            L.tmax = split;
        }
        if (L.cur == 0) break;
    }
    if (is_leaf(L.node)) {
        if (COUNT) c_nodes++;
        if constexpr (DEFER) {
            *df = Defer{L.node.x >> 2, L.node.y, kDoneIfCloser};
            return false;
        }
        test_leaf<COUNT, ANY>(V, L.node, L.o, L.d, L.best, L.best_id, c_refs, L.lim);
        if (L.best < L.tmax || (ANY && L.best < L.lim)) return true;
    }
    return false;
}

// one leg of the full stack (KDTreeCPU::searchKDTree, KDTreeCPU.cpp:285-361 ==
// GPUTrace.cl:6-90; far children pushed only when they exist), run until a leaf
// has been tested; true = finished
template <bool COUNT, bool ANY, bool DEFER = false>
__device__ __forceinline__ bool leg_fullstack(const TraceArgs &A, const SceneView &V, LaneState &L, uint2 root, float *st_s, float *st_e,
                                              uint32_t *st_n, int max_stack, uint32_t &c_nodes, uint32_t &c_refs,
                                              uint32_t &steps, Defer *df = nullptr) {
    while (true) {
        if (L.best < L.tmin) return true;
        if (COUNT) c_nodes++;
        if (++steps > A.max_steps) {
            atomicOr(A.err, 1u);
            return true;
        }
        bool tested = false;
        if (is_leaf(L.node)) {
            if constexpr (DEFER) {
                // the stack pop below does not depend on the test's outcome
                *df = Defer{L.node.x >> 2, L.node.y, kGoOn};
            } else {
                test_leaf<COUNT, ANY>(V, L.node, L.o, L.d, L.best, L.best_id, c_refs, L.lim);
                if (ANY && L.best < L.lim) return true;
            }
            L.cur = 0;
            tested = true;
        } else {
            uint32_t axis = L.node.x & 3u, pair = L.node.x >> 2;
            float pl = __int_as_float(L.node.y);
            float rs = comp(L.o, axis), dc = comp(L.d, axis);
            float split = __fmul_rn(__fsub_rn(pl, rs), comp(L.inv, axis));
            bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
            if (split > L.tmax || split <= 0.0f) {
                pick_child(V.nodes, pair, below_first, L.cur, L.node, root);
            } else if (split < L.tmin) {
                pick_child(V.nodes, pair, !below_first, L.cur, L.node, root);
            } else {
                uint32_t second = sentinel_to_root(V.nodes, below_first ? pair + 1 : pair);
                if (second != 0 && L.size < max_stack) {
                    st_n[L.size] = second;
                    st_s[L.size] = split;
                    st_e[L.size] = L.tmax;
                    L.size++;
                }
                pick_child(V.nodes, pair, below_first, L.cur, L.node, root);
                L.tmax = split;
            }
        }
        if (L.cur == 0 && L.size > 0) {
            L.size--;
            L.tmin = st_s[L.size];
            L.tmax = st_e[L.size];
            L.cur = st_n[L.size];
            L.node = V.nodes[L.cur];
        }
        if (L.cur == 0) {
            if (DEFER && tested) df->after = kDone;
            return true;
        }
        if (tested) return false;
    }
}

// one leg of kd-restart (GPUTrace_stackless.cl:53-117 with every leaf resident;
// EARLY adds the resume path's exit once the closest hit precedes tmax); true = finished
template <bool EARLY, bool COUNT, bool ANY, bool DEFER = false>
__device__ __forceinline__ bool leg_restart(const TraceArgs &A, const SceneView &V, LaneState &L, uint2 root, uint32_t &c_nodes,
                                            uint32_t &c_refs, uint32_t &steps, Defer *df = nullptr) {
    if (!(L.tmax < L.te)) return true;
    L.tmin = L.tmax;
    L.tmax = L.te;
    L.cur = 0;
    L.node = root;
    while (!is_leaf(L.node)) {
        if (COUNT) c_nodes++;
        if (++steps > A.max_steps) {
            atomicOr(A.err, 1u);
            return true;
        }
        uint32_t axis = L.node.x & 3u, pair = L.node.x >> 2;
        float pl = __int_as_float(L.node.y);
        float rs = comp(L.o, axis), dc = comp(L.d, axis);
        float split = __fmul_rn(__fsub_rn(pl, rs), comp(L.inv, axis));
        bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
        if (split >= L.tmax || split <= 0.0f) {
            pick_child(V.nodes, pair, below_first, L.cur, L.node, root);
        } else if (split <= L.tmin) {
            pick_child(V.nodes, pair, !below_first, L.cur, L.node, root);
        } else {
            pick_child(V.nodes, pair, below_first, L.cur, L.node, root);
            L.tmax = split;
        }
        if (L.cur == 0) break;
    }
    if (is_leaf(L.node)) {
        if (COUNT) c_nodes++;
        if constexpr (DEFER) {
            *df = Defer{L.node.x >> 2, L.node.y, EARLY ? kDoneIfCloser : kGoOn};
            return false;
        }
        test_leaf<COUNT, ANY>(V, L.node, L.o, L.d, L.best, L.best_id, c_refs, L.lim);
        if ((EARLY && L.best < L.tmax) || (ANY && L.best < L.lim)) return true;
    }
    return false;
}

// one leg of the ropes traversal (no reference counterpart; restated in the
// oracle's search_ropes): locate the leaf cell holding o + d*tentry from the
// current node (ties on a plane go to the side the ray moves into), test it,
// stop when the closest hit precedes the cell's exit, else follow the rope of
// the exit face. Legs are bounded by 4 * nodes + 8. ropes_locate does the
// descent and the exit face (true = the leg bound ran out), the leaf test
// follows, ropes_advance decides and follows the rope (true = finished).
template <bool COUNT>
__device__ __forceinline__ bool ropes_locate(const SceneView &A, LaneState &L, uint32_t legs_max, uint32_t &c_nodes,
                                             uint32_t &lstart, uint32_t &lcnt, float &texit, int &face) {
    if (++L.size > (int)legs_max) return true;
    float p[3] = {__fadd_rn(L.o.x, __fmul_rn(L.d.x, L.tmin)), __fadd_rn(L.o.y, __fmul_rn(L.d.y, L.tmin)),
                  __fadd_rn(L.o.z, __fmul_rn(L.d.z, L.tmin))};
    uint2 node = A.nodes[L.cur];
    while (!is_leaf(node)) {
        if (COUNT) c_nodes++;
        uint32_t axis = node.x & 3u, pair = node.x >> 2;
        float pl = __int_as_float(node.y);
        float pc = axis == 0 ? p[0] : (axis == 1 ? p[1] : p[2]);
        bool below = (pc < pl) || (pc == pl && comp(L.d, axis) <= 0.0f);
        L.cur = below ? pair : pair + 1;
        node = A.nodes[L.cur];
    }
    const float4 blo = A.cbox[2 * (size_t)L.cur], bhi = A.cbox[2 * (size_t)L.cur + 1];
    texit = L.te;
    face = -1;
    const float o3[3] = {L.o.x, L.o.y, L.o.z}, d3[3] = {L.d.x, L.d.y, L.d.z}, i3[3] = {L.inv.x, L.inv.y, L.inv.z};
    const float lo3[3] = {blo.x, blo.y, blo.z}, hi3[3] = {bhi.x, bhi.y, bhi.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (d3[k] > 0.0f) {
            float tt = __fmul_rn(__fsub_rn(hi3[k], o3[k]), i3[k]);
            if (tt < texit) {
                texit = tt;
                face = 2 * k + 1;
            }
        } else if (d3[k] < 0.0f) {
            float tt = __fmul_rn(__fsub_rn(lo3[k], o3[k]), i3[k]);
            if (tt < texit) {
                texit = tt;
                face = 2 * k;
            }
        }
    }
    if (COUNT) c_nodes++;
    lstart = node.x >> 2;
    lcnt = node.y;
    return false;
}

template <bool ANY>
__device__ __forceinline__ bool ropes_advance(const SceneView &A, LaneState &L, uint32_t lcnt, float texit, int face) {
    if (lcnt && (L.best < texit || (ANY && L.best < L.lim))) return true;
    if (face < 0) return true;
    uint32_t r = A.ropes[6 * (size_t)L.cur + face];
    if (r == 0xffffffffu) return true;
    L.tmin = texit > L.tmin ? texit : L.tmin;
    L.cur = r;
    return false;
}

// the whole leg with the in-order leaf test (occlusion rays, batches)
template <bool COUNT, bool ANY>
__device__ __forceinline__ bool leg_ropes(const SceneView &A, LaneState &L, uint32_t legs_max, uint32_t &c_nodes,
                                          uint32_t &c_refs) {
    if (++L.size > (int)legs_max) return true;
    float p[3] = {__fadd_rn(L.o.x, __fmul_rn(L.d.x, L.tmin)), __fadd_rn(L.o.y, __fmul_rn(L.d.y, L.tmin)),
                  __fadd_rn(L.o.z, __fmul_rn(L.d.z, L.tmin))};
    uint2 node = A.nodes[L.cur];
    while (!is_leaf(node)) {
        if (COUNT) c_nodes++;
        uint32_t axis = node.x & 3u, pair = node.x >> 2;
        float pl = __int_as_float(node.y);
        float pc = axis == 0 ? p[0] : (axis == 1 ? p[1] : p[2]);
        bool below = (pc < pl) || (pc == pl && comp(L.d, axis) <= 0.0f);
        L.cur = below ? pair : pair + 1;
        node = A.nodes[L.cur];
    }
    const float4 blo = A.cbox[2 * (size_t)L.cur], bhi = A.cbox[2 * (size_t)L.cur + 1];
    float texit = L.te;
    int face = -1;
    const float o3[3] = {L.o.x, L.o.y, L.o.z}, d3[3] = {L.d.x, L.d.y, L.d.z}, i3[3] = {L.inv.x, L.inv.y, L.inv.z};
    const float lo3[3] = {blo.x, blo.y, blo.z}, hi3[3] = {bhi.x, bhi.y, bhi.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (d3[k] > 0.0f) {
            float tt = __fmul_rn(__fsub_rn(hi3[k], o3[k]), i3[k]);
            if (tt < texit) {
                texit = tt;
                face = 2 * k + 1;
            }
        } else if (d3[k] < 0.0f) {
            float tt = __fmul_rn(__fsub_rn(lo3[k], o3[k]), i3[k]);
            if (tt < texit) {
                texit = tt;
                face = 2 * k;
            }
        }
    }
    if (COUNT) c_nodes++;
    if (node.y) {
        test_leaf<COUNT, ANY>(A, node, L.o, L.d, L.best, L.best_id, c_refs, L.lim);
        if (L.best < texit || (ANY && L.best < L.lim)) return true;
    }
    if (face < 0) return true;
    uint32_t r = A.ropes[6 * (size_t)L.cur + face];
    if (r == 0xffffffffu) return true;
    L.tmin = texit > L.tmin ? texit : L.tmin;
    L.cur = r;
    return false;
}

// The leaf tests of a whole warp shared out over its 32 lanes (all lanes call
// it; lane k brings its leaf's reference run start, cnt, with cnt = 0 when it
// has nothing to test). The warp's (ray, triangle) pairs are numbered in lane
// order, then leaf order; lane l takes pairs l, l + 32, ... and tests each
// against its ray's closest hit so far. Each ray keeps the least key
// (t without its sign bit, position in the leaf, sign bit) in a shared slot:
// t does not depend on the best hit it is tested against (that only culls),
// so this is the hit the in-order loop keeps -- the closest, the first in
// leaf order among equal t -- bit for bit.
__device__ __forceinline__ void coop_leaf(const SceneView &V, LaneState &L, uint32_t start, uint32_t cnt,
                                          unsigned long long *slot) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t P = cnt;   // inclusive prefix of the counts over the lanes
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, P, dd);
        if ((int)lane >= dd) P += u;
    }
    const uint32_t W = __shfl_sync(0xffffffffu, P, 31);
    if (W == 0) return;   // the same on every lane
    const uint32_t E = P - cnt;
    for (uint32_t base = 0; base < W; base += 32) {
        const uint32_t w = base + lane;
        // owner: the number of lanes whose inclusive prefix is <= w (P rises
        // and lane 31's exceeds every valid w, so this stays below 32)
        uint32_t owner = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1) {
            const uint32_t pv = __shfl_sync(0xffffffffu, P, owner + step - 1);
            if (pv <= w) owner += step;
        }
        const uint32_t j = w - __shfl_sync(0xffffffffu, E, owner);
        const uint32_t st = __shfl_sync(0xffffffffu, start, owner);
        const float3 o = make_float3(__shfl_sync(0xffffffffu, L.o.x, owner), __shfl_sync(0xffffffffu, L.o.y, owner),
                                     __shfl_sync(0xffffffffu, L.o.z, owner));
        const float3 d = make_float3(__shfl_sync(0xffffffffu, L.d.x, owner), __shfl_sync(0xffffffffu, L.d.y, owner),
                                     __shfl_sync(0xffffffffu, L.d.z, owner));
        const float best = __shfl_sync(0xffffffffu, L.best, owner);
        if (w < W) {
            const uint32_t tri = __ldg(&V.refs[st + j]);
            const float t = isect_tri(&V.tris[tri], o, d, best);
            if (t < best) {
                const uint32_t tb = __float_as_uint(t);
                const unsigned long long key =
                    ((unsigned long long)(tb & 0x7fffffffu) << 32) | ((unsigned long long)j << 1) | (tb >> 31);
                atomicMin(&slot[owner], key);
            }
        }
    }
    __syncwarp();
    const unsigned long long k = slot[lane];
    if (k != ~0ull) {
        slot[lane] = ~0ull;
        const uint32_t j = (uint32_t)(k >> 1) & 0x7fffffffu;
        L.best = __uint_as_float((uint32_t)(k >> 32) | ((uint32_t)(k & 1u) << 31));
        L.best_id = (int32_t)__ldg(&V.refs[start + j]);
    }
    __syncwarp();
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// scene of a ray in a batch: the last s with ray_offsets[s] <= rid
__device__ __forceinline__ uint32_t scene_of(const uint32_t *off, uint32_t nscenes, uint32_t rid) {
    uint32_t lo = 0, hi = nscenes;  // invariant off[lo] <= rid < off[hi]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(&off[mid]) <= rid) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ANY: occlusion rays (origin w = distance to the light). A ray stops at the
// first hit closer than that distance; until then its state is the closest-hit
// traversal's, so "some hit closer than the light" is found exactly when the
// closest-hit traversal's answer is closer than the light, in every variant.
template <int VARIANT, bool COUNT, bool BATCH, bool ANY>
__global__ void __launch_bounds__(kTraceMaxBlock, BATCH ? 4 : ((VARIANT != HK_TRACE_BRUTE && !ANY) ? 5 : 6))
    k_trace(TraceArgs A) {
    extern __shared__ float smem[];
    const bool smem_ring = (VARIANT == HK_TRACE_SMEMSTACK);
    float *s_s = smem;
    float *s_e = smem + A.stack_depth * blockDim.x;
    uint32_t *s_n = reinterpret_cast<uint32_t *>(smem + 2 * A.stack_depth * blockDim.x);
    constexpr int kLocal = (VARIANT == HK_TRACE_FULLSTACK) ? 64 : ((VARIANT == HK_TRACE_SHORTSTACK) ? 16 : 1);
    float l_s[kLocal], l_e[kLocal];
    uint32_t l_n[kLocal];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t c_nodes = 0, c_refs = 0;
    // single-scene closest-hit ropes: leaf tests shared out over the warp
    // (coop_leaf), one 8-byte slot per lane in dynamic shared memory. Occlusion
    // rays keep the in-order test, which stops at the first hit closer than
    // the light.
    constexpr bool COOP = VARIANT == HK_TRACE_ROPES && trace_coop_slots(VARIANT, BATCH, ANY);
    // the stack variants defer their leaf test to the same warp-wide pass
    constexpr bool COOP_LEG = VARIANT != HK_TRACE_ROPES && trace_coop_slots(VARIANT, BATCH, ANY);
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(
                                   smem + (smem_ring ? 3 * A.stack_depth * blockDim.x : 0u)) +
                               (threadIdx.x & ~31u);
    if (COOP || COOP_LEG) {
        slot[lane] = ~0ull;
        __syncwarp();
    }
    const uint32_t n = A.n_dev ? *A.n_dev : A.n;
    if (BATCH && threadIdx.x == 0) atomicMin(A.start_ns, global_ns());
    // scene arrays: launch-uniform for one scene, per lane in a batch
    SceneView V{A.nodes, A.refs, A.tris, A.ropes, A.cbox};
    float bmin[3], bmax[3];
    uint2 root = make_uint2(kLeafTag, 0);
    uint32_t legs_max = 0, ntris = A.ntris, scene = 0;
    if (!BATCH) {
        for (int k = 0; k < 3; k++) {
            bmin[k] = A.box[k];
            bmax[k] = A.box[4 + k];
        }
        root = A.nodes[0];
        legs_max = VARIANT == HK_TRACE_ROPES ? 4u * (A.rope_nn_dev ? *A.rope_nn_dev : A.rope_nn) + 8u : 0u;
    }
    LaneState L;
    if (COOP || COOP_LEG) {
        // an idle lane's ray fields are shuffled (and ignored) in coop_leaf
        L.o = L.d = make_float3(0.0f, 0.0f, 0.0f);
        L.best = kInf;
    }
    bool active = false, drained = false;
    uint32_t steps = 0;
    while (true) {
        // refill idle lanes
        uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (idle && !drained) {
            uint32_t want = __popc(idle);
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(A.fetch, want);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base + want >= n) drained = true;
            if (!active) {
                uint32_t rid = base + __popc(idle & lt_mask);
                if (rid < n) {
                    if (BATCH) {
                        // only the scene index stays with the lane; the scene's
                        // arrays are looked up again at every leg (L1-resident)
                        scene = scene_of(A.ray_offsets, A.nscenes, rid);
                        const SceneDesc &D = A.scenes[scene];
                        for (int k = 0; k < 3; k++) {
                            bmin[k] = D.box[k];
                            bmax[k] = D.box[4 + k];
                        }
                        // the full stack starts its ray at this scene's root
                        if (VARIANT == HK_TRACE_FULLSTACK) root = D.nodes[0];
                    }
                    float4 ro = A.rays[2 * (size_t)rid], rd = A.rays[2 * (size_t)rid + 1];
                    L.o = make_float3(ro.x, ro.y, ro.z);
                    L.d = make_float3(rd.x, rd.y, rd.z);
                    L.ray = rid;
                    L.best = kInf;
                    L.best_id = -1;
                    L.lim = ANY ? ro.w : 0.0f;
                    steps = 0;
                    if (VARIANT == HK_TRACE_BRUTE) {
                        active = true;
                    } else {
                        float ts = 0.0f, te = kInf;
                        if (ray_box(bmin, bmax, L.o, L.d, ts, te)) {
                            // invDir = 1 / rayDir (KDTreeCPU.cpp:293): correctly rounded reciprocal
                            L.inv = make_float3(__frcp_rn(L.d.x), __frcp_rn(L.d.y), __frcp_rn(L.d.z));
                            L.te = te;
                            L.size = 0;
                            L.idx = 0;
                            if (VARIANT == HK_TRACE_FULLSTACK) {
                                L.tmin = ts;
                                L.tmax = te;
                                L.cur = 0;
                                L.node = root;
                            } else if (VARIANT == HK_TRACE_ROPES) {
                                L.tmin = ts;  // entry distance
                                L.cur = 0;
                                // an occlusion ray may name in its direction's w lane a
                                // leaf to start from: taken when the start point lies
                                // strictly inside the leaf's cell, where the descent
                                // from the root would end as well
                                const uint32_t hint = __float_as_uint(rd.w);
                                if (ANY && hint != 0u && hint < (legs_max - 8u) / 4u && is_leaf(V.nodes[hint])) {
                                    const float4 c0 = V.cbox[2 * (size_t)hint], c1 = V.cbox[2 * (size_t)hint + 1];
                                    const float px = __fadd_rn(L.o.x, __fmul_rn(L.d.x, ts));
                                    const float py = __fadd_rn(L.o.y, __fmul_rn(L.d.y, ts));
                                    const float pz = __fadd_rn(L.o.z, __fmul_rn(L.d.z, ts));
                                    if (c0.x < px && px < c1.x && c0.y < py && py < c1.y && c0.z < pz && pz < c1.z)
                                        L.cur = hint;
                                }
                            } else if (VARIANT == HK_TRACE_RESTART || VARIANT == HK_TRACE_RESTART_EARLY) {
                                L.tmin = 0.0f;   // ThreadContext starts zeroed (GPUTrace_stackless.cl:98-100)
                                L.tmax = 0.0f;
                            } else {
                                L.tmin = ts;
                                L.tmax = ts;
                            }
                            active = true;
                        } else {
                            A.hits[rid] = hk_hit{kInf, -1};
                            if (BATCH && atomicSub(&A.remaining[scene], 1u) == 1u) A.done_ns[scene] = global_ns();
                        }
                    }
                }
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0) {
            if (drained) break;
            continue;
        }
        if (!COOP && !COOP_LEG && !active) continue;
        if (COOP) {
            // every lane takes part in the warp's leaf tests
            uint32_t lstart = 0, lcnt = 0;
            float texit = 0.0f;
            int face = -1;
            bool fin = false;
            if (active) fin = ropes_locate<COUNT>(V, L, legs_max, c_nodes, lstart, lcnt, texit, face);
            const uint32_t work = (active && !fin) ? lcnt : 0u;
            coop_leaf(V, L, lstart, work, slot);
            if (COUNT) c_refs += work;
            if (!active) continue;
            if (fin || ropes_advance<ANY>(V, L, lcnt, texit, face)) {
                A.hits[L.ray] = hk_hit{L.best, L.best_id};
                if (A.leaf_out) A.leaf_out[L.ray] = L.cur;
                active = false;
            }
            continue;
        }
        if (COOP_LEG) {
            // the leg runs up to its leaf, the warp tests every lane's leaf,
            // then each lane applies what its leg said follows the test
            Defer df{0u, 0u, kNoTest};
            bool fin = false;
            if (active) {
                if (VARIANT == HK_TRACE_FULLSTACK)
                    fin = leg_fullstack<COUNT, ANY, true>(A, V, L, root, l_s, l_e, l_n, kLocal, c_nodes, c_refs,
                                                          steps, &df);
                else if (VARIANT == HK_TRACE_RESTART)
                    fin = leg_restart<false, COUNT, ANY, true>(A, V, L, root, c_nodes, c_refs, steps, &df);
                else if (VARIANT == HK_TRACE_RESTART_EARLY)
                    fin = leg_restart<true, COUNT, ANY, true>(A, V, L, root, c_nodes, c_refs, steps, &df);
                else
                    fin = leg_shortstack<smem_ring, COUNT, ANY, true>(A, V, L, root, s_s, s_e, s_n, l_s, l_e, l_n,
                                                                      c_nodes, c_refs, steps, &df);
            }
            const uint32_t work = (active && df.after != kNoTest) ? df.cnt : 0u;
            coop_leaf(V, L, df.start, work, slot);
            if (COUNT) c_refs += work;
            if (!active) continue;
            if (fin || df.after == kDone || (df.after == kDoneIfCloser && L.best < L.tmax)) {
                A.hits[L.ray] = hk_hit{L.best, L.best_id};
                active = false;
            }
            continue;
        }
        if (BATCH) {
            const SceneDesc &D = A.scenes[scene];
            V = SceneView{D.nodes, D.refs, D.tris, D.ropes, D.cbox};
            legs_max = 4u * D.nn + 8u;
            ntris = D.ntris;
            if (VARIANT != HK_TRACE_ROPES && VARIANT != HK_TRACE_BRUTE) root = V.nodes[0];
        }
        bool done;
        if (VARIANT == HK_TRACE_BRUTE) {
            // GPUTrace_bruteforce.cl:30-42: every triangle in index order
            for (uint32_t t = 0; t < ntris; t++) {
                float h = isect_tri(&V.tris[t], L.o, L.d, L.best);
                if (h < L.best) {
                    L.best = h;
                    L.best_id = (int32_t)t;
                    if (ANY && L.best < L.lim) break;
                }
            }
            if (COUNT) c_refs += ntris;
            done = true;
        } else if (VARIANT == HK_TRACE_FULLSTACK) {
            done = leg_fullstack<COUNT, ANY>(A, V, L, root, l_s, l_e, l_n, kLocal, c_nodes, c_refs, steps);
        } else if (VARIANT == HK_TRACE_ROPES) {
            done = leg_ropes<COUNT, ANY>(V, L, legs_max, c_nodes, c_refs);
        } else if (VARIANT == HK_TRACE_RESTART) {
            done = leg_restart<false, COUNT, ANY>(A, V, L, root, c_nodes, c_refs, steps);
        } else if (VARIANT == HK_TRACE_RESTART_EARLY) {
            done = leg_restart<true, COUNT, ANY>(A, V, L, root, c_nodes, c_refs, steps);
        } else {
            done = leg_shortstack<smem_ring, COUNT, ANY>(A, V, L, root, s_s, s_e, s_n, l_s, l_e, l_n, c_nodes, c_refs,
                                                    steps);
        }
        if (done) {
            A.hits[L.ray] = hk_hit{L.best, L.best_id};
            if (VARIANT == HK_TRACE_ROPES && !BATCH && A.leaf_out) A.leaf_out[L.ray] = L.cur;
            active = false;
            if (BATCH && atomicSub(&A.remaining[scene], 1u) == 1u) A.done_ns[scene] = global_ns();
        }
    }
    if (COUNT) {
        atomicAdd(&A.counters[0], (unsigned long long)c_nodes);
        atomicAdd(&A.counters[1], (unsigned long long)c_refs);
        atomicAdd(&A.counters[2], (unsigned long long)c_refs);
    }
}

// occlusion launches take the any-hit instantiation unless they count (the
// counting one is the closest-hit kernel, which gives the same shading)
template <int V>
static cudaError_t launch_v(const TraceArgs &a, bool count, bool occlusion, int grid, int block, size_t smem,
                            cudaStream_t s) {
    if (a.scenes) {
        if (count)
            k_trace<V, true, true, false><<<grid, block, smem, s>>>(a);
        else
            k_trace<V, false, true, false><<<grid, block, smem, s>>>(a);
    } else if (count) {
        k_trace<V, true, false, false><<<grid, block, smem, s>>>(a);
    } else if (occlusion) {
        k_trace<V, false, false, true><<<grid, block, smem, s>>>(a);
    } else {
        k_trace<V, false, false, false><<<grid, block, smem, s>>>(a);
    }
    return cudaGetLastError();
}

template <int V>
static cudaError_t preload_v() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_trace<V, false, false, false>);
    return e == cudaSuccess ? cudaFuncGetAttributes(&fa, k_trace<V, false, false, true>) : e;
}

cudaError_t preload_trace_kernels(int variant) {
    switch (variant) {
    case HK_TRACE_FULLSTACK: return preload_v<HK_TRACE_FULLSTACK>();
    case HK_TRACE_SHORTSTACK: return preload_v<HK_TRACE_SHORTSTACK>();
    case HK_TRACE_SMEMSTACK: return preload_v<HK_TRACE_SMEMSTACK>();
    case HK_TRACE_RESTART: return preload_v<HK_TRACE_RESTART>();
    case HK_TRACE_RESTART_EARLY: return preload_v<HK_TRACE_RESTART_EARLY>();
    case HK_TRACE_ROPES: return preload_v<HK_TRACE_ROPES>();
    case HK_TRACE_BRUTE: return preload_v<HK_TRACE_BRUTE>();
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_trace(const TraceLaunch &L, cudaStream_t s) {
    TraceArgs a;
    a.nodes = L.nodes;
    a.refs = L.refs;
    a.tris = L.tris;
    a.rays = L.rays;
    a.hits = L.hits;
    a.n = L.n;
    a.n_dev = L.n_dev;
    a.ntris = L.ntris;
    a.box = L.box;
    a.fetch = L.fetch;
    a.counters = L.counters;
    a.err = L.err;
    a.stack_depth = L.stack_depth;
    a.max_steps = L.max_steps;
    a.ropes = L.ropes;
    a.cbox = L.cbox;
    a.rope_nn = L.rope_nn;
    a.rope_nn_dev = L.rope_nn_dev;
    a.leaf_out = L.leaf_out;
    a.scenes = L.scenes;
    a.ray_offsets = L.ray_offsets;
    a.nscenes = L.nscenes;
    a.remaining = L.remaining;
    a.done_ns = L.done_ns;
    a.start_ns = L.start_ns;
    cudaError_t e = cudaMemsetAsync(L.fetch, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (L.n == 0 && L.n_dev == nullptr) return cudaSuccess;
    int block = L.block;
    int grid = L.grid;
    const size_t smem =
        trace_smem_bytes(L.variant, (uint32_t)block, L.stack_depth, L.scenes != nullptr, L.occlusion, L.count);
    if (block < 32 || (uint32_t)block > kTraceMaxBlock || smem > kTraceMaxSmem) return cudaErrorInvalidConfiguration;
    switch (L.variant) {
    case HK_TRACE_FULLSTACK: return launch_v<HK_TRACE_FULLSTACK>(a, L.count, L.occlusion, grid, block, smem, s);
    case HK_TRACE_SHORTSTACK: return launch_v<HK_TRACE_SHORTSTACK>(a, L.count, L.occlusion, grid, block, smem, s);
    case HK_TRACE_SMEMSTACK: return launch_v<HK_TRACE_SMEMSTACK>(a, L.count, L.occlusion, grid, block, smem, s);
    case HK_TRACE_RESTART: return launch_v<HK_TRACE_RESTART>(a, L.count, L.occlusion, grid, block, smem, s);
    case HK_TRACE_RESTART_EARLY: return launch_v<HK_TRACE_RESTART_EARLY>(a, L.count, L.occlusion, grid, block, smem, s);
    case HK_TRACE_ROPES:
        if (!L.scenes && (!L.ropes || !L.cbox)) return cudaErrorInvalidValue;
        return launch_v<HK_TRACE_ROPES>(a, L.count, L.occlusion, grid, block, smem, s);
    case HK_TRACE_BRUTE: return launch_v<HK_TRACE_BRUTE>(a, L.count, L.occlusion, grid, block, smem, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace hk
