// hk_trace.cu -- KD-tree traversal kernels (sm_100a).
//
// One persistent kernel per traversal variant. Each warp takes 32 rays at a
// time from a global counter (atomicAdd by lane 0, broadcast with
// __shfl_sync), so the grid is sized to the SM count rather than the ray
// count and uneven ray batches balance themselves. Traversal semantics follow
// the reference kernels exactly (comparison operators, near/far rule, the
// "child 0" sentinel, strict < between hits in leaf order); see the comments
// at each variant.
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
};

// ---------------------------------------------------------------------------
// leaf test: KDTreeCPU::testNodePolygons (KDTreeCPU.cpp:255-283): triangles
// in leaf order, a hit replaces the best only when strictly closer.
// ---------------------------------------------------------------------------
template <bool COUNT>
__device__ __forceinline__ void test_leaf(const TraceArgs &A, uint2 leaf, float3 o, float3 d,
                                          float &best, int32_t &best_id, uint32_t &c_refs) {
    uint32_t start = leaf.x >> 2, cnt = leaf.y;
    for (uint32_t i = 0; i < cnt; i++) {
        uint32_t tri = __ldg(&A.refs[start + i]);
        float t = isect_tri(&A.tris[tri], o, d, best);
        if (t < best) {
            best = t;
            best_id = (int32_t)tri;
        }
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
// ring short stack: KDTreeCPU::searchKDTreeStackless (KDTreeCPU.cpp:363-447),
// GPUTrace_shortStack.cl:6-105 and GPUTrace_LDSshortStack.cl:7-105. The ring
// lives in local memory (SMEM = false) or in shared memory, one column per
// thread (SMEM = true).
// ---------------------------------------------------------------------------
template <bool SMEM, bool COUNT>
__device__ void trace_shortstack(const TraceArgs &A, float3 o, float3 d, float3 inv, float ts, float te,
                                 float &best, int32_t &best_id, uint32_t &c_nodes, uint32_t &c_refs,
                                 float *s_s, float *s_e, uint32_t *s_n) {
    constexpr int kMaxRing = 16;
    float l_s[SMEM ? 1 : kMaxRing], l_e[SMEM ? 1 : kMaxRing];
    uint32_t l_n[SMEM ? 1 : kMaxRing];
    const uint32_t D = A.stack_depth;
    const uint32_t stride = blockDim.x;
    const uint32_t tid = threadIdx.x;
    int size = 0, idx = 0;
    float tmin = ts, tmax = ts;
    const uint2 root = A.nodes[0];
    uint32_t steps = 0;
    while (tmax < te) {
        uint32_t cur;
        uint2 node;
        if (size == 0) {
            cur = 0;
            node = root;
            tmin = tmax;
            tmax = te;
        } else {
            --size;
            --idx;
            if (idx == -1) idx += (int)D;
            if (SMEM) {
                tmin = s_s[idx * stride + tid];
                tmax = s_e[idx * stride + tid];
                cur = s_n[idx * stride + tid];
            } else {
                tmin = l_s[idx];
                tmax = l_e[idx];
                cur = l_n[idx];
            }
            node = A.nodes[cur];
        }
        while (!is_leaf(node)) {
            if (COUNT) c_nodes++;
            if (++steps > A.max_steps) {
                atomicOr(A.err, 1u);
                return;
            }
            uint32_t axis = node.x & 3u, pair = node.x >> 2;
            float pl = __int_as_float(node.y);
            float rs = comp(o, axis), dc = comp(d, axis);
            float split = __fmul_rn(__fsub_rn(pl, rs), comp(inv, axis));
            bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
            if (split >= tmax || split <= 0.0f) {
                pick_child(A.nodes, pair, below_first, cur, node, root);
            } else if (split <= tmin) {
                pick_child(A.nodes, pair, !below_first, cur, node, root);
            } else {
                uint32_t second = sentinel_to_root(A.nodes, below_first ? pair + 1 : pair);
                if (SMEM) {
                    s_s[idx * stride + tid] = split;
                    s_e[idx * stride + tid] = tmax;
                    s_n[idx * stride + tid] = second;
                } else {
                    l_s[idx] = split;
                    l_e[idx] = tmax;
                    l_n[idx] = second;
                }
                idx = (idx + 1) % (int)D;
                size++;
                size = size > (int)D ? (int)D : size;
                pick_child(A.nodes, pair, below_first, cur, node, root);
                tmax = split;
            }
            if (cur == 0) break;
        }
        if (is_leaf(node)) {
            if (COUNT) c_nodes++;
            test_leaf<COUNT>(A, node, o, d, best, best_id, c_refs);
            if (best < tmax) break;
        }
    }
}

// ---------------------------------------------------------------------------
// full stack: KDTreeCPU::searchKDTree (KDTreeCPU.cpp:285-361) == GPUTrace.cl:
// 6-90. Far children are pushed only when they exist.
// ---------------------------------------------------------------------------
template <bool COUNT>
__device__ void trace_fullstack(const TraceArgs &A, float3 o, float3 d, float3 inv, float ts, float te,
                                float &best, int32_t &best_id, uint32_t &c_nodes, uint32_t &c_refs) {
    constexpr int kMaxStack = 64;
    float st_s[kMaxStack], st_e[kMaxStack];
    uint32_t st_n[kMaxStack];
    int todo = 0;
    float tmin = ts, tmax = te;
    const uint2 root = A.nodes[0];
    uint32_t cur = 0;
    uint2 node = root;
    uint32_t steps = 0;
    do {
        if (best < tmin) break;
        if (COUNT) c_nodes++;
        if (++steps > A.max_steps) {
            atomicOr(A.err, 1u);
            return;
        }
        if (is_leaf(node)) {
            test_leaf<COUNT>(A, node, o, d, best, best_id, c_refs);
            cur = 0;
        } else {
            uint32_t axis = node.x & 3u, pair = node.x >> 2;
            float pl = __int_as_float(node.y);
            float rs = comp(o, axis), dc = comp(d, axis);
            float split = __fmul_rn(__fsub_rn(pl, rs), comp(inv, axis));
            bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
            if (split > tmax || split <= 0.0f) {
                pick_child(A.nodes, pair, below_first, cur, node, root);
            } else if (split < tmin) {
                pick_child(A.nodes, pair, !below_first, cur, node, root);
            } else {
                uint32_t second = sentinel_to_root(A.nodes, below_first ? pair + 1 : pair);
                if (second != 0 && todo < kMaxStack) {
                    st_n[todo] = second;
                    st_s[todo] = split;
                    st_e[todo] = tmax;
                    todo++;
                }
                pick_child(A.nodes, pair, below_first, cur, node, root);
                tmax = split;
            }
        }
        if (cur == 0 && todo > 0) {
            todo--;
            tmin = st_s[todo];
            tmax = st_e[todo];
            cur = st_n[todo];
            node = A.nodes[cur];
        }
    } while (cur != 0);
}

// ---------------------------------------------------------------------------
// kd-restart: GPUTrace_stackless.cl:53-117 with every leaf resident. The
// ThreadContext starts zeroed, so the first descent runs with tmin = tmax = 0;
// EARLY adds the exit the resume path performs (closest hit before tmax).
// ---------------------------------------------------------------------------
template <bool EARLY, bool COUNT>
__device__ void trace_restart(const TraceArgs &A, float3 o, float3 d, float3 inv, float te, float &best,
                              int32_t &best_id, uint32_t &c_nodes, uint32_t &c_refs) {
    float tmax = 0.0f, tmin = 0.0f;
    const uint2 root = A.nodes[0];
    uint32_t steps = 0;
    while (tmax < te) {
        tmin = tmax;
        tmax = te;
        uint32_t cur = 0;
        uint2 node = root;
        while (!is_leaf(node)) {
            if (COUNT) c_nodes++;
            if (++steps > A.max_steps) {
                atomicOr(A.err, 1u);
                return;
            }
            uint32_t axis = node.x & 3u, pair = node.x >> 2;
            float pl = __int_as_float(node.y);
            float rs = comp(o, axis), dc = comp(d, axis);
            float split = __fmul_rn(__fsub_rn(pl, rs), comp(inv, axis));
            bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
            if (split >= tmax || split <= 0.0f) {
                pick_child(A.nodes, pair, below_first, cur, node, root);
            } else if (split <= tmin) {
                pick_child(A.nodes, pair, !below_first, cur, node, root);
            } else {
                pick_child(A.nodes, pair, below_first, cur, node, root);
                tmax = split;
            }
            if (cur == 0) break;
        }
        if (is_leaf(node)) {
            if (COUNT) c_nodes++;
            test_leaf<COUNT>(A, node, o, d, best, best_id, c_refs);
            if (EARLY && best < tmax) break;
        }
    }
}

// ---------------------------------------------------------------------------
// persistent driver
// ---------------------------------------------------------------------------
template <int VARIANT, bool COUNT>
__global__ void __launch_bounds__(1024) k_trace(TraceArgs A) {
    extern __shared__ float smem[];
    float *s_s = smem;
    float *s_e = smem + A.stack_depth * blockDim.x;
    uint32_t *s_n = reinterpret_cast<uint32_t *>(smem + 2 * A.stack_depth * blockDim.x);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t c_nodes = 0, c_refs = 0;
    const uint32_t n = A.n_dev ? *A.n_dev : A.n;
    const float bmin[3] = {A.box[0], A.box[1], A.box[2]};
    const float bmax[3] = {A.box[4], A.box[5], A.box[6]};
    while (true) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(A.fetch, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= n) break;
        uint32_t i = base + lane;
        if (i >= n) continue;
        float4 ro = A.rays[2 * (size_t)i], rd = A.rays[2 * (size_t)i + 1];
        float3 o = make_float3(ro.x, ro.y, ro.z), d = make_float3(rd.x, rd.y, rd.z);
        float best = kInf;
        int32_t best_id = -1;
        if (VARIANT == HK_TRACE_BRUTE) {
            // GPUTrace_bruteforce.cl:30-42: every triangle in index order
            for (uint32_t t = 0; t < A.ntris; t++) {
                float h = isect_tri(&A.tris[t], o, d, best);
                if (h < best) {
                    best = h;
                    best_id = (int32_t)t;
                }
            }
            if (COUNT) c_refs += A.ntris;
        } else {
            float ts = 0.0f, te = kInf;
            if (ray_box(bmin, bmax, o, d, ts, te)) {
                // invDir = 1 / rayDir (KDTreeCPU.cpp:293)
                float3 inv = make_float3(__fdiv_rn(1.0f, d.x), __fdiv_rn(1.0f, d.y), __fdiv_rn(1.0f, d.z));
                if (VARIANT == HK_TRACE_SHORTSTACK)
                    trace_shortstack<false, COUNT>(A, o, d, inv, ts, te, best, best_id, c_nodes, c_refs, s_s, s_e, s_n);
                else if (VARIANT == HK_TRACE_SMEMSTACK)
                    trace_shortstack<true, COUNT>(A, o, d, inv, ts, te, best, best_id, c_nodes, c_refs, s_s, s_e, s_n);
                else if (VARIANT == HK_TRACE_FULLSTACK)
                    trace_fullstack<COUNT>(A, o, d, inv, ts, te, best, best_id, c_nodes, c_refs);
                else if (VARIANT == HK_TRACE_RESTART)
                    trace_restart<false, COUNT>(A, o, d, inv, te, best, best_id, c_nodes, c_refs);
                else if (VARIANT == HK_TRACE_RESTART_EARLY)
                    trace_restart<true, COUNT>(A, o, d, inv, te, best, best_id, c_nodes, c_refs);
            }
        }
        hk_hit h;
        h.t = best;
        h.tri = best_id;
        A.hits[i] = h;
    }
    if (COUNT) {
        atomicAdd(&A.counters[0], (unsigned long long)c_nodes);
        atomicAdd(&A.counters[1], (unsigned long long)c_refs);
        atomicAdd(&A.counters[2], (unsigned long long)c_refs);
    }
}

template <int V>
static cudaError_t launch_v(const TraceArgs &a, bool count, int grid, int block, size_t smem, cudaStream_t s) {
    if (count)
        k_trace<V, true><<<grid, block, smem, s>>>(a);
    else
        k_trace<V, false><<<grid, block, smem, s>>>(a);
    return cudaGetLastError();
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
    cudaError_t e = cudaMemsetAsync(L.fetch, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (L.n == 0 && L.n_dev == nullptr) return cudaSuccess;
    int block = L.block;
    int grid = L.grid;
    size_t smem = 0;
    if (L.variant == HK_TRACE_SMEMSTACK) smem = (size_t)L.stack_depth * block * 12;
    switch (L.variant) {
    case HK_TRACE_FULLSTACK: return launch_v<HK_TRACE_FULLSTACK>(a, L.count, grid, block, smem, s);
    case HK_TRACE_SHORTSTACK: return launch_v<HK_TRACE_SHORTSTACK>(a, L.count, grid, block, smem, s);
    case HK_TRACE_SMEMSTACK: return launch_v<HK_TRACE_SMEMSTACK>(a, L.count, grid, block, smem, s);
    case HK_TRACE_RESTART: return launch_v<HK_TRACE_RESTART>(a, L.count, grid, block, smem, s);
    case HK_TRACE_RESTART_EARLY: return launch_v<HK_TRACE_RESTART_EARLY>(a, L.count, grid, block, smem, s);
    case HK_TRACE_BRUTE: return launch_v<HK_TRACE_BRUTE>(a, L.count, grid, block, smem, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace hk
