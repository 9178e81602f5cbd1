// hk_stream.cu -- out-of-core leaf geometry (sm_100a).
//
// The reference's residency protocol (GPUTrace_stackless.cl:6-120,
// GLVisitorGPUTrace::launchTraceIterations, GLVisitorGPUTrace.cpp:412-502):
// a kd-restart traversal tests a leaf only when its geometry is resident;
// otherwise it marks the leaf requested, saves its resume point (the
// ThreadContext: tmin, tmax and the leaf's node) and stops; the host pages the
// requested leaves into a ring of device memory, evicting the oldest ones
// (at most half the ring per round, as there), and relaunches until no ray
// waits for a leaf.
//
// Here the leaves' triangle records live in pinned host memory that the
// device maps: a page-in is one kernel in which warps copy the requested
// leaves' records straight from host memory into the pool (no per-leaf
// copies issued by the host). Residency and pool offsets are per compact
// cell. The hits equal HK_TRACE_RESTART's bit for bit whatever the pool size:
// the traversal takes the same steps, except that a ray stops once its closest
// hit precedes the exit of the leaf it tested (as HK_TRACE_RESTART_EARLY does;
// that changes no hit). Stopping there also keeps the leaves behind the hit
// out of the pool, so a warm pool pages nothing in.
// Unlike the reference, the first leaf of a round is always loaded even when
// that needs more than half the ring, so every round makes progress, and the
// rounds are bounded (HK_E_CAPACITY when the ring cannot hold a leaf).
#include <algorithm>
#include <cstring>
#include <string>

#include "hk_stream.h"

namespace hk {

namespace {

__device__ __forceinline__ float comp3(float3 v, uint32_t a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// child 0 (an empty cell) is the reference's "no child": the root
__device__ __forceinline__ void child(const uint2 *nodes, uint32_t pair, bool below, uint32_t &cur, uint2 &node,
                                      uint2 root) {
    const uint32_t c = below ? pair : pair + 1;
    const uint2 n = nodes[c];
    if (is_leaf(n) && n.y == 0) {
        cur = 0;
        node = root;
    } else {
        cur = c;
        node = n;
    }
}

// the leaf's triangles from the pool, in leaf order; strictly closer wins
__device__ __forceinline__ void test_pool_leaf(const TriRec *__restrict__ pool, uint32_t off, const uint32_t *refs,
                                               uint2 leaf, float3 o, float3 d, float &best, int32_t &best_id) {
    const uint32_t start = leaf.x >> 2, cnt = leaf.y;
    for (uint32_t i = 0; i < cnt; i++) {
        const float t = isect_tri(&pool[off + i], o, d, best);
        if (t < best) {
            best = t;
            best_id = (int32_t)refs[start + i];
        }
    }
}

// one launch: every unfinished ray resumes where it stopped and runs until it
// finishes or reaches a leaf that is not resident
__global__ void __launch_bounds__(256) k_stream_trace(StreamTraceArgs A, const TriRec *__restrict__ pool,
                                                      uint32_t *res, const uint32_t *__restrict__ pool_off,
                                                      float *s_tmin, float *s_tmax, uint32_t *s_node,
                                                      uint32_t *done) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= A.n || done[r]) return;
    const float4 ro = A.rays[2 * (size_t)r], rd = A.rays[2 * (size_t)r + 1];
    const float3 o = make_float3(ro.x, ro.y, ro.z), d = make_float3(rd.x, rd.y, rd.z);
    float bmin[3] = {A.box[0], A.box[1], A.box[2]}, bmax[3] = {A.box[4], A.box[5], A.box[6]};
    float ts = 0.0f, te = kInf;
    if (!ray_box(bmin, bmax, o, d, ts, te)) {
        A.hits[r] = hk_hit{kInf, -1};
        done[r] = 1;
        return;
    }
    const float3 inv = make_float3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
    const uint2 root = A.nodes[0];
    float tmin = s_tmin[r], tmax = s_tmax[r];
    hk_hit h = A.hits[r];
    float best = h.t;
    int32_t best_id = h.tri;
    uint32_t steps = 0;
    const uint32_t resume = s_node[r];
    if (resume != 0) {
        // the leaf this ray stopped at (GPUTrace_stackless.cl:28-46)
        if (res[resume] != 2u) {
            atomicCAS(&res[resume], 0u, 1u);
            return;
        }
        test_pool_leaf(pool, pool_off[resume], A.refs, A.nodes[resume], o, d, best, best_id);
        s_node[r] = 0;
    }
    if (!(best < tmax)) {
        while (tmax < te) {
            tmin = tmax;
            tmax = te;
            uint32_t cur = 0;
            uint2 node = root;
            while (!is_leaf(node)) {
                if (++steps > A.max_steps) {
                    atomicOr(A.err, 1u);
                    break;
                }
                const uint32_t axis = node.x & 3u, pair = node.x >> 2;
                const float pl = __int_as_float(node.y);
                const float rs = comp3(o, axis), dc = comp3(d, axis);
                const float split = __fmul_rn(__fsub_rn(pl, rs), comp3(inv, axis));
                const bool below_first = (rs < pl) || (rs == pl && dc <= 0.0f);
                if (split >= tmax || split <= 0.0f) {
                    child(A.nodes, pair, below_first, cur, node, root);
                } else if (split <= tmin) {
                    child(A.nodes, pair, !below_first, cur, node, root);
                } else {
                    child(A.nodes, pair, below_first, cur, node, root);
                    tmax = split;
                }
                if (cur == 0) break;
            }
            if (steps > A.max_steps) break;
            if (is_leaf(node)) {
                if (res[cur] != 2u) {
                    // request the leaf and keep the resume point
                    atomicCAS(&res[cur], 0u, 1u);
                    s_tmin[r] = tmin;
                    s_tmax[r] = tmax;
                    s_node[r] = cur;
                    A.hits[r] = hk_hit{best, best_id};
                    return;
                }
                test_pool_leaf(pool, pool_off[cur], A.refs, node, o, d, best, best_id);
                if (best < tmax) break;
            }
        }
    }
    A.hits[r] = hk_hit{best, best_id};
    done[r] = 1;
}

__global__ void k_stream_init(float *tmin, float *tmax, uint32_t *node, uint32_t *done, hk_hit *hits, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        tmin[i] = 0.0f;   // ThreadContext starts zeroed
        tmax[i] = 0.0f;
        node[i] = 0;
        done[i] = 0;
        hits[i] = hk_hit{kInf, -1};
    }
}

// requested cells, compacted (order arbitrary; the host sorts them)
__global__ void k_stream_collect(const uint32_t *res, uint32_t nn, uint32_t *req) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nn && res[c] == 1u) req[atomicAdd(&req[nn], 1u)] = c;
}

__global__ void k_stream_evict(uint32_t *res, const uint32_t *cells, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) res[cells[i]] = 0u;
}

// one warp per leaf: its records from mapped host memory into the pool
__global__ void k_stream_load(const uint4 *loads, uint32_t n, const TriRec *__restrict__ hrecs, TriRec *pool,
                              uint32_t *res, uint32_t *pool_off) {
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (w >= n) return;
    const uint4 L = loads[w];   // cell, pool offset, record start, count
    for (uint32_t i = lane; i < L.w; i += 32) pool[L.y + i] = hrecs[L.z + i];
    if (lane == 0) {
        pool_off[L.x] = L.y;
        res[L.x] = 2u;
    }
}

inline unsigned blocks(size_t n, unsigned t = 256) { return (unsigned)std::max<size_t>(1, (n + t - 1) / t); }

// ring allocation of s contiguous records: used region [head, tail), or
// [head, cap) + [0, tail) once wrapped
bool ring_alloc(StreamState &S, uint32_t s, uint32_t &off) {
    if (S.fifo.empty()) {
        S.head = S.tail = 0;
        S.wrapped = false;
    }
    if (!S.wrapped) {
        if (S.cap - S.tail >= s) {
            off = S.tail;
            S.tail += s;
            return true;
        }
        if (S.head >= s) {
            S.wrapped = true;
            off = 0;
            S.tail = s;
            return true;
        }
        return false;
    }
    if (S.head - S.tail >= s) {
        off = S.tail;
        S.tail += s;
        return true;
    }
    return false;
}

// the oldest resident leaf leaves the ring
StreamEntry ring_evict(StreamState &S) {
    const StreamEntry e = S.fifo.front();
    S.fifo.pop_front();
    if (S.fifo.empty()) {
        S.head = S.tail = 0;
        S.wrapped = false;
    } else {
        const uint32_t next = S.fifo.front().off;
        if (S.wrapped && next < e.off) S.wrapped = false;   // the used region no longer wraps
        S.head = next;
    }
    return e;
}

template <class T>
cudaError_t dalloc(T *&p, size_t n) {
    return cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T));
}

}  // namespace

void StreamState::release() {
    if (h_recs) cudaFreeHost(h_recs);
    h_recs = nullptr;
    d_hrecs = nullptr;
    for (void *p : {(void *)pool, (void *)res, (void *)pool_off, (void *)req, (void *)loads, (void *)evicts,
                    (void *)tmin, (void *)tmax, (void *)rnode, (void *)done})
        if (p) cudaFree(p);
    pool = nullptr;
    res = pool_off = req = evicts = rnode = done = nullptr;
    loads = nullptr;
    tmin = tmax = nullptr;
    cap_rays = 0;
    fifo.clear();
    nodes.clear();
    ready = false;
}

#define ST_CHECK(x)                                                              \
    do {                                                                         \
        cudaError_t e_ = (x);                                                    \
        if (e_ != cudaSuccess) {                                                 \
            if (err) *err = std::string(#x) + ": " + cudaGetErrorString(e_);    \
            return HK_E_CUDA;                                                    \
        }                                                                        \
    } while (0)

hk_status stream_setup(StreamState &S, const uint2 *d_nodes, uint32_t nn, const uint32_t *d_refs, uint32_t nr,
                       const TriRec *d_recs, uint32_t cap, cudaStream_t st, std::string *err) {
    S.release();
    if (cap == 0) {
        if (err) *err = "pool capacity must be at least one triangle record";
        return HK_E_ILLEGAL_INPUT;
    }
    S.nodes.resize(nn);
    std::vector<uint32_t> refs(nr);
    ST_CHECK(cudaMemcpyAsync(S.nodes.data(), d_nodes, (size_t)nn * 8, cudaMemcpyDeviceToHost, st));
    if (nr) ST_CHECK(cudaMemcpyAsync(refs.data(), d_refs, (size_t)nr * 4, cudaMemcpyDeviceToHost, st));
    ST_CHECK(cudaStreamSynchronize(st));
    // every leaf's records in reference order: leaf (start, count) reads
    // records start .. start + count - 1
    uint32_t ntris = 0;
    for (uint32_t r : refs) ntris = std::max(ntris, r + 1);
    std::vector<TriRec> recs(ntris);
    if (ntris) ST_CHECK(cudaMemcpyAsync(recs.data(), d_recs, (size_t)ntris * sizeof(TriRec), cudaMemcpyDeviceToHost, st));
    ST_CHECK(cudaStreamSynchronize(st));
    ST_CHECK(cudaHostAlloc((void **)&S.h_recs, std::max<size_t>(nr, 1) * sizeof(TriRec), cudaHostAllocMapped));
    for (uint32_t k = 0; k < nr; k++) S.h_recs[k] = recs[refs[k]];
    ST_CHECK(cudaHostGetDevicePointer((void **)&S.d_hrecs, S.h_recs, 0));
    S.nrecs = nr;
    S.nn = nn;
    S.cap = cap;
    ST_CHECK(dalloc(S.pool, cap));
    ST_CHECK(dalloc(S.res, nn));
    ST_CHECK(dalloc(S.pool_off, nn));
    ST_CHECK(dalloc(S.req, (size_t)nn + 1));
    ST_CHECK(dalloc(S.loads, nn));
    ST_CHECK(dalloc(S.evicts, nn));
    ST_CHECK(cudaMemsetAsync(S.res, 0, (size_t)nn * 4, st));
    ST_CHECK(cudaStreamSynchronize(st));
    S.ready = true;
    return HK_OK;
}

hk_status stream_trace(StreamState &S, const StreamTraceArgs &a, cudaStream_t st, hk_stream_stats *stats,
                       std::string *err) {
    if (!S.ready) {
        if (err) *err = "hk_stream_setup first";
        return HK_E_STATE;
    }
    hk_stream_stats out;
    memset(&out, 0, sizeof out);
    if (a.n > S.cap_rays) {
        for (void *p : {(void *)S.tmin, (void *)S.tmax, (void *)S.rnode, (void *)S.done})
            if (p) cudaFree(p);
        S.tmin = S.tmax = nullptr;
        S.rnode = S.done = nullptr;
        ST_CHECK(dalloc(S.tmin, a.n));
        ST_CHECK(dalloc(S.tmax, a.n));
        ST_CHECK(dalloc(S.rnode, a.n));
        ST_CHECK(dalloc(S.done, a.n));
        S.cap_rays = a.n;
    }
    cudaEvent_t e0, e1;
    ST_CHECK(cudaEventCreate(&e0));
    ST_CHECK(cudaEventCreate(&e1));
    ST_CHECK(cudaEventRecord(e0, st));
    k_stream_init<<<blocks(a.n), 256, 0, st>>>(S.tmin, S.tmax, S.rnode, S.done, a.hits, a.n);
    uint32_t nleaves = 0;
    for (const uint2 &n : S.nodes)
        if (is_leaf(n) && n.y) nleaves++;
    // every round loads at least one requested leaf, and a loaded leaf serves
    // every ray waiting for it; the bound is far above what that needs
    const uint32_t max_rounds = 8 * nleaves + 1024;
    std::vector<uint32_t> req(S.nn);
    std::vector<uint4> loads;
    std::vector<uint32_t> evicts;
    hk_status result = HK_OK;
    for (uint32_t round = 0;; round++) {
        if (round >= max_rounds) {
            if (err) *err = "leaf paging made no progress (rounds exhausted)";
            result = HK_E_CAPACITY;
            break;
        }
        k_stream_trace<<<blocks(a.n), 256, 0, st>>>(a, S.pool, S.res, S.pool_off, S.tmin, S.tmax, S.rnode, S.done);
        out.launches++;
        ST_CHECK(cudaMemsetAsync(S.req + S.nn, 0, 4, st));
        k_stream_collect<<<blocks(S.nn), 256, 0, st>>>(S.res, S.nn, S.req);
        uint32_t nreq = 0;
        ST_CHECK(cudaMemcpyAsync(&nreq, S.req + S.nn, 4, cudaMemcpyDeviceToHost, st));
        ST_CHECK(cudaStreamSynchronize(st));
        if (nreq == 0) break;
        ST_CHECK(cudaMemcpyAsync(req.data(), S.req, (size_t)nreq * 4, cudaMemcpyDeviceToHost, st));
        ST_CHECK(cudaStreamSynchronize(st));
        std::sort(req.begin(), req.begin() + nreq);
        // page in, oldest leaves out first; at most half the ring is evicted
        // per round (the reference's bound), except for the round's first leaf
        loads.clear();
        evicts.clear();
        uint32_t evicted = 0;
        for (uint32_t k = 0; k < nreq; k++) {
            const uint32_t cell = req[k];
            const uint32_t size = S.nodes[cell].y, start = S.nodes[cell].x >> 2;
            if (size > S.cap) {
                if (err) *err = "a leaf holds more triangles than the pool";
                result = HK_E_CAPACITY;
                break;
            }
            uint32_t off = 0;
            bool ok = true;
            while (!ring_alloc(S, size, off)) {
                // the leaves loaded in this round sit at the back of the FIFO
                // and are never evicted in it
                if (S.fifo.size() <= loads.size() || (evicted > S.cap / 2 && !loads.empty())) {
                    ok = false;
                    break;
                }
                const StreamEntry e = ring_evict(S);
                evicts.push_back(e.cell);
                evicted += e.size;
            }
            if (!ok) break;
            S.fifo.push_back(StreamEntry{cell, off, size});
            loads.push_back(make_uint4(cell, off, start, size));
        }
        if (result != HK_OK) break;
        if (!evicts.empty()) {
            ST_CHECK(cudaMemcpyAsync(S.evicts, evicts.data(), evicts.size() * 4, cudaMemcpyHostToDevice, st));
            k_stream_evict<<<blocks(evicts.size()), 256, 0, st>>>(S.res, S.evicts, (uint32_t)evicts.size());
        }
        if (!loads.empty()) {
            ST_CHECK(cudaMemcpyAsync(S.loads, loads.data(), loads.size() * 16, cudaMemcpyHostToDevice, st));
            k_stream_load<<<blocks(loads.size() * 32), 256, 0, st>>>(S.loads, (uint32_t)loads.size(), S.d_hrecs,
                                                                       S.pool, S.res, S.pool_off);
        }
        out.leaves_loaded += (uint32_t)loads.size();
        out.leaves_evicted += (uint32_t)evicts.size();
        for (const uint4 &l : loads) out.bytes_paged += (uint64_t)l.w * sizeof(TriRec);
        ST_CHECK(cudaGetLastError());
    }
    ST_CHECK(cudaEventRecord(e1, st));
    ST_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out.ms = ms;
    out.resident = (uint32_t)S.fifo.size();
    if (stats) *stats = out;
    return result;
}

}  // namespace hk
