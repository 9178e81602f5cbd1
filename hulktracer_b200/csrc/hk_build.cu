// hk_build.cu -- GPU KD-tree builder: exact binned SAH (sm_100a).
//
// Breadth-first and level-synchronous. Per level:
//   prep/scan     which nodes are "large" and how many histogram chunks each has
//   hist_large    one CTA per chunk of a large node: shared-memory histograms
//                 (3 axes x {lo bin, hi bin, flat-on-plane}) of the clipped
//                 reference bounds, flushed to global memory with atomics
//   sah_large     one warp per large node: warp scans over the 32 bins, exact
//                 SAH at the 31 planes of each axis, warp argmin
//   small         one warp per small node: histogram in warp-private shared
//                 memory, then the same SAH evaluation
//   plan/scan     leaf refs, child pairs, next-level nodes, child refs
//   guard         capacity check (the whole level stops splitting on overflow)
//   emit          compact node entries and next-level node records
//   scan/scatter  stable partition of the references (global exclusive scan of
//                 below/above flags), leaf references to the output list
//   advance       level counters
// Every kernel reads its work size from device memory, so the whole build is
// a fixed launch sequence (graph-capturable, no host round trips).
//
// The algorithm is restated serially in the CPU oracle (hko_build_binned); the
// two produce identical trees. The plane / bin / cost arithmetic below is
// written with explicit IEEE round-to-nearest intrinsics for that reason.
#include <algorithm>
#include <cstdio>

#include "hk_build.h"
#include "hk_common.cuh"
#include "hk_internal.h"

namespace hk {

constexpr uint32_t kBins = 32;
constexpr uint32_t kSmall = 256;     // nodes with <= kSmall refs: one warp per node
constexpr uint32_t kChunk = 2048;    // refs per histogram CTA of a large node
constexpr uint32_t kHist = 3 * 3 * kBins;
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr uint32_t kTile = kScanThreads * kScanItems;

// ---------------------------------------------------------------------------
// small vector types for the scans
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint2 vadd(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ uint4 vadd(uint4 a, uint4 b) { return make_uint4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
template <class T> __device__ __forceinline__ T vzero();
template <> __device__ __forceinline__ uint2 vzero<uint2>() { return make_uint2(0, 0); }
template <> __device__ __forceinline__ uint4 vzero<uint4>() { return make_uint4(0, 0, 0, 0); }
__device__ __forceinline__ uint2 shfl_up(uint2 v, int d) {
    return make_uint2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ uint4 shfl_up(uint4 v, int d) {
    return make_uint4(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d),
                      __shfl_up_sync(0xffffffffu, v.z, d), __shfl_up_sync(0xffffffffu, v.w, d));
}

// inclusive warp scan
template <class T>
__device__ __forceinline__ T warp_incl(T v) {
    const int lane = threadIdx.x & 31;
    for (int d = 1; d < 32; d <<= 1) {
        T u = shfl_up(v, d);
        if (lane >= d) v = vadd(v, u);
    }
    return v;
}

__device__ __forceinline__ uint2 vsub(uint2 a, uint2 b) { return make_uint2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ uint4 vsub(uint4 a, uint4 b) { return make_uint4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }

// exclusive block scan of one value per thread (kScanThreads threads); returns
// the thread's exclusive prefix and the block total
template <class T>
__device__ __forceinline__ T block_excl(T v, T *sh_warp, T &total) {
    constexpr int NW = kScanThreads / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_incl(v);
    if (lane == 31) sh_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < NW ? sh_warp[lane] : vzero<T>();
        T wi = warp_incl(w);
        if (lane < NW) sh_warp[lane] = wi;
    }
    __syncthreads();
    T wbase = warp ? sh_warp[warp - 1] : vzero<T>();
    total = sh_warp[NW - 1];
    __syncthreads();
    return vadd(wbase, vsub(inc, v));
}

// scan phase 1: per-tile sums
template <class T, class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(Load ld, T *partials) {
    __shared__ T sh[kScanThreads / 32 + 1];
    const uint32_t n = ld.count();
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        T s = vzero<T>();
        uint32_t base = tile * kTile + threadIdx.x * kScanItems;
        for (int k = 0; k < kScanItems; k++)
            if (base + k < n) s = vadd(s, ld(base + k));
        T tot;
        block_excl(s, sh, tot);
        if (threadIdx.x == 0) partials[tile] = tot;
    }
}

// scan phase 2: one CTA scans the tile sums (exclusive) and writes the total
template <class T, class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_partials(Load ld, T *partials, T *total) {
    __shared__ T sh[kScanThreads / 32 + 1];
    const uint32_t n = ld.count();
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    T carry = vzero<T>();
    for (uint32_t b = 0; b < ntiles; b += kScanThreads) {
        uint32_t i = b + threadIdx.x;
        T v = i < ntiles ? partials[i] : vzero<T>();
        T tot;
        T ex = block_excl(v, sh, tot);
        if (i < ntiles) partials[i] = vadd(carry, ex);
        carry = vadd(carry, tot);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *total = carry;
        ld.on_total(carry);
    }
}

// scan phase 3: exclusive prefix of every element
template <class T, class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(Load ld, const T *partials, T *out) {
    __shared__ T sh[kScanThreads / 32 + 1];
    const uint32_t n = ld.count();
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint32_t base = tile * kTile + threadIdx.x * kScanItems;
        T v[kScanItems];
        T s = vzero<T>();
        for (int k = 0; k < kScanItems; k++) {
            v[k] = (base + k < n) ? ld(base + k) : vzero<T>();
            s = vadd(s, v[k]);
        }
        T tot;
        T ex = vadd(partials[tile], block_excl(s, sh, tot));
        for (int k = 0; k < kScanItems; k++) {
            if (base + k < n) {
                out[base + k] = ex;
                ld.on_prefix(base + k, ex);
            }
            ex = vadd(ex, v[k]);
        }
    }
}

template <class T, class Load>
static cudaError_t scan(const Load &ld, T *partials, T *out, T *total, int grid, cudaStream_t s) {
    k_scan_reduce<T, Load><<<grid, kScanThreads, 0, s>>>(ld, partials);
    k_scan_partials<T, Load><<<1, kScanThreads, 0, s>>>(ld, partials, total);
    k_scan_apply<T, Load><<<grid, kScanThreads, 0, s>>>(ld, partials, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// exact-order helpers shared with the oracle restatement
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float mnf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float c3(float4 v, uint32_t a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ void s3(float4 &v, uint32_t a, float x) {
    if (a == 0) v.x = x;
    else if (a == 1) v.y = x;
    else v.z = x;
}

// p_k = min + ext * (k / bins)
__device__ __forceinline__ float plane_k(float blo, float ext, uint32_t k) {
    return __fadd_rn(blo, __fmul_rn(ext, __fmul_rn((float)k, 0.03125f)));
}

__device__ __forceinline__ float surf(float4 lo, float4 hi) {
    float sx = __fsub_rn(hi.x, lo.x), sy = __fsub_rn(hi.y, lo.y), sz = __fsub_rn(hi.z, lo.z);
    return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(sx, sy), __fmul_rn(sz, sy)), __fmul_rn(sx, sz)));
}

// bins of a clipped interval [lo, hi] on one axis: p_b <= lo < p_{b+1},
// p_c < hi <= p_{c+1}; on = the interval is flat and lies on plane b
__device__ __forceinline__ void bin_interval(float lo, float hi, float blo, float ext, float inv, int &b, int &c,
                                             bool &on) {
    b = __float2int_rz(__fmul_rn(__fsub_rn(lo, blo), inv));
    b = b < 0 ? 0 : (b > (int)kBins - 1 ? (int)kBins - 1 : b);
    while (b > 0 && lo < plane_k(blo, ext, b)) b--;
    while (b < (int)kBins - 1 && lo >= plane_k(blo, ext, b + 1)) b++;
    c = __float2int_rz(__fmul_rn(__fsub_rn(hi, blo), inv));
    c = c < 0 ? 0 : (c > (int)kBins - 1 ? (int)kBins - 1 : c);
    while (c > 0 && hi <= plane_k(blo, ext, c)) c--;
    while (c < (int)kBins - 1 && hi > plane_k(blo, ext, c + 1)) c++;
    on = (lo == hi) && b >= 1 && lo == plane_k(blo, ext, b);
}

// histogram contribution of one reference (shared-memory counters)
__device__ __forceinline__ void hist_ref(uint32_t *H, float4 tlo, float4 thi, float4 blo, float4 bhi) {
#pragma unroll
    for (uint32_t a = 0; a < 3; a++) {
        float l = c3(blo, a), h = c3(bhi, a);
        float ext = __fsub_rn(h, l);
        if (!(ext > 0.0f)) continue;
        float inv = __fdiv_rn(32.0f, ext);
        float lo = mxf(c3(tlo, a), l), hi = mnf(c3(thi, a), h);
        int b, c;
        bool on;
        bin_interval(lo, hi, l, ext, inv, b, c, on);
        atomicAdd(&H[a * 96 + b], 1u);
        atomicAdd(&H[a * 96 + 32 + c], 1u);
        if (on) atomicAdd(&H[a * 96 + 64 + b], 1u);
    }
}

struct Decision {
    int axis;
    float plane;
    uint32_t nb, na;
    float cost;
    int bin;      // plane index k of the chosen plane
};

// Warp-wide SAH over the node's histograms (all 32 lanes call it). The
// first minimum in (axis, plane) order wins, as in the serial loop.
template <class HistPtr>
__device__ Decision sah_warp(HistPtr H, float4 blo, float4 bhi, uint32_t cnt, float ct, float ci) {
    const uint32_t lane = threadIdx.x & 31u;
    float A = surf(blo, bhi);
    Decision best{-1, 0.0f, 0, 0, kInf, 0};
    for (uint32_t a = 0; a < 3; a++) {
        float l = c3(blo, a), h = c3(bhi, a);
        float ext = __fsub_rn(h, l);
        if (!(ext > 0.0f)) continue;
        uint32_t hlo = H[a * 96 + lane], hhi = H[a * 96 + 32 + lane];
        // exclusive prefix over bins < lane
        uint32_t slo = hlo, shi = hhi;
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t u = __shfl_up_sync(0xffffffffu, slo, d), w = __shfl_up_sync(0xffffffffu, shi, d);
            if ((int)lane >= d) {
                slo += u;
                shi += w;
            }
        }
        uint32_t below = slo - hlo;          // sum_{b < k} hlo[b]
        uint32_t above = cnt - (shi - hhi);  // sum_{c >= k} hhi[c]
        uint32_t on = H[a * 96 + 64 + lane];
        float pk = plane_k(l, ext, lane), pk1 = plane_k(l, ext, lane + 1);
        bool valid = lane >= 1 && pk > l && pk < h && (lane == 31 || pk < pk1);
        float cost = kInf;
        uint32_t nb = below + on, na = above + on;
        if (valid) {
            float4 bb = bhi, ba = blo;
            s3(bb, a, pk);
            s3(ba, a, pk);
            float sb = surf(blo, bb), sa = surf(ba, bhi);
            cost = __fadd_rn(ct, __fmul_rn(ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)nb), __fmul_rn(sa, (float)na)), A)));
            if (!(cost < kInf)) cost = kInf;  // NaN / inf never win
        }
        // argmin with ties to the lower plane index
        float mc = cost;
        uint32_t mk = lane;
        for (int off = 16; off; off >>= 1) {
            float oc = __shfl_xor_sync(0xffffffffu, mc, off);
            uint32_t ok = __shfl_xor_sync(0xffffffffu, mk, off);
            if (oc < mc || (oc == mc && ok < mk)) {
                mc = oc;
                mk = ok;
            }
        }
        if (mc < best.cost) {
            best.cost = mc;
            best.axis = (int)a;
            best.plane = __shfl_sync(0xffffffffu, pk, mk);
            best.nb = __shfl_sync(0xffffffffu, nb, mk);
            best.na = __shfl_sync(0xffffffffu, na, mk);
            best.bin = (int)mk;
        }
    }
    if (best.axis >= 0 && !(best.cost < __fmul_rn(ci, (float)cnt))) best.axis = -1;
    return best;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
struct LevelArgs {
    const float4 *tb_lo, *tb_hi;
    const float4 *n_lo, *n_hi;
    const uint4 *n_info;
    float4 *nx_lo, *nx_hi;
    uint4 *nx_info;
    int32_t *axis;
    float *plane;
    uint2 *cnt;
    uint4 *plan;
    uint2 *chunks;          // (large rank, chunk index within the node)
    uint32_t *large_slot;
    uint32_t *hist;
    uint32_t *done;
    const uint32_t *refs;
    const uint32_t *ref_node;
    uint32_t *nx_refs, *nx_ref_node;
    const uint2 *rscan;
    uint2 *out_nodes;
    uint32_t *out_refs;
    uint32_t *out_ropes;
    float4 *out_cbox;
    BuildCounters *ctr;
    LevelCounters *lc, *nlc;
    uint32_t *err;
    uint32_t level;
    float ct, ci;
    uint32_t max_depth, leaf_size;
    uint32_t cap_refs, cap_nodes, cap_level, cap_large, cap_chunks;
    // learned proposer
    int learned, record;
    uint32_t *lrank;        // node slot -> proposer row (0xffffffff: none)
    float *feat, *logits;
    float *rec_X;
    int32_t *rec_y;
    uint32_t *rec_rows, rec_cap;
    float fallback_ratio;
    uint32_t topk;
};

__global__ void k_tri_bounds(const float4 *__restrict__ V, const uint4 *__restrict__ T, uint32_t nt, float4 *lo,
                             float4 *hi) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    uint4 t = T[i];
    float4 a = V[t.x], b = V[t.y], c = V[t.z];
    lo[i] = make_float4(mnf(mnf(a.x, b.x), c.x), mnf(mnf(a.y, b.y), c.y), mnf(mnf(a.z, b.z), c.z), 0.0f);
    hi[i] = make_float4(mxf(mxf(a.x, b.x), c.x), mxf(mxf(a.y, b.y), c.y), mxf(mxf(a.z, b.z), c.z), 0.0f);
}

// root node + references of level 0 (the counters were zeroed by a memset)
__global__ void k_root(LevelArgs A, const float *box, uint32_t nt) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        LevelCounters *l0 = &A.ctr->lvl[0];
        l0->nodes = 1;
        l0->refs = nt;
        l0->nodes_total = 2;
        l0->leafrefs_total = 0;
        A.nx_lo[0] = make_float4(box[0], box[1], box[2], 0.0f);
        A.nx_hi[0] = make_float4(box[4], box[5], box[6], 0.0f);
        A.nx_info[0] = make_uint4(0, nt, 0, 0);
        A.out_nodes[1] = make_uint2(kLeafTag, 0);
        A.out_nodes[0] = make_uint2(kLeafTag, 0);
        // root cell = scene box, no ropes (every face is the scene boundary)
        A.out_cbox[0] = A.nx_lo[0];
        A.out_cbox[1] = A.nx_hi[0];
        for (int f = 0; f < 6; f++) A.out_ropes[f] = 0xffffffffu;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        const_cast<uint32_t *>(A.refs)[i] = i;
        const_cast<uint32_t *>(A.ref_node)[i] = 0;
    }
}

__device__ __forceinline__ bool decidable(const LevelArgs &A, uint32_t cnt) {
    return cnt > A.leaf_size && A.level < A.max_depth;
}

// large nodes take ranks and chunk ranges (atomics: the histogram sums do not
// depend on their order)
__global__ void k_prep(LevelArgs A) {
    const uint32_t n = A.lc->nodes;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        uint32_t cnt = A.n_info[s].y;
        if (A.learned) A.lrank[s] = 0xffffffffu;
        if (!(decidable(A, cnt) && cnt > kSmall)) continue;
        uint32_t nch = (cnt + kChunk - 1) / kChunk;
        uint32_t rank = atomicAdd(&A.lc->n_large, 1u);
        uint32_t first = atomicAdd(&A.lc->n_chunks, nch);
        if (rank >= A.cap_large || first + nch > A.cap_chunks) {
            atomicOr(A.err, 2u);
            continue;
        }
        A.large_slot[rank] = s;
        if (A.learned) A.lrank[s] = rank;   // the proposer row of the node
        for (uint32_t k = 0; k < nch; k++) A.chunks[first + k] = make_uint2(rank, k);
        uint32_t *H = A.hist + (size_t)rank * kHist;
        for (uint32_t k = 0; k < kHist; k++) H[k] = 0;
        A.done[rank] = 0;
    }
}

__device__ __forceinline__ void write_decision(const LevelArgs &A, uint32_t s, const Decision &d) {
    A.axis[s] = d.axis;
    A.plane[s] = d.plane;
    A.cnt[s] = make_uint2(d.nb, d.na);
}

// global histogram read past L1 (other CTAs wrote it with atomics)
struct GHist {
    const uint32_t *p;
    __device__ uint32_t operator[](uint32_t i) const { return __ldcg(p + i); }
};

// ---------------------------------------------------------------------------
// proposer features of one node (one warp): from at most 64 references taken
// at a fixed stride, per axis a 32-bin histogram of clipped centroids and
// 16-bin histograms of clipped lower / upper bounds (fractions of the sample),
// the extents over the largest extent, depth / max_depth, 4 zeros = 200.
// Counts are exact small integers, so the order of the shared atomics does
// not matter.
// ---------------------------------------------------------------------------
constexpr uint32_t kFeatSample = 64;

__device__ void node_features(const LevelArgs &A, uint4 info, float4 blo, float4 bhi, float *sh, float *out) {
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t i = lane; i < 200; i += 32) sh[i] = 0.0f;
    __syncwarp();
    const uint32_t cnt = info.y;
    const uint32_t S = cnt < kFeatSample ? cnt : kFeatSample;
    for (uint32_t i = lane; i < S; i += 32) {
        uint32_t r = info.x + (uint32_t)(((uint64_t)i * cnt) / S);
        uint32_t tri = A.refs[r];
        float4 tlo = A.tb_lo[tri], thi = A.tb_hi[tri];
        for (uint32_t a = 0; a < 3; a++) {
            float l = c3(blo, a), h = c3(bhi, a), ext = h - l;
            if (!(ext > 0.0f)) continue;
            float lo = mxf(c3(tlo, a), l), hi = mnf(c3(thi, a), h);
            float c = (lo + hi) * 0.5f;
            int b32 = (int)((c - l) * (32.0f / ext));
            int blo16 = (int)((lo - l) * (16.0f / ext));
            int bhi16 = (int)((hi - l) * (16.0f / ext));
            b32 = b32 < 0 ? 0 : (b32 > 31 ? 31 : b32);
            blo16 = blo16 < 0 ? 0 : (blo16 > 15 ? 15 : blo16);
            bhi16 = bhi16 < 0 ? 0 : (bhi16 > 15 ? 15 : bhi16);
            atomicAdd(&sh[a * 32 + b32], 1.0f);
            atomicAdd(&sh[96 + a * 32 + blo16], 1.0f);
            atomicAdd(&sh[96 + a * 32 + 16 + bhi16], 1.0f);
        }
    }
    __syncwarp();
    const float inv = S ? 1.0f / (float)S : 0.0f;
    for (uint32_t i = lane; i < 192; i += 32) out[i] = sh[i] * inv;
    if (lane == 0) {
        float ex = bhi.x - blo.x, ey = bhi.y - blo.y, ez = bhi.z - blo.z;
        float m = fmaxf(ex, fmaxf(ey, ez));
        float im = m > 0.0f ? 1.0f / m : 0.0f;
        out[192] = ex * im;
        out[193] = ey * im;
        out[194] = ez * im;
        out[195] = (float)A.level / (float)A.max_depth;
        out[196] = out[197] = out[198] = out[199] = 0.0f;
    }
    __syncwarp();
}

// binned mode, recording: (features, label) of a node the exact SAH split
__device__ void record_node(const LevelArgs &A, uint4 info, float4 blo, float4 bhi, const Decision &d, float *sh) {
    if (!A.record || d.axis < 0 || info.y <= kSmall) return;
    uint32_t row = 0;
    if ((threadIdx.x & 31u) == 0) row = atomicAdd(A.rec_rows, 1u);
    row = __shfl_sync(0xffffffffu, row, 0);
    if (row >= A.rec_cap) return;
    node_features(A, info, blo, bhi, sh, A.rec_X + (size_t)row * 200);
    if ((threadIdx.x & 31u) == 0) A.rec_y[row] = d.axis * 32 + d.bin;
}

// Work items: first the chunks of large nodes (one CTA each; the CTA that
// finishes a node's last chunk evaluates its SAH), then groups of 8 small
// nodes (one warp each: warp-private histogram + SAH).
__global__ void __launch_bounds__(256) k_work(LevelArgs A) {
    __shared__ uint32_t H[kHist];
    __shared__ uint32_t HS[8][kHist];
    __shared__ int s_last;
    const uint32_t wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nch = min(A.lc->n_chunks, A.cap_chunks);
    const uint32_t nodes = A.lc->nodes;
    const uint32_t ngroups = (nodes + 7) / 8;
    for (uint32_t item = blockIdx.x; item < nch + ngroups; item += gridDim.x) {
        if (item < nch) {
            if (A.learned) continue;  // learned mode: chunks are costed by k_propose
            uint2 ck = A.chunks[item];
            uint32_t rank = ck.x;
            if (rank >= A.cap_large) continue;  // uniform per CTA
            uint32_t s = A.large_slot[rank];
            if (s >= nodes) continue;
            uint4 info = A.n_info[s];
            uint32_t r0 = info.x + ck.y * kChunk, r1 = min(info.x + info.y, r0 + kChunk);
            float4 blo = A.n_lo[s], bhi = A.n_hi[s];
            for (uint32_t i = threadIdx.x; i < kHist; i += blockDim.x) H[i] = 0;
            __syncthreads();
            for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
                uint32_t tri = A.refs[r];
                hist_ref(H, A.tb_lo[tri], A.tb_hi[tri], blo, bhi);
            }
            __syncthreads();
            uint32_t *G = A.hist + (size_t)rank * kHist;
            for (uint32_t i = threadIdx.x; i < kHist; i += blockDim.x)
                if (H[i]) atomicAdd(&G[i], H[i]);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t nchunks = (info.y + kChunk - 1) / kChunk;
                s_last = (atomicAdd(&A.done[rank], 1u) == nchunks - 1) ? 1 : 0;
            }
            __syncthreads();
            if (s_last && wib == 0) {
                __threadfence();
                Decision d = sah_warp(GHist{G}, blo, bhi, info.y, A.ct, A.ci);
                if (lane == 0) write_decision(A, s, d);
                record_node(A, info, blo, bhi, d, reinterpret_cast<float *>(HS[0]));
            }
            __syncthreads();
        } else {
            uint32_t s = (item - nch) * 8 + wib;
            if (s >= nodes) continue;
            uint4 info = A.n_info[s];
            uint32_t cnt = info.y;
            bool dec = decidable(A, cnt);
            if (dec && cnt > kSmall) {
                // learned mode: the proposer's features instead of histograms
                if (A.learned) {
                    uint32_t row = A.lrank[s];
                    if (row < A.cap_large)
                        node_features(A, info, A.n_lo[s], A.n_hi[s], reinterpret_cast<float *>(HS[wib]),
                                      A.feat + (size_t)row * 200);
                }
                continue;  // binned mode: handled by its chunks
            }
            if (!dec) {
                if (lane == 0) write_decision(A, s, Decision{-1, 0.0f, 0, 0, kInf, 0});
                continue;
            }
            uint32_t *Hw = HS[wib];
            for (uint32_t i = lane; i < kHist; i += 32) Hw[i] = 0;
            __syncwarp();
            float4 blo = A.n_lo[s], bhi = A.n_hi[s];
            for (uint32_t r = info.x + lane; r < info.x + cnt; r += 32) {
                uint32_t tri = A.refs[r];
                hist_ref(Hw, A.tb_lo[tri], A.tb_hi[tri], blo, bhi);
            }
            __syncwarp();
            Decision d = sah_warp(Hw, blo, bhi, cnt, A.ct, A.ci);
            if (lane == 0) write_decision(A, s, d);
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------------------
// learned proposals. Per proposer row (a large node), the valid planes (those
// the binned search would cost) with the top-k logits, plus a reference plane
// -- the middle plane of the node's longest axis -- are costed exactly with
// the partition's own classification. The references are counted in the
// node's chunks (one CTA each, counts summed with global atomics); the CTA
// that finishes the node's last chunk costs the candidates. The cheapest
// proposal wins unless it costs more than fallback_ratio x the reference
// plane, in which case that CTA runs the full binned SAH on the node.
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool plane_valid(float l, float ext, float h, uint32_t k, float &pk) {
    if (!(ext > 0.0f) || k < 1 || k > 31) return false;
    pk = plane_k(l, ext, k);
    float pk1 = plane_k(l, ext, k + 1);
    return pk > l && pk < h && (k == 31 || pk < pk1);
}

constexpr int kMaxCand = 9;   // top-k (k <= 8) + the reference plane

struct Candidates {
    int n;          // proposals
    int has_ref;    // candidate n is the reference plane
    int axis[kMaxCand];
    int bin[kMaxCand];
    float plane[kMaxCand];
};

// warp 0: the top-k valid planes by logit (ties: lowest index) + reference
__device__ void select_candidates(const LevelArgs &A, const float *__restrict__ L, float4 blo, float4 bhi,
                                  Candidates &C) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t K = A.topk < 8 ? A.topk : 8;
    float v[3];
    float pk[3];
    for (int j = 0; j < 3; j++) {
        uint32_t c = lane + 32u * j, a = c / 32u, k = c % 32u;
        float l = c3(blo, a), h = c3(bhi, a);
        float x = L[c];
        v[j] = plane_valid(l, __fsub_rn(h, l), h, k, pk[j]) ? (x == x ? x : -INFINITY) : NAN;
    }
    int n = 0;
    for (uint32_t r = 0; r < K; r++) {
        // lane-local best (NaN = invalid or taken)
        float bv = NAN;
        int bc = 1 << 30;
        for (int j = 0; j < 3; j++)
            if (v[j] == v[j] && (bv != bv || v[j] > bv)) {
                bv = v[j];
                bc = (int)lane + 32 * j;
            }
        for (int o = 16; o; o >>= 1) {
            float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            int oc = __shfl_xor_sync(0xffffffffu, bc, o);
            bool take = (ov == ov) && (bv != bv || ov > bv || (ov == bv && oc < bc));
            if (take) {
                bv = ov;
                bc = oc;
            }
        }
        if (bv != bv) break;  // no valid plane left (uniform across the warp)
        if ((uint32_t)(bc & 31) == lane) {
            int j = bc >> 5;
            C.axis[n] = bc / 32;
            C.bin[n] = bc % 32;
            C.plane[n] = pk[j];
            v[j] = NAN;
        }
        n++;
    }
    if (lane == 0) {
        float ex = __fsub_rn(bhi.x, blo.x), ey = __fsub_rn(bhi.y, blo.y), ez = __fsub_rn(bhi.z, blo.z);
        uint32_t la = (ex >= ey && ex >= ez) ? 0 : (ey >= ez ? 1 : 2);
        float p;
        C.has_ref = plane_valid(c3(blo, la), __fsub_rn(c3(bhi, la), c3(blo, la)), c3(bhi, la), 16, p) ? 1 : 0;
        if (C.has_ref) {
            C.axis[n] = (int)la;
            C.plane[n] = p;
            C.bin[n] = 16;
        }
        C.n = n;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(256) k_propose(LevelArgs A) {
    __shared__ uint32_t H[kHist];
    __shared__ Candidates C;
    __shared__ uint32_t s_cnt[2 * kMaxCand];
    __shared__ int s_last, s_fallback;
    const uint32_t nch = min(A.lc->n_chunks, A.cap_chunks);
    const uint32_t nodes = A.lc->nodes;
    for (uint32_t item = blockIdx.x; item < nch; item += gridDim.x) {
        const uint2 ck = A.chunks[item];
        const uint32_t rank = ck.x;
        if (rank >= A.cap_large) continue;  // uniform per CTA
        const uint32_t s = A.large_slot[rank];
        if (s >= nodes) continue;
        const uint4 info = A.n_info[s];
        const float4 blo = A.n_lo[s], bhi = A.n_hi[s];
        if (threadIdx.x < 32) select_candidates(A, A.logits + (size_t)rank * kMlpOut, blo, bhi, C);
        if (threadIdx.x < 2 * kMaxCand) s_cnt[threadIdx.x] = 0;
        __syncthreads();
        const int nc = C.n + C.has_ref;
        // exact below / above counts of every candidate over this chunk
        const uint32_t r0 = info.x + ck.y * kChunk, r1 = min(info.x + info.y, r0 + kChunk);
        uint32_t nb[kMaxCand], na[kMaxCand];
#pragma unroll
        for (int i = 0; i < kMaxCand; i++) nb[i] = na[i] = 0;
        for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
            const uint32_t tri = A.refs[r];
            const float4 tlo = A.tb_lo[tri], thi = A.tb_hi[tri];
#pragma unroll
            for (int i = 0; i < kMaxCand; i++) {
                if (i >= nc) break;
                const uint32_t a = (uint32_t)C.axis[i];
                const float l = c3(blo, a), h = c3(bhi, a), p = C.plane[i];
                const float lo = mxf(c3(tlo, a), l), hi = mnf(c3(thi, a), h);
                const bool flat_on = (lo == hi) && lo == p;
                nb[i] += (lo < p || flat_on) ? 1u : 0u;
                na[i] += (hi > p || flat_on) ? 1u : 0u;
            }
        }
#pragma unroll
        for (int i = 0; i < kMaxCand; i++) {
            if (i >= nc) break;
            uint32_t b = nb[i], a = na[i];
            for (int o = 16; o; o >>= 1) {
                b += __shfl_xor_sync(0xffffffffu, b, o);
                a += __shfl_xor_sync(0xffffffffu, a, o);
            }
            if ((threadIdx.x & 31u) == 0) {
                atomicAdd(&s_cnt[2 * i], b);
                atomicAdd(&s_cnt[2 * i + 1], a);
            }
        }
        __syncthreads();
        uint32_t *G = A.hist + (size_t)rank * kHist;   // 2 x 9 counters of the row
        if (threadIdx.x < 2 * (uint32_t)nc && s_cnt[threadIdx.x]) atomicAdd(&G[threadIdx.x], s_cnt[threadIdx.x]);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t nchunks = (info.y + kChunk - 1) / kChunk;
            s_last = (atomicAdd(&A.done[rank], 1u) == nchunks - 1) ? 1 : 0;
        }
        __syncthreads();
        if (!s_last) continue;
        __threadfence();
        if (threadIdx.x == 0) {
            uint32_t cb[kMaxCand], ca[kMaxCand];
            for (int i = 0; i < nc; i++) {
                cb[i] = __ldcg(G + 2 * i);
                ca[i] = __ldcg(G + 2 * i + 1);
            }
            const float Anode = surf(blo, bhi);
            auto cost = [&](int i) {
                float4 bb = bhi, ba = blo;
                s3(bb, (uint32_t)C.axis[i], C.plane[i]);
                s3(ba, (uint32_t)C.axis[i], C.plane[i]);
                float sb = surf(blo, bb), sa = surf(ba, bhi);
                return __fadd_rn(A.ct, __fmul_rn(A.ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)cb[i]),
                                                                            __fmul_rn(sa, (float)ca[i])), Anode)));
            };
            int bi = -1;
            float bc = INFINITY;
            for (int i = 0; i < C.n; i++) {
                float ci = cost(i);
                if (ci < bc) {
                    bc = ci;
                    bi = i;
                }
            }
            bool fb = bi < 0 || (C.has_ref && bc > A.fallback_ratio * cost(C.n));
            s_fallback = fb ? 1 : 0;
            if (!fb) {
                Decision d{C.axis[bi], C.plane[bi], cb[bi], ca[bi], bc, C.bin[bi]};
                if (!(bc < __fmul_rn(A.ci, (float)info.y))) d.axis = -1;
                write_decision(A, s, d);
                atomicAdd(&A.ctr->learned_nodes, 1u);
            } else {
                atomicAdd(&A.ctr->fallback_nodes, 1u);
            }
        }
        __syncthreads();
        if (s_fallback) {
            // the full binned SAH on this node
            for (uint32_t i = threadIdx.x; i < kHist; i += blockDim.x) H[i] = 0;
            __syncthreads();
            for (uint32_t r = info.x + threadIdx.x; r < info.x + info.y; r += blockDim.x) {
                uint32_t tri = A.refs[r];
                hist_ref(H, A.tb_lo[tri], A.tb_hi[tri], blo, bhi);
            }
            __syncthreads();
            if (threadIdx.x < 32) {
                Decision d = sah_warp(H, blo, bhi, info.y, A.ct, A.ci);
                if (threadIdx.x == 0) write_decision(A, s, d);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// plan scan: (leaf refs, child pairs, next-level nodes, child refs) per node.
// on_total (one thread, after the tile sums) is the capacity guard and writes
// the next level's counters; on_prefix emits node s's compact entry and its
// children's next-level records.
struct LoadPlan {
    LevelArgs A;
    __device__ uint32_t count() const { return A.lc->nodes; }
    __device__ uint4 operator()(uint32_t s) const {
        if (A.axis[s] < 0) return make_uint4(A.n_info[s].y, 0, 0, 0);
        uint2 c = A.cnt[s];
        return make_uint4(0, 1, (c.x > 0) + (c.y > 0), c.x + c.y);
    }
    __device__ void on_total(uint4 t) const {
        LevelCounters *l = A.lc, *nx = A.nlc;
        nx->n_large = 0;
        nx->n_chunks = 0;
        if (l->nodes == 0) {
            nx->nodes = 0;
            nx->refs = 0;
            nx->nodes_total = l->nodes_total;
            nx->leafrefs_total = l->leafrefs_total;
            return;
        }
        uint64_t child_refs = t.w, leaf_refs = t.x, splits = t.y;
        bool over = child_refs > A.cap_refs || (uint64_t)l->leafrefs_total + leaf_refs + child_refs > A.cap_refs ||
                    (uint64_t)l->nodes_total + 2 * splits > A.cap_nodes || t.z > A.cap_level;
        l->stop = over ? 1u : 0u;
        if (over) A.ctr->capacity_hit = 1;
        nx->nodes = over ? 0u : t.z;
        nx->refs = over ? 0u : t.w;
        nx->nodes_total = l->nodes_total + (over ? 0u : 2u * t.y);
        nx->leafrefs_total = l->leafrefs_total + (over ? l->refs : t.x);
        if (!over && t.z) A.ctr->depth = A.level + 1;
    }
    __device__ void on_prefix(uint32_t s, uint4 pl) const {
        const LevelCounters *l = A.lc;
        const bool stop = l->stop != 0;
        uint4 info = A.n_info[s];
        int ax = stop ? -1 : A.axis[s];
        if (ax < 0) {
            uint32_t off = l->leafrefs_total + (stop ? info.x : pl.x);
            A.out_nodes[info.z] = make_uint2((off << 2) | kLeafTag, info.y);
            if (info.y) atomicAdd(&A.ctr->leaves, 1u);
            return;
        }
        uint32_t pair = l->nodes_total + 2 * pl.y;
        float p = A.plane[s];
        uint2 ct = A.cnt[s];
        A.out_nodes[info.z] = make_uint2((pair << 2) | (uint32_t)ax, __float_as_uint(p));
        uint32_t ns = pl.z, co = pl.w;
        float4 lo = A.n_lo[s], hi = A.n_hi[s];
        {
            // cells and ropes of both children: the parent's ropes, with the
            // face on the split plane pointing at the sibling
            float4 bh = hi, al = lo;
            s3(bh, ax, p);
            s3(al, ax, p);
            A.out_cbox[2 * (size_t)pair] = lo;
            A.out_cbox[2 * (size_t)pair + 1] = bh;
            A.out_cbox[2 * (size_t)pair + 2] = al;
            A.out_cbox[2 * (size_t)pair + 3] = hi;
            const uint32_t *pr = A.out_ropes + 6 * (size_t)info.z;
            uint32_t *rb = A.out_ropes + 6 * (size_t)pair, *ra = rb + 6;
            for (int f = 0; f < 6; f++) {
                uint32_t r = pr[f];
                rb[f] = r;
                ra[f] = r;
            }
            rb[2 * ax + 1] = pair + 1;
            ra[2 * ax] = pair;
        }
        if (ct.x) {
            float4 h2 = hi;
            s3(h2, ax, p);
            A.nx_lo[ns] = lo;
            A.nx_hi[ns] = h2;
            A.nx_info[ns] = make_uint4(co, ct.x, pair, 0);
            ns++;
        } else {
            A.out_nodes[pair] = make_uint2(kLeafTag, 0);
        }
        if (ct.y) {
            float4 l2 = lo;
            s3(l2, ax, p);
            A.nx_lo[ns] = l2;
            A.nx_hi[ns] = hi;
            A.nx_info[ns] = make_uint4(co + ct.x, ct.y, pair + 1, 0);
        } else {
            A.out_nodes[pair + 1] = make_uint2(kLeafTag, 0);
        }
    }
};

__device__ __forceinline__ uint2 ref_flags(const LevelArgs &A, uint32_t r, uint32_t s, int ax) {
    uint32_t tri = A.refs[r];
    float l = c3(A.n_lo[s], ax), h = c3(A.n_hi[s], ax), p = A.plane[s];
    float lo = mxf(c3(A.tb_lo[tri], ax), l), hi = mnf(c3(A.tb_hi[tri], ax), h);
    bool flat_on = (lo == hi) && lo == p;
    return make_uint2((lo < p || flat_on) ? 1u : 0u, (hi > p || flat_on) ? 1u : 0u);
}

struct LoadRefFlags {
    LevelArgs A;
    __device__ uint32_t count() const { return A.lc->refs; }
    __device__ uint2 operator()(uint32_t r) const {
        if (A.lc->stop) return make_uint2(0, 0);
        uint32_t s = A.ref_node[r];
        int ax = A.axis[s];
        if (ax < 0) return make_uint2(0, 0);
        return ref_flags(A, r, s, ax);
    }
    __device__ void on_total(uint2) const {}
    __device__ void on_prefix(uint32_t, uint2) const {}
};

__global__ void k_scatter(LevelArgs A) {
    const LevelCounters *l = A.lc;
    const uint32_t n = l->refs;
    const bool stop = l->stop != 0;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        uint32_t s = A.ref_node[r];
        uint4 info = A.n_info[s];
        int ax = stop ? -1 : A.axis[s];
        uint32_t tri = A.refs[r];
        if (ax < 0) {
            uint32_t off = l->leafrefs_total + (stop ? info.x : A.plan[s].x) + (r - info.x);
            if (off < A.cap_refs) A.out_refs[off] = tri;
            else atomicOr(A.err, 2u);
            continue;
        }
        uint2 f = ref_flags(A, r, s, ax);
        uint2 base = A.rscan[info.x], mine = A.rscan[r];
        uint4 pl = A.plan[s];
        uint2 ct = A.cnt[s];
        if (f.x) {
            uint32_t pos = pl.w + (mine.x - base.x);
            if (pos < A.cap_refs && pos < pl.w + ct.x) {
                A.nx_refs[pos] = tri;
                A.nx_ref_node[pos] = pl.z;
            } else {
                atomicOr(A.err, 2u);
            }
        }
        if (f.y) {
            uint32_t pos = pl.w + ct.x + (mine.y - base.y);
            if (pos < A.cap_refs && pos < pl.w + ct.x + ct.y) {
                A.nx_refs[pos] = tri;
                A.nx_ref_node[pos] = pl.z + (ct.x ? 1u : 0u);
            } else {
                atomicOr(A.err, 2u);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
template <class T>
static cudaError_t dalloc(T *&p, size_t n) {
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T));
}

void build_release(BuildState &S) {
    auto f = [](void *p) {
        if (p) cudaFree(p);
    };
    f(S.tb_lo); f(S.tb_hi);
    for (int k = 0; k < 2; k++) {
        f(S.n_lo[k]); f(S.n_hi[k]); f(S.n_info[k]); f(S.refs[k]); f(S.ref_node[k]);
        S.n_lo[k] = S.n_hi[k] = nullptr; S.n_info[k] = nullptr; S.refs[k] = S.ref_node[k] = nullptr;
    }
    f(S.d_axis); f(S.d_plane); f(S.d_cnt); f(S.plan); f(S.plan_tot); f(S.prep); f(S.prep_tot);
    f(S.chunks); f(S.hist); f(S.done); f(S.lrank); f(S.feat); f(S.logits);
    S.lrank = nullptr; S.feat = nullptr; S.logits = nullptr; f(S.rscan); f(S.rscan_tot); f(S.scan_partials); f(S.ctr); f(S.err);
    f(S.out_nodes); f(S.out_refs); f(S.out_ropes); f(S.out_cbox);
    S.tb_lo = S.tb_hi = nullptr;
    S.d_axis = nullptr; S.d_plane = nullptr; S.d_cnt = nullptr; S.plan = nullptr; S.plan_tot = nullptr;
    S.prep = nullptr; S.prep_tot = nullptr; S.chunks = nullptr; S.hist = nullptr; S.done = nullptr; S.rscan = nullptr;
    S.rscan_tot = nullptr; S.scan_partials = nullptr; S.ctr = nullptr; S.err = nullptr;
    S.out_nodes = nullptr; S.out_refs = nullptr; S.out_ropes = nullptr; S.out_cbox = nullptr;
    S.nt = S.cap_refs = S.cap_nodes = S.cap_level = 0;
    S.active = false;
}

hk_status build_prepare(BuildState &S, const BuildParams &p, uint32_t nt, int sm_count) {
    // leaf starts and child-pair indices are stored shifted left by 2 bits
    const uint64_t kMaxIndex = (1ull << 30) - 64;
    if ((uint64_t)nt > kMaxIndex / 16) return HK_E_CAPACITY;
    uint32_t cap_refs = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(p.max_refs, nt), kMaxIndex);
    uint32_t cap_nodes = (uint32_t)std::min<uint64_t>(std::max<uint64_t>(12ull * nt, 1024ull), kMaxIndex);
    S.p = p;
    S.sm_count = sm_count;
    if (S.ctr && S.nt == nt && S.cap_refs == cap_refs && S.cap_nodes == cap_nodes) return HK_OK;
    build_release(S);
    S.nt = nt;
    S.cap_refs = cap_refs;
    S.cap_nodes = cap_nodes;
    S.cap_level = std::min(cap_refs, cap_nodes) + 1;
    S.cap_large = cap_refs / kSmall + 2;
    S.cap_chunks = cap_refs / kChunk + S.cap_large + 2;
    uint32_t tiles = (std::max(cap_refs, S.cap_level) + kTile - 1) / kTile + 1;
    S.cap_partials = tiles;
    bool bad = false;
    bad |= dalloc(S.tb_lo, nt) != cudaSuccess;
    bad |= dalloc(S.tb_hi, nt) != cudaSuccess;
    for (int k = 0; k < 2; k++) {
        bad |= dalloc(S.n_lo[k], S.cap_level) != cudaSuccess;
        bad |= dalloc(S.n_hi[k], S.cap_level) != cudaSuccess;
        bad |= dalloc(S.n_info[k], S.cap_level) != cudaSuccess;
        bad |= dalloc(S.refs[k], cap_refs) != cudaSuccess;
        bad |= dalloc(S.ref_node[k], cap_refs) != cudaSuccess;
    }
    bad |= dalloc(S.d_axis, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.d_plane, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.d_cnt, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.plan, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.plan_tot, 1) != cudaSuccess;
    bad |= dalloc(S.prep, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.prep_tot, 1) != cudaSuccess;
    bad |= dalloc(S.chunks, S.cap_chunks + S.cap_large) != cudaSuccess;  // tail holds large_slot
    bad |= dalloc(S.hist, (size_t)S.cap_large * kHist) != cudaSuccess;
    bad |= dalloc(S.done, S.cap_large) != cudaSuccess;
    bad |= dalloc(S.lrank, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.feat, (size_t)S.cap_large * 200) != cudaSuccess;
    bad |= dalloc(S.logits, (size_t)S.cap_large * kMlpOut) != cudaSuccess;
    bad |= dalloc(S.rscan, cap_refs) != cudaSuccess;
    bad |= dalloc(S.rscan_tot, 1) != cudaSuccess;
    {
        uint4 *pp = nullptr;
        bad |= dalloc(pp, tiles) != cudaSuccess;
        S.scan_partials = pp;
    }
    bad |= dalloc(S.ctr, 1) != cudaSuccess;
    bad |= dalloc(S.err, 1) != cudaSuccess;
    bad |= dalloc(S.out_nodes, cap_nodes) != cudaSuccess;
    bad |= dalloc(S.out_refs, cap_refs) != cudaSuccess;
    bad |= dalloc(S.out_ropes, (size_t)cap_nodes * 6) != cudaSuccess;
    bad |= dalloc(S.out_cbox, (size_t)cap_nodes * 2) != cudaSuccess;
    if (bad) {
        build_release(S);
        return HK_E_ALLOC;
    }
    cudaMemset(S.err, 0, 4);
    cudaMemset(S.ctr, 0, sizeof(BuildCounters));
    return HK_OK;
}

hk_status build_ensure_outputs(BuildState &S, BuildOutputs *o) {
    if (!S.out_nodes || !S.out_refs) return HK_E_ALLOC;
    if (o) {
        o->nodes = S.out_nodes;
        o->refs = S.out_refs;
    }
    return HK_OK;
}

cudaError_t build_launch(BuildState &S, const float4 *verts, const uint4 *tris, uint32_t nt, const float *box,
                         cudaStream_t st) {
    const int G = S.sm_count * 4;
    LevelArgs A;
    memset(&A, 0, sizeof(A));
    A.tb_lo = S.tb_lo;
    A.tb_hi = S.tb_hi;
    A.axis = S.d_axis;
    A.plane = S.d_plane;
    A.cnt = S.d_cnt;
    A.plan = S.plan;
    A.chunks = S.chunks;
    A.large_slot = reinterpret_cast<uint32_t *>(S.chunks + S.cap_chunks);
    A.hist = S.hist;
    A.done = S.done;
    A.rscan = S.rscan;
    A.out_nodes = S.out_nodes;
    A.out_refs = S.out_refs;
    A.out_ropes = S.out_ropes;
    A.out_cbox = S.out_cbox;
    A.ctr = S.ctr;
    A.err = S.err;
    A.ct = S.p.ct;
    A.ci = S.p.ci;
    A.max_depth = S.p.max_depth;
    A.leaf_size = S.p.leaf_size;
    A.cap_refs = S.cap_refs;
    A.cap_nodes = S.cap_nodes;
    A.cap_level = S.cap_level;
    A.cap_large = S.cap_large;
    A.cap_chunks = S.cap_chunks;
    A.learned = (S.p.mode == HK_BUILD_LEARNED) ? 1 : 0;
    A.record = (S.p.mode == HK_BUILD_BINNED && S.p.record && S.learn && S.learn->rec_X) ? 1 : 0;
    A.lrank = S.lrank;
    A.feat = S.feat;
    A.logits = S.logits;
    A.fallback_ratio = S.p.fallback_ratio;
    A.topk = S.p.topk;
    if (S.learn) {
        A.rec_X = S.learn->rec_X;
        A.rec_y = S.learn->rec_y;
        A.rec_rows = S.learn->rec_rows;
        A.rec_cap = S.learn->rec_cap;
    }
    if (A.learned && !(S.learn && S.learn->have_mlp)) return cudaErrorInvalidValue;
    cudaMemsetAsync(S.ctr, 0, sizeof(BuildCounters), st);
    if (nt) k_tri_bounds<<<(nt + 255) / 256, 256, 0, st>>>(verts, tris, nt, S.tb_lo, S.tb_hi);
    A.nx_lo = S.n_lo[0];
    A.nx_hi = S.n_hi[0];
    A.nx_info = S.n_info[0];
    A.refs = S.refs[0];
    A.ref_node = S.ref_node[0];
    k_root<<<G, 256, 0, st>>>(A, box, nt);
    for (uint32_t L = 0; L <= S.p.max_depth; L++) {
        int cur = L & 1, nxt = cur ^ 1;
        A.level = L;
        A.lc = &S.ctr->lvl[L];
        A.nlc = &S.ctr->lvl[L + 1];
        A.n_lo = S.n_lo[cur];
        A.n_hi = S.n_hi[cur];
        A.n_info = S.n_info[cur];
        A.nx_lo = S.n_lo[nxt];
        A.nx_hi = S.n_hi[nxt];
        A.nx_info = S.n_info[nxt];
        A.refs = S.refs[cur];
        A.ref_node = S.ref_node[cur];
        A.nx_refs = S.refs[nxt];
        A.nx_ref_node = S.ref_node[nxt];
        k_prep<<<G, 256, 0, st>>>(A);
        k_work<<<G * 2, 256, 0, st>>>(A);
        if (A.learned) {
            mlp_infer(S.learn->mlp, S.feat, &A.lc->n_large, S.cap_large, S.logits, G, st);
            k_propose<<<G * 2, 256, 0, st>>>(A);
        }
        scan<uint4>(LoadPlan{A}, reinterpret_cast<uint4 *>(S.scan_partials), S.plan, S.plan_tot, G, st);
        scan<uint2>(LoadRefFlags{A}, reinterpret_cast<uint2 *>(S.scan_partials), S.rscan, S.rscan_tot, G, st);
        k_scatter<<<G, 256, 0, st>>>(A);
    }
    S.active = true;
    S.last_level = S.p.max_depth + 1;
    return cudaGetLastError();
}

const uint32_t *build_nodes_total_ptr(const BuildState &S) {
    return &S.ctr->lvl[S.p.max_depth + 1].nodes_total;
}

hk_status build_read_stats(BuildState &S, cudaStream_t st, hk_tree_stats *out) {
    BuildCounters c;
    uint32_t err = 0;
    if (cudaMemcpyAsync(&c, S.ctr, sizeof(c), cudaMemcpyDeviceToHost, st) != cudaSuccess) return HK_E_CUDA;
    if (cudaMemcpyAsync(&err, S.err, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess) return HK_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return HK_E_CUDA;
    if (err) {
        cudaMemsetAsync(S.err, 0, 4, st);
        return HK_E_CAPACITY;
    }
    const LevelCounters &fin = c.lvl[S.last_level];
    out->nodes = fin.nodes_total;
    out->refs = fin.leafrefs_total;
    out->leaves = c.leaves;
    out->depth = c.depth;
    out->capacity_hit = c.capacity_hit;
    out->learned_nodes = c.learned_nodes;
    out->fallback_nodes = c.fallback_nodes;
    return HK_OK;
}

}  // namespace hk
