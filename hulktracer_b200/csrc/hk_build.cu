// hk_build.cu -- GPU KD-tree builder: exact binned SAH (sm_100a).
//
// Breadth-first and level-synchronous for nodes of more than 32 references:
// two launches per level in the binned mode (k_decide, k_plan_refs), three
// with exact_max or the proposer (k_hist on a second stream beside k_small,
// then k_plan_refs; the proposer adds its chain after k_hist); smaller nodes
// are deferred subtrees (below; hk_config subtree_max / subtree_depth /
// level_streams choose the layout). Splits are searched over 32 bins per
// axis, or, with exact_max (32..1024), over every clipped reference bound for
// nodes of at most exact_max references (one warp in registers up to 32, one
// CTA above):
//   work      large nodes (> 256 references): one CTA per chunk of 1024
//             references builds shared-memory histograms (3 axes x {lo bin,
//             hi bin, flat-on-plane}) of the clipped reference bounds and
//             flushes them with atomics; the CTA that finishes a node's last
//             chunk runs the SAH (one warp: scans over the 32 bins, exact cost
//             at the 31 planes per axis, argmin). Small nodes: one warp per
//             node, warp-private histogram, same SAH. Every decision is also
//             tallied into the level totals (leaf refs, splits, next-level
//             nodes, child refs) that the capacity guard needs.
//   [learn]   learned mode: nodes of 33..1024 references get the binned SAH
//             and their histogram features in the small-node kernel; then
//             k_learn runs the tensor-core MLP on them (64-node tiles), takes
//             the top-k (axis, bin) proposals and costs every clipped
//             reference bound inside the proposed bins exactly (the exact
//             SAH restricted to those bins); the cheaper of that and the
//             binned optimum splits the node
//   plan      single-pass scan over nodes (decoupled look-back): leaf
//             reference offsets, child pairs, next-level slots, child
//             reference offsets; emits compact node entries, cells and ropes,
//             next-level node records and the next level's large-node
//             chunks. The guard (the whole level stops splitting on overflow)
//             is decided from the tallies before anything is emitted.
//   refs      single-pass scan of the below/above flags of every reference,
//             fused with the stable partition into the next level and the
//             leaf reference list.
//   subtrees  a decidable node of 2..32 references is not split by the
//             levels: it is recorded (with its references) as a deferred
//             root. After the last level one warp per root builds its whole
//             subtree depth first in registers (one reference per lane, the
//             node's references a lane mask, the same SAH), a scan over the
//             subtrees' sizes places them after the levels' nodes and leaf
//             references, and a last pass moves them there. On the 200k-triangle
//             animated frame, deferring at any depth, 94% of the split
//             decisions are taken this way.
// Every kernel reads its work size from device memory, so the whole build is
// a fixed launch sequence (graph-capturable, no host round trips). Look-back
// waits are bounded: a wait that runs out sets an error bit and the build
// reports failure instead of hanging.
//
// The algorithm is restated serially in the CPU oracle (hko_build_binned); the
// two produce identical trees. The plane / bin / cost arithmetic below is
// written with explicit IEEE round-to-nearest intrinsics for that reason.
#include <algorithm>
#include <cstdio>
#include <type_traits>

#include "hk_build.h"
#include "hk_common.cuh"
#include "hk_internal.h"
#include "hk_mlp_tc.cuh"
#include "hk_mlp_tile.cuh"

namespace hk {

constexpr uint32_t kBins = 32;
constexpr uint32_t kSmall = 256;     // nodes with <= kSmall refs: one warp per node
constexpr uint32_t kChunk = 1024;    // refs per histogram CTA of a large node (4 per thread)
constexpr uint32_t kWarpExact = 32;  // exact-SAH nodes up to this size: one warp, in registers
constexpr uint32_t kLearnMax = 1024; // learned mode: nodes of kWarpExact + 1 .. kLearnMax refs are proposer rows
constexpr uint32_t kHist = 3 * 3 * kBins;
static_assert(kHist % 4 == 0 && kHist / 4 > 64 && kHist / 4 <= 96, "k_small clears its histogram with 16-byte stores");
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr uint32_t kTile = kScanThreads * kScanItems;
constexpr int kPlanItems = 1;                                 // nodes per thread of a plan tile
constexpr uint32_t kPlanTile = kScanThreads * kPlanItems;

// ---------------------------------------------------------------------------
// scan value types: uint2 (reference below/above flags; subtree sizes) and U7
// (node plan: leaf refs, splits, next-level nodes, child refs, below child
// refs, deferred-subtree refs, deferred-subtree roots)
// ---------------------------------------------------------------------------
struct U7 {
    uint32_t x, y, z, w, v, d, e;
};
__device__ __forceinline__ uint2 vadd(uint2 a, uint2 b) { return make_uint2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ U7 vadd(U7 a, U7 b) {
    return U7{a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w, a.v + b.v, a.d + b.d, a.e + b.e};
}
__device__ __forceinline__ uint2 vsub(uint2 a, uint2 b) { return make_uint2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ U7 vsub(U7 a, U7 b) {
    return U7{a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w, a.v - b.v, a.d - b.d, a.e - b.e};
}
template <class T> __device__ __forceinline__ T vzero();
template <> __device__ __forceinline__ uint2 vzero<uint2>() { return make_uint2(0, 0); }
template <> __device__ __forceinline__ U7 vzero<U7>() { return U7{0, 0, 0, 0, 0, 0, 0}; }
__device__ __forceinline__ uint2 shfl_up(uint2 v, int d) {
    return make_uint2(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ U7 shfl_up(U7 v, int d) {
    return U7{__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d),
              __shfl_up_sync(0xffffffffu, v.z, d), __shfl_up_sync(0xffffffffu, v.w, d),
              __shfl_up_sync(0xffffffffu, v.v, d), __shfl_up_sync(0xffffffffu, v.d, d),
              __shfl_up_sync(0xffffffffu, v.e, d)};
}
__device__ __forceinline__ uint2 shfl_xor(uint2 v, int d) {
    return make_uint2(__shfl_xor_sync(0xffffffffu, v.x, d), __shfl_xor_sync(0xffffffffu, v.y, d));
}
__device__ __forceinline__ U7 shfl_xor(U7 v, int d) {
    return U7{__shfl_xor_sync(0xffffffffu, v.x, d), __shfl_xor_sync(0xffffffffu, v.y, d),
              __shfl_xor_sync(0xffffffffu, v.z, d), __shfl_xor_sync(0xffffffffu, v.w, d),
              __shfl_xor_sync(0xffffffffu, v.v, d), __shfl_xor_sync(0xffffffffu, v.d, d),
              __shfl_xor_sync(0xffffffffu, v.e, d)};
}
// loads past L1 (values other CTAs of the same kernel published)
__device__ __forceinline__ uint2 ldcg(const uint2 *p) { return __ldcg(p); }
__device__ __forceinline__ U7 ldcg(const U7 *p) {
    const uint32_t *q = reinterpret_cast<const uint32_t *>(p);
    return U7{__ldcg(q), __ldcg(q + 1), __ldcg(q + 2), __ldcg(q + 3), __ldcg(q + 4), __ldcg(q + 5), __ldcg(q + 6)};
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

// ---------------------------------------------------------------------------
// single-pass scan with decoupled look-back. Tiles are taken in order from an
// atomic ticket, so every tile a CTA waits for belongs to a CTA that is
// already running and publishes its aggregate without waiting. A tile's flag
// is (tag << 2) | status, status 1 = aggregate, 2 = inclusive prefix; the tag
// (build epoch x 64 + level) makes flags of earlier levels and builds stale,
// so the flag arrays are never cleared. Waits are bounded (the build's spin
// limit, kSpinLimit polls by default): one that runs out sets error bit 4 and
// counts the tile as zero; every later kernel of the build then returns at
// once (level_aborted), so the inconsistent level is never read.
// ---------------------------------------------------------------------------
constexpr uint32_t kSpinLimit = 1u << 22;
// error bits after which the build's data may be inconsistent: a wait ran
// out (4), a partition / decision count mismatch (8), a plan bound (16)
constexpr uint32_t kErrAbort = 4u | 8u | 16u | kErrTensorWait;

// Kernels launched as programmatic dependents (launch_pdl) start before their
// predecessor in the stream has finished; this waits until it has, with its
// writes visible. Without the launch attribute it returns at once.
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <class T>
__device__ T lookback(const uint32_t *flags, const T *aggs, const T *incls, uint32_t tile, uint32_t tag,
                      uint32_t *err, uint32_t spin_limit) {
    const int lane = threadIdx.x & 31;
    T excl = vzero<T>();
    int32_t p = (int32_t)tile - 1;
    for (;;) {
        const int32_t q = p - lane;
        uint32_t st = 2;    // before tile 0: an inclusive prefix of zero
        bool have = false;
        if (q >= 0) {
            have = true;
            for (uint32_t spins = 0;; spins++) {
                const uint32_t f = __ldcv(flags + q);
                if ((f >> 2) == tag && (f & 3u)) {
                    st = f & 3u;
                    break;
                }
                if (spins >= spin_limit) {
                    atomicOr(err, 4u);
                    have = false;
                    st = 2;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        const uint32_t m2 = __ballot_sync(0xffffffffu, st == 2);
        const int stop = m2 ? __ffs(m2) - 1 : 32;
        T v = vzero<T>();
        if (have && lane <= stop) v = lane == stop ? ldcg(incls + q) : ldcg(aggs + q);
        for (int o = 16; o; o >>= 1) v = vadd(v, shfl_xor(v, o));
        excl = vadd(excl, v);
        if (m2) break;
        p -= 32;
    }
    return excl;
}

// Op: T (scan value), Item (what load caches for apply), Ctx (per-CTA
// constants), kItems (consecutive elements per thread); load(i) -> Item,
// value(Item) -> T, apply_first / apply(i, exclusive prefix, Item, Ctx),
// err(). One tile of a single-pass scan: load, block scan, publish the
// aggregate, look back for the tile's exclusive prefix, then apply_first every
// element with its global prefix, run between() (all threads), and apply every
// element.
template <class Op, class Between>
__device__ __forceinline__ void scan_tile(const Op &op, uint32_t tile, uint32_t n, uint32_t tag,
                                          const typename Op::Ctx &cx, uint32_t *flags, typename Op::T *aggs,
                                          typename Op::T *incls, typename Op::T *sh, typename Op::T &s_excl,
                                          const Between &between) {
    using T = typename Op::T;
    constexpr int kItems = Op::kItems;
    constexpr uint32_t kTileN = kScanThreads * kItems;
    const uint32_t base = tile * kTileN + threadIdx.x * kItems;
    typename Op::Item it[kItems];
    T s = vzero<T>();
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        it[k] = op.load(base + k < n ? base + k : 0xffffffffu, cx);
        s = vadd(s, op.value(it[k]));
    }
    T tot;
    const T ex = block_excl(s, sh, tot);
    if (threadIdx.x == 0) {
        if (tile == 0) incls[0] = tot;
        else aggs[tile] = tot;
        __threadfence();
        *reinterpret_cast<volatile uint32_t *>(flags + tile) = (tag << 2) | (tile == 0 ? 2u : 1u);
    }
    if (threadIdx.x < 32) {
        const T e = tile ? lookback(flags, aggs, incls, tile, tag, op.err(), op.A.spin_limit) : vzero<T>();
        if (threadIdx.x == 0) {
            if (tile) {
                incls[tile] = vadd(e, tot);
                __threadfence();
                *reinterpret_cast<volatile uint32_t *>(flags + tile) = (tag << 2) | 2u;
            }
            s_excl = e;
        }
    }
    __syncthreads();
    const T pre0 = vadd(s_excl, ex);
    T pre = pre0;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        if (base + k < n) op.apply_first(base + k, pre, it[k], cx);
        pre = vadd(pre, op.value(it[k]));
    }
    between();
    pre = pre0;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        if (base + k < n) op.apply(base + k, pre, it[k], cx);
        pre = vadd(pre, op.value(it[k]));
    }
    __syncthreads();
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

// bins per unit length of the node on each axis (32 / extent). It only seeds
// bin_interval's first guess, whose corrections end on the one bin b with
// p_b <= lo < p_{b+1} from any start in [0, 31], so a fast division serves.
__device__ __forceinline__ float4 bin_scale(float4 blo, float4 bhi) {
    float4 r;
    r.x = __fdividef(32.0f, __fsub_rn(bhi.x, blo.x));
    r.y = __fdividef(32.0f, __fsub_rn(bhi.y, blo.y));
    r.z = __fdividef(32.0f, __fsub_rn(bhi.z, blo.z));
    r.w = 0.0f;
    return r;
}

// histogram contribution of one reference (shared-memory counters); inv3 =
// bin_scale(blo, bhi)
__device__ __forceinline__ void hist_ref(uint32_t *H, float4 tlo, float4 thi, float4 blo, float4 bhi, float4 inv3) {
#pragma unroll
    for (uint32_t a = 0; a < 3; a++) {
        float l = c3(blo, a), h = c3(bhi, a);
        float ext = __fsub_rn(h, l);
        if (!(ext > 0.0f)) continue;
        float inv = c3(inv3, a);
        float lo = mxf(c3(tlo, a), l), hi = mnf(c3(thi, a), h);
        int b, c;
        bool on;
        bin_interval(lo, hi, l, ext, inv, b, c, on);
        atomicAdd(&H[a * 96 + b], 1u);
        atomicAdd(&H[a * 96 + 32 + c], 1u);
        if (on) atomicAdd(&H[a * 96 + 64 + b], 1u);
    }
}

// The node's planes p_k (k = 0..31) of each axis in P[a * 32 + k], so the bin
// corrections read them instead of recomputing them (the same values): one
// warp (lane k writes plane k of the three axes) or threads 0..95 of a CTA;
// the caller syncs before reading.
constexpr uint32_t kPlanes = 3 * kBins;
__device__ __forceinline__ void node_planes_warp(float *P, float4 blo, float4 bhi) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t a = 0; a < 3; a++) {
        const float l = c3(blo, a);
        P[a * 32 + lane] = plane_k(l, __fsub_rn(c3(bhi, a), l), lane);
    }
}
__device__ __forceinline__ void node_planes_cta(float *P, float4 blo, float4 bhi) {
    if (threadIdx.x < kPlanes) {
        const uint32_t a = threadIdx.x >> 5, k = threadIdx.x & 31u;
        const float l = c3(blo, a);
        P[threadIdx.x] = plane_k(l, __fsub_rn(c3(bhi, a), l), k);
    }
}

// bin_interval with the planes of the axis read from Pa
__device__ __forceinline__ void bin_interval_tab(float lo, float hi, float blo, float inv, const float *Pa, int &b,
                                                 int &c, bool &on) {
    b = __float2int_rz(__fmul_rn(__fsub_rn(lo, blo), inv));
    b = b < 0 ? 0 : (b > (int)kBins - 1 ? (int)kBins - 1 : b);
    while (b > 0 && lo < Pa[b]) b--;
    while (b < (int)kBins - 1 && lo >= Pa[b + 1]) b++;
    c = __float2int_rz(__fmul_rn(__fsub_rn(hi, blo), inv));
    c = c < 0 ? 0 : (c > (int)kBins - 1 ? (int)kBins - 1 : c);
    while (c > 0 && hi <= Pa[c]) c--;
    while (c < (int)kBins - 1 && hi > Pa[c + 1]) c++;
    on = (lo == hi) && b >= 1 && lo == Pa[b];
}

// hist_ref with the node's plane table P (node_planes_*)
__device__ __forceinline__ void hist_ref_tab(uint32_t *H, float4 tlo, float4 thi, float4 blo, float4 bhi, float4 inv3,
                                             const float *P) {
#pragma unroll
    for (uint32_t a = 0; a < 3; a++) {
        float l = c3(blo, a), h = c3(bhi, a);
        float ext = __fsub_rn(h, l);
        if (!(ext > 0.0f)) continue;
        float inv = c3(inv3, a);
        float lo = mxf(c3(tlo, a), l), hi = mnf(c3(thi, a), h);
        int b, c;
        bool on;
        bin_interval_tab(lo, hi, l, inv, P + a * 32, b, c, on);
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

// Warp-wide SAH over the node's histograms (all 32 lanes call it): lane k
// costs plane k of every axis, keeps its cheapest, and one warp argmin over
// (cost, axis, plane) picks the first minimum in (axis, plane) order, as the
// serial loop does. Below / above counts come from exclusive scans over the
// bins (packed 16 + 16 bits when the node has fewer than 65536 references).
template <class HistPtr>
__device__ Decision sah_warp(HistPtr H, float4 blo, float4 bhi, uint32_t cnt, float ct, float ci) {
    const uint32_t lane = threadIdx.x & 31u;
    const float A = surf(blo, bhi);
    const bool packed = cnt < 65536u;
    float mc = kInf;
    uint32_t mkey = 0xffffffffu, m_nb = 0, m_na = 0;
    float m_pk = 0.0f;
#pragma unroll
    for (uint32_t a = 0; a < 3; a++) {
        const float l = c3(blo, a), h = c3(bhi, a);
        const float ext = __fsub_rn(h, l);
        if (!(ext > 0.0f)) continue;
        const uint32_t hlo = H[a * 96 + lane], hhi = H[a * 96 + 32 + lane];
        uint32_t slo, shi;
        if (packed) {
            uint32_t v = hlo | (hhi << 16);
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
                if ((int)lane >= d) v += u;
            }
            slo = v & 0xffffu;
            shi = v >> 16;
        } else {
            slo = hlo;
            shi = hhi;
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t u = __shfl_up_sync(0xffffffffu, slo, d), w = __shfl_up_sync(0xffffffffu, shi, d);
                if ((int)lane >= d) {
                    slo += u;
                    shi += w;
                }
            }
        }
        const uint32_t below = slo - hlo;          // sum_{b < k} hlo[b]
        const uint32_t above = cnt - (shi - hhi);  // sum_{c >= k} hhi[c]
        const uint32_t on = H[a * 96 + 64 + lane];
        const float pk = plane_k(l, ext, lane);
        const float pk1 = __shfl_down_sync(0xffffffffu, pk, 1);   // plane k + 1 (lane 31: unused)
        const bool valid = lane >= 1 && pk > l && pk < h && (lane == 31 || pk < pk1);
        if (!valid) continue;
        const uint32_t nb = below + on, na = above + on;
        float4 bb = bhi, ba = blo;
        s3(bb, a, pk);
        s3(ba, a, pk);
        const float sb = surf(blo, bb), sa = surf(ba, bhi);
        const float cost =
            __fadd_rn(ct, __fmul_rn(ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)nb), __fmul_rn(sa, (float)na)), A)));
        if (cost < mc) {   // NaN / inf never win; an earlier axis keeps ties
            mc = cost;
            mkey = a * 32u + lane;
            m_nb = nb;
            m_na = na;
            m_pk = pk;
        }
    }
    // argmin over (cost, axis, plane): costs are +0 .. +inf (ct >= 0, ci > 0,
    // surfaces and counts >= 0; NaN never replaced kInf), so their bit
    // patterns order as the values do: the least cost, then the least key
    const uint32_t cbits = __float_as_uint(mc);
    const uint32_t mbits = __reduce_min_sync(0xffffffffu, cbits);
    const uint32_t bk = __reduce_min_sync(0xffffffffu, cbits == mbits ? mkey : 0xffffffffu);
    const float bc = __uint_as_float(mbits);
    Decision best{-1, 0.0f, 0, 0, kInf, 0};
    const uint32_t src = bk & 31u;
    const float pk = __shfl_sync(0xffffffffu, m_pk, src);
    const uint32_t nb = __shfl_sync(0xffffffffu, m_nb, src), na = __shfl_sync(0xffffffffu, m_na, src);
    if (bc < kInf) {
        best.axis = (int)(bk >> 5);
        best.plane = pk;
        best.nb = nb;
        best.na = na;
        best.cost = bc;
        best.bin = (int)src;
    }
    if (best.axis >= 0 && !(best.cost < __fmul_rn(ci, (float)cnt))) best.axis = -1;
    return best;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
struct LevelArgs {
    const float4 *tb_lo, *tb_hi;
    // the level's nodes and references, ping-pong by level parity: level L
    // reads buffer L & 1 and writes the other (the accessors below)
    float4 *lo_buf[2], *hi_buf[2];
    uint4 *info_buf[2];
    uint32_t *refs_buf[2], *ref_node_buf[2];
    int32_t *axis;
    float *plane;
    uint2 *cnt;
    float4 *split;          // per node: axis (int bits, -1 = leaf), plane, node min / max on the axis
    uint4 *scat;            // per node: where its references go (written by the plan scan)
    uint2 *chunks;          // (large rank, chunk index within the node)
    uint32_t *large_slot;
    uint32_t *medium_slot;
    uint32_t *hist;
    uint32_t *done;
    uint2 *out_nodes;
    uint32_t *out_refs;
    uint32_t *out_ropes;
    float4 *out_cbox;
    BuildCounters *ctr;
    LevelCounters *lc, *nlc;
    uint32_t *err;
    uint32_t *epoch;        // build counter (k_root increments it)
    uint32_t level;
    float ct, ci;
    uint32_t max_depth, leaf_size;
    uint32_t cap_refs, cap_nodes, cap_level, cap_large, cap_chunks, cap_medium;
    uint32_t exact_max;     // 0: binned everywhere; else nodes <= exact_max refs take the exact SAH
    // learned proposer
    int learned, record;
    uint32_t *learn_slot;   // proposer row -> node slot
    LearnBin *learn_bin;    // proposer row -> binned decision
    uint2 *learn_prop;      // proposer row -> proposed bins, one byte each (0xff: none)
    float *feat;            // proposer row -> features
    int32_t *prop_log;      // optional: compact node -> its 8 proposed bins
    uint32_t cap_learn;
    MlpDevice mlp;
    float *rec_X;
    int32_t *rec_y;
    uint32_t *rec_rows, rec_cap;
    float fallback_ratio;
    uint32_t topk;
    uint32_t spin_limit;       // polls before a bounded wait gives up
    uint32_t withhold_level;   // test aid: at this level plan tile 0 never publishes its done flag
    // deferred subtrees: a decidable node of 2..defer (<= kDeferMax)
    // references is recorded (d_root: compact index, reference offset, count,
    // depth; d_lo / d_hi: its cell; defer_refs: its references) and built
    // after the levels; 0: none
    uint32_t defer;
    uint32_t defer_level;      // the first level whose nodes may be deferred
    uint4 *d_root;
    float4 *d_lo, *d_hi;
    uint32_t *defer_refs;
    uint32_t cap_defer;
    uint2 *sc_key, *sc_node;   // subtree scratch node slots: (subtree, local index), entry
    float4 *sc_cbox;           // 2 per node slot
    uint32_t *sc_rope;         // 6 per node slot
    uint4 *sc_ref;             // subtree scratch reference slots: (subtree, local index, triangle, -)
    uint32_t cap_sc_nodes, cap_sc_refs;
    uint2 *st_cnt, *st_root, *st_base;   // per subtree: (nodes, refs), root entry, place

    // (selects rather than indexing: a copy of the struct whose level changes
    // stays in registers)
    __device__ __forceinline__ bool odd() const { return (level & 1u) != 0; }
    __device__ __forceinline__ float4 *n_lo() const { return odd() ? lo_buf[1] : lo_buf[0]; }
    __device__ __forceinline__ float4 *n_hi() const { return odd() ? hi_buf[1] : hi_buf[0]; }
    __device__ __forceinline__ uint4 *n_info() const { return odd() ? info_buf[1] : info_buf[0]; }
    __device__ __forceinline__ uint32_t *refs() const { return odd() ? refs_buf[1] : refs_buf[0]; }
    __device__ __forceinline__ uint32_t *ref_node() const { return odd() ? ref_node_buf[1] : ref_node_buf[0]; }
    __device__ __forceinline__ float4 *nx_lo() const { return odd() ? lo_buf[0] : lo_buf[1]; }
    __device__ __forceinline__ float4 *nx_hi() const { return odd() ? hi_buf[0] : hi_buf[1]; }
    __device__ __forceinline__ uint4 *nx_info() const { return odd() ? info_buf[0] : info_buf[1]; }
    __device__ __forceinline__ uint32_t *nx_refs() const { return odd() ? refs_buf[0] : refs_buf[1]; }
    __device__ __forceinline__ uint32_t *nx_ref_node() const { return odd() ? ref_node_buf[0] : ref_node_buf[1]; }
};

// true (on every thread of the CTA alike) when an earlier kernel of this build
// hit an error after which its data may be inconsistent; the kernel then does
// nothing. Called after wait_prior_grid by every thread.
__device__ __forceinline__ bool level_aborted(const LevelArgs &A) {
    __shared__ uint32_t s_abort;
    __syncthreads();
    if (threadIdx.x == 0) s_abort = __ldcg(A.err) & kErrAbort;
    __syncthreads();
    return s_abort != 0;
}

__global__ void k_tri_bounds(const float4 *__restrict__ V, const uint4 *__restrict__ T, uint32_t nt, float4 *lo,
                             float4 *hi) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    uint4 t = T[i];
    float4 a = V[t.x], b = V[t.y], c = V[t.z];
    lo[i] = make_float4(mnf(mnf(a.x, b.x), c.x), mnf(mnf(a.y, b.y), c.y), mnf(mnf(a.z, b.z), c.z), 0.0f);
    hi[i] = make_float4(mxf(mxf(a.x, b.x), c.x), mxf(mxf(a.y, b.y), c.y), mxf(mxf(a.z, b.z), c.z), 0.0f);
}

__device__ __forceinline__ bool decidable(const LevelArgs &A, uint32_t cnt) {
    return cnt > A.leaf_size && A.level < A.max_depth;
}

// classes of a splittable node by its reference count: small (one warp,
// k_small), medium (exact SAH, one CTA, when exact_max reaches it) and large
// (chunked binned histograms, or the proposer)
__device__ __forceinline__ bool is_medium(const LevelArgs &A, uint32_t c) {
    return A.exact_max >= kWarpExact && c > kWarpExact && c <= A.exact_max;
}
// learned mode: a proposer row (33..1024 references)
__device__ __forceinline__ bool is_learn(const LevelArgs &A, uint32_t c) {
    return A.learned && c > kWarpExact && c <= kLearnMax;
}
// large: k_hist's chunked histograms (in learned mode the proposer rows too, so
// that the proposer's chain needs nothing from k_small)
__device__ __forceinline__ bool is_large(const LevelArgs &A, uint32_t c) {
    return (c > kSmall || is_learn(A, c)) && !is_medium(A, c);
}
// a decidable node of 2..A.defer references roots a deferred subtree
constexpr uint32_t kDeferMax = 32;   // one reference per lane
constexpr int kDeferAxis = -2;       // the decision that records a deferred root
__device__ __forceinline__ bool is_deferred(const LevelArgs &A, uint32_t c) {
    return c >= 2 && c <= A.defer && A.level >= A.defer_level;
}

// root node + references of level 0 (the counters were zeroed by a memset);
// a root with more than 256 references is the first large node
__global__ void k_root(LevelArgs A, const float *box, uint32_t nt) {
    const bool dec = nt > A.leaf_size && A.max_depth > 0;
    const bool medium = dec && is_medium(A, nt);
    const bool large = dec && is_large(A, nt);
    const uint32_t nch = large ? (nt + kChunk - 1) / kChunk : 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *A.epoch += 1u;
        LevelCounters *l0 = &A.ctr->lvl[0];
        l0->nodes = 1;
        l0->refs = nt;
        l0->nodes_total = 2;
        l0->leafrefs_total = 0;
        l0->n_large = large ? 1u : 0u;
        l0->n_chunks = nch;
        l0->n_medium = medium ? 1u : 0u;
        if (large) A.large_slot[0] = 0;
        if (medium) A.medium_slot[0] = 0;
        // level 0's node buffers (A.level is 0)
        A.n_lo()[0] = make_float4(box[0], box[1], box[2], 0.0f);
        A.n_hi()[0] = make_float4(box[4], box[5], box[6], 0.0f);
        A.n_info()[0] = make_uint4(0, nt, 0, 0);
        A.out_nodes[1] = make_uint2(kLeafTag, 0);
        A.out_nodes[0] = make_uint2(kLeafTag, 0);
        // root cell = scene box, no ropes (every face is the scene boundary)
        A.out_cbox[0] = make_float4(box[0], box[1], box[2], 0.0f);
        A.out_cbox[1] = make_float4(box[4], box[5], box[6], 0.0f);
        for (int f = 0; f < 6; f++) A.out_ropes[f] = 0xffffffffu;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nt; i += gridDim.x * blockDim.x) {
        A.refs()[i] = i;
        A.ref_node()[i] = 0;
    }
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nch; k += gridDim.x * blockDim.x)
        A.chunks[k] = make_uint2(0, k);
}



// level totals of the decisions (what the capacity guard needs), kept per
// thread and flushed once per CTA
struct Tally {
    uint32_t leafrefs = 0, leafnodes = 0, splits = 0, next = 0, childrefs = 0, deferrefs = 0, defernodes = 0;
    __device__ void add(const Decision &d, uint32_t cnt) {
        if (d.axis == kDeferAxis) {
            deferrefs += cnt;
            defernodes += 1;
        } else if (d.axis < 0) {
            leafrefs += cnt;
            leafnodes += cnt ? 1u : 0u;
        } else {
            splits += 1;
            next += (d.nb > 0 ? 1u : 0u) + (d.na > 0 ? 1u : 0u);
            childrefs += d.nb + d.na;
        }
    }
};

// all threads of the CTA call it once, at the end of the kernel
constexpr int kTallies = 7;
__device__ void tally_flush(const LevelArgs &A, const Tally &t, uint32_t *sh) {
    if (threadIdx.x < kTallies) sh[threadIdx.x] = 0;
    __syncthreads();
    if (t.leafrefs) atomicAdd(&sh[0], t.leafrefs);
    if (t.leafnodes) atomicAdd(&sh[1], t.leafnodes);
    if (t.splits) atomicAdd(&sh[2], t.splits);
    if (t.next) atomicAdd(&sh[3], t.next);
    if (t.childrefs) atomicAdd(&sh[4], t.childrefs);
    if (t.deferrefs) atomicAdd(&sh[5], t.deferrefs);
    if (t.defernodes) atomicAdd(&sh[6], t.defernodes);
    __syncthreads();
    // t_leafrefs .. t_defernodes are consecutive fields of LevelCounters
    if (threadIdx.x < kTallies && sh[threadIdx.x]) atomicAdd(&A.lc->t_leafrefs + threadIdx.x, sh[threadIdx.x]);
}

// the node's bounds blo / bhi, when the caller has them
__device__ __forceinline__ void write_decision(const LevelArgs &A, uint32_t s, const Decision &d, float4 blo,
                                              float4 bhi) {
    A.axis[s] = d.axis;
    A.plane[s] = d.plane;
    A.cnt[s] = make_uint2(d.nb, d.na);
    // the partition's view of the decision in one 16-byte record
    float l = 0.0f, h = 0.0f;
    if (d.axis >= 0) {
        l = c3(blo, (uint32_t)d.axis);
        h = c3(bhi, (uint32_t)d.axis);
    }
    A.split[s] = make_float4(__int_as_float(d.axis), d.plane, l, h);
}

__device__ __forceinline__ void write_decision(const LevelArgs &A, uint32_t s, const Decision &d) {
    if (d.axis >= 0) write_decision(A, s, d, A.n_lo()[s], A.n_hi()[s]);
    else write_decision(A, s, d, make_float4(0, 0, 0, 0), make_float4(0, 0, 0, 0));
}

// global histogram read past L1 (other CTAs wrote it with atomics)
struct GHist {
    const uint32_t *p;
    __device__ uint32_t operator[](uint32_t i) const { return __ldcg(p + i); }
};

// ---------------------------------------------------------------------------
// proposer features of one node (one warp), from the node's binned histogram
// (the counts the binned SAH itself uses, exact integers, so every kernel that
// builds the histogram gives the same features): per axis the 32 lower-bound
// bin counts and the 32 upper-bound bin counts as fractions of the node's
// references (192), the extents over the largest extent (3), depth /
// max_depth, references / 1024, 3 zeros = 200.
// ---------------------------------------------------------------------------
template <class HistPtr>
__device__ void hist_features(HistPtr H, uint32_t cnt, float4 blo, float4 bhi, uint32_t level, uint32_t max_depth,
                              float *out) {
    const uint32_t lane = threadIdx.x & 31u;
    const float inv = cnt ? 1.0f / (float)cnt : 0.0f;
#pragma unroll
    for (uint32_t k = 0; k < 6; k++) {
        const uint32_t i = lane + 32u * k;                 // 0..191
        const uint32_t a = i >> 6, j = i & 63u;
        out[i] = (float)H[a * 96 + j] * inv;               // j < 32: lower-bound bins, else upper-bound bins
    }
    if (lane == 0) {
        const float ex = bhi.x - blo.x, ey = bhi.y - blo.y, ez = bhi.z - blo.z;
        const float m = fmaxf(ex, fmaxf(ey, ez));
        const float im = m > 0.0f ? 1.0f / m : 0.0f;
        out[192] = ex * im;
        out[193] = ey * im;
        out[194] = ez * im;
        out[195] = (float)level / (float)max_depth;
        out[196] = (float)cnt * (1.0f / 1024.0f);
        out[197] = out[198] = out[199] = 0.0f;
    }
    __syncwarp();
}

// training label of an exactly searched node: axis * 32 + the bin b of the
// chosen plane p on its axis (p_b <= p < p_{b+1}, p_k = min + ext * k / 32)
__device__ __forceinline__ int32_t exact_label(int axis, float p, float4 blo, float4 bhi) {
    const float l = c3(blo, (uint32_t)axis), h = c3(bhi, (uint32_t)axis), ext = __fsub_rn(h, l);
    int b = __float2int_rz(__fmul_rn(__fsub_rn(p, l), __fdividef(32.0f, ext)));
    b = b < 0 ? 0 : (b > (int)kBins - 1 ? (int)kBins - 1 : b);
    while (b > 0 && p < plane_k(l, ext, (uint32_t)b)) b--;
    while (b < (int)kBins - 1 && p >= plane_k(l, ext, (uint32_t)b + 1)) b++;
    return axis * 32 + b;
}

// ---------------------------------------------------------------------------
// exact SAH (no reference counterpart; the oracle restates it): every clipped
// reference bound on every axis with a positive extent is a candidate plane p
// (+0.0f turns a -0 bound into +0), with
//   below = #(lo < p) + #(flat at p),  above = #(hi > p) + #(flat at p)
// -- the partition's own classification -- from sorted copies of the lower
// bounds, upper bounds and flat references' bounds; the lowest cost wins,
// ties to the lower axis, then the lower plane, as in the oracle's loop.
// ---------------------------------------------------------------------------
// sorted ascending across the warp, one value per lane
__device__ __forceinline__ float warp_sort32(float v) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const float o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
            v = keep_min ? (o < v ? o : v) : (o > v ? o : v);
        }
    return v;
}

// #(sorted lane values < p) (LT) or <= p, over the warp's 32 sorted values
template <bool LE>
__device__ __forceinline__ uint32_t warp_rank32(float sorted, float p) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t step = 16; step; step >>= 1) {
        const float v = __shfl_sync(0xffffffffu, sorted, (int)(pos + step - 1));
        if (LE ? v <= p : v < p) pos += step;
    }
    // [0, pos) pass; lane pos is untested only when pos == 31
    const float v = __shfl_sync(0xffffffffu, sorted, (int)pos);
    if (LE ? v <= p : v < p) pos += 1;
    return pos;
}

// a node of at most 32 references, one warp, registers only: the lanes with
// have set hold its references' bounds (cnt of them, in any lanes)
__device__ Decision sah_exact_lanes(bool have, float4 tlo, float4 thi, uint32_t cnt, float4 blo, float4 bhi,
                                    float ct, float ci) {
    const uint32_t lane = threadIdx.x & 31u;
    const float Anode = surf(blo, bhi);
    float mc = kInf, m_pk = 0.0f;
    uint32_t m_ax = 3, m_nb = 0, m_na = 0;
#pragma unroll 1
    for (uint32_t a = 0; a < 3; a++) {
        const float l = c3(blo, a), h = c3(bhi, a);
        if (!(__fsub_rn(h, l) > 0.0f)) continue;
        const float lo = have ? mxf(c3(tlo, a), l) : kInf, hi = have ? mnf(c3(thi, a), h) : kInf;
        const float slo = warp_sort32(lo), shi = warp_sort32(hi);
        // references flat on this axis (often none: then no sort, no search)
        const bool any_flat = __ballot_sync(0xffffffffu, have && lo == hi) != 0u;
        const float sfl = any_flat ? warp_sort32(lo == hi ? lo : kInf) : kInf;
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const float pk = __fadd_rn(side ? hi : lo, 0.0f);
            const uint32_t fon = any_flat ? warp_rank32<true>(sfl, pk) - warp_rank32<false>(sfl, pk) : 0u;
            const uint32_t nb = warp_rank32<false>(slo, pk) + fon;
            const uint32_t na = (cnt - warp_rank32<true>(shi, pk)) + fon;
            if (!(have && pk > l && pk < h)) continue;
            float4 bb = bhi, ba = blo;
            s3(bb, a, pk);
            s3(ba, a, pk);
            const float sb = surf(blo, bb), sa = surf(ba, bhi);
            const float cost = __fadd_rn(
                ct, __fmul_rn(ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)nb), __fmul_rn(sa, (float)na)), Anode)));
            if (cost < mc || (cost == mc && a == m_ax && pk < m_pk)) {
                mc = cost;
                m_ax = a;
                m_pk = pk;
                m_nb = nb;
                m_na = na;
            }
        }
    }
    float bc = mc, bp = m_pk;
    uint32_t bax = m_ax, blane = lane;
    for (int off = 16; off; off >>= 1) {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, off), op = __shfl_xor_sync(0xffffffffu, bp, off);
        const uint32_t oax = __shfl_xor_sync(0xffffffffu, bax, off), ol = __shfl_xor_sync(0xffffffffu, blane, off);
        if (oc < bc || (oc == bc && (oax < bax || (oax == bax && (op < bp || (op == bp && ol < blane)))))) {
            bc = oc;
            bp = op;
            bax = oax;
            blane = ol;
        }
    }
    Decision best{-1, 0.0f, 0, 0, kInf, 0};
    const uint32_t nb = __shfl_sync(0xffffffffu, m_nb, blane), na = __shfl_sync(0xffffffffu, m_na, blane);
    if (bc < kInf) {
        best.axis = (int)bax;
        best.plane = bp;
        best.nb = nb;
        best.na = na;
        best.cost = bc;
    }
    if (best.axis >= 0 && !(best.cost < __fmul_rn(ci, (float)cnt))) best.axis = -1;
    return best;
}

// a node of at most 32 references of the level, one per lane
__device__ Decision sah_exact_warp32(const LevelArgs &A, uint4 info, float4 blo, float4 bhi, float ct, float ci) {
    const uint32_t lane = threadIdx.x & 31u;
    const bool have = lane < info.y;
    float4 tlo = make_float4(0, 0, 0, 0), thi = tlo;
    if (have) {
        const uint32_t tri = A.refs()[info.x + lane];
        tlo = A.tb_lo[tri];
        thi = A.tb_hi[tri];
    }
    return sah_exact_lanes(have, tlo, thi, info.y, blo, bhi, ct, ci);
}

// first index in sorted v[0, n) with v[i] >= p (lower) or v[i] > p (upper)
__device__ __forceinline__ uint32_t lower_bound_f(const float *v, uint32_t n, float p) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (v[m] < p) lo = m + 1;
        else hi = m;
    }
    return lo;
}
__device__ __forceinline__ uint32_t upper_bound_f(const float *v, uint32_t n, float p) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (v[m] <= p) lo = m + 1;
        else hi = m;
    }
    return lo;
}

// Exact SAH of a medium node (33..1024 references), one CTA: the same
// algorithm with the three sorts (bitonic, shared memory) and the candidates
// spread over the CTA, then a CTA argmin over (cost, axis, plane).
struct ExactCtaSmem {
    float lo[kChunk], hi[kChunk], fl[kChunk];
    uint32_t nflat;
    float w_cost[8], w_pk[8];
    uint32_t w_ax[8], w_nb[8], w_na[8], w_key[8];
};

__device__ Decision sah_exact_cta(const LevelArgs &A, uint4 info, float4 blo, float4 bhi, float ct, float ci,
                                  ExactCtaSmem &S) {
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5;
    const uint32_t cnt = info.y;
    uint32_t n2 = 1;
    while (n2 < cnt) n2 <<= 1;
    const float Anode = surf(blo, bhi);
    float mc = kInf, m_pk = 0.0f;
    uint32_t m_ax = 3, m_nb = 0, m_na = 0;
    for (uint32_t a = 0; a < 3; a++) {
        const float l = c3(blo, a), h = c3(bhi, a);
        if (!(__fsub_rn(h, l) > 0.0f)) continue;
        if (tid == 0) S.nflat = 0;
        __syncthreads();
        for (uint32_t i = tid; i < n2; i += blockDim.x) {
            float lo = kInf, hi = kInf;
            if (i < cnt) {
                const uint32_t tri = A.refs()[info.x + i];
                lo = mxf(c3(A.tb_lo[tri], a), l);
                hi = mnf(c3(A.tb_hi[tri], a), h);
                if (lo == hi) S.fl[atomicAdd(&S.nflat, 1u)] = lo;   // flat references, any order
            }
            S.lo[i] = lo;
            S.hi[i] = hi;
        }
        __syncthreads();
        const uint32_t nfl = S.nflat;
        uint32_t nf2 = nfl ? 1u : 0u;
        while (nf2 < nfl) nf2 <<= 1;
        for (uint32_t i = nfl + tid; i < nf2; i += blockDim.x) S.fl[i] = kInf;
        __syncthreads();
        for (uint32_t k = 2; k <= n2; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = tid; i < n2; i += blockDim.x) {
                    const uint32_t ixj = i ^ j;
                    if (ixj > i) {
                        const bool up = (i & k) == 0;
                        float x = S.lo[i], y = S.lo[ixj];
                        if ((x > y) == up) {
                            S.lo[i] = y;
                            S.lo[ixj] = x;
                        }
                        x = S.hi[i];
                        y = S.hi[ixj];
                        if ((x > y) == up) {
                            S.hi[i] = y;
                            S.hi[ixj] = x;
                        }
                        if (i < nf2 && ixj < nf2 && k <= nf2) {
                            x = S.fl[i];
                            y = S.fl[ixj];
                            if ((x > y) == up) {
                                S.fl[i] = y;
                                S.fl[ixj] = x;
                            }
                        }
                    }
                }
                __syncthreads();
            }
        for (uint32_t q = tid; q < 2 * cnt; q += blockDim.x) {
            const float pk = __fadd_rn(q < cnt ? S.lo[q] : S.hi[q - cnt], 0.0f);
            if (!(pk > l && pk < h)) continue;
            const uint32_t fon = nfl ? upper_bound_f(S.fl, nfl, pk) - lower_bound_f(S.fl, nfl, pk) : 0u;
            const uint32_t nb = lower_bound_f(S.lo, cnt, pk) + fon;
            const uint32_t na = (cnt - upper_bound_f(S.hi, cnt, pk)) + fon;
            float4 bb = bhi, ba = blo;
            s3(bb, a, pk);
            s3(ba, a, pk);
            const float sb = surf(blo, bb), sa = surf(ba, bhi);
            const float cost = __fadd_rn(
                ct, __fmul_rn(ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)nb), __fmul_rn(sa, (float)na)), Anode)));
            if (cost < mc || (cost == mc && a == m_ax && pk < m_pk)) {
                mc = cost;
                m_ax = a;
                m_pk = pk;
                m_nb = nb;
                m_na = na;
            }
        }
        __syncthreads();
    }
    // argmin over (cost, axis, plane): warps, then warp 0 over the warps
    float bc = mc, bp = m_pk;
    uint32_t bax = m_ax, bkey = tid;
    for (int off = 16; off; off >>= 1) {
        const float oc = __shfl_xor_sync(0xffffffffu, bc, off), op = __shfl_xor_sync(0xffffffffu, bp, off);
        const uint32_t oax = __shfl_xor_sync(0xffffffffu, bax, off), ok = __shfl_xor_sync(0xffffffffu, bkey, off);
        if (oc < bc || (oc == bc && (oax < bax || (oax == bax && (op < bp || (op == bp && ok < bkey)))))) {
            bc = oc;
            bp = op;
            bax = oax;
            bkey = ok;
        }
    }
    if (lane == 0) {
        S.w_cost[wid] = bc;
        S.w_pk[wid] = bp;
        S.w_ax[wid] = bax;
        S.w_key[wid] = bkey;
    }
    // the winning thread of each warp publishes its counts
    if (tid == bkey) {
        S.w_nb[wid] = m_nb;
        S.w_na[wid] = m_na;
    }
    __syncthreads();
    const uint32_t nw = blockDim.x >> 5;
    float fc = S.w_cost[0], fp = S.w_pk[0];
    uint32_t fax = S.w_ax[0], fw = 0;
    for (uint32_t w = 1; w < nw; w++) {
        const float oc = S.w_cost[w], op = S.w_pk[w];
        const uint32_t oax = S.w_ax[w];
        if (oc < fc || (oc == fc && (oax < fax || (oax == fax && op < fp)))) {
            fc = oc;
            fp = op;
            fax = oax;
            fw = w;
        }
    }
    Decision best{-1, 0.0f, 0, 0, kInf, 0};
    if (fc < kInf) {
        best.axis = (int)fax;
        best.plane = fp;
        best.nb = S.w_nb[fw];
        best.na = S.w_na[fw];
        best.cost = fc;
        best.bin = 0;
    }
    if (best.axis >= 0 && !(best.cost < __fmul_rn(ci, (float)cnt))) best.axis = -1;
    __syncthreads();
    return best;
}

// Large nodes, binned mode: one CTA per chunk of 1024 references builds the
// chunk's histograms in shared memory and adds them to the node's global
// histogram; the CTA that finishes the node's last chunk evaluates the SAH.
// the binned SAH of a large node from its complete histogram (one warp): a
// proposer row keeps the binned decision and the features for k_refine_cta /
// k_refine_warp, every other node is decided here
template <class HistPtr>
__device__ __forceinline__ void finish_large(const LevelArgs &A, uint32_t s, const uint4 &info, float4 blo,
                                             float4 bhi, HistPtr H, Tally &tally) {
    const uint32_t lane = threadIdx.x & 31u;
    const Decision d = sah_warp(H, blo, bhi, info.y, A.ct, A.ci);
    if (is_learn(A, info.y)) {
        uint32_t row = 0;
        if (lane == 0) row = atomicAdd(&A.lc->n_learn, 1u);
        row = __shfl_sync(0xffffffffu, row, 0);
        if (row < A.cap_learn) {
            if (lane == 0) {
                A.learn_slot[row] = s;
                A.learn_bin[row] = LearnBin{d.cost, d.plane, d.axis, d.nb, d.na, {info.y, 0, 0}};
            }
            hist_features(H, info.y, blo, bhi, A.level, A.max_depth, A.feat + (size_t)row * 200);
            return;
        }
    }
    if (lane == 0) {
        write_decision(A, s, d);
        tally.add(d, info.y);
    }
}

// shared memory of a CTA's large-node work
struct HistSmem {
    uint32_t H[kHist];
    float P[kPlanes];
    int last;
};

// k_hist's work for one level (every CTA of the grid calls it): the chunks of
// the large nodes and, with MEDIUM, the medium nodes (exact SAH, XS)
template <bool MEDIUM>
__device__ __forceinline__ void hist_body(const LevelArgs &A, HistSmem &SH, ExactCtaSmem *XSp, Tally &tally) {
    uint32_t *H = SH.H;
    int &s_last = SH.last;
    const uint32_t wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nch = min(A.lc->n_chunks, A.cap_chunks);
    const uint32_t nmed = MEDIUM ? min(A.lc->n_medium, A.cap_medium) : 0u;
    const uint32_t nodes = A.lc->nodes;
    for (uint32_t item = blockIdx.x; item < nch + nmed; item += gridDim.x) {
        if (MEDIUM && item >= nch) {
            // a medium node: the exact SAH in this CTA
            const uint32_t s = A.medium_slot[item - nch];
            if (s >= nodes) continue;
            const uint4 info = A.n_info()[s];
            const float4 blo = A.n_lo()[s], bhi = A.n_hi()[s];
            const Decision d = sah_exact_cta(A, info, blo, bhi, A.ct, A.ci, *XSp);
            if (threadIdx.x == 0) {
                write_decision(A, s, d);
                tally.add(d, info.y);
            }
            if (A.record && d.axis >= 0 && info.y <= kLearnMax) {
                // a training row: the node's binned histogram as features, the
                // bin of the exact plane as label (every thread holds d)
                for (uint32_t i = threadIdx.x; i < kHist; i += blockDim.x) H[i] = 0;
                __syncthreads();
                const float4 inv3 = bin_scale(blo, bhi);
                for (uint32_t r = info.x + threadIdx.x; r < info.x + info.y; r += blockDim.x) {
                    const uint32_t tri = A.refs()[r];
                    hist_ref(H, A.tb_lo[tri], A.tb_hi[tri], blo, bhi, inv3);
                }
                __syncthreads();
                if (wib == 0) {
                    uint32_t row = 0;
                    if (lane == 0) row = atomicAdd(A.rec_rows, 1u);
                    row = __shfl_sync(0xffffffffu, row, 0);
                    if (row < A.rec_cap) {
                        hist_features(H, info.y, blo, bhi, A.level, A.max_depth, A.rec_X + (size_t)row * 200);
                        if (lane == 0) A.rec_y[row] = exact_label(d.axis, d.plane, blo, bhi);
                    }
                }
                __syncthreads();
            }
            continue;
        }
        const uint2 ck = A.chunks[item];
        const uint32_t rank = ck.x;
        if (rank >= A.cap_large) continue;  // uniform per CTA
        const uint32_t s = A.large_slot[rank];
        if (s >= nodes) continue;
        const uint4 info = A.n_info()[s];
        const float4 blo = A.n_lo()[s], bhi = A.n_hi()[s];
        const uint32_t r0 = info.x + ck.y * kChunk, r1 = min(info.x + info.y, r0 + kChunk);
        for (uint32_t i = threadIdx.x; i < kHist; i += blockDim.x) H[i] = 0;
        node_planes_cta(SH.P, blo, bhi);
        __syncthreads();
        {
            // all of the thread's references and bounds loaded first
            constexpr int kPer = kChunk / 256;
            const float4 inv3 = bin_scale(blo, bhi);
            uint32_t tri[kPer];
            float4 tlo[kPer], thi[kPer];
#pragma unroll
            for (int k = 0; k < kPer; k++) {
                const uint32_t r = r0 + threadIdx.x + 256u * k;
                tri[k] = r < r1 ? A.refs()[r] : 0xffffffffu;
            }
#pragma unroll
            for (int k = 0; k < kPer; k++)
                if (tri[k] != 0xffffffffu) {
                    tlo[k] = A.tb_lo[tri[k]];
                    thi[k] = A.tb_hi[tri[k]];
                }
#pragma unroll
            for (int k = 0; k < kPer; k++)
                if (tri[k] != 0xffffffffu) hist_ref_tab(H, tlo[k], thi[k], blo, bhi, inv3, SH.P);
        }
        __syncthreads();
        if (info.y <= kChunk) {
            // the node's only chunk: its histogram is complete in shared memory
            if (wib == 0) finish_large(A, s, info, blo, bhi, H, tally);
            __syncthreads();
            continue;
        }
        uint32_t *G = A.hist + (size_t)rank * kHist;
        for (uint32_t i = threadIdx.x; i < kHist; i += blockDim.x)
            if (H[i]) atomicAdd(&G[i], H[i]);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t nchunks = (info.y + kChunk - 1) / kChunk;
            s_last = (atomicAdd(&A.done[rank], 1u) == nchunks - 1) ? 1 : 0;
        }
        __syncthreads();
        if (s_last && wib == 0) {
            __threadfence();
            finish_large(A, s, info, blo, bhi, GHist{G}, tally);
            // clean the histogram and the done counter for the next level
            __syncwarp();
            for (uint32_t i = lane; i < kHist; i += 32) G[i] = 0;
            if (lane == 0) A.done[rank] = 0;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256, 3) k_hist(LevelArgs A) {
    __shared__ HistSmem SH;
    __shared__ ExactCtaSmem XS;
    __shared__ uint32_t s_tally[kTallies];
    if (level_aborted(A)) return;
    Tally tally;
    hist_body<true>(A, SH, &XS, tally);
    tally_flush(A, tally, s_tally);
}

// Small nodes (not splittable, or splittable and neither medium nor large):
// one warp per node; the exact SAH in registers for nodes of at most 32
// references when exact_max >= 32 or in learned mode (the WARP_EXACT
// instantiations), else a warp-private histogram + the binned SAH. In learned
// mode (LEARNED) a node of 33..1024 references becomes a proposer row: its
// binned decision and histogram features are stored for k_learn, which
// decides it (a node past the row capacity keeps the binned decision).
template <bool WARP_EXACT, bool LEARNED>
__device__ __forceinline__ void small_body(const LevelArgs &A, uint32_t (*HS)[kHist], float (*PS)[kPlanes],
                                           Tally &tally) {
    const uint32_t wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t nodes = A.lc->nodes;
    const uint32_t ngroups = (nodes + 7) / 8;
    for (uint32_t g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const uint32_t s = g * 8 + wib;
        if (s >= nodes) continue;
        const uint4 info = A.n_info()[s];
        const uint32_t cnt = info.y;
        const bool dec = decidable(A, cnt);
        if (dec && (is_large(A, cnt) || is_medium(A, cnt))) continue;   // k_hist
        if (!dec || is_deferred(A, cnt)) {
            // a leaf, or the root of a subtree built after the levels
            if (lane == 0) {
                const Decision leaf{dec ? kDeferAxis : -1, 0.0f, 0, 0, kInf, 0};
                write_decision(A, s, leaf);
                tally.add(leaf, cnt);
            }
            continue;
        }
        const float4 blo = A.n_lo()[s], bhi = A.n_hi()[s];
        Decision d;
        if (WARP_EXACT && cnt <= kWarpExact) {
            d = sah_exact_warp32(A, info, blo, bhi, A.ct, A.ci);
        } else {
            uint32_t *Hw = HS[wib];
            float *Pw = PS[wib];
            __syncwarp();   // the previous node's readers are done
            {
                // 288 counters = 72 16-byte stores
                uint4 *H4 = reinterpret_cast<uint4 *>(Hw);
                H4[lane] = make_uint4(0, 0, 0, 0);
                H4[lane + 32] = make_uint4(0, 0, 0, 0);
                if (lane < kHist / 4 - 64) H4[lane + 64] = make_uint4(0, 0, 0, 0);
            }
            node_planes_warp(Pw, blo, bhi);
            __syncwarp();
            const float4 inv3 = bin_scale(blo, bhi);
            for (uint32_t r = info.x + lane; r < info.x + cnt; r += 32) {
                const uint32_t tri = A.refs()[r];
                hist_ref_tab(Hw, A.tb_lo[tri], A.tb_hi[tri], blo, bhi, inv3, Pw);
            }
            __syncwarp();
            d = sah_warp(Hw, blo, bhi, cnt, A.ct, A.ci);
            if (LEARNED && is_learn(A, cnt)) {
                uint32_t row = 0;
                if (lane == 0) row = atomicAdd(&A.lc->n_learn, 1u);
                row = __shfl_sync(0xffffffffu, row, 0);
                if (row < A.cap_learn) {
                    if (lane == 0) {
                        A.learn_slot[row] = s;
                        A.learn_bin[row] = LearnBin{d.cost, d.plane, d.axis, d.nb, d.na, {info.y, 0, 0}};
                    }
                    hist_features(Hw, cnt, blo, bhi, A.level, A.max_depth, A.feat + (size_t)row * 200);
                    continue;   // decided and tallied by k_learn
                }
            }
        }
        if (lane == 0) {
            write_decision(A, s, d, blo, bhi);
            tally.add(d, cnt);
        }
        __syncwarp();
    }
}

template <bool WARP_EXACT, bool LEARNED>
__global__ void __launch_bounds__(256, 5) k_small(LevelArgs A) {
    __shared__ __align__(16) uint32_t HS[8][kHist];
    __shared__ float PS[8][kPlanes];
    __shared__ uint32_t s_tally[kTallies];
    wait_prior_grid();
    if (level_aborted(A)) return;
    Tally tally;
    small_body<WARP_EXACT, LEARNED>(A, HS, PS, tally);
    tally_flush(A, tally, s_tally);
}

// Binned mode (no medium nodes, no proposer): a level's large-node chunks and
// small nodes in one launch on the build's stream, PDL-chained to the plan
// (no second stream, no fork and join per level)
union DecideSmem {
    HistSmem hist;
    struct {
        uint32_t HS[8][kHist];
        float PS[8][kPlanes];
    } small;
};

__global__ void __launch_bounds__(256, 4) k_decide(LevelArgs A) {
    __shared__ __align__(16) DecideSmem sm;
    __shared__ uint32_t s_tally[kTallies];
    wait_prior_grid();
    if (level_aborted(A)) return;
    Tally tally;
    hist_body<false>(A, sm.hist, nullptr, tally);
    __syncthreads();
    small_body<false, false>(A, sm.small.HS, sm.small.PS, tally);
    tally_flush(A, tally, s_tally);
}

constexpr int kLearnMaxK = 8;
constexpr uint32_t kLearnScratch = 2048;   // floats of list space per warp
constexpr size_t kRefineSmem = (size_t)kLearnScratch * 4;   // the lists of one row, 8 KB

// list capacity per (proposal, list): the largest power of two with 3 k of
// them in one warp's space (128 for k = 4), so a list sorts in place
__host__ __device__ constexpr uint32_t learn_list_cap(uint32_t K) {
    uint32_t c = 1;
    while (2 * c * 3 * K <= kLearnScratch) c *= 2;
    return c;
}
// lists of up to 32 x kLearnSortRegs values sort in registers (every list
// with k >= 4 proposals); longer ones in shared memory
constexpr int kLearnSortRegs = 4;

// warp-aggregated append of val (where pred) to list[n ..); n counts past cap
__device__ __forceinline__ void list_append(float *list, uint32_t cap, uint32_t &n, bool pred, float val) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t m = __ballot_sync(0xffffffffu, pred);
    if (pred) {
        const uint32_t pos = n + __popc(m & ((1u << lane) - 1u));
        if (pos < cap) list[pos] = val;
    }
    n += __popc(m);
}

// ascending bitonic sort of v[0, n) in shared memory by one warp; the list's
// capacity is a power of two >= n, the padding up to the next power of two
// is filled with +inf
__device__ __forceinline__ void warp_sort_smem(float *v, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t n2 = 1;
    while (n2 < n) n2 <<= 1;
    for (uint32_t i = n + lane; i < n2; i += 32) v[i] = kInf;
    __syncwarp();
    for (uint32_t k = 2; k <= n2; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < n2; i += 32) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const float x = v[i], y = v[ixj];
                    if ((x > y) == up) {
                        v[i] = y;
                        v[ixj] = x;
                    }
                }
            }
            __syncwarp();
        }
}

// ascending bitonic sort of v[0, n) by one warp, done in registers: element
// r * 32 + lane of the list padded with +inf to the next power of two in x[r]
// of that lane (R registers, up to 32 R elements), every compare-exchange a
// shuffle (partner in another lane) or a swap between two of the lane's
// registers; the sorted list is written back to v[0, n)
template <int R>
__device__ __forceinline__ void warp_sort_regs(float *v, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t n2 = 1;
    while (n2 < n) n2 <<= 1;
    const uint32_t nr = (n2 + 31u) >> 5;
    float x[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
        const uint32_t i = (uint32_t)r * 32u + lane;
        x[r] = i < n ? v[i] : kInf;
    }
    for (uint32_t k = 2; k <= n2; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const uint32_t rj = j >> 5;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    if ((uint32_t)r >= nr || ((uint32_t)r & rj)) continue;
                    const int r2 = r | (int)rj;
                    const bool up = (((uint32_t)r * 32u + lane) & k) == 0;
                    const float a = x[r], b = x[r2];
                    if ((a > b) == up) {
                        x[r] = b;
                        x[r2] = a;
                    }
                }
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    if ((uint32_t)r >= nr) continue;
                    const float p = __shfl_xor_sync(0xffffffffu, x[r], (int)j);
                    const bool up = (((uint32_t)r * 32u + lane) & k) == 0;
                    const float mn = x[r] < p ? x[r] : p, mx = x[r] < p ? p : x[r];
                    x[r] = (lower == up) ? mn : mx;
                }
            }
        }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < R; r++) {
        const uint32_t i = (uint32_t)r * 32u + lane;
        if (i < n) v[i] = x[r];
    }
    __syncwarp();
}

__device__ __forceinline__ void warp_sort_list(float *v, uint32_t n) {
    if (n <= 32u * kLearnSortRegs) warp_sort_regs<kLearnSortRegs>(v, n);
    else warp_sort_smem(v, n);
}

// ---------------------------------------------------------------------------
// learned split search (no reference counterpart), two launches per level.
// k_learn: the network on the level's proposer rows (tcgen05: 128-row tiles,
// hk_mlp_tc.cuh; else mma.sync: 64-row tiles, hk_mlp_tile.cuh), then per row
// the top-k valid bins by logit (ties to the lower index; an axis of zero
// extent has no valid bin), one byte each (axis * 32 + bin, 0xff: none) in
// learn_prop.
// ---------------------------------------------------------------------------
template <bool TC>
__global__ void __launch_bounds__(256, 1) k_learn(LevelArgs A) {
    extern __shared__ __align__(1024) unsigned char learn_smem[];
    constexpr uint32_t kRows = TC ? (uint32_t)kTcRows : (uint32_t)kTileRows;
    wait_prior_grid();
    if (level_aborted(A)) return;
    const uint32_t rows = min(A.lc->n_learn, A.cap_learn);
    if (blockIdx.x * kRows >= rows) return;   // no tile: no TMEM taken (the CTA takes part in no barrier)
    const TileSmem S = tile_smem(learn_smem);
    const TcSmem T = tc_smem(learn_smem);
    uint32_t tmem = 0, g = 0;
    if (TC) tmem = tc_setup(T);
    const uint32_t K = A.topk < (uint32_t)kLearnMaxK ? (A.topk ? A.topk : 1u) : (uint32_t)kLearnMaxK;
    const float *logits = TC ? T.logits : S.logits;
    for (uint32_t row0 = blockIdx.x * kRows; row0 < rows; row0 += gridDim.x * kRows) {
        if constexpr (TC) {
            if (!tc_tile_forward(A.mlp, A.feat, row0, rows, T, tmem, g, A.err)) break;
        } else {
            tile_forward(A.mlp, A.feat, row0, rows, S);
        }
        // one thread per row (rr = threadIdx.x): a row's candidates are the
        // bins of its node's axes of nonzero extent, a NaN logit counting as
        // -inf, taken as the logits' bits in an order-preserving unsigned form
        // (-inf maps to 0x007fffff; an empty slot holds 0, below every
        // candidate). The candidates pass in index order through a sorted
        // list of NS slots, a candidate moving ahead of a slot only when its
        // key is strictly greater: the k best by (logit, then the lower index).
        constexpr uint32_t kStride = TC ? kTcLogitStride : (uint32_t)kMlpOut;
        const uint32_t rr = threadIdx.x;
        if (rr < kRows && row0 + rr < rows) {
            const uint32_t row = row0 + rr;
            const uint32_t slot = A.learn_slot[row];
            const float4 blo = A.n_lo()[slot], bhi = A.n_hi()[slot];
            const float *Lg = logits + rr * kStride;
            uint32_t tk[kLearnMaxK], tix[kLearnMaxK];
#pragma unroll
            for (int i = 0; i < kLearnMaxK; i++) tk[i] = 0u, tix[i] = 0xffu;
            auto select = [&](auto ns_tag) {
                constexpr int NS = decltype(ns_tag)::value;
#pragma unroll
                for (uint32_t j = 0; j < 3; j++) {
                    if (!(__fsub_rn(c3(bhi, j), c3(blo, j)) > 0.0f)) continue;
#pragma unroll 4
                    for (uint32_t k = 0; k < 32; k++) {
                        float x = Lg[32u * j + k];
                        if (x != x) x = -INFINITY;
                        if (x == 0.0f) x = 0.0f;   // -0 ties with +0, as the values compare
                        const uint32_t u = __float_as_uint(x);
                        uint32_t key = (u & 0x80000000u) ? ~u : (u | 0x80000000u), c = 32u * j + k;
#pragma unroll
                        for (int i = 0; i < NS; i++) {
                            const bool sw = key > tk[i];
                            const uint32_t k2 = sw ? tk[i] : key, c2 = sw ? tix[i] : c;
                            tk[i] = sw ? key : tk[i];
                            tix[i] = sw ? c : tix[i];
                            key = k2;
                            c = c2;
                        }
                    }
                }
            };
            if (K <= 4) select(std::integral_constant<int, 4>{});
            else select(std::integral_constant<int, kLearnMaxK>{});
            uint32_t packed[2] = {0xffffffffu, 0xffffffffu};
#pragma unroll
            for (uint32_t r = 0; r < (uint32_t)kLearnMaxK; r++)
                if (r < K && tk[r] != 0u) {
                    const uint32_t sh = 8u * (r & 3u);
                    packed[r >> 2] = (packed[r >> 2] & ~(0xffu << sh)) | (tix[r] << sh);
                }
            A.learn_prop[row] = make_uint2(packed[0], packed[1]);
            if (A.prop_log) {
                const uint32_t cidx = A.n_info()[slot].z;
                if (cidx < A.cap_nodes)
#pragma unroll
                    for (uint32_t r = 0; r < 8; r++) {
                        const uint32_t bb = (packed[r >> 2] >> (8u * (r & 3u))) & 0xffu;
                        A.prop_log[(size_t)cidx * 8 + r] = bb == 0xffu ? -1 : (int32_t)bb;
                    }
            }
        }
        __syncthreads();   // the logits are rewritten by the next tile
    }
    if (TC) tc_teardown(tmem);
}

// ---------------------------------------------------------------------------
// k_refine_cta: one CTA per proposer row of more than kRefineWarpMax
// references, grid-striding over the level's rows (k_refine_warp takes the
// others).
//   1. the 256 threads pass over the node's references once: per proposed bin
//      (axis a, bin b, the closed interval [P0, P1] = [p_b, p_{b+1}] with p_0
//      the node's minimum and p_32 its maximum) the references whose clipped
//      lower bound lies below P0 and those whose clipped upper bound lies
//      above P1 are counted, and the lower bounds, upper bounds and flat
//      references inside [P0, P1] are listed in shared memory (slots taken
//      per warp with one shared atomic: the order of a list is arbitrary, its
//      contents are not);
//   2. each warp sorts some of the lists (in registers);
//   3. every listed bound p strictly inside the node is a candidate -- the
//      exact SAH's candidates that fall in the bin -- with
//        below = #(lo < P0) + #(listed lo < p) + #(listed flat at p),
//        above = #(hi > P1) + #(listed hi > p) + #(listed flat at p)
//      (binary searches in the sorted lists), the exact SAH's own counts; the
//      threads share the candidates and the cheapest by (cost, axis, plane)
//      wins (equal keys are the same plane with the same counts);
//   4. that plane is taken unless it costs more than fallback_ratio x the
//      binned optimum k_small found for the node (then the binned plane); the
//      usual leaf test follows.
// A bin whose lists overflow their capacity (learn_list_cap) is not costed.
// ---------------------------------------------------------------------------
constexpr uint32_t kRefineThreads = 256;
constexpr uint32_t kRefineWarpMax = 128;   // rows up to this many references: one warp each
constexpr uint32_t kRefineRowWarps = 8;
constexpr size_t kRefineWarpSmem = (size_t)kRefineRowWarps * kLearnScratch * 4;   // 64 KB
// k_refine_warp's grid in CTAs per SM: more than are resident (two, by its
// registers), so that CTAs finishing early are replaced by new ones
constexpr int kRefineWarpGrid = 3;

__device__ __forceinline__ bool refine_better(float c, uint32_t a, float p, float bc, uint32_t ba, float bp) {
    return c < bc || (c == bc && (a < ba || (a == ba && p < bp)));
}

__global__ void __launch_bounds__(kRefineThreads) k_refine_cta(LevelArgs A) {
    extern __shared__ __align__(16) float refine_smem[];
    __shared__ uint32_t s_tally[kTallies];
    __shared__ uint32_t s_stat[2];
    __shared__ uint32_t s_n[3 * kLearnMaxK], s_bl[kLearnMaxK], s_ab[kLearnMaxK];
    __shared__ float s_wc[kRefineThreads / 32], s_wp[kRefineThreads / 32];
    __shared__ uint32_t s_wa[kRefineThreads / 32], s_wnb[kRefineThreads / 32], s_wna[kRefineThreads / 32];
    wait_prior_grid();
    if (level_aborted(A)) return;
    Tally tally;
    uint32_t n_learned = 0, n_fallback = 0;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, wib = tid >> 5;
    constexpr uint32_t kWarps = kRefineThreads / 32;
    const uint32_t rows = min(A.lc->n_learn, A.cap_learn);
    const uint32_t K = A.topk < (uint32_t)kLearnMaxK ? (A.topk ? A.topk : 1u) : (uint32_t)kLearnMaxK;
    const uint32_t cap = learn_list_cap(K);
    for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x) {
        const LearnBin lb = A.learn_bin[row];
        if (lb.pad[0] <= kRefineWarpMax) continue;   // k_refine_warp's row (uniform over the CTA)
        const uint32_t s = A.learn_slot[row];
        const uint4 info = A.n_info()[s];
        const float4 blo = A.n_lo()[s], bhi = A.n_hi()[s];
        const uint32_t cnt = info.y;
        const uint2 pp = A.learn_prop[row];
        uint32_t pax[kLearnMaxK];
        float p0[kLearnMaxK], p1[kLearnMaxK];
        uint32_t np = 0;
#pragma unroll
        for (int r = 0; r < kLearnMaxK; r++) {
            const uint32_t b8 = ((r < 4 ? pp.x : pp.y) >> (8 * (r & 3))) & 0xffu;
            if (b8 == 0xffu || (uint32_t)r >= K) break;
            const uint32_t a = b8 >> 5, b = b8 & 31u;
            const float l = c3(blo, a), h = c3(bhi, a), ext = __fsub_rn(h, l);
            pax[r] = a;
            p0[r] = b == 0 ? l : plane_k(l, ext, b);
            p1[r] = b == kBins - 1 ? h : plane_k(l, ext, b + 1);
            np++;
        }
        if (tid < 3 * kLearnMaxK) s_n[tid] = 0;
        if (tid < kLearnMaxK) s_bl[tid] = s_ab[tid] = 0;
        __syncthreads();
        // 1. counts and lists over the node's references
        uint32_t bl[kLearnMaxK], ab[kLearnMaxK];
#pragma unroll
        for (int i = 0; i < kLearnMaxK; i++) bl[i] = ab[i] = 0;
        for (uint32_t base = 0; base < cnt; base += kRefineThreads) {
            const bool have = base + tid < cnt;
            float4 tlo = make_float4(0, 0, 0, 0), thi = tlo;
            if (have) {
                const uint32_t tri = A.refs()[info.x + base + tid];
                tlo = A.tb_lo[tri];
                thi = A.tb_hi[tri];
            }
#pragma unroll
            for (int i = 0; i < kLearnMaxK; i++) {
                if ((uint32_t)i >= np) break;
                const uint32_t a = pax[i];
                const float l = c3(blo, a), h = c3(bhi, a);
                const float lo = mxf(c3(tlo, a), l), hi = mnf(c3(thi, a), h);
                bl[i] += (have && lo < p0[i]) ? 1u : 0u;
                ab[i] += (have && hi > p1[i]) ? 1u : 0u;
                const bool inL = have && p0[i] <= lo && lo <= p1[i];
                const bool inH = have && p0[i] <= hi && hi <= p1[i];
                const bool inF = inL && lo == hi;
                float *Ls = refine_smem + (size_t)i * 3 * cap;
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const bool pred = q == 0 ? inL : (q == 1 ? inH : inF);
                    const uint32_t m = __ballot_sync(0xffffffffu, pred);
                    if (!m) continue;
                    uint32_t pos0 = 0;
                    if (lane == (uint32_t)(__ffs(m) - 1)) pos0 = atomicAdd(&s_n[3 * i + q], (uint32_t)__popc(m));
                    pos0 = __shfl_sync(0xffffffffu, pos0, __ffs(m) - 1);
                    if (pred) {
                        const uint32_t pos = pos0 + __popc(m & ((1u << lane) - 1u));
                        if (pos < cap) Ls[(size_t)q * cap + pos] = q == 1 ? hi : lo;
                    }
                }
            }
        }
#pragma unroll
        for (int i = 0; i < kLearnMaxK; i++) {
            if ((uint32_t)i >= np) break;
            uint32_t b0 = bl[i], a0 = ab[i];
            for (int o = 16; o; o >>= 1) {
                b0 += __shfl_xor_sync(0xffffffffu, b0, o);
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            }
            if (lane == 0) {
                if (b0) atomicAdd(&s_bl[i], b0);
                if (a0) atomicAdd(&s_ab[i], a0);
            }
        }
        __syncthreads();
        // 2. sort the lists of the bins that did not overflow
        for (uint32_t j = wib; j < 3 * np; j += kWarps) {
            const uint32_t i = j / 3;
            if (s_n[3 * i] > cap || s_n[3 * i + 1] > cap || s_n[3 * i + 2] > cap) continue;
            const uint32_t n = s_n[j];
            if (n > 1) warp_sort_list(refine_smem + (size_t)j * cap, n);
        }
        __syncthreads();
        // 3. exact costs of the listed candidates
        const float Anode = surf(blo, bhi);
        float mc = kInf, m_pk = 0.0f;
        uint32_t m_ax = 3, m_nb = 0, m_na = 0;
        for (uint32_t i = 0; i < np; i++) {
            const uint32_t nl = s_n[3 * i], nh = s_n[3 * i + 1], nf = s_n[3 * i + 2];
            if (nl > cap || nh > cap || nf > cap) continue;   // overflowed: not costed
            const uint32_t a = pax[i], b0 = s_bl[i], a0 = s_ab[i];
            const float l = c3(blo, a), h = c3(bhi, a);
            const float *Ls = refine_smem + (size_t)i * 3 * cap, *Hs = Ls + cap, *Fs = Ls + 2 * cap;
            for (uint32_t q = tid; q < nl + nh; q += kRefineThreads) {
                const float x = q < nl ? Ls[q] : Hs[q - nl];
                if (!(x > l && x < h)) continue;
                const float pk = __fadd_rn(x, 0.0f);
                const uint32_t fon = nf ? upper_bound_f(Fs, nf, pk) - lower_bound_f(Fs, nf, pk) : 0u;
                const uint32_t nb = b0 + lower_bound_f(Ls, nl, pk) + fon;
                const uint32_t na = a0 + (nh - upper_bound_f(Hs, nh, pk)) + fon;
                float4 bb = bhi, ba = blo;
                s3(bb, a, pk);
                s3(ba, a, pk);
                const float sb = surf(blo, bb), sa = surf(ba, bhi);
                const float cost = __fadd_rn(
                    A.ct,
                    __fmul_rn(A.ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)nb), __fmul_rn(sa, (float)na)), Anode)));
                if (refine_better(cost, a, pk, mc, m_ax, m_pk)) {
                    mc = cost;
                    m_ax = a;
                    m_pk = pk;
                    m_nb = nb;
                    m_na = na;
                }
            }
        }
        // 4. the cheapest over the CTA
        for (int off = 16; off; off >>= 1) {
            const float oc = __shfl_xor_sync(0xffffffffu, mc, off), op = __shfl_xor_sync(0xffffffffu, m_pk, off);
            const uint32_t oa = __shfl_xor_sync(0xffffffffu, m_ax, off);
            const uint32_t onb = __shfl_xor_sync(0xffffffffu, m_nb, off), ona = __shfl_xor_sync(0xffffffffu, m_na, off);
            if (refine_better(oc, oa, op, mc, m_ax, m_pk)) {
                mc = oc;
                m_pk = op;
                m_ax = oa;
                m_nb = onb;
                m_na = ona;
            }
        }
        if (lane == 0) {
            s_wc[wib] = mc;
            s_wp[wib] = m_pk;
            s_wa[wib] = m_ax;
            s_wnb[wib] = m_nb;
            s_wna[wib] = m_na;
        }
        __syncthreads();
        if (tid == 0) {
            float bc = s_wc[0], bp = s_wp[0];
            uint32_t bax = s_wa[0], nb = s_wnb[0], na = s_wna[0];
            for (uint32_t w = 1; w < kWarps; w++)
                if (refine_better(s_wc[w], s_wa[w], s_wp[w], bc, bax, bp)) {
                    bc = s_wc[w];
                    bp = s_wp[w];
                    bax = s_wa[w];
                    nb = s_wnb[w];
                    na = s_wna[w];
                }
            // 5. the proposal's plane, or the binned optimum
            const bool take = bc < kInf && bc <= __fmul_rn(A.fallback_ratio, lb.cost);
            Decision d;
            if (take) {
                d = Decision{(int)bax, bp, nb, na, bc, 0};
                if (!(bc < __fmul_rn(A.ci, (float)cnt))) d.axis = -1;
            } else {
                d = Decision{lb.axis, lb.plane, lb.nb, lb.na, lb.cost, 0};
            }
            write_decision(A, s, d, blo, bhi);
            tally.add(d, cnt);
            if (take) n_learned++;
            else n_fallback++;
        }
        __syncthreads();
    }
    if (threadIdx.x < 2) s_stat[threadIdx.x] = 0;
    __syncthreads();
    if (n_learned) atomicAdd(&s_stat[0], n_learned);
    if (n_fallback) atomicAdd(&s_stat[1], n_fallback);
    __syncthreads();
    if (threadIdx.x == 0 && s_stat[0]) atomicAdd(&A.ctr->learned_nodes, s_stat[0]);
    if (threadIdx.x == 1 && s_stat[1]) atomicAdd(&A.ctr->fallback_nodes, s_stat[1]);
    tally_flush(A, tally, s_tally);
}

// rows of at most kRefineWarpMax references: one warp per row, eight rows per
// CTA, the same three steps with the lists in the warp's own shared memory
__global__ void __launch_bounds__(256) k_refine_warp(LevelArgs A) {
    extern __shared__ __align__(16) float refine_smem[];
    __shared__ uint32_t s_tally[kTallies];
    __shared__ uint32_t s_stat[2];
    wait_prior_grid();
    if (level_aborted(A)) return;
    Tally tally;
    uint32_t n_learned = 0, n_fallback = 0;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t rows = min(A.lc->n_learn, A.cap_learn);
    const uint32_t K = A.topk < (uint32_t)kLearnMaxK ? (A.topk ? A.topk : 1u) : (uint32_t)kLearnMaxK;
    const uint32_t cap = learn_list_cap(K);
    float *scratch = refine_smem + (size_t)wib * kLearnScratch;
    for (uint32_t row = blockIdx.x * kRefineRowWarps + wib; row < rows; row += gridDim.x * kRefineRowWarps) {
        const LearnBin lb = A.learn_bin[row];
        if (lb.pad[0] > kRefineWarpMax) continue;   // k_refine_cta's row
        const uint32_t s = A.learn_slot[row];
        const uint4 info = A.n_info()[s];
        const float4 blo = A.n_lo()[s], bhi = A.n_hi()[s];
        const uint32_t cnt = info.y;
        const uint2 pp = A.learn_prop[row];
        uint32_t pax[kLearnMaxK];
        float p0[kLearnMaxK], p1[kLearnMaxK];
        uint32_t np = 0;
#pragma unroll
        for (int r = 0; r < kLearnMaxK; r++) {
            const uint32_t b8 = ((r < 4 ? pp.x : pp.y) >> (8 * (r & 3))) & 0xffu;
            if (b8 == 0xffu || (uint32_t)r >= K) break;
            const uint32_t a = b8 >> 5, b = b8 & 31u;
            const float l = c3(blo, a), h = c3(bhi, a), ext = __fsub_rn(h, l);
            pax[r] = a;
            p0[r] = b == 0 ? l : plane_k(l, ext, b);
            p1[r] = b == kBins - 1 ? h : plane_k(l, ext, b + 1);
            np++;
        }
        // 1. counts and lists over the node's references
        uint32_t bl[kLearnMaxK], ab[kLearnMaxK], nL[kLearnMaxK], nH[kLearnMaxK], nF[kLearnMaxK];
#pragma unroll
        for (int i = 0; i < kLearnMaxK; i++) bl[i] = ab[i] = nL[i] = nH[i] = nF[i] = 0;
        // four references per lane per pass: their loads are issued together
        for (uint32_t base = 0; base < cnt; base += 128) {
            float4 tlo[4], thi[4];
            bool have[4];
            uint32_t tri[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                have[u] = base + 32u * u + lane < cnt;
                tri[u] = have[u] ? A.refs()[info.x + base + 32u * u + lane] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                tlo[u] = have[u] ? A.tb_lo[tri[u]] : make_float4(0, 0, 0, 0);
                thi[u] = have[u] ? A.tb_hi[tri[u]] : make_float4(0, 0, 0, 0);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                if (base + 32u * u >= cnt) break;   // uniform across the warp
#pragma unroll
                for (int i = 0; i < kLearnMaxK; i++) {
                    if ((uint32_t)i >= np) break;
                    const uint32_t a = pax[i];
                    const float l = c3(blo, a), h = c3(bhi, a);
                    const float lo = mxf(c3(tlo[u], a), l), hi = mnf(c3(thi[u], a), h);
                    bl[i] += (have[u] && lo < p0[i]) ? 1u : 0u;
                    ab[i] += (have[u] && hi > p1[i]) ? 1u : 0u;
                    const bool inL = have[u] && p0[i] <= lo && lo <= p1[i];
                    const bool inH = have[u] && p0[i] <= hi && hi <= p1[i];
                    float *Ls = scratch + (size_t)i * 3 * cap;
                    list_append(Ls, cap, nL[i], inL, lo);
                    list_append(Ls + cap, cap, nH[i], inH, hi);
                    list_append(Ls + 2 * cap, cap, nF[i], inL && lo == hi, lo);
                }
            }
        }
        __syncwarp();
        // 2. exact costs of the listed candidates
        const float Anode = surf(blo, bhi);
        float mc = kInf, m_pk = 0.0f;
        uint32_t m_ax = 3, m_nb = 0, m_na = 0;
#pragma unroll
        for (int i = 0; i < kLearnMaxK; i++) {
            if ((uint32_t)i >= np) break;
            uint32_t b0 = bl[i], a0 = ab[i];
            for (int o = 16; o; o >>= 1) {
                b0 += __shfl_xor_sync(0xffffffffu, b0, o);
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            }
            if (nL[i] > cap || nH[i] > cap || nF[i] > cap) continue;   // overflowed: not costed
            const uint32_t a = pax[i];
            const float l = c3(blo, a), h = c3(bhi, a);
            float *Ls = scratch + (size_t)i * 3 * cap, *Hs = Ls + cap, *Fs = Ls + 2 * cap;
            const uint32_t nl = nL[i], nh = nH[i], nf = nF[i];
            warp_sort_list(Ls, nl);
            warp_sort_list(Hs, nh);
            if (nf) warp_sort_list(Fs, nf);
            for (uint32_t q = lane; q < nl + nh; q += 32) {
                const float x = q < nl ? Ls[q] : Hs[q - nl];
                if (!(x > l && x < h)) continue;
                const float pk = __fadd_rn(x, 0.0f);
                const uint32_t fon = nf ? upper_bound_f(Fs, nf, pk) - lower_bound_f(Fs, nf, pk) : 0u;
                const uint32_t nb = b0 + lower_bound_f(Ls, nl, pk) + fon;
                const uint32_t na = a0 + (nh - upper_bound_f(Hs, nh, pk)) + fon;
                float4 bb = bhi, ba = blo;
                s3(bb, a, pk);
                s3(ba, a, pk);
                const float sb = surf(blo, bb), sa = surf(ba, bhi);
                const float cost = __fadd_rn(
                    A.ct,
                    __fmul_rn(A.ci, __fdiv_rn(__fadd_rn(__fmul_rn(sb, (float)nb), __fmul_rn(sa, (float)na)), Anode)));
                if (cost < mc || (cost == mc && (a < m_ax || (a == m_ax && pk < m_pk)))) {
                    mc = cost;
                    m_ax = a;
                    m_pk = pk;
                    m_nb = nb;
                    m_na = na;
                }
            }
        }
        float bc = mc, bp = m_pk;
        uint32_t bax = m_ax, blane = lane;
        for (int off = 16; off; off >>= 1) {
            const float oc = __shfl_xor_sync(0xffffffffu, bc, off), op = __shfl_xor_sync(0xffffffffu, bp, off);
            const uint32_t oax = __shfl_xor_sync(0xffffffffu, bax, off), ol = __shfl_xor_sync(0xffffffffu, blane, off);
            if (oc < bc || (oc == bc && (oax < bax || (oax == bax && (op < bp || (op == bp && ol < blane)))))) {
                bc = oc;
                bp = op;
                bax = oax;
                blane = ol;
            }
        }
        const uint32_t nb = __shfl_sync(0xffffffffu, m_nb, blane), na = __shfl_sync(0xffffffffu, m_na, blane);
        // 3. the proposal's plane, or the binned optimum
        const bool take = bc < kInf && bc <= __fmul_rn(A.fallback_ratio, lb.cost);
        Decision d;
        if (take) {
            d = Decision{(int)bax, bp, nb, na, bc, 0};
            if (!(bc < __fmul_rn(A.ci, (float)cnt))) d.axis = -1;
        } else {
            d = Decision{lb.axis, lb.plane, lb.nb, lb.na, lb.cost, 0};
        }
        if (lane == 0) {
            write_decision(A, s, d, blo, bhi);
            tally.add(d, cnt);
            if (take) n_learned++;
            else n_fallback++;
        }
        __syncwarp();
    }
    if (threadIdx.x < 2) s_stat[threadIdx.x] = 0;
    __syncthreads();
    if (n_learned) atomicAdd(&s_stat[0], n_learned);
    if (n_fallback) atomicAdd(&s_stat[1], n_fallback);
    __syncthreads();
    if (threadIdx.x == 0 && s_stat[0]) atomicAdd(&A.ctr->learned_nodes, s_stat[0]);
    if (threadIdx.x == 1 && s_stat[1]) atomicAdd(&A.ctr->fallback_nodes, s_stat[1]);
    tally_flush(A, tally, s_tally);
}

// ---------------------------------------------------------------------------
// plan: single-pass scan over the level's nodes of (leaf refs, splits,
// next-level nodes, child refs, below child refs); the guard is decided from
// the decision tallies, block 0 writes the next level's counters, and every
// node emits its compact entry, its children's cells / ropes / next-level
// records and the next level's large-node chunks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t level_tag(const LevelArgs &A) {
    return (*A.epoch * 64u + A.level) & 0x3fffffffu;
}

// the capacity guard: true when splitting this level would overflow
__device__ __forceinline__ bool level_over(const LevelArgs &A) {
    const LevelCounters *l = A.lc;
    const uint64_t child_refs = l->t_childrefs, splits = l->t_splits;
    // deferred-subtree references count as leaf references (a root that
    // cannot be expanded stays a leaf)
    const uint64_t leaf_refs = (uint64_t)l->t_leafrefs + l->t_deferrefs;
    return child_refs > A.cap_refs ||
           (uint64_t)l->leafrefs_total + l->defer_refs_total + leaf_refs + child_refs > A.cap_refs ||
           (uint64_t)l->nodes_total + 2 * splits > A.cap_nodes || l->t_next > A.cap_level;
}

// a child of count c in next-level slot ns: large nodes take a rank and
// their chunks (few per level, so plain atomics)
__device__ void child_setup(const LevelArgs &A, uint32_t ns, uint32_t c) {
    const bool dec = c > A.leaf_size && A.level + 1 < A.max_depth;
    if (dec && is_medium(A, c)) {
        const uint32_t m = atomicAdd(&A.nlc->n_medium, 1u);
        if (m < A.cap_medium) A.medium_slot[m] = ns;
        else atomicOr(A.err, 2u);
        return;
    }
    if (!(dec && is_large(A, c))) return;
    const uint32_t nch = (c + kChunk - 1) / kChunk;
    const uint32_t rank = atomicAdd(&A.nlc->n_large, 1u);
    const uint32_t first = atomicAdd(&A.nlc->n_chunks, nch);
    if (rank >= A.cap_large || first + nch > A.cap_chunks) {
        atomicOr(A.err, 2u);
        return;
    }
    A.large_slot[rank] = ns;
    for (uint32_t k = 0; k < nch; k++) A.chunks[first + k] = make_uint2(rank, k);
}

struct PlanCtx {
    uint32_t stop, nodes_total, leafrefs_total, defer_refs_total, defer_nodes_total;
};

struct PlanItem {
    uint4 info;     // start, count, compact index
    uint2 cnt;      // below, above
    int axis;
};

struct PlanOp {
    using T = U7;
    using Item = PlanItem;
    using Ctx = PlanCtx;
    static constexpr int kItems = kPlanItems;
    LevelArgs A;
    __device__ uint32_t count() const { return A.lc->nodes; }
    __device__ uint32_t tag() const { return level_tag(A); }
    __device__ uint32_t *err() const { return A.err; }
    __device__ Ctx ctx() const {
        LevelCounters *l = A.lc, *nx = A.nlc;
        const bool over = level_over(A);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            l->stop = over ? 1u : 0u;
            if (over) A.ctr->capacity_hit = 1;
            nx->nodes = over ? 0u : l->t_next;
            nx->refs = over ? 0u : l->t_childrefs;
            nx->nodes_total = l->nodes_total + (over ? 0u : 2u * l->t_splits);
            nx->leafrefs_total = l->leafrefs_total + (over ? l->refs : l->t_leafrefs);
            nx->defer_refs_total = l->defer_refs_total + (over ? 0u : l->t_deferrefs);
            nx->defer_nodes_total = l->defer_nodes_total + (over ? 0u : l->t_defernodes);
            A.ctr->leaves += over ? l->nodes : l->t_leafnodes;
            if (!over && l->t_next) A.ctr->depth = A.level + 1;
        }
        return Ctx{over ? 1u : 0u, l->nodes_total, l->leafrefs_total, l->defer_refs_total, l->defer_nodes_total};
    }
    __device__ Item load(uint32_t s, const Ctx &) const {
        if (s == 0xffffffffu) return Item{make_uint4(0, 0, 0, 0), make_uint2(0, 0), -1};
        return Item{A.n_info()[s], A.cnt[s], A.axis[s]};
    }
    __device__ T value(const Item &it) const {
        if (it.axis == kDeferAxis) return U7{0, 0, 0, 0, 0, it.info.y, 1};
        if (it.axis < 0) return U7{it.info.y, 0, 0, 0, 0, 0, 0};
        const uint2 c = it.cnt;
        return U7{0, 1, (c.x > 0 ? 1u : 0u) + (c.y > 0 ? 1u : 0u), c.x + c.y, c.x, 0, 0};
    }
    // where the node's references go (what the reference tiles wait for)
    __device__ void apply_first(uint32_t s, U7 pl, const Item &it, const Ctx &cx) const {
        const uint4 info = it.info;
        if (info.z >= A.cap_nodes) return;   // apply flags it
        if (!cx.stop && it.axis == kDeferAxis) {
            // reference r of this deferred root goes to defer_refs[off - start + r]
            const uint32_t off = cx.defer_refs_total + pl.d;
            A.scat[s] = make_uint4(off - info.x, 0, 0, 2u);
        } else if (cx.stop || it.axis < 0) {
            // reference r of this leaf goes to out_refs[off - start + r]
            const uint32_t off = cx.leafrefs_total + (cx.stop ? info.x : pl.x);
            A.scat[s] = make_uint4(off - info.x, 0, 0, 0);
        } else {
            // the node's below references go to nx_refs[pl.w ..), its above ones
            // right after them, each in its order within the node (its rank among
            // the node's flagged references), as next-level slots pl.z and pl.z +
            // (cnt.x > 0); w = above count << 2 | has-below << 1 | split
            const uint2 c2 = it.cnt;
            A.scat[s] = make_uint4(pl.w, pl.w + c2.x, pl.z, (c2.y << 2) | 1u | (c2.x ? 2u : 0u));
        }
    }
    // the node's compact entry, its children's cells / ropes / records
    __device__ void apply(uint32_t s, U7 pl, const Item &it, const Ctx &cx) const {
        const uint4 info = it.info;
        const int ax = cx.stop ? -1 : it.axis;
        if (info.z >= A.cap_nodes) {
            atomicOr(A.err, 16u);
            return;
        }
        if (ax == kDeferAxis) {
            // the subtree pass writes the node's entry; its cell and ropes are
            // already written (by its parent's plan)
            const uint32_t did = cx.defer_nodes_total + pl.e;
            if (did < A.cap_defer) {
                A.d_root[did] = make_uint4(info.z, cx.defer_refs_total + pl.d, info.y, A.level);
                A.d_lo[did] = A.n_lo()[s];
                A.d_hi[did] = A.n_hi()[s];
            } else {
                atomicOr(A.err, 2u);
            }
            return;
        }
        if (ax < 0) {
            const uint32_t off = cx.leafrefs_total + (cx.stop ? info.x : pl.x);
            A.out_nodes[info.z] = make_uint2((off << 2) | kLeafTag, info.y);
            return;
        }
        const uint32_t pair = cx.nodes_total + 2 * pl.y;
        const uint2 ct = it.cnt;
        // the tallies that passed the guard and this scan sum the same
        // decisions; these checks only keep an inconsistent level in bounds
        if ((uint64_t)pair + 1 >= A.cap_nodes ||
            (uint64_t)pl.z + (ct.x ? 1u : 0u) + (ct.y ? 1u : 0u) > A.cap_level) {
            atomicOr(A.err, 16u);
            return;
        }
        const float p = A.plane[s];
        const float4 lo = A.n_lo()[s], hi = A.n_hi()[s];
        uint32_t r[6];
        {
            // the parent's ropes: 6 words at a 24-byte stride (8-byte aligned)
            const uint2 *pr2 = reinterpret_cast<const uint2 *>(A.out_ropes + 6 * (size_t)info.z);
            const uint2 a0 = pr2[0], a1 = pr2[1], a2 = pr2[2];
            r[0] = a0.x; r[1] = a0.y; r[2] = a1.x; r[3] = a1.y; r[4] = a2.x; r[5] = a2.y;
        }
        A.out_nodes[info.z] = make_uint2((pair << 2) | (uint32_t)ax, __float_as_uint(p));
        uint32_t ns = pl.z;
        const uint32_t co = pl.w;
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
            uint32_t rb[6], ra[6];
#pragma unroll
            for (int f = 0; f < 6; f++) {
                rb[f] = f == 2 * ax + 1 ? pair + 1 : r[f];
                ra[f] = f == 2 * ax ? pair : r[f];
            }
            // the pair's 12 rope words start at 24 * pair bytes, pair even
            // (nodes_total starts at 2 and grows by pairs): 16-byte aligned
            uint4 *dst = reinterpret_cast<uint4 *>(A.out_ropes + 6 * (size_t)pair);
            dst[0] = make_uint4(rb[0], rb[1], rb[2], rb[3]);
            dst[1] = make_uint4(rb[4], rb[5], ra[0], ra[1]);
            dst[2] = make_uint4(ra[2], ra[3], ra[4], ra[5]);
        }
        if (ct.x) {
            float4 h2 = hi;
            s3(h2, ax, p);
            A.nx_lo()[ns] = lo;
            A.nx_hi()[ns] = h2;
            A.nx_info()[ns] = make_uint4(co, ct.x, pair, 0);
            child_setup(A, ns, ct.x);
            ns++;
        } else {
            A.out_nodes[pair] = make_uint2(kLeafTag, 0);
        }
        if (ct.y) {
            float4 l2 = lo;
            s3(l2, ax, p);
            A.nx_lo()[ns] = l2;
            A.nx_hi()[ns] = hi;
            A.nx_info()[ns] = make_uint4(co + ct.x, ct.y, pair + 1, 0);
            child_setup(A, ns, ct.y);
        } else {
            A.out_nodes[pair + 1] = make_uint2(kLeafTag, 0);
        }
    }
};

// refs: single-pass scan of the below / above flags, segmented by node, fused
// with the stable partition: a reference's rank among its node's below (above)
// references, added to where the plan scan put the node's children, is its
// place in the next level.
struct RefItem {
    uint2 f;        // below / above flags
    uint32_t s;     // node slot
    uint32_t tri;
};

struct RefOp {
    using T = uint2;
    using Item = RefItem;
    using Ctx = uint32_t;   // the level stopped splitting
    static constexpr int kItems = 4;
    LevelArgs A;
    __device__ uint32_t count() const { return A.lc->refs; }
    __device__ uint32_t tag() const { return level_tag(A); }
    __device__ uint32_t *err() const { return A.err; }
    __device__ Ctx ctx() const { return A.lc->stop; }
    __device__ Item load(uint32_t r, const Ctx &stop) const {
        if (r == 0xffffffffu) return Item{make_uint2(0, 0), 0, 0};
        const uint32_t s = A.ref_node()[r];
        const uint32_t tri = A.refs()[r];
        const float4 sp = A.split[s];
        const int ax = stop ? -1 : __float_as_int(sp.x);
        if (ax < 0) return Item{make_uint2(0, 0), s, tri};
        const float p = sp.y, l = sp.z, h = sp.w;
        const float lo = mxf(c3(A.tb_lo[tri], ax), l), hi = mnf(c3(A.tb_hi[tri], ax), h);
        const bool flat_on = (lo == hi) && lo == p;
        return Item{make_uint2((lo < p || flat_on) ? 1u : 0u, (hi > p || flat_on) ? 1u : 0u), s, tri};
    }
    __device__ T value(const Item &it) const { return it.f; }
    // R: the reference's rank among its node's below / above references
    __device__ void apply(uint32_t r, uint2 R, const Item &it, const Ctx &) const {
        const uint4 sc = __ldcg(A.scat + it.s);   // written by a plan tile of this launch
        if (!(sc.w & 1u)) {
            const uint32_t off = sc.x + r;   // leaf, or a deferred root (w = 2)
            if (off < A.cap_refs) (sc.w & 2u ? A.defer_refs : A.out_refs)[off] = it.tri;
            else atomicOr(A.err, 2u);
            return;
        }
        if (it.f.x) {
            const uint32_t pos = sc.x + R.x;
            if (pos < A.cap_refs && R.x < sc.y - sc.x) {
                A.nx_refs()[pos] = it.tri;
                A.nx_ref_node()[pos] = sc.z;
            } else {
                atomicOr(A.err, 8u);
            }
        }
        if (it.f.y) {
            const uint32_t pos = sc.y + R.y;
            if (pos < A.cap_refs && R.y < (sc.w >> 2)) {
                A.nx_refs()[pos] = it.tri;
                A.nx_ref_node()[pos] = sc.z + ((sc.w & 2u) ? 1u : 0u);
            } else {
                atomicOr(A.err, 8u);
            }
        }
    }
};

// segmented scan values: the flag counts since the last node start, and
// whether a node starts in the span
struct SegV {
    uint2 v;
    uint32_t h;
};
__device__ __forceinline__ SegV seg_join(SegV a, SegV b) {   // a before b
    return SegV{b.h ? b.v : vadd(a.v, b.v), a.h | b.h};
}
__device__ __forceinline__ SegV seg_shfl_up(SegV x, int d) {
    return SegV{make_uint2(__shfl_up_sync(0xffffffffu, x.v.x, d), __shfl_up_sync(0xffffffffu, x.v.y, d)),
                __shfl_up_sync(0xffffffffu, x.h, d)};
}

struct RefTileSmem {
    SegV w_tot[kScanThreads / 32];
    uint32_t w_last[kScanThreads / 32];   // node of each warp's last reference
    uint2 carry;                          // the tile's first segment: flags in earlier tiles
};

// One reference tile (kTile references, kScanItems per thread). The scan is
// segmented by node: a tile in which a node starts publishes its last
// segment's counts as complete (status 2) at once; only its first segment,
// when it continues a node of earlier tiles, needs the look-back, which ends at
// the tile where that node starts. wait_plan() runs (all threads) before the
// scatter.
template <class Wait>
__device__ void ref_tile(const RefOp &R, uint32_t rt, uint32_t nr, uint32_t tag, uint32_t stop, uint32_t *flags,
                         uint2 *aggs, uint2 *incls, RefTileSmem &sh, const Wait &wait_plan) {
    const LevelArgs &A = R.A;
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const uint32_t r0 = rt * kTile;
    const uint32_t base = r0 + threadIdx.x * kScanItems;
    RefItem it[kScanItems];
    bool hd[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; k++) it[k] = R.load(base + k < nr ? base + k : 0xffffffffu, stop);
    // node of the reference before this thread's first one
    uint32_t prev = __shfl_up_sync(0xffffffffu, it[kScanItems - 1].s, 1);
    if (lane == 31) sh.w_last[wid] = it[kScanItems - 1].s;
    const uint32_t first_prev = (threadIdx.x == 0 && r0 > 0) ? A.ref_node()[r0 - 1] : 0xffffffffu;
    __syncthreads();
    if (lane == 0) prev = wid ? sh.w_last[wid - 1] : first_prev;
    SegV t{make_uint2(0, 0), 0u};
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        const bool valid = base + k < nr;
        hd[k] = !valid || it[k].s != (k ? it[k - 1].s : prev);
        t = seg_join(t, SegV{it[k].f, hd[k] ? 1u : 0u});
    }
    // warp and block segmented scans
    SegV inc = t;
    for (int d = 1; d < 32; d <<= 1) {
        const SegV o = seg_shfl_up(inc, d);
        if ((int)lane >= d) inc = seg_join(o, inc);
    }
    SegV ex = seg_shfl_up(inc, 1);
    if (lane == 0) ex = SegV{make_uint2(0, 0), 0u};
    if (lane == 31) sh.w_tot[wid] = inc;
    __syncthreads();
    SegV wp{make_uint2(0, 0), 0u}, tot{make_uint2(0, 0), 0u};
    for (uint32_t w = 0; w < kScanThreads / 32; w++) {
        if (w < wid) wp = seg_join(wp, sh.w_tot[w]);
        tot = seg_join(tot, sh.w_tot[w]);
    }
    ex = seg_join(wp, ex);
    // the tile's first reference starts a node: no earlier tile matters
    const bool starts = r0 == 0 || first_prev != it[0].s;
    if (threadIdx.x == 0) {
        if (tot.h) incls[rt] = tot.v;
        else aggs[rt] = tot.v;
        __threadfence();
        *reinterpret_cast<volatile uint32_t *>(flags + rt) = (tag << 2) | (tot.h ? 2u : 1u);
    }
    if (threadIdx.x < 32) {
        // the tile-0 rule is kept for the look-back: before tile 0 is zero
        const uint2 c = (rt && !__shfl_sync(0xffffffffu, starts ? 1u : 0u, 0))
                            ? lookback(flags, aggs, incls, rt, tag, A.err, A.spin_limit)
                            : make_uint2(0, 0);
        if (threadIdx.x == 0) {
            if (!tot.h) {
                incls[rt] = vadd(c, tot.v);
                __threadfence();
                *reinterpret_cast<volatile uint32_t *>(flags + rt) = (tag << 2) | 2u;
            }
            sh.carry = c;
        }
    }
    __syncthreads();
    if (!wait_plan()) return;   // uniform: the scatter needs the plan's destinations
    uint2 run = ex.h ? ex.v : vadd(ex.v, sh.carry);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (hd[k]) run = make_uint2(0, 0);
        if (base + k < nr) R.apply(base + k, run, it[k], stop);
        run = vadd(run, it[k].f);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// plan + refs of one level in one launch. Tickets 0 .. node tiles - 1 are plan
// tiles (kPlanTile nodes), the rest reference tiles (kTile refs). A plan tile
// publishes a done flag once its nodes' reference destinations are written,
// then emits the rest; a reference tile computes its flags, scans and looks
// back, then waits (bounded) for the plan tiles of its nodes (its references
// belong to a contiguous run of nodes) before it scatters. Plan tiles take
// their tickets before any reference tile and wait for nothing but earlier
// plan tiles, so every wait ends.
// ---------------------------------------------------------------------------
struct PlanSmem {
    U7 shp[kScanThreads / 32 + 1];
    U7 sxp;
    RefTileSmem shr_seg;
    uint32_t tile, wait_ok;
};

__device__ __forceinline__ void plan_refs_body(const LevelArgs &A, PlanSmem &SM, uint32_t *pflags, U7 *paggs,
                                               U7 *pincls, uint32_t *rflags, uint2 *raggs, uint2 *rincls,
                                               uint32_t *pdone, uint32_t *ticket) {
    U7 *shp = SM.shp;
    U7 &sxp = SM.sxp;
    RefTileSmem &shr_seg = SM.shr_seg;
    uint32_t &s_tile = SM.tile;
    uint32_t &s_wait_ok = SM.wait_ok;
    const PlanOp P{A};
    const RefOp R{A};
    const uint32_t tag = level_tag(A);
    const PlanCtx pc = P.ctx();                 // block 0 also writes the next level's counters
    const uint32_t stop = pc.stop;              // the guard, decided from the tallies by every CTA
    const uint32_t nn = A.lc->nodes, nr = A.lc->refs;
    const uint32_t ntn = (nn + kPlanTile - 1) / kPlanTile;
    const uint32_t ntr = (nr + kTile - 1) / kTile;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t < ntn) {
            // the done flag follows the tile's reference destinations; the
            // rest of its emission overlaps the reference tiles' scatter
            scan_tile(P, t, nn, tag, pc, pflags, paggs, pincls, shp, sxp, [&] {
                __threadfence();
                __syncthreads();
                if (threadIdx.x == 0 && !(t == 0 && A.level == A.withhold_level))
                    *reinterpret_cast<volatile uint32_t *>(pdone + t) = tag;
            });
        } else if (t < ntn + ntr) {
            const uint32_t rt = t - ntn;
            // true when every plan tile of this tile's nodes has published
            // its reference destinations; a wait that runs out leaves the
            // tile's scatter undone (error bit 4, the build reports failure)
            auto wait_plan = [&]() -> bool {
                if (threadIdx.x == 0) {
                    uint32_t ok = 1;
                    const uint32_t r0 = rt * kTile, r1 = min(nr, r0 + kTile) - 1;
                    const uint32_t k0 = A.ref_node()[r0] / kPlanTile, k1 = A.ref_node()[r1] / kPlanTile;
                    for (uint32_t k = k0; k <= k1 && k < ntn && ok; k++) {
                        for (uint32_t spins = 0; __ldcv(pdone + k) != tag; spins++) {
                            if (spins >= A.spin_limit) {
                                atomicOr(A.err, 4u);
                                ok = 0;
                                break;
                            }
                            __nanosleep(32);
                        }
                    }
                    __threadfence();
                    s_wait_ok = ok;
                }
                __syncthreads();
                return s_wait_ok != 0;
            };
            ref_tile(R, rt, nr, tag, stop, rflags, raggs, rincls, shr_seg, wait_plan);
        } else {
            break;
        }
    }
}

__global__ void __launch_bounds__(kScanThreads, 6) k_plan_refs(LevelArgs A, uint32_t *pflags, U7 *paggs, U7 *pincls,
                                                            uint32_t *rflags, uint2 *raggs, uint2 *rincls,
                                                            uint32_t *pdone, uint32_t *ticket) {
    __shared__ PlanSmem SM;
    wait_prior_grid();
    if (level_aborted(A)) return;
    plan_refs_body(A, SM, pflags, paggs, pincls, rflags, raggs, rincls, pdone, ticket);
}

// ---------------------------------------------------------------------------
// deferred subtrees. After the levels, one warp builds each subtree rooted at
// a recorded node of at most kDeferMax references, depth first, with one
// reference per lane (a node's references are a mask of the warp's lanes, in
// the root's order), deciding every node with the levels' SAH (the binned
// histograms, or the exact search in registers). Nodes are numbered locally:
// a split takes the next pair of local indices (below, above); the below
// child is built next and the above child waits on a stack in shared memory.
// Entries, cells and ropes go to scratch slots keyed (subtree, local index),
// references to slots keyed (subtree, local index); slots are handed out per
// warp in chunks. A single-pass scan over the subtrees' sizes places subtree
// i after the levels' nodes and leaf references and after subtrees 0 .. i-1,
// and the last pass moves every slot to its place. When the subtrees do not
// fit the node or reference capacity (or a scratch arena ran out), every root
// stays a leaf holding its references instead. The oracle's
// hko_build_binned restates this order.
// ---------------------------------------------------------------------------
constexpr uint32_t kLocalRope = 0x80000000u;   // a rope to a local index of the same subtree
constexpr uint32_t kNoSlot = 0xffffffffu;
constexpr uint32_t kScNodeChunk = 64;          // node slots per chunk (pairs never straddle)
constexpr uint32_t kScRefChunk = 256;          // reference slots per chunk
constexpr int kSubWarps = 8;

// entries of a warp's stack of waiting (above) children: one per depth below
// the root, an even count (the per-warp shared-memory regions stay 16-byte
// aligned)
__host__ __device__ constexpr uint32_t sub_stack_entries(uint32_t max_depth) { return (max_depth + 3u) & ~1u; }
// per warp: the binned histograms, the plane table, then the stack (cells lo,
// hi; meta: lane mask, depth, scratch slot; 6 rope words per entry)
__host__ __device__ constexpr size_t sub_warp_smem(uint32_t entries) {
    return kHist * 4 + kPlanes * 4 + (size_t)72 * entries;
}

// a scratch entry moved to its place: child pairs and leaf starts shifted by
// the subtree's first node / reference; an empty cell keeps start 0
__device__ __forceinline__ uint2 sub_relocate(uint2 e, uint32_t nb, uint32_t rb) {
    if ((e.x & 3u) == kLeafTag) return e.y ? make_uint2((((e.x >> 2) + rb) << 2) | kLeafTag, e.y) : e;
    return make_uint2((((e.x >> 2) + nb) << 2) | (e.x & 3u), e.y);
}

// the rest of a warp's scratch chunk marked unused
__device__ __forceinline__ void sub_close_chunks(const LevelArgs &A, uint32_t nbase, uint32_t nused, uint32_t rbase,
                                                 uint32_t rused) {
    const uint32_t lane = threadIdx.x & 31u;
    if (nbase != kNoSlot)
        for (uint32_t k = nused + lane; k < kScNodeChunk; k += 32) A.sc_key[nbase + k] = make_uint2(kNoSlot, 0);
    if (rbase != kNoSlot)
        for (uint32_t k = rused + lane; k < kScRefChunk; k += 32) A.sc_ref[rbase + k] = make_uint4(kNoSlot, 0, 0, 0);
}

// a new chunk of `chunk` slots from the counter (all lanes; kNoSlot when the
// arena is spent)
__device__ __forceinline__ uint32_t sub_chunk(uint32_t *ctr, uint32_t chunk, uint32_t cap) {
    uint32_t b = 0;
    if ((threadIdx.x & 31u) == 0) b = atomicAdd(ctr, chunk);
    b = __shfl_sync(0xffffffffu, b, 0);
    return (uint64_t)b + chunk <= cap ? b : kNoSlot;
}

// true (CTA-uniform) when the build has any error bit: the subtree pass reads
// records and references that a capacity error may have left unwritten
__device__ __forceinline__ bool sub_aborted(const LevelArgs &A) {
    __shared__ uint32_t s_err;
    __syncthreads();
    if (threadIdx.x == 0) s_err = __ldcg(A.err);
    __syncthreads();
    return s_err != 0;
}

// The subtrees of roots A.lc->defer_nodes_total .. A.nlc->defer_nodes_total,
// one warp per subtree taken by ticket from A.lc (E stack entries per warp).
// Lane r holds reference r of the root; lanes 0..11 hold the current node's
// ropes, word lane % 6, so a child's cell, ropes and stack entry are written
// by parallel lanes.
template <bool WARP_EXACT>
__global__ void __launch_bounds__(kSubWarps * 32, 4) k_subtree(LevelArgs A, uint32_t E) {
    extern __shared__ __align__(16) unsigned char sub_smem[];
    wait_prior_grid();
    if (sub_aborted(A)) return;
    const uint32_t wib = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    unsigned char *wbase = sub_smem + (size_t)wib * sub_warp_smem(E);
    uint32_t *Hw = reinterpret_cast<uint32_t *>(wbase);
    float *Pw = reinterpret_cast<float *>(wbase + kHist * 4);
    float4 *s_lo = reinterpret_cast<float4 *>(wbase + kHist * 4 + kPlanes * 4);
    float4 *s_hi = s_lo + E;
    uint4 *s_meta = reinterpret_cast<uint4 *>(s_hi + E);
    uint32_t *s_rope = reinterpret_cast<uint32_t *>(s_meta + E);
    const uint32_t r0 = min(A.lc->defer_nodes_total, A.cap_defer);
    const uint32_t r1 = min(A.nlc->defer_nodes_total, A.cap_defer);
    const uint32_t f6 = lane % 6u, child6 = lane / 6u;   // rope word; child of a pair (lanes 0..11)
    uint32_t nbase = kNoSlot, nused = kScNodeChunk, rbase = kNoSlot, rused = kScRefChunk;
    uint32_t leaves = 0, maxdepth = 0;
    bool dead = false;
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = r0 + atomicAdd(&A.lc->sub_ticket, 1u);
        i = __shfl_sync(0xffffffffu, i, 0);
        if (i >= r1 || dead) break;
        const uint4 rt = A.d_root[i];   // compact index, reference offset, count, depth
        float4 lo = A.d_lo[i], hi = A.d_hi[i];
        const uint32_t cnt0 = min(rt.z, 32u);
        if ((uint64_t)rt.y + cnt0 > A.cap_refs || rt.x >= A.cap_nodes) {
            dead = true;   // an inconsistent record: the roots stay leaves
            break;
        }
        uint32_t tri = 0;
        float4 tlo = make_float4(0, 0, 0, 0), thi = tlo;
        if (lane < cnt0) {
            tri = A.defer_refs[rt.y + lane];
            tlo = A.tb_lo[tri];
            thi = A.tb_hi[tri];
        }
        uint32_t rr = lane < 12 ? A.out_ropes[6 * (size_t)rt.x + f6] : 0u;
        uint32_t mask = cnt0 >= 32 ? 0xffffffffu : ((1u << cnt0) - 1u);
        uint32_t depth = rt.w, slot = kNoSlot, sp = 0, npair = 0, nref = 0;
        uint2 root_entry = make_uint2(kLeafTag, 0);
        for (;;) {
            const bool in = (mask >> lane) & 1u;
            const uint32_t c = __popc(mask);
            Decision d{-1, 0.0f, 0, 0, kInf, 0};
            if (c > A.leaf_size && depth < A.max_depth) {
                if (WARP_EXACT) {
                    d = sah_exact_lanes(in, tlo, thi, c, lo, hi, A.ct, A.ci);
                } else {
                    __syncwarp();
                    uint4 *H4 = reinterpret_cast<uint4 *>(Hw);
                    H4[lane] = make_uint4(0, 0, 0, 0);
                    H4[lane + 32] = make_uint4(0, 0, 0, 0);
                    if (lane < kHist / 4 - 64) H4[lane + 64] = make_uint4(0, 0, 0, 0);
                    node_planes_warp(Pw, lo, hi);
                    __syncwarp();
                    if (in) hist_ref_tab(Hw, tlo, thi, lo, hi, bin_scale(lo, hi), Pw);
                    __syncwarp();
                    d = sah_warp(Hw, lo, hi, c, A.ct, A.ci);
                }
            }
            if (d.axis < 0) {
                // a leaf: its references in the subtree's next local slots
                const uint2 entry = make_uint2((nref << 2) | kLeafTag, c);
                if (slot == kNoSlot) root_entry = entry;
                else if (lane == 0) A.sc_node[slot] = entry;
                if (rused + c > kScRefChunk) {
                    sub_close_chunks(A, kNoSlot, 0, rbase, rused);
                    rbase = sub_chunk(&A.ctr->sc_ref_ctr, kScRefChunk, A.cap_sc_refs);
                    rused = 0;
                    if (rbase == kNoSlot) {
                        dead = true;
                        break;
                    }
                }
                if (in) {
                    const uint32_t rank = __popc(mask & ((1u << lane) - 1u));
                    A.sc_ref[rbase + rused + rank] = make_uint4(i, nref + rank, tri, 0);
                }
                rused += c;
                nref += c;
                leaves++;
            } else {
                const uint32_t ax = (uint32_t)d.axis;
                const float p = d.plane;
                const uint32_t pair = npair;
                npair += 2;
                const uint2 entry = make_uint2((pair << 2) | ax, __float_as_uint(p));
                if (slot == kNoSlot) root_entry = entry;
                else if (lane == 0) A.sc_node[slot] = entry;
                // the partition of the levels (checkPolygonToAAPlane on the
                // clipped bounds), as lane masks
                const float l = c3(lo, ax), h = c3(hi, ax);
                const float clo = mxf(c3(tlo, ax), l), chi = mnf(c3(thi, ax), h);
                const bool flat_on = (clo == chi) && clo == p;
                const uint32_t bm = __ballot_sync(0xffffffffu, in && (clo < p || flat_on));
                const uint32_t am = __ballot_sync(0xffffffffu, in && (chi > p || flat_on));
                if (nused + 2 > kScNodeChunk) {
                    sub_close_chunks(A, nbase, nused, kNoSlot, 0);
                    nbase = sub_chunk(&A.ctr->sc_node_ctr, kScNodeChunk, A.cap_sc_nodes);
                    nused = 0;
                    if (nbase == kNoSlot) {
                        dead = true;
                        break;
                    }
                }
                const uint32_t sb = nbase + nused;
                nused += 2;
                float4 bhi = hi, alo = lo;
                s3(bhi, ax, p);
                s3(alo, ax, p);
                // the pair's scratch slots: keys (lanes 0, 1; an empty child is
                // an empty leaf, a non-empty one's entry is written when it is
                // decided), cells (lane = 2 child + corner), ropes (lane = 6
                // child + face: the parent's, with the face on the plane
                // pointing at the sibling)
                if (lane < 2) {
                    A.sc_key[sb + lane] = make_uint2(i, pair + lane);
                    if ((lane ? am : bm) == 0) A.sc_node[sb + lane] = make_uint2(kLeafTag, 0);
                }
                if (lane < 4) {
                    const float4 v = lane == 0 ? lo : (lane == 1 ? bhi : (lane == 2 ? alo : hi));
                    A.sc_cbox[2 * (size_t)sb + lane] = v;
                }
                uint32_t rb = rr, ra = rr;
                if (f6 == 2 * ax + 1) rb = kLocalRope | (pair + 1);
                if (f6 == 2 * ax) ra = kLocalRope | pair;
                if (lane < 12) A.sc_rope[6 * (size_t)sb + lane] = child6 ? ra : rb;
                if (bm | am) maxdepth = max(maxdepth, depth + 1);
                if (am) {
                    if (sp >= E) {
                        dead = true;
                        break;
                    }
                    if (lane == 0) {
                        s_lo[sp] = alo;
                        s_hi[sp] = hi;
                        s_meta[sp] = make_uint4(am, depth + 1, sb + 1, 0);
                    }
                    if (lane < 6) s_rope[6 * sp + lane] = ra;
                    sp++;
                }
                if (bm) {
                    mask = bm;
                    hi = bhi;
                    depth++;
                    slot = sb;
                    rr = rb;
                    continue;
                }
            }
            if (sp == 0) break;
            __syncwarp();
            sp--;
            lo = s_lo[sp];
            hi = s_hi[sp];
            const uint4 m = s_meta[sp];
            rr = lane < 12 ? s_rope[6 * sp + f6] : 0u;
            __syncwarp();
            mask = m.x;
            depth = m.y;
            slot = m.z;
        }
        if (!dead && lane == 0) {
            A.st_cnt[i] = make_uint2(npair, nref);
            A.st_root[i] = root_entry;
        }
    }
    if (dead) {
        if (lane == 0) atomicExch(&A.ctr->sub_overflow, 1u);
    } else {
        sub_close_chunks(A, nbase, nused, rbase, rused);
    }
    if (lane == 0 && leaves) {
        atomicAdd(&A.ctr->sub_leaves, leaves);
        atomicMax(&A.ctr->sub_depth, maxdepth);
    }
}

// subtree sizes -> places (exclusive prefix over the subtrees); the thread of
// the last subtree decides whether they fit and writes the build's totals
struct SubScanOp {
    using T = uint2;
    using Item = uint2;
    using Ctx = uint32_t;
    static constexpr int kItems = kScanItems;
    LevelArgs A;
    uint32_t n;
    __device__ uint32_t *err() const { return A.err; }
    __device__ Item load(uint32_t i, const Ctx &) const { return i == 0xffffffffu ? make_uint2(0, 0) : A.st_cnt[i]; }
    __device__ T value(const Item &it) const { return it; }
    __device__ void apply_first(uint32_t i, uint2 pre, const Item &, const Ctx &) const { A.st_base[i] = pre; }
    __device__ void apply(uint32_t i, uint2 pre, const Item &it, const Ctx &) const {
        if (i + 1 != n) return;
        LevelCounters *fin = A.lc;
        BuildCounters *c = A.ctr;
        const uint2 tot = vadd(pre, it);
        const uint32_t N0 = fin->nodes_total, R0 = fin->leafrefs_total;
        const bool fits = !c->sub_overflow && (uint64_t)N0 + tot.x <= A.cap_nodes &&
                          (uint64_t)R0 + tot.y <= A.cap_refs;
        c->sub_n0 = N0;
        c->sub_r0 = R0;
        c->sub_fits = fits ? 1u : 0u;
        if (fits) {
            fin->nodes_total = N0 + tot.x;
            fin->leafrefs_total = R0 + tot.y;
            c->sub_nodes = tot.x;
            c->sub_refs = tot.y;
            c->leaves += c->sub_leaves;
            c->depth = max(c->depth, c->sub_depth);
        } else {
            // every root a leaf over its references (they were counted as
            // leaf references by the levels' guard, so they fit)
            fin->leafrefs_total = R0 + fin->defer_refs_total;
            c->leaves += n;
            c->capacity_hit = 1;
        }
    }
};

__global__ void __launch_bounds__(kScanThreads) k_sub_scan(LevelArgs A, uint32_t *flags, uint2 *aggs,
                                                           uint2 *incls) {
    __shared__ uint2 sh[kScanThreads / 32 + 1];
    __shared__ uint2 sx;
    __shared__ uint32_t s_tile;
    wait_prior_grid();
    if (sub_aborted(A)) return;
    const uint32_t n = min(A.lc->defer_nodes_total, A.cap_defer);
    const uint32_t ntiles = (n + kTile - 1) / kTile;
    const SubScanOp op{A, n};
    const uint32_t tag = level_tag(A);
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&A.ctr->sub_ticket, 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles) break;
        scan_tile(op, t, n, tag, 0u, flags, aggs, incls, sh, sx, [] {});
    }
}

// every scratch slot to its place (or, when the subtrees do not fit, every
// root a leaf)
__global__ void __launch_bounds__(256) k_sub_place(LevelArgs A) {
    wait_prior_grid();
    if (sub_aborted(A)) return;
    const uint32_t n = min(A.lc->defer_nodes_total, A.cap_defer);
    if (n == 0) return;
    const BuildCounters *c = A.ctr;
    const uint32_t N0 = c->sub_n0, R0 = c->sub_r0;
    const uint32_t stride = gridDim.x * blockDim.x, t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (!c->sub_fits) {
        for (uint32_t i = t0; i < n; i += stride) {
            const uint4 rt = A.d_root[i];
            A.out_nodes[rt.x] = make_uint2(((R0 + rt.y) << 2) | kLeafTag, rt.z);
        }
        const uint32_t nr = min(A.lc->defer_refs_total, A.cap_refs);
        for (uint32_t k = t0; k < nr; k += stride) {
            if ((uint64_t)R0 + k < A.cap_refs) A.out_refs[R0 + k] = A.defer_refs[k];
            else atomicOr(A.err, 2u);
        }
        return;
    }
    const uint32_t nsn = min(c->sc_node_ctr, A.cap_sc_nodes), nsr = min(c->sc_ref_ctr, A.cap_sc_refs);
    for (uint32_t j = t0; j < nsn; j += stride) {
        const uint2 key = A.sc_key[j];
        if (key.x >= n) continue;   // an unused slot
        const uint2 base = A.st_base[key.x];
        const uint32_t nb = N0 + base.x, g = nb + key.y;
        if (g >= A.cap_nodes) {
            atomicOr(A.err, 16u);
            continue;
        }
        A.out_nodes[g] = sub_relocate(A.sc_node[j], nb, R0 + base.y);
        A.out_cbox[2 * (size_t)g] = A.sc_cbox[2 * (size_t)j];
        A.out_cbox[2 * (size_t)g + 1] = A.sc_cbox[2 * (size_t)j + 1];
#pragma unroll
        for (int f = 0; f < 6; f++) {
            uint32_t r = A.sc_rope[6 * (size_t)j + f];
            if (r != kNoSlot && (r & kLocalRope)) r = nb + (r & ~kLocalRope);
            A.out_ropes[6 * (size_t)g + f] = r;
        }
    }
    for (uint32_t j = t0; j < nsr; j += stride) {
        const uint4 q = A.sc_ref[j];
        if (q.x >= n) continue;
        const uint32_t pos = R0 + A.st_base[q.x].y + q.y;
        if (pos < A.cap_refs) A.out_refs[pos] = q.z;
        else atomicOr(A.err, 16u);
    }
    for (uint32_t i = t0; i < n; i += stride) {
        const uint2 base = A.st_base[i];
        A.out_nodes[A.d_root[i].x] = sub_relocate(A.st_root[i], N0 + base.x, R0 + base.y);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// k_subtree's grid: four CTAs of kSubWarps warps per SM, one wave
static unsigned sub_grid(int sm_count) { return (unsigned)sm_count * 4u; }

// a launch that may start while the stream's previous kernel finishes
// (programmatic stream serialization); the kernel calls wait_prior_grid()
// before it reads anything that kernel wrote
template <class... KArgs, class... Args>
static cudaError_t launch_pdl(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                              Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

template <class T>
static cudaError_t dalloc(T *&p, size_t n) {
    if (p) cudaFree(p);
    p = nullptr;
    return cudaMalloc((void **)&p, std::max<size_t>(n, 1) * sizeof(T));
}

void build_release(BuildState &S) {
    auto f = [](auto *&p) {
        if (p) cudaFree((void *)p);
        p = nullptr;
    };
    f(S.tb_lo); f(S.tb_hi);
    for (int k = 0; k < 2; k++) {
        f(S.n_lo[k]); f(S.n_hi[k]); f(S.n_info[k]); f(S.refs[k]); f(S.ref_node[k]);
    }
    f(S.d_axis); f(S.d_plane); f(S.d_cnt); f(S.d_split); f(S.d_scat);
    f(S.chunks); f(S.hist); f(S.done); f(S.medium_slot); f(S.learn_slot); f(S.learn_bin); f(S.learn_prop); f(S.feat); f(S.prop_log);
    f(S.plan_flags); f(S.ref_flags); f(S.plan_done); f(S.plan_agg); f(S.plan_incl); f(S.ref_agg); f(S.ref_incl); f(S.epoch);
    f(S.ctr); f(S.err);
    f(S.out_nodes); f(S.out_refs); f(S.out_ropes); f(S.out_cbox);
    f(S.d_root); f(S.d_lo); f(S.d_hi); f(S.defer_refs);
    f(S.sc_key); f(S.sc_node); f(S.sc_cbox); f(S.sc_rope); f(S.sc_ref);
    f(S.st_cnt); f(S.st_root); f(S.st_base); f(S.sub_flags); f(S.sub_agg); f(S.sub_incl);
    S.cap_defer = S.cap_sc_nodes = S.cap_sc_refs = S.sub_tiles = 0;
    if (S.ev_fork) cudaEventDestroy(S.ev_fork);
    if (S.ev_join) cudaEventDestroy(S.ev_join);
    if (S.ev_learn) cudaEventDestroy(S.ev_learn);
    if (S.ev_join2) cudaEventDestroy(S.ev_join2);
    if (S.aux) cudaStreamDestroy(S.aux);
    if (S.aux2) cudaStreamDestroy(S.aux2);
    S.ev_fork = S.ev_join = S.ev_learn = S.ev_join2 = nullptr;
    S.aux = S.aux2 = nullptr;
    S.nt = S.cap_refs = S.cap_nodes = S.cap_level = 0;
    S.plan_tiles = S.ref_tiles = 0;
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
    if (S.ctr && S.nt == nt && S.cap_refs == cap_refs && S.cap_nodes == cap_nodes && p.max_depth <= S.alloc_depth) {
        if (p.prop_log && !S.prop_log && dalloc(S.prop_log, (size_t)S.cap_nodes * 8) != cudaSuccess) return HK_E_ALLOC;
        return HK_OK;
    }
    build_release(S);
    S.nt = nt;
    S.cap_refs = cap_refs;
    S.cap_nodes = cap_nodes;
    S.alloc_depth = p.max_depth;
    S.cap_level = std::min(cap_refs, cap_nodes) + 1;
    S.cap_large = cap_refs / (kWarpExact + 1) + 2;   // learned mode: every node above 32 references
    S.cap_chunks = cap_refs / kChunk + S.cap_large + 2;
    S.cap_medium = cap_refs / (kWarpExact + 1) + 2;
    S.cap_learn = cap_refs / (kWarpExact + 1) + 2;
    S.plan_tiles = S.cap_level / kPlanTile + 2;
    S.ref_tiles = cap_refs / kTile + 2;
    // a deferred root holds 2..32 references, all within the reference arena
    S.cap_defer = cap_refs / 2 + 2;
    // subtree scratch: the arenas' own capacities, plus one open chunk per
    // warp of k_subtree, plus the reference slots a chunk can leave unused at
    // its end (fewer than a 32-reference leaf, per 256)
    {
        const uint64_t warps = (uint64_t)sub_grid(sm_count) * kSubWarps;
        S.cap_sc_nodes = (uint32_t)std::min<uint64_t>((uint64_t)cap_nodes + warps * kScNodeChunk, kMaxIndex);
        S.cap_sc_refs =
            (uint32_t)std::min<uint64_t>((uint64_t)cap_refs + cap_refs / 7 + warps * kScRefChunk, kMaxIndex);
    }
    S.sub_tiles = S.cap_defer / kTile + 2;
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
    bad |= dalloc(S.d_split, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.d_scat, S.cap_level) != cudaSuccess;
    bad |= dalloc(S.chunks, S.cap_chunks + S.cap_large) != cudaSuccess;  // tail holds large_slot
    bad |= dalloc(S.hist, (size_t)S.cap_large * kHist) != cudaSuccess;
    bad |= dalloc(S.done, S.cap_large) != cudaSuccess;
    bad |= dalloc(S.medium_slot, S.cap_medium) != cudaSuccess;
    bad |= dalloc(S.learn_slot, S.cap_learn) != cudaSuccess;
    bad |= dalloc(S.learn_bin, S.cap_learn) != cudaSuccess;
    bad |= dalloc(S.learn_prop, S.cap_learn) != cudaSuccess;
    bad |= dalloc(S.feat, (size_t)S.cap_learn * kMlpIn) != cudaSuccess;
    if (p.prop_log) bad |= dalloc(S.prop_log, (size_t)cap_nodes * 8) != cudaSuccess;
    bad |= dalloc(S.plan_flags, S.plan_tiles) != cudaSuccess;
    bad |= dalloc(S.ref_flags, S.ref_tiles) != cudaSuccess;
    bad |= dalloc(S.plan_done, S.plan_tiles) != cudaSuccess;
    {
        U7 *pa = nullptr, *pi = nullptr;
        bad |= dalloc(pa, S.plan_tiles) != cudaSuccess;
        bad |= dalloc(pi, S.plan_tiles) != cudaSuccess;
        S.plan_agg = pa;
        S.plan_incl = pi;
    }
    bad |= dalloc(S.ref_agg, S.ref_tiles) != cudaSuccess;
    bad |= dalloc(S.ref_incl, S.ref_tiles) != cudaSuccess;
    bad |= dalloc(S.epoch, 1) != cudaSuccess;
    bad |= dalloc(S.ctr, 1) != cudaSuccess;
    bad |= dalloc(S.err, 1) != cudaSuccess;
    bad |= dalloc(S.out_nodes, cap_nodes) != cudaSuccess;
    bad |= dalloc(S.out_refs, cap_refs) != cudaSuccess;
    bad |= dalloc(S.out_ropes, (size_t)cap_nodes * 6) != cudaSuccess;
    bad |= dalloc(S.out_cbox, (size_t)cap_nodes * 2) != cudaSuccess;
    bad |= dalloc(S.d_root, S.cap_defer) != cudaSuccess;
    bad |= dalloc(S.d_lo, S.cap_defer) != cudaSuccess;
    bad |= dalloc(S.d_hi, S.cap_defer) != cudaSuccess;
    bad |= dalloc(S.defer_refs, cap_refs) != cudaSuccess;
    bad |= dalloc(S.sc_key, S.cap_sc_nodes) != cudaSuccess;
    bad |= dalloc(S.sc_node, S.cap_sc_nodes) != cudaSuccess;
    bad |= dalloc(S.sc_cbox, (size_t)S.cap_sc_nodes * 2) != cudaSuccess;
    bad |= dalloc(S.sc_rope, (size_t)S.cap_sc_nodes * 6) != cudaSuccess;
    bad |= dalloc(S.sc_ref, S.cap_sc_refs) != cudaSuccess;
    bad |= dalloc(S.st_cnt, S.cap_defer) != cudaSuccess;
    bad |= dalloc(S.st_root, S.cap_defer) != cudaSuccess;
    bad |= dalloc(S.st_base, S.cap_defer) != cudaSuccess;
    bad |= dalloc(S.sub_flags, S.sub_tiles) != cudaSuccess;
    bad |= dalloc(S.sub_agg, S.sub_tiles) != cudaSuccess;
    bad |= dalloc(S.sub_incl, S.sub_tiles) != cudaSuccess;
    bad |= cudaStreamCreateWithFlags(&S.aux, cudaStreamNonBlocking) != cudaSuccess;
    bad |= cudaEventCreateWithFlags(&S.ev_fork, cudaEventDisableTiming) != cudaSuccess;
    bad |= cudaEventCreateWithFlags(&S.ev_join, cudaEventDisableTiming) != cudaSuccess;
    bad |= cudaStreamCreateWithFlags(&S.aux2, cudaStreamNonBlocking) != cudaSuccess;
    bad |= cudaEventCreateWithFlags(&S.ev_learn, cudaEventDisableTiming) != cudaSuccess;
    bad |= cudaEventCreateWithFlags(&S.ev_join2, cudaEventDisableTiming) != cudaSuccess;
    if (bad) {
        build_release(S);
        return HK_E_ALLOC;
    }
    cudaMemset(S.err, 0, 4);
    cudaMemset(S.epoch, 0, 4);
    cudaMemset(S.hist, 0, (size_t)S.cap_large * kHist * sizeof(uint32_t));
    cudaMemset(S.done, 0, (size_t)S.cap_large * sizeof(uint32_t));
    cudaMemset(S.plan_flags, 0, (size_t)S.plan_tiles * 4);
    cudaMemset(S.ref_flags, 0, (size_t)S.ref_tiles * 4);
    cudaMemset(S.plan_done, 0, (size_t)S.plan_tiles * 4);
    cudaMemset(S.sub_flags, 0, (size_t)S.sub_tiles * 4);

    cudaMemset(S.ctr, 0, sizeof(BuildCounters));
    // these run on the legacy stream, which does not order against the
    // context's own stream: every one is finished before a build may start
    if (cudaDeviceSynchronize() != cudaSuccess) return HK_E_ALLOC;
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

cudaError_t build_learn_setup() {
    static uint64_t attr_set = 0;   // the shared-memory opt-in is per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || !((attr_set >> dev) & 1u)) {
        e = cudaFuncSetAttribute(k_learn<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_learn<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_refine_cta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRefineSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_refine_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRefineWarpSmem);
        if (e != cudaSuccess) return e;
        if (dev < 64) attr_set |= 1ull << dev;
    }
    return cudaSuccess;
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
    A.split = S.d_split;
    A.scat = S.d_scat;
    A.chunks = S.chunks;
    A.large_slot = reinterpret_cast<uint32_t *>(S.chunks + S.cap_chunks);
    A.hist = S.hist;
    A.done = S.done;
    A.out_nodes = S.out_nodes;
    A.out_refs = S.out_refs;
    A.out_ropes = S.out_ropes;
    A.out_cbox = S.out_cbox;
    A.ctr = S.ctr;
    A.err = S.err;
    A.epoch = S.epoch;
    A.ct = S.p.ct;
    A.ci = S.p.ci;
    A.max_depth = S.p.max_depth;
    A.leaf_size = S.p.leaf_size;
    A.cap_refs = S.cap_refs;
    A.cap_nodes = S.cap_nodes;
    A.cap_level = S.cap_level;
    A.cap_large = S.cap_large;
    A.cap_chunks = S.cap_chunks;
    A.cap_medium = S.cap_medium;
    A.medium_slot = S.medium_slot;
    A.learned = (S.p.mode == HK_BUILD_LEARNED) ? 1 : 0;
    // learned mode: nodes up to 32 references take the warp's exact SAH,
    // 33..1024 the proposer, larger ones the binned SAH (exact_max unused)
    A.exact_max = A.learned ? 0u : S.p.exact_max;
    A.record = (S.p.mode == HK_BUILD_BINNED && S.p.record && S.learn && S.learn->rec_X) ? 1 : 0;
    A.learn_slot = S.learn_slot;
    A.learn_bin = S.learn_bin;
    A.learn_prop = S.learn_prop;
    A.feat = S.feat;
    A.cap_learn = S.cap_learn;
    A.prop_log = (A.learned && S.p.prop_log) ? S.prop_log : nullptr;
    A.fallback_ratio = S.p.fallback_ratio;
    A.topk = S.p.topk;
    A.spin_limit = S.p.spin_limit ? S.p.spin_limit : kSpinLimit;
    A.withhold_level = (S.p.debug_flags & 1u) ? 1u : 0xffffffffu;
    A.defer = std::min<uint32_t>(S.p.defer, kDeferMax);
    A.defer_level = (S.p.defer_margin && S.p.defer_margin < S.p.max_depth) ? S.p.max_depth - S.p.defer_margin : 0u;
    A.d_root = S.d_root;
    A.d_lo = S.d_lo;
    A.d_hi = S.d_hi;
    A.defer_refs = S.defer_refs;
    A.cap_defer = S.cap_defer;
    A.sc_key = S.sc_key;
    A.sc_node = S.sc_node;
    A.sc_cbox = S.sc_cbox;
    A.sc_rope = S.sc_rope;
    A.sc_ref = S.sc_ref;
    A.cap_sc_nodes = S.cap_sc_nodes;
    A.cap_sc_refs = S.cap_sc_refs;
    A.st_cnt = S.st_cnt;
    A.st_root = S.st_root;
    A.st_base = S.st_base;
    if (S.learn) {
        A.rec_X = S.learn->rec_X;
        A.rec_y = S.learn->rec_y;
        A.rec_rows = S.learn->rec_rows;
        A.rec_cap = S.learn->rec_cap;
    }
    if (A.learned) {
        if (!(S.learn && S.learn->have_mlp)) return cudaErrorInvalidValue;
        A.mlp = S.learn->mlp;
        const cudaError_t e = build_learn_setup();
        if (e != cudaSuccess) return e;
    }
    cudaMemsetAsync(S.ctr, 0, sizeof(BuildCounters), st);
    if (A.prop_log) cudaMemsetAsync(A.prop_log, 0xff, (size_t)S.cap_nodes * 8 * sizeof(int32_t), st);
    // the per-rank histograms and done counters are zero here: zeroed at
    // allocation, cleaned by the kernel that used them, and zeroed again by
    // build_read_stats after a build that stopped on an error
    if (nt) k_tri_bounds<<<(nt + 255) / 256, 256, 0, st>>>(verts, tris, nt, S.tb_lo, S.tb_hi);
    for (int k = 0; k < 2; k++) {
        A.lo_buf[k] = S.n_lo[k];
        A.hi_buf[k] = S.n_hi[k];
        A.info_buf[k] = S.n_info[k];
        A.refs_buf[k] = S.refs[k];
        A.ref_node_buf[k] = S.ref_node[k];
    }
    A.level = 0;
    k_root<<<G, 256, 0, st>>>(A, box, nt);
    const bool exact_small = A.learned || A.exact_max >= kWarpExact;
    const uint32_t sub_E = sub_stack_entries(S.p.max_depth);
    const size_t sub_smem = kSubWarps * sub_warp_smem(sub_E);
    const bool binned_only = !A.learned && A.exact_max == 0 && S.p.level_streams != 2;
    for (uint32_t L = 0; L <= S.p.max_depth; L++) {
        A.level = L;
        A.lc = &S.ctr->lvl[L];
        A.nlc = &S.ctr->lvl[L + 1];
        if (binned_only) {
            // one wave (four CTAs per SM resident), grid-stride over the work
            launch_pdl(k_decide, S.sm_count * 4, 256, 0, st, A);
            launch_pdl(k_plan_refs, S.sm_count * 6, kScanThreads, 0, st, A, S.plan_flags,
                       static_cast<U7 *>(S.plan_agg), static_cast<U7 *>(S.plan_incl), S.ref_flags, S.ref_agg,
                       S.ref_incl, S.plan_done, &A.lc->plan_ticket);
            continue;
        }
        // large (and medium) nodes on the second stream, beside the small
        // nodes (independent nodes; both only add to the level tallies):
        // binned histograms, or the proposer's features, inference and costing
        cudaEventRecord(S.ev_fork, st);
        cudaStreamWaitEvent(S.aux, S.ev_fork, 0);
        k_hist<<<S.sm_count * 3, 256, 0, S.aux>>>(A);   // one wave: three CTAs per SM resident
        if (A.learned) {
            // the proposer's chain on the second stream after the histograms
            // (every proposer row comes from k_hist), beside the small nodes
            if (mlp_use_tcgen05() && A.mlp.tcw) launch_pdl(k_learn<true>, S.sm_count, 256, kTcSmem, S.aux, A);
            else launch_pdl(k_learn<false>, S.sm_count, 256, kTileSmem, S.aux, A);
            // the two costing kernels take disjoint rows (by reference count)
            // and only add to the tallies: the warp-costed rows on a third
            // stream, beside the CTA-costed ones
            cudaEventRecord(S.ev_learn, S.aux);
            cudaStreamWaitEvent(S.aux2, S.ev_learn, 0);
            k_refine_warp<<<S.sm_count * kRefineWarpGrid, 256, kRefineWarpSmem, S.aux2>>>(A);
            cudaEventRecord(S.ev_join2, S.aux2);
            launch_pdl(k_refine_cta, S.sm_count * 8, kRefineThreads, kRefineSmem, S.aux, A);
        }
        cudaEventRecord(S.ev_join, S.aux);
        if (A.learned) {
            launch_pdl(k_small<true, true>, S.sm_count * 5, 256, 0, st, A);
        } else if (A.exact_max >= kWarpExact) {
            launch_pdl(k_small<true, false>, S.sm_count * 5, 256, 0, st, A);
        } else {
            launch_pdl(k_small<false, false>, S.sm_count * 5, 256, 0, st, A);
        }
        cudaStreamWaitEvent(st, S.ev_join, 0);
        if (A.learned) cudaStreamWaitEvent(st, S.ev_join2, 0);
        launch_pdl(k_plan_refs, S.sm_count * 6, kScanThreads, 0, st, A, S.plan_flags, static_cast<U7 *>(S.plan_agg),
                   static_cast<U7 *>(S.plan_incl), S.ref_flags, S.ref_agg, S.ref_incl, S.plan_done,
                   &A.lc->plan_ticket);
    }
    if (A.defer) {
        // every subtree (roots 0 .. the last level's total, tickets of level
        // 0's counter: the earliest roots, with the largest subtrees, first),
        // then their places and the final layout; tag level 63 keeps the
        // scan's flags apart from the levels'
        A.lc = &S.ctr->lvl[0];
        A.nlc = &S.ctr->lvl[S.p.max_depth + 1];
        if (exact_small)
            launch_pdl(k_subtree<true>, sub_grid(S.sm_count), kSubWarps * 32, sub_smem, st, A, sub_E);
        else
            launch_pdl(k_subtree<false>, sub_grid(S.sm_count), kSubWarps * 32, sub_smem, st, A, sub_E);
        A.level = 63;
        A.lc = &S.ctr->lvl[S.p.max_depth + 1];
        launch_pdl(k_sub_scan, S.sm_count * 2, kScanThreads, 0, st, A, S.sub_flags, S.sub_agg, S.sub_incl);
        launch_pdl(k_sub_place, S.sm_count * 8, 256, 0, st, A);
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
    S.last_err = err;
    if (err) {
        cudaMemsetAsync(S.err, 0, 4, st);
        // a stopped build may leave partial histograms behind
        cudaMemsetAsync(S.hist, 0, (size_t)S.cap_large * kHist * sizeof(uint32_t), st);
        cudaMemsetAsync(S.done, 0, (size_t)S.cap_large * sizeof(uint32_t), st);
        if (err & (4u | kErrTensorWait)) return HK_E_DEVICE_TIMEOUT;   // a bounded wait ran out
        if (err & (8u | 16u)) return HK_E_BOUNDS;       // a partition / plan check fired
        return HK_E_CAPACITY;                           // an arena or list was too small
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
