// hk_build_resort.cu -- the reference's per-node re-sampling SAH builder
// (--treeType=SAH: KDTreeCPU::buildKDTreeSAH / buildNodeSAH,
// HulkEngine/src/KDTreeSAH.cpp:9-244) on the GPU, one level at a time.
//
// The reference recurses depth-first; every node takes every sample-th
// polygon of its own list, clips the triangle's bounds to the node box, makes
// one co-planar candidate (clipped extent <= FLT_EPSILON) or a begin and an
// end candidate per axis, sorts each axis, and sweeps the sorted values with
// running counts (below += previous group's co-planar + begin counts;
// co-planar = previous group's co-planar count; above -= this group's
// co-planar + end counts; the first group starts from list size / sample).
// Nodes are independent, so here all nodes of a level are processed at once:
//
//   keys     one 64-bit key per candidate slot: segment (node x 3 + axis),
//            the value as an order-preserving integer, the marker; each
//            segment occupies a fixed range (two slots per sampled polygon,
//            an unused slot sorts last in its segment)
//   sort     LSD radix sort of the level's keys, 8 bits per pass (so each
//            segment ends up sorted in place)
//   sweep    the running counts of the sequential sweep are prefix sums over
//            the sorted keys, taken with device-wide scans and read back at
//            every group of equal values; each group's SAH cost is computed
//            with the reference's float expression and the first minimum in
//            sweep order (axis, then value) wins through a 64-bit atomicMin
//            of (cost, key position)
//   split    checkPolygonToAAPlane by vertex coordinates on every polygon of
//            a split node; a stable partition (scans) writes the next level's
//            lists in the reference's list order, below child then above
//
// The output is the compact tree the traversal kernels read (child pairs in
// breadth-first order: below, above; an absent child is an empty leaf cell),
// with the ropes and cell boxes of every cell. It is the tree of the
// reference's builder in the layout hk_tree_import makes of it.
#include <algorithm>
#include <cfloat>
#include <string>

#include "hk_common.cuh"
#include "hk_resort.h"

namespace hk {

template <class T>
cudaError_t RBuf<T>::ensure(size_t n) {
    if (n <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t c = n < 16 ? 16 : n + n / 4;
    cudaError_t e = cudaMalloc((void **)&p, c * sizeof(T));
    if (e == cudaSuccess) cap = c;
    return e;
}

template <class T>
void RBuf<T>::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

namespace {

typedef unsigned long long u64;

// grow an output array keeping its first `keep` elements
template <class T>
cudaError_t grow_keep(RBuf<T> &b, size_t n, size_t keep, cudaStream_t st) {
    if (n <= b.cap && b.p) return cudaSuccess;
    const size_t c = n + n / 2 + 64;
    T *q = nullptr;
    cudaError_t e = cudaMalloc((void **)&q, c * sizeof(T));
    if (e != cudaSuccess) return e;
    if (b.p && keep) {
        e = cudaMemcpyAsync(q, b.p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) {
            cudaFree(q);
            return e;
        }
        cudaStreamSynchronize(st);
    }
    if (b.p) cudaFree(b.p);
    b.p = q;
    b.cap = c;
    return cudaSuccess;
}

// ---------------------------------------------------------------- scans ----
constexpr int kSB = 512;  // threads per scan block
constexpr int kSI = 8;    // elements per thread

template <class T>
__device__ __forceinline__ T warp_incl(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// exclusive block scan; *total (if given) receives the block's sum
template <class T>
__device__ T block_excl(T v, T *sw, T *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const T inc = warp_incl(v);
    if (lane == 31) sw[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? sw[lane] : T(0);
        s = warp_incl(s);
        sw[lane] = s;
    }
    __syncthreads();
    const T base = w ? sw[w - 1] : T(0);
    if (total) *total = sw[nw - 1];
    __syncthreads();
    return base + inc - v;
}

template <class T>
__global__ void __launch_bounds__(kSB) k_scan_reduce(const T *__restrict__ in, uint32_t n, T *part) {
    __shared__ T sw[32];
    const size_t base = (size_t)blockIdx.x * kSB * kSI;
    T s = 0;
#pragma unroll
    for (int k = 0; k < kSI; k++) {
        const size_t i = base + (size_t)k * kSB + threadIdx.x;
        if (i < n) s += in[i];
    }
    T tot;
    block_excl(s, sw, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

template <class T>
__global__ void __launch_bounds__(kSB) k_scan_part(T *part, uint32_t nb) {
    __shared__ T sw[32];
    T carry = 0;
    for (uint32_t b0 = 0; b0 < nb; b0 += kSB) {
        const uint32_t i = b0 + threadIdx.x;
        const T v = i < nb ? part[i] : T(0);
        T tot;
        const T e = block_excl(v, sw, &tot);
        if (i < nb) part[i] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) part[nb] = carry;
}

template <class T>
__global__ void __launch_bounds__(kSB) k_scan_down(const T *in, uint32_t n, const T *__restrict__ part, T *out) {
    __shared__ T sw[32];
    const size_t base = (size_t)blockIdx.x * kSB * kSI + (size_t)threadIdx.x * kSI;
    T v[kSI];
    T s = 0;
#pragma unroll
    for (int k = 0; k < kSI; k++) {
        const size_t i = base + k;
        v[k] = i < n ? in[i] : T(0);
        s += v[k];
    }
    T e = block_excl(s, sw, (T *)nullptr) + part[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kSI; k++) {
        const size_t i = base + k;
        if (i < n) out[i] = e;
        e += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = part[gridDim.x];
}

// out[0..n] = exclusive prefix sums of in[0..n) and the total; out may be in
template <class T>
cudaError_t scan_excl(const T *in, T *out, uint32_t n, RBuf<T> &part, cudaStream_t st) {
    const uint32_t per = (uint32_t)(kSB * kSI);
    uint32_t nb = (n + per - 1) / per;
    if (nb == 0) nb = 1;
    cudaError_t e = part.ensure(nb + 1);
    if (e != cudaSuccess) return e;
    k_scan_reduce<T><<<nb, kSB, 0, st>>>(in, n, part.p);
    k_scan_part<T><<<1, kSB, 0, st>>>(part.p, nb);
    k_scan_down<T><<<nb, kSB, 0, st>>>(in, n, part.p, out);
    return cudaGetLastError();
}

// ----------------------------------------------------------- radix sort ----
constexpr int kRT = 256;                     // threads per sort tile
constexpr int kRI = 16;                      // keys per thread
constexpr uint32_t kTile = kRT * kRI;        // 4096 keys per tile

__global__ void __launch_bounds__(kRT) k_rs_hist(const u64 *__restrict__ keys, uint32_t n, int shift,
                                                 uint32_t ntiles, uint32_t *hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * kTile;
    for (int r = 0; r < kRI; r++) {
        const size_t i = base + (size_t)r * kRT + threadIdx.x;
        if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// stable scatter: within a tile keys are ranked in index order (rounds of
// 256 consecutive keys; warps in order; lanes by __match_any_sync)
__global__ void __launch_bounds__(kRT) k_rs_scatter(const u64 *__restrict__ in, u64 *__restrict__ out, uint32_t n,
                                                    int shift, uint32_t ntiles, const uint32_t *__restrict__ offs) {
    __shared__ uint32_t run[256];
    __shared__ uint32_t wc[kRT / 32][256];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    run[threadIdx.x] = 0;
    const size_t base = (size_t)blockIdx.x * kTile;
    for (int r = 0; r < kRI; r++) {
        for (uint32_t q = threadIdx.x; q < (kRT / 32) * 256; q += kRT) (&wc[0][0])[q] = 0;
        __syncthreads();
        const size_t i = base + (size_t)r * kRT + threadIdx.x;
        const bool have = i < n;
        const u64 k = have ? in[i] : 0ull;
        const uint32_t d = have ? ((uint32_t)(k >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if (have && lane == (uint32_t)(__ffs(peers) - 1)) wc[w][d] = __popc(peers);
        __syncthreads();
        size_t dst = 0;
        if (have) {
            uint32_t pre = 0;
            for (uint32_t q = 0; q < w; q++) pre += wc[q][d];
            dst = (size_t)offs[(size_t)d * ntiles + blockIdx.x] + run[d] + pre + rank;
        }
        __syncthreads();
        uint32_t tot = 0;
        for (int q = 0; q < kRT / 32; q++) tot += wc[q][threadIdx.x];
        run[threadIdx.x] += tot;
        if (have) out[dst] = k;
        __syncthreads();
    }
}

// ------------------------------------------------------------- helpers ----
constexpr uint32_t kNone = 3u;      // marker of an unused key slot
constexpr uint32_t kDecLeaf = 3u;   // decision: leaf (else the split axis)

__device__ __forceinline__ float c3(const float4 &v, uint32_t a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }
__device__ __forceinline__ void s3(float4 &v, uint32_t a, float x) {
    if (a == 0) v.x = x;
    else if (a == 1) v.y = x;
    else v.z = x;
}
// _mm_min_ps / _mm_max_ps lanes
__device__ __forceinline__ float mnf(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float mxf(float a, float b) { return a > b ? a : b; }

__device__ __forceinline__ uint32_t f2o(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}
__device__ __forceinline__ u64 make_key(uint32_t seg, float v, uint32_t marker) {
    return ((u64)seg << 34) | ((u64)f2o(v) << 2) | marker;
}
__device__ __forceinline__ float key_value(u64 k) { return o2f((uint32_t)(k >> 2)); }
__device__ __forceinline__ uint32_t lo32(u64 x) { return (uint32_t)x; }
__device__ __forceinline__ uint32_t hi32(u64 x) { return (uint32_t)(x >> 32); }

struct LevelPtrs {
    // this level
    uint32_t n;
    const float4 *lo, *hi;
    const float *surf;
    const uint32_t *off, *cnt, *ropes, *refs, *ref_node;
    // scratch
    uint32_t *nkeys, *koff, *jflag, *jrank, *leafcnt, *loff, *efirst, *decision, *gfirst;
    float *plane, *surf_lo, *surf_hi;
    u64 *best, *keys, *f1, *f2, *rflag, *rscan;
    uint32_t *maxseg;   // longest candidate segment of the level
    // next level
    float4 *nlo, *nhi;
    float *nsurf;
    uint32_t *noff, *ncnt, *nropes, *nrefs, *nref_node;
    // output
    uint2 *nodes;
    uint32_t *out_refs, *out_ropes;
    float4 *out_cbox;
    uint32_t cbase, nbase, rbase;
    ResortParams p;
    uint32_t depth;
};

__device__ __forceinline__ bool forced_leaf(const LevelPtrs &L, uint32_t c) {
    return c == 0 || c <= L.p.leaf_size || L.depth >= L.p.max_depth;
}

__global__ void k_r_init(LevelPtrs L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    const uint32_t c = L.cnt[i];
    const uint32_t s = forced_leaf(L, c) ? 0u : (c + L.p.sample - 1) / L.p.sample;
    L.nkeys[i] = 6u * s;
    if (s) atomicMax(L.maxseg, 2u * s);
    L.best[i] = ~0ull;
    L.efirst[3 * i] = L.efirst[3 * i + 1] = L.efirst[3 * i + 2] = 0;
}

// KDTreeSAH.cpp:51-82: candidates of the sampled polygons
__global__ void k_r_emit(LevelPtrs L, uint32_t Q, const float4 *__restrict__ V, const uint4 *__restrict__ T) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    uint32_t a = 0, b = L.n;   // node: koff[i] / 6 <= q < koff[i + 1] / 6
    while (a < b) {
        const uint32_t m = (a + b) >> 1;
        if (L.koff[m + 1] / 6u <= q) a = m + 1;
        else b = m;
    }
    const uint32_t i = a;
    const uint32_t s = (L.koff[i + 1] - L.koff[i]) / 6u, j = q - L.koff[i] / 6u;
    const uint32_t poly = L.refs[L.off[i] + j * L.p.sample];
    const uint4 t = T[poly];
    const float4 p1 = V[t.x], p2 = V[t.y], p3 = V[t.z];
    const float4 bl = L.lo[i], bh = L.hi[i];
#pragma unroll
    for (uint32_t ax = 0; ax < 3; ax++) {
        float lo = mnf(mnf(c3(p1, ax), c3(p2, ax)), c3(p3, ax));
        float hi = mxf(mxf(c3(p1, ax), c3(p2, ax)), c3(p3, ax));
        lo = mxf(lo, c3(bl, ax));
        hi = mnf(hi, c3(bh, ax));
        const uint32_t seg = 3 * i + ax;
        const size_t k = (size_t)L.koff[i] + (size_t)ax * 2 * s + 2 * (size_t)j;
        if (fabsf(__fsub_rn(lo, hi)) <= FLT_EPSILON) {
            L.keys[k] = make_key(seg, lo, 1);
            L.keys[k + 1] = ((u64)seg << 34) | (0xffffffffull << 2) | kNone;
        } else {
            L.keys[k] = make_key(seg, lo, 0);
            L.keys[k + 1] = make_key(seg, hi, 2);
        }
    }
}

__device__ __forceinline__ void seg_range(const LevelPtrs &L, uint32_t seg, uint32_t &i, uint32_t &ax, uint32_t &s0,
                                          uint32_t &s1) {
    i = seg / 3;
    ax = seg - 3 * i;
    const uint32_t s = (L.koff[i + 1] - L.koff[i]) / 6u;
    s0 = L.koff[i] + ax * 2 * s;
    s1 = s0 + 2 * s;
}

// Levels whose candidate segments are all short sort each segment on its own
// instead of the whole level: a warp in registers up to kSegWarpMax keys
// (8 per lane), a CTA in shared memory up to kSegCtaMax. Segments hold their
// keys in fixed ranges, so either way every segment ends up sorted in place.
constexpr uint32_t kSegWarpMax = 256, kSegCtaMax = 4096;

template <int RJ>
__device__ __forceinline__ void reg_exchange(u64 (&x)[kSegWarpMax / 32], uint32_t nr, uint32_t lane, uint32_t k) {
#pragma unroll
    for (int r = 0; r < (int)(kSegWarpMax / 32); r++) {
        if ((r & RJ) || (uint32_t)r >= nr) continue;
        const bool up = (((uint32_t)r * 32u + lane) & k) == 0;
        const u64 a = x[r], b = x[r | RJ];
        if ((a > b) == up) {
            x[r] = b;
            x[r | RJ] = a;
        }
    }
}

__global__ void k_seg_sort_warp(LevelPtrs L, uint32_t nseg) {
    const uint32_t lane = threadIdx.x & 31u, seg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (seg >= nseg) return;   // uniform over the warp
    uint32_t i, ax, s0, s1;
    seg_range(L, seg, i, ax, s0, s1);
    const uint32_t n = s1 - s0;
    if (n <= 1 || n > kSegWarpMax) return;
    uint32_t n2 = 1;
    while (n2 < n) n2 <<= 1;
    const uint32_t nr = (n2 + 31u) >> 5;
    u64 x[kSegWarpMax / 32];
#pragma unroll
    for (int r = 0; r < (int)(kSegWarpMax / 32); r++) {
        const uint32_t e = (uint32_t)r * 32u + lane;
        x[r] = e < n ? L.keys[s0 + e] : ~0ull;
    }
    for (uint32_t k = 2; k <= n2; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                // partners in the lane's own registers (compile-time indices)
                if (j == 32) reg_exchange<1>(x, nr, lane, k);
                else if (j == 64) reg_exchange<2>(x, nr, lane, k);
                else reg_exchange<4>(x, nr, lane, k);
            } else {
                const bool lower = (lane & j) == 0;
#pragma unroll
                for (int r = 0; r < (int)(kSegWarpMax / 32); r++) {
                    if ((uint32_t)r >= nr) continue;
                    const u64 o = __shfl_xor_sync(0xffffffffu, x[r], (int)j);
                    const bool up = (((uint32_t)r * 32u + lane) & k) == 0;
                    const u64 mn = x[r] < o ? x[r] : o, mx = x[r] < o ? o : x[r];
                    x[r] = (lower == up) ? mn : mx;
                }
            }
        }
#pragma unroll
    for (int r = 0; r < (int)(kSegWarpMax / 32); r++) {
        const uint32_t e = (uint32_t)r * 32u + lane;
        if (e < n) L.keys[s0 + e] = x[r];
    }
}

__global__ void __launch_bounds__(256) k_seg_sort_cta(LevelPtrs L, uint32_t nseg) {
    __shared__ u64 sk[kSegCtaMax];
    for (uint32_t seg = blockIdx.x; seg < nseg; seg += gridDim.x) {
        uint32_t i, ax, s0, s1;
        seg_range(L, seg, i, ax, s0, s1);
        const uint32_t n = s1 - s0;
        if (n <= kSegWarpMax || n > kSegCtaMax) continue;   // uniform over the CTA
        uint32_t n2 = 1;
        while (n2 < n) n2 <<= 1;
        for (uint32_t e = threadIdx.x; e < n2; e += blockDim.x) sk[e] = e < n ? L.keys[s0 + e] : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= n2; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t e = threadIdx.x; e < n2; e += blockDim.x) {
                    const uint32_t p = e ^ j;
                    if (p > e) {
                        const bool up = (e & k) == 0;
                        const u64 a = sk[e], b = sk[p];
                        if ((a > b) == up) {
                            sk[e] = b;
                            sk[p] = a;
                        }
                    }
                }
                __syncthreads();
            }
        for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) L.keys[s0 + e] = sk[e];
        __syncthreads();
    }
}

// group heads and the counters the sweep accumulates:
//   f1 = [begin or co-planar] | [co-planar] << 32, f2 = [end] | [head] << 32
__global__ void k_r_heads(LevelPtrs L, uint32_t K) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= K) return;
    const u64 k = L.keys[p];
    const uint32_t m = (uint32_t)k & 3u;
    const bool real = m != kNone;
    bool head = false;
    if (real) {
        uint32_t i, ax, s0, s1;
        seg_range(L, (uint32_t)(k >> 34), i, ax, s0, s1);
        const float v = key_value(k);
        head = p == s0 || !(key_value(L.keys[p - 1]) == v);
        // ends in the segment's first group are never subtracted (:164-169)
        if (m == 2 && key_value(L.keys[s0]) == v) atomicAdd(&L.efirst[(uint32_t)(k >> 34)], 1u);
    }
    L.f1[p] = (u64)(real && m != 2) | ((u64)(real && m == 1) << 32);
    L.f2[p] = (u64)(real && m == 2) | ((u64)head << 32);
}

__global__ void k_r_gfirst(LevelPtrs L, uint32_t K) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) L.gfirst[hi32(L.f2[K])] = K;   // f2 holds the scan: total groups
    if (p >= K) return;
    const u64 a = L.f2[p], b = L.f2[p + 1];
    if (hi32(b) != hi32(a)) L.gfirst[hi32(a)] = p;
}

// (cost, key position) of the group that starts at key p, or ~0 when p
// starts no group or its cost is not below FLT_MAX
__device__ u64 r_group_cost(const LevelPtrs &L, uint32_t p) {
    const u64 g2 = L.f2[p], g2n = L.f2[p + 1];
    if (hi32(g2n) == hi32(g2)) return ~0ull;   // not a group head
    const uint32_t g = hi32(g2);
    const u64 k = L.keys[p];
    const uint32_t seg = (uint32_t)(k >> 34);
    uint32_t i, ax, s0, s1;
    seg_range(L, seg, i, ax, s0, s1);
    const uint32_t real_end = s0 + (lo32(L.f1[s1]) - lo32(L.f1[s0])) + (lo32(L.f2[s1]) - lo32(L.f2[s0]));
    const uint32_t nxt = L.gfirst[g + 1];
    const uint32_t l1 = nxt < real_end ? nxt : real_end;
    const uint32_t cop_here = hi32(L.f1[l1]) - hi32(L.f1[p]);
    const uint32_t cop = p == s0 ? cop_here : hi32(L.f1[p]) - hi32(L.f1[L.gfirst[g - 1]]);
    const uint32_t below = lo32(L.f1[p]) - lo32(L.f1[s0]);
    const uint32_t N = L.cnt[i] / L.p.sample;
    const uint32_t above = N - (hi32(L.f1[l1]) - hi32(L.f1[s0])) - ((lo32(L.f2[l1]) - lo32(L.f2[s0])) - L.efirst[seg]);
    const float v = key_value(k);
    const float4 bl = L.lo[i], bh = L.hi[i];
    const float dim[3] = {__fsub_rn(bh.x, bl.x), __fsub_rn(bh.y, bl.y), __fsub_rn(bh.z, bl.z)};
    const float x = dim[(ax + 1) % 3], y = dim[(ax + 2) % 3];
    const float xpy = __fadd_rn(x, y), area = __fmul_rn(x, y);
    const float upper = __fadd_rn(area, __fmul_rn(__fsub_rn(c3(bh, ax), v), xpy));
    const float lower = __fadd_rn(area, __fmul_rn(__fsub_rn(v, c3(bl, ax)), xpy));
    const float cb = __fmul_rn(lower, (float)below), ca = __fmul_rn(upper, (float)above);
    const float ci = __fmul_rn(area, (float)cop);
    const float inv = __fdiv_rn(1.0f, L.surf[i]);
    const float score =
        __fadd_rn(L.p.ct, __fmul_rn(L.p.ci, __fmul_rn(__fadd_rn(__fadd_rn(ci, cb), ca), inv)));
    return score < FLT_MAX ? ((u64)f2o(score) << 32) | p : ~0ull;
}

// the SAH of every group (KDTreeSAH.cpp:147-175); the node's minimum of
// (cost, position) is taken over the warp first (keys are sorted by node, so
// a warp's lanes span few nodes), then with one atomicMin per node and warp
__global__ void k_r_cost(LevelPtrs L, uint32_t K) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    u64 packed = ~0ull;
    uint32_t node = 0xffffffffu;
    if (p < K) {
        node = (uint32_t)(L.keys[p] >> 34) / 3u;
        packed = r_group_cost(L, p);
    }
    // segmented minimum over runs of equal node in lane order
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const u64 o = __shfl_down_sync(0xffffffffu, packed, off);
        const uint32_t on = __shfl_down_sync(0xffffffffu, node, off);
        if (lane + off < 32 && on == node && o < packed) packed = o;
    }
    const uint32_t prev = __shfl_up_sync(0xffffffffu, node, 1);
    const bool first = lane == 0 || prev != node;
    if (p < K && first && packed != ~0ull) atomicMin(&L.best[node], packed);
}


// leaf test (KDTreeSAH.cpp:186-191) and the split's child surfaces
__global__ void k_r_decide(LevelPtrs L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    const uint32_t c = L.cnt[i];
    const u64 b = L.best[i];
    bool leaf = forced_leaf(L, c) || b == ~0ull;
    if (!leaf) {
        const float score = o2f(hi32(b));
        const float leafcost = __fmul_rn(L.p.ci, (float)(c / L.p.sample));
        leaf = score >= leafcost;
    }
    if (leaf) {
        L.decision[i] = kDecLeaf;
        L.jflag[i] = 0;
        L.leafcnt[i] = c;
        return;
    }
    const u64 k = L.keys[lo32(b)];
    const uint32_t ax = (uint32_t)(k >> 34) % 3u;
    const float v = key_value(k);
    const float4 bl = L.lo[i], bh = L.hi[i];
    const float dim[3] = {__fsub_rn(bh.x, bl.x), __fsub_rn(bh.y, bl.y), __fsub_rn(bh.z, bl.z)};
    const float x = dim[(ax + 1) % 3], y = dim[(ax + 2) % 3];
    const float xpy = __fadd_rn(x, y), area = __fmul_rn(x, y);
    L.surf_hi[i] = __fadd_rn(area, __fmul_rn(__fsub_rn(c3(bh, ax), v), xpy));
    L.surf_lo[i] = __fadd_rn(area, __fmul_rn(__fsub_rn(v, c3(bl, ax)), xpy));
    L.plane[i] = v;
    L.decision[i] = ax;
    L.jflag[i] = 1;
    L.leafcnt[i] = 0;
}

// KDTreeCPU::checkPolygonToAAPlane (KDTreeCPU.cpp:450-477) on the polygons of
// split nodes: rflag = [goes below] | [goes above] << 32
__global__ void k_r_classify(LevelPtrs L, uint32_t R, const float4 *__restrict__ V, const uint4 *__restrict__ T) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= R) return;
    const uint32_t i = L.ref_node[q];
    const uint32_t d = L.decision[i];
    if (d == kDecLeaf) {
        L.rflag[q] = 0;
        return;
    }
    const float v = L.plane[i];
    const uint4 t = T[L.refs[q]];
    const float a = c3(V[t.x], d), b = c3(V[t.y], d), c = c3(V[t.z], d);
    const bool cop = (a == v) & (b == v) & (c == v);
    const bool above = (a >= v) & (b >= v) & (c >= v);
    const bool below = (a <= v) & (b <= v) & (c <= v);
    const bool goA = cop || above || !below;   // above, intersecting, co-planar
    const bool goB = cop || !above;            // below, intersecting, co-planar
    L.rflag[q] = (u64)goB | ((u64)goA << 32);
}

// cells of this level, and the next level's nodes
__global__ void k_r_nodes(LevelPtrs L) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= L.n) return;
    const uint32_t cell = L.cbase + i;
    const uint32_t c = L.cnt[i], d = L.decision[i];
    const float4 bl = L.lo[i], bh = L.hi[i];
    for (int f = 0; f < 6; f++) L.out_ropes[6 * (size_t)cell + f] = L.ropes[6 * (size_t)i + f];
    L.out_cbox[2 * (size_t)cell] = make_float4(bl.x, bl.y, bl.z, 0.0f);
    L.out_cbox[2 * (size_t)cell + 1] = make_float4(bh.x, bh.y, bh.z, 0.0f);
    if (d == kDecLeaf) {
        L.nodes[cell] = c ? make_uint2(((L.rbase + L.loff[i]) << 2) | kLeafTag, c) : make_uint2(kLeafTag, 0u);
        return;
    }
    const uint32_t k = L.jrank[i], pair = L.nbase + 2 * k;
    const float v = L.plane[i];
    L.nodes[cell] = make_uint2((pair << 2) | d, __float_as_uint(v));
    const u64 r0 = L.rscan[L.off[i]], r1 = L.rscan[L.off[i] + c];
    const uint32_t cB = lo32(r1) - lo32(r0), cA = hi32(r1) - hi32(r0);
    const uint32_t oB = lo32(r0) + hi32(r0);
    // below child (pair), above child (pair + 1)
    float4 hB = bh, lA = bl;
    s3(hB, d, v);
    s3(lA, d, v);
    L.nlo[2 * k] = bl;
    L.nhi[2 * k] = hB;
    L.nlo[2 * k + 1] = lA;
    L.nhi[2 * k + 1] = bh;
    L.nsurf[2 * k] = L.surf_lo[i];
    L.nsurf[2 * k + 1] = L.surf_hi[i];
    L.noff[2 * k] = oB;
    L.ncnt[2 * k] = cB;
    L.noff[2 * k + 1] = oB + cB;
    L.ncnt[2 * k + 1] = cA;
    for (int f = 0; f < 6; f++) {
        const uint32_t r = L.ropes[6 * (size_t)i + f];
        L.nropes[12 * (size_t)k + f] = r;
        L.nropes[12 * (size_t)k + 6 + f] = r;
    }
    L.nropes[12 * (size_t)k + 2 * d + 1] = pair + 1;
    L.nropes[12 * (size_t)k + 6 + 2 * d] = pair;
}

// leaf references out; split references into the next level (stable)
__global__ void k_r_scatter(LevelPtrs L, uint32_t R) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= R) return;
    const uint32_t i = L.ref_node[q];
    const uint32_t ref = L.refs[q];
    if (L.decision[i] == kDecLeaf) {
        L.out_refs[L.rbase + L.loff[i] + (q - L.off[i])] = ref;
        return;
    }
    const uint32_t k = L.jrank[i];
    const u64 f = L.rflag[q], rq = L.rscan[q], r0 = L.rscan[L.off[i]], r1 = L.rscan[L.off[i] + L.cnt[i]];
    const uint32_t oB = lo32(r0) + hi32(r0), cB = lo32(r1) - lo32(r0);
    if (lo32(f)) {
        const uint32_t dst = oB + (lo32(rq) - lo32(r0));
        L.nrefs[dst] = ref;
        L.nref_node[dst] = 2 * k;
    }
    if (hi32(f)) {
        const uint32_t dst = oB + cB + (hi32(rq) - hi32(r0));
        L.nrefs[dst] = ref;
        L.nref_node[dst] = 2 * k + 1;
    }
}

__global__ void k_r_iota(uint32_t *refs, uint32_t *ref_node, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        refs[i] = i;
        ref_node[i] = 0;
    }
}

__global__ void k_r_pad(uint2 *nodes, uint32_t *ropes, float4 *cbox) {
    const int f = threadIdx.x;
    if (f == 0) nodes[1] = make_uint2(kLeafTag, 0u);
    if (f < 6) ropes[6 + f] = 0xffffffffu;
    if (f < 2) cbox[2 + f] = make_float4(0, 0, 0, 0);
}

__global__ void k_r_copy3(const uint32_t *a, const u64 *b, uint32_t ia, uint32_t ib, const uint32_t *c, uint32_t ic,
                          uint32_t *out) {
    out[0] = a[ia];
    out[1] = lo32(b[ib]) + hi32(b[ib]);
    out[2] = c[ic];
}

inline unsigned blocks(uint32_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t) ? (unsigned)((n + t - 1) / t) : 1u; }

}  // namespace

void ResortState::release() {
    for (int b = 0; b < 2; b++) {
        lo[b].release();
        hi[b].release();
        surf[b].release();
        off[b].release();
        cnt[b].release();
        ropes[b].release();
        refs[b].release();
        ref_node[b].release();
        keys[b].release();
    }
    nkeys.release();
    koff.release();
    jflag.release();
    jrank.release();
    leafcnt.release();
    loff.release();
    efirst.release();
    decision.release();
    plane.release();
    surf_lo.release();
    surf_hi.release();
    best.release();
    kscan_a.release();
    kscan_b.release();
    rscan.release();
    rflag.release();
    hist.release();
    gfirst.release();
    scan_part.release();
    scan_part64.release();
    dev_u32.release();
    nodes.release();
    out_refs.release();
    out_ropes.release();
    out_cbox.release();
}

#define RS_CHECK(x)                                                 \
    do {                                                            \
        cudaError_t e_ = (x);                                       \
        if (e_ != cudaSuccess) {                                    \
            if (err) *err = std::string(#x) + ": " + cudaGetErrorString(e_); \
            return HK_E_CUDA;                                       \
        }                                                           \
    } while (0)

hk_status resort_build(ResortState &S, const ResortParams &p, const float4 *verts, const uint4 *tris, uint32_t nt,
                       const float *hbox, cudaStream_t st, std::string *err) {
    if (p.sample == 0 || p.max_depth > 64) {
        if (err) *err = "sample must be >= 1 and max_depth <= 64";
        return HK_E_ILLEGAL_INPUT;
    }
    // level 0: the root (cell 0) over every polygon; cell 1 is padding
    // cells [cbase, cbase + n) hold the current level; `written` cells exist
    uint32_t n = 1, R = nt, cbase = 0, rbase = 0, written = 2, depth = 0;
    RS_CHECK(S.lo[0].ensure(1));
    RS_CHECK(S.hi[0].ensure(1));
    RS_CHECK(S.surf[0].ensure(1));
    RS_CHECK(S.off[0].ensure(1));
    RS_CHECK(S.cnt[0].ensure(1));
    RS_CHECK(S.ropes[0].ensure(6));
    RS_CHECK(S.refs[0].ensure(R));
    RS_CHECK(S.ref_node[0].ensure(R));
    RS_CHECK(S.dev_u32.ensure(4));
    RS_CHECK(grow_keep(S.nodes, 2, 0, st));
    RS_CHECK(grow_keep(S.out_ropes, 12, 0, st));
    RS_CHECK(grow_keep(S.out_cbox, 4, 0, st));
    RS_CHECK(grow_keep(S.out_refs, 1, 0, st));
    {
        // root box and half surface (getHalfBoxSurface, SharedFunctions.hpp:40-44)
        const float4 lo = make_float4(hbox[0], hbox[1], hbox[2], hbox[3]);
        const float4 hi = make_float4(hbox[4], hbox[5], hbox[6], hbox[7]);
        const float sx = hbox[4] - hbox[0], sy = hbox[5] - hbox[1], sz = hbox[6] - hbox[2];
        const float half = sx * sy + sz * sy + sx * sz;
        const uint32_t zero = 0, ropes[6] = {~0u, ~0u, ~0u, ~0u, ~0u, ~0u};
        RS_CHECK(cudaMemcpyAsync(S.lo[0].p, &lo, sizeof lo, cudaMemcpyHostToDevice, st));
        RS_CHECK(cudaMemcpyAsync(S.hi[0].p, &hi, sizeof hi, cudaMemcpyHostToDevice, st));
        RS_CHECK(cudaMemcpyAsync(S.surf[0].p, &half, sizeof half, cudaMemcpyHostToDevice, st));
        RS_CHECK(cudaMemcpyAsync(S.off[0].p, &zero, sizeof zero, cudaMemcpyHostToDevice, st));
        RS_CHECK(cudaMemcpyAsync(S.cnt[0].p, &nt, sizeof nt, cudaMemcpyHostToDevice, st));
        RS_CHECK(cudaMemcpyAsync(S.ropes[0].p, ropes, sizeof ropes, cudaMemcpyHostToDevice, st));
        if (R) k_r_iota<<<blocks(R), 256, 0, st>>>(S.refs[0].p, S.ref_node[0].p, R);
        k_r_pad<<<1, 32, 0, st>>>(S.nodes.p, S.out_ropes.p, S.out_cbox.p);
        RS_CHECK(cudaStreamSynchronize(st));
    }
    for (uint32_t level = 0; n > 0; level++) {
        const int cur = level & 1, nxt = cur ^ 1;
        depth = level;
        // per-node scratch
        RS_CHECK(S.nkeys.ensure(n));
        RS_CHECK(S.koff.ensure(n + 1));
        RS_CHECK(S.jflag.ensure(n));
        RS_CHECK(S.jrank.ensure(n + 1));
        RS_CHECK(S.leafcnt.ensure(n));
        RS_CHECK(S.loff.ensure(n + 1));
        RS_CHECK(S.efirst.ensure(3 * (size_t)n));
        RS_CHECK(S.decision.ensure(n));
        RS_CHECK(S.plane.ensure(n));
        RS_CHECK(S.surf_lo.ensure(n));
        RS_CHECK(S.surf_hi.ensure(n));
        RS_CHECK(S.best.ensure(n));
        // this level's cells in the output
        RS_CHECK(grow_keep(S.nodes, (size_t)cbase + n, written, st));
        RS_CHECK(grow_keep(S.out_ropes, 6 * ((size_t)cbase + n), 6 * (size_t)written, st));
        RS_CHECK(grow_keep(S.out_cbox, 2 * ((size_t)cbase + n), 2 * (size_t)written, st));
        LevelPtrs L;
        memset(&L, 0, sizeof L);
        L.n = n;
        L.lo = S.lo[cur].p;
        L.hi = S.hi[cur].p;
        L.surf = S.surf[cur].p;
        L.off = S.off[cur].p;
        L.cnt = S.cnt[cur].p;
        L.ropes = S.ropes[cur].p;
        L.refs = S.refs[cur].p;
        L.ref_node = S.ref_node[cur].p;
        L.nkeys = S.nkeys.p;
        L.koff = S.koff.p;
        L.jflag = S.jflag.p;
        L.jrank = S.jrank.p;
        L.leafcnt = S.leafcnt.p;
        L.loff = S.loff.p;
        L.efirst = S.efirst.p;
        L.decision = S.decision.p;
        L.plane = S.plane.p;
        L.surf_lo = S.surf_lo.p;
        L.surf_hi = S.surf_hi.p;
        L.best = S.best.p;
        L.p = p;
        L.depth = level;
        L.cbase = cbase;
        L.nbase = level == 0 ? 2u : cbase + n;   // the next level's first cell
        L.rbase = rbase;
        // 1. candidates
        L.maxseg = S.dev_u32.p + 3;
        RS_CHECK(cudaMemsetAsync(L.maxseg, 0, 4, st));
        k_r_init<<<blocks(n), 256, 0, st>>>(L);
        RS_CHECK(scan_excl<uint32_t>(S.nkeys.p, S.koff.p, n, S.scan_part, st));
        uint32_t K = 0, maxseg = 0;
        RS_CHECK(cudaMemcpyAsync(&K, S.koff.p + n, 4, cudaMemcpyDeviceToHost, st));
        RS_CHECK(cudaMemcpyAsync(&maxseg, L.maxseg, 4, cudaMemcpyDeviceToHost, st));
        RS_CHECK(cudaStreamSynchronize(st));
        RS_CHECK(S.keys[0].ensure(K ? K : 1));
        RS_CHECK(S.keys[1].ensure(K ? K : 1));
        RS_CHECK(S.kscan_a.ensure((size_t)K + 1));
        RS_CHECK(S.kscan_b.ensure((size_t)K + 1));
        RS_CHECK(S.gfirst.ensure((size_t)K + 2));
        RS_CHECK(S.rscan.ensure((size_t)R + 1));
        RS_CHECK(S.rflag.ensure(R ? R : 1));
        int kc = 0;
        L.keys = S.keys[kc].p;
        if (K) {
            k_r_emit<<<blocks(K / 6), 256, 0, st>>>(L, K / 6, verts, tris);
            // 2. sort by (segment, value, marker)
            if (maxseg <= kSegCtaMax) {
                const uint32_t nseg = 3 * n;
                k_seg_sort_warp<<<(unsigned)(((size_t)nseg * 32 + 255) / 256), 256, 0, st>>>(L, nseg);
                if (maxseg > kSegWarpMax) k_seg_sort_cta<<<std::min<uint32_t>(nseg, 148u * 8u), 256, 0, st>>>(L, nseg);
            } else {
                uint32_t segbits = 1;
                while (segbits < 30 && (1ull << segbits) < 3ull * n) segbits++;
                const int nbits = 34 + (int)segbits;
                const uint32_t ntiles = (K + kTile - 1) / kTile;
                RS_CHECK(S.hist.ensure(256 * (size_t)ntiles + 1));
                for (int shift = 0; shift < nbits; shift += 8) {
                    k_rs_hist<<<ntiles, kRT, 0, st>>>(S.keys[kc].p, K, shift, ntiles, S.hist.p);
                    RS_CHECK(scan_excl<uint32_t>(S.hist.p, S.hist.p, 256 * ntiles, S.scan_part, st));
                    k_rs_scatter<<<ntiles, kRT, 0, st>>>(S.keys[kc].p, S.keys[kc ^ 1].p, K, shift, ntiles,
                                                         S.hist.p);
                    kc ^= 1;
                }
            }
            L.keys = S.keys[kc].p;
            // 3. sweep
            L.f1 = S.kscan_a.p;
            L.f2 = S.kscan_b.p;
            L.gfirst = S.gfirst.p;
            k_r_heads<<<blocks(K), 256, 0, st>>>(L, K);
            RS_CHECK(scan_excl<u64>(S.kscan_a.p, S.kscan_a.p, K, S.scan_part64, st));
            RS_CHECK(scan_excl<u64>(S.kscan_b.p, S.kscan_b.p, K, S.scan_part64, st));
            k_r_gfirst<<<blocks(K), 256, 0, st>>>(L, K);
            k_r_cost<<<blocks(K), 256, 0, st>>>(L, K);
        }
        // 4. decisions, ranks, leaf offsets
        k_r_decide<<<blocks(n), 256, 0, st>>>(L);
        RS_CHECK(scan_excl<uint32_t>(S.jflag.p, S.jrank.p, n, S.scan_part, st));
        RS_CHECK(scan_excl<uint32_t>(S.leafcnt.p, S.loff.p, n, S.scan_part, st));
        // 5. classification and stable partition
        L.rflag = S.rflag.p;
        L.rscan = S.rscan.p;
        k_r_classify<<<blocks(R), 256, 0, st>>>(L, R, verts, tris);
        RS_CHECK(scan_excl<u64>(L.rflag, S.rscan.p, R, S.scan_part64, st));
        k_r_copy3<<<1, 1, 0, st>>>(S.jrank.p, S.rscan.p, n, R, S.loff.p, n, S.dev_u32.p);
        uint32_t h3[3];
        RS_CHECK(cudaMemcpyAsync(h3, S.dev_u32.p, sizeof h3, cudaMemcpyDeviceToHost, st));
        RS_CHECK(cudaStreamSynchronize(st));
        const uint32_t J = h3[0], R2 = h3[1], Lrefs = h3[2];
        const uint32_t n2 = 2 * J;
        // 6. emit cells, next level
        RS_CHECK(grow_keep(S.out_refs, (size_t)rbase + Lrefs, rbase, st));
        RS_CHECK(S.lo[nxt].ensure(n2));
        RS_CHECK(S.hi[nxt].ensure(n2));
        RS_CHECK(S.surf[nxt].ensure(n2));
        RS_CHECK(S.off[nxt].ensure(n2));
        RS_CHECK(S.cnt[nxt].ensure(n2));
        RS_CHECK(S.ropes[nxt].ensure(6 * (size_t)n2));
        RS_CHECK(S.refs[nxt].ensure(R2));
        RS_CHECK(S.ref_node[nxt].ensure(R2));
        L.nodes = S.nodes.p;
        L.out_refs = S.out_refs.p;
        L.out_ropes = S.out_ropes.p;
        L.out_cbox = S.out_cbox.p;
        L.nlo = S.lo[nxt].p;
        L.nhi = S.hi[nxt].p;
        L.nsurf = S.surf[nxt].p;
        L.noff = S.off[nxt].p;
        L.ncnt = S.cnt[nxt].p;
        L.nropes = S.ropes[nxt].p;
        L.nrefs = S.refs[nxt].p;
        L.nref_node = S.ref_node[nxt].p;
        k_r_nodes<<<blocks(n), 256, 0, st>>>(L);
        k_r_scatter<<<blocks(R), 256, 0, st>>>(L, R);
        RS_CHECK(cudaGetLastError());
        written = L.nbase;
        cbase = L.nbase;
        rbase += Lrefs;
        n = n2;
        R = R2;
    }
    RS_CHECK(cudaStreamSynchronize(st));
    S.nn = written;
    S.nr = rbase;
    S.depth = depth;
    return HK_OK;
}

template struct RBuf<float4>;
template struct RBuf<float>;
template struct RBuf<uint32_t>;
template struct RBuf<u64>;
template struct RBuf<uint2>;

}  // namespace hk
