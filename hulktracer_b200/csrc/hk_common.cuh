// hk_common.cuh -- device data layout and exact-order arithmetic shared by the
// trace, shade and build kernels.
//
// Compiled with -fmad=false: every float expression below rounds after each
// operation, in the order written, so results match the reference's SSE code
// (HulkEngine/public/SPMatrix.hpp) bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hk {

// ---------------------------------------------------------------------------
// Compact KD node: 8 bytes (uint2).
//   junction: x = (pair << 2) | axis (axis 0..2), y = split plane (float bits);
//             children are nodes[pair] (below) and nodes[pair + 1] (above).
//   leaf:     x = (ref_start << 2) | 3, y = ref count. count == 0 marks an empty
//             cell: the reference's child index 0 (KDTreeNode links to the
//             root when a side has no polygons, KDTreeSAH.cpp:494-520).
// nodes[0] is the root, nodes[1] is padding so that every pair starts at an
// even index and both children load as one 16-byte uint4.
// ---------------------------------------------------------------------------
constexpr uint32_t kLeafTag = 3u;

__host__ __device__ inline bool is_leaf(uint2 n) { return (n.x & 3u) == kLeafTag; }

// Triangle record, 64 bytes: the reference PolyToRayCache (SharedStructs.hpp:
// 80-90) with p1 folded in. Normal, e0, e1 have w == 0 and p1 has w == 1 in
// the reference layout, so their w lanes carry the scalars instead:
//   a = {n.x, n.y, n.z, e00}   b = {p1.x, p1.y, p1.z, e01}
//   c = {e0.x, e0.y, e0.z, e11} d = {e1.x, e1.y, e1.z, det}
struct alignas(16) TriRec {
    float4 a, b, c, d;
};

struct Ray4 {
    float4 o, d;
};

// 4-lane dot product in the reference's reduction order (SPMatrix.hpp:284-289):
// (p3 + p1) + (p2 + p0).
__device__ __forceinline__ float dot4(float ax, float ay, float az, float aw, float bx, float by,
                                      float bz, float bw) {
    float p0 = __fmul_rn(ax, bx), p1 = __fmul_rn(ay, by), p2 = __fmul_rn(az, bz), p3 = __fmul_rn(aw, bw);
    return __fadd_rn(__fadd_rn(p3, p1), __fadd_rn(p2, p0));
}

// IEEE normalisation: v * (1 / sqrt(dot4(v, v))), w lane included.
__device__ __forceinline__ float4 normalize4(float4 v) {
    float l2 = dot4(v.x, v.y, v.z, v.w, v.x, v.y, v.z, v.w);
    float s = __fdiv_rn(1.0f, __fsqrt_rn(l2));
    return make_float4(__fmul_rn(v.x, s), __fmul_rn(v.y, s), __fmul_rn(v.z, s), __fmul_rn(v.w, s));
}

// isRayToAbovePlane / isRayToBelowPlane (SharedFunctions.hpp:154-220)
__device__ __forceinline__ bool above_plane(float p0, float d0, float e0, float &t0, float &t1) {
    if (d0 > 0.0f) {
        float ti = __fdiv_rn(__fsub_rn(e0, p0), d0);
        if (ti > t1) return false;
        if (ti > t0) t0 = ti;
        return true;
    } else if (d0 < 0.0f) {
        float ti = __fdiv_rn(__fsub_rn(e0, p0), d0);
        if (ti < t0) return false;
        if (ti < t1) t1 = ti;
        return true;
    }
    return e0 < p0;
}
__device__ __forceinline__ bool below_plane(float p0, float d0, float e0, float &t0, float &t1) {
    if (d0 < 0.0f) {
        float ti = __fdiv_rn(__fsub_rn(e0, p0), d0);
        if (ti > t1) return false;
        if (ti > t0) t0 = ti;
        return true;
    } else if (d0 > 0.0f) {
        float ti = __fdiv_rn(__fsub_rn(e0, p0), d0);
        if (ti < t0) return false;
        if (ti < t1) t1 = ti;
        return true;
    }
    return e0 > p0;
}

// checkRayToBoundingBoxGPU (SharedFunctions.hpp:245-264): all six slab tests run
// (non short-circuit &), t in [0, FLT_MAX].
__device__ __forceinline__ bool ray_box(const float *bmin, const float *bmax, float3 o, float3 d,
                                        float &ts, float &te) {
    float t0 = 0.0f, t1 = 3.402823466e+38f;
    bool r = above_plane(o.x, d.x, bmin[0], t0, t1);
    r &= below_plane(o.x, d.x, bmax[0], t0, t1);
    r &= above_plane(o.y, d.y, bmin[1], t0, t1);
    r &= below_plane(o.y, d.y, bmax[1], t0, t1);
    r &= above_plane(o.z, d.z, bmin[2], t0, t1);
    r &= below_plane(o.z, d.z, bmax[2], t0, t1);
    if (r) {
        te = t1;
        ts = t0;
    }
    return r;
}

// checkRayToPolyACC (SharedFunctions.hpp:105-150) for a ray with o.w == d.w == 0:
//   den = n.d (the w lane adds n.w*d.w = +0), t = (n.(p1-o)) / den (w lane:
//   n.w*(1-0) = +0), hit = o + d t, q = e.(hit-p1) (w lane e.w*(0-1) = -0,
//   which leaves the sum unchanged). Returns t when the triangle is hit and
//   t < best, else +inf. The remaining loads are skipped once the plane test
//   fails or t cannot beat `best` (the reference would discard that hit).
__device__ __forceinline__ float isect_tri(const TriRec *__restrict__ tri, float3 o, float3 d,
                                           float best) {
    // a and b share one 32-byte sector: load both before the first test
    const float4 a = __ldg(&tri->a);
    const float4 b = __ldg(&tri->b);
    float den = __fadd_rn(__fadd_rn(__fmul_rn(a.y, d.y), 0.0f),
                          __fadd_rn(__fmul_rn(a.z, d.z), __fmul_rn(a.x, d.x)));
    if (fabsf(den) < 1.192092896e-07f) return __int_as_float(0x7f800000);
    den = __frcp_rn(den);  // == 1.0f / den, correctly rounded
    float vx = __fsub_rn(b.x, o.x), vy = __fsub_rn(b.y, o.y), vz = __fsub_rn(b.z, o.z);
    float num = __fadd_rn(__fadd_rn(__fmul_rn(a.y, vy), 0.0f),
                          __fadd_rn(__fmul_rn(a.z, vz), __fmul_rn(a.x, vx)));
    float t = __fmul_rn(num, den);
    if (t < 0.0f) return __int_as_float(0x7f800000);
    if (!(t < best)) return __int_as_float(0x7f800000);
    const float4 c = __ldg(&tri->c);
    const float4 e = __ldg(&tri->d);
    float hx = __fsub_rn(__fadd_rn(o.x, __fmul_rn(d.x, t)), b.x);
    float hy = __fsub_rn(__fadd_rn(o.y, __fmul_rn(d.y, t)), b.y);
    float hz = __fsub_rn(__fadd_rn(o.z, __fmul_rn(d.z, t)), b.z);
    float q0 = __fadd_rn(__fmul_rn(c.y, hy), __fadd_rn(__fmul_rn(c.z, hz), __fmul_rn(c.x, hx)));
    float q1 = __fadd_rn(__fmul_rn(e.y, hy), __fadd_rn(__fmul_rn(e.z, hz), __fmul_rn(e.x, hx)));
    float s1 = __fsub_rn(__fmul_rn(c.w, q0), __fmul_rn(b.w, q1));
    float s2 = __fsub_rn(__fmul_rn(a.w, q1), __fmul_rn(b.w, q0));
    if (s1 >= 0.0f && s2 >= 0.0f && __fadd_rn(s1, s2) <= e.w) return t;
    return __int_as_float(0x7f800000);
}

constexpr float kInf = __builtin_huge_valf();

}  // namespace hk
