// hk_shade.cu -- per-frame geometry and shading kernels (sm_100a):
// rigid transform + scene box, triangle records, primary rays, shadow rays
// and the two shading semantics of the reference.
#include <cfloat>

#include "hk_common.cuh"
#include "hk_internal.h"

namespace hk {

static inline int blocks_for(uint32_t n, int b) { return (int)((n + b - 1) / b); }

// order-preserving float <-> uint mapping for atomicMin / atomicMax
__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// ---------------------------------------------------------------------------
// triangle record: KDTreeCPU::buildPolygonCache (KDTreeCPU.cpp:479-507) with
// IEEE normalisation. Vertices carry w == 1, so edges and the normal have
// w == 0 and every 4-lane dot has a +0 w term.
// ---------------------------------------------------------------------------
__global__ void k_precompute(const float4 *__restrict__ V, const uint4 *__restrict__ T, uint32_t nt,
                             TriRec *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    uint4 t = T[i];
    float4 p1 = V[t.x], p2 = V[t.y], p3 = V[t.z];
    float a1x = __fsub_rn(p2.x, p1.x), a1y = __fsub_rn(p2.y, p1.y), a1z = __fsub_rn(p2.z, p1.z);
    float a2x = __fsub_rn(p3.x, p2.x), a2y = __fsub_rn(p3.y, p2.y), a2z = __fsub_rn(p3.z, p2.z);
    float a3x = __fsub_rn(p1.x, p3.x), a3y = __fsub_rn(p1.y, p3.y), a3z = __fsub_rn(p1.z, p3.z);
    // cross (SPMatrix.hpp:269-278): (A1B2 - A2B1, A2B0 - A0B2, A0B1 - A1B0)
#define HK_CROSS(Ax, Ay, Az, Bx, By, Bz, ox, oy, oz)                  \
    float ox = __fsub_rn(__fmul_rn(Ay, Bz), __fmul_rn(Az, By));       \
    float oy = __fsub_rn(__fmul_rn(Az, Bx), __fmul_rn(Ax, Bz));       \
    float oz = __fsub_rn(__fmul_rn(Ax, By), __fmul_rn(Ay, Bx));
    HK_CROSS(a1x, a1y, a1z, a2x, a2y, a2z, c1x, c1y, c1z)
    HK_CROSS(a2x, a2y, a2z, a3x, a3y, a3z, c2x, c2y, c2z)
    HK_CROSS(a3x, a3y, a3z, a1x, a1y, a1z, c3x, c3y, c3z)
#undef HK_CROSS
    float4 n = make_float4(__fadd_rn(__fadd_rn(c1x, c2x), c3x), __fadd_rn(__fadd_rn(c1y, c2y), c3y),
                           __fadd_rn(__fadd_rn(c1z, c2z), c3z), 0.0f);
    n = normalize4(n);
    float e0x = a1x, e0y = a1y, e0z = a1z;
    float e1x = __fsub_rn(p3.x, p1.x), e1y = __fsub_rn(p3.y, p1.y), e1z = __fsub_rn(p3.z, p1.z);
    float e00 = dot4(e0x, e0y, e0z, 0.0f, e0x, e0y, e0z, 0.0f);
    float e01 = dot4(e0x, e0y, e0z, 0.0f, e1x, e1y, e1z, 0.0f);
    float e11 = dot4(e1x, e1y, e1z, 0.0f, e1x, e1y, e1z, 0.0f);
    // (e00 * e11) - pow(e01, 2): float product, double subtraction
    float det = __double2float_rn(
        __dsub_rn((double)__fmul_rn(e00, e11), __dmul_rn((double)e01, (double)e01)));
    TriRec r;
    r.a = make_float4(n.x, n.y, n.z, e00);
    r.b = make_float4(p1.x, p1.y, p1.z, e01);
    r.c = make_float4(e0x, e0y, e0z, e11);
    r.d = make_float4(e1x, e1y, e1z, det);
    out[i] = r;
}

cudaError_t launch_precompute(const float4 *verts, const uint4 *tris, uint32_t nt, TriRec *out, cudaStream_t s) {
    if (nt) k_precompute<<<blocks_for(nt, 256), 256, 0, s>>>(verts, tris, nt, out);
    return cudaGetLastError();
}

// imported PolyToRayCache (16 floats) + p1 -> record
__global__ void k_cache_to_rec(const float *__restrict__ C, const float4 *__restrict__ V,
                               const uint4 *__restrict__ T, uint32_t nt, TriRec *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    const float *c = C + 16 * (size_t)i;
    float4 p1 = V[T[i].x];
    TriRec r;
    r.a = make_float4(c[0], c[1], c[2], c[12]);
    r.b = make_float4(p1.x, p1.y, p1.z, c[13]);
    r.c = make_float4(c[4], c[5], c[6], c[14]);
    r.d = make_float4(c[8], c[9], c[10], c[15]);
    out[i] = r;
}

cudaError_t launch_cache_to_rec(const float *cache16, const float4 *verts, const uint4 *tris, uint32_t nt,
                                TriRec *out, cudaStream_t s) {
    if (nt) k_cache_to_rec<<<blocks_for(nt, 256), 256, 0, s>>>(cache16, verts, tris, nt, out);
    return cudaGetLastError();
}

__global__ void k_rec_to_cache(const TriRec *__restrict__ R, uint32_t nt, float *__restrict__ C) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nt) return;
    TriRec r = R[i];
    float *c = C + 16 * (size_t)i;
    // the reference's normal w is 0 * (1/|n|): NaN exactly when the normal is
    c[0] = r.a.x; c[1] = r.a.y; c[2] = r.a.z; c[3] = isnan(r.a.x) ? r.a.x : 0.0f;
    c[4] = r.c.x; c[5] = r.c.y; c[6] = r.c.z; c[7] = 0.0f;
    c[8] = r.d.x; c[9] = r.d.y; c[10] = r.d.z; c[11] = 0.0f;
    c[12] = r.a.w; c[13] = r.b.w; c[14] = r.c.w; c[15] = r.d.w;
}

cudaError_t launch_rec_to_cache(const TriRec *rec, uint32_t nt, float *cache16, cudaStream_t s) {
    if (nt) k_rec_to_cache<<<blocks_for(nt, 256), 256, 0, s>>>(rec, nt, cache16);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// rigid transform v' = M[part] (x, y, z, 1) fused with the scene-box
// reduction (BoundingBoxVisitor, HulkEngine/src/BoundingBoxVisitor.cpp:72-80)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void box_accumulate(float x, float y, float z, uint32_t *box_ord) {
    // warp-reduce before the atomics
    uint32_t lo[3] = {f2ord(x), f2ord(y), f2ord(z)}, hi[3] = {lo[0], lo[1], lo[2]};
    for (int off = 16; off; off >>= 1)
        for (int k = 0; k < 3; k++) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = max(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
    if ((threadIdx.x & 31u) == 0)
        for (int k = 0; k < 3; k++) {
            atomicMin(&box_ord[k], lo[k]);
            atomicMax(&box_ord[4 + k], hi[k]);
        }
}

__device__ __forceinline__ float3 xform(const float *m, float4 v) {
    float x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], v.x), __fmul_rn(m[1], v.y)), __fmul_rn(m[2], v.z)), m[3]);
    float y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], v.x), __fmul_rn(m[5], v.y)), __fmul_rn(m[6], v.z)), m[7]);
    float z = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[8], v.x), __fmul_rn(m[9], v.y)), __fmul_rn(m[10], v.z)), m[11]);
    return make_float3(x, y, z);
}

__global__ void k_transform(const float4 *__restrict__ R, const uint32_t *__restrict__ P, uint32_t nv,
                            const float *__restrict__ M, float4 *__restrict__ out, uint32_t *box_ord) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // lanes past the end repeat the block's first vertex (a no-op for min/max)
    uint32_t j = i < nv ? i : blockIdx.x * blockDim.x;
    float3 p = xform(M + 12 * (size_t)P[j], R[j]);
    if (i < nv) out[i] = make_float4(p.x, p.y, p.z, 1.0f);
    box_accumulate(p.x, p.y, p.z, box_ord);
}

__global__ void k_box(const float4 *__restrict__ V, uint32_t nv, uint32_t *box_ord) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float4 v = V[i < nv ? i : blockIdx.x * blockDim.x];
    box_accumulate(v.x, v.y, v.z, box_ord);
}

__global__ void k_box_init(uint32_t *box_ord) {
    int k = threadIdx.x;
    if (k < 8) box_ord[k] = (k < 4) ? 0xffffffffu : 0u;
}

__global__ void k_box_finish(const uint32_t *box_ord, float *box) {
    int k = threadIdx.x;
    if (k < 3) {
        box[k] = ord2f(box_ord[k]);
        box[4 + k] = ord2f(box_ord[4 + k]);
    } else if (k == 3 || k == 7) {
        box[k] = 1.0f;
    }
}

cudaError_t launch_transform(const float4 *rest, const uint32_t *part, uint32_t nv, const float *mats12,
                             float4 *out, uint32_t *box_ord, cudaStream_t s) {
    k_box_init<<<1, 32, 0, s>>>(box_ord);
    if (nv) k_transform<<<blocks_for(nv, 256), 256, 0, s>>>(rest, part, nv, mats12, out, box_ord);
    return cudaGetLastError();
}

cudaError_t launch_box_finish(const uint32_t *box_ord, float *box, cudaStream_t s) {
    k_box_finish<<<1, 32, 0, s>>>(box_ord, box);
    return cudaGetLastError();
}

cudaError_t launch_box(const float4 *verts, uint32_t nv, uint32_t *box_ord, float *box, cudaStream_t s) {
    k_box_init<<<1, 32, 0, s>>>(box_ord);
    if (nv) k_box<<<blocks_for(nv, 256), 256, 0, s>>>(verts, nv, box_ord);
    k_box_finish<<<1, 32, 0, s>>>(box_ord, box);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// primary rays: castRay (GLVisitorCPUTrace.cpp:201-216) with IEEE normalise:
// dir = ((lowerLeft + vertical * x/W) + horizontal * y/H) - from
// ---------------------------------------------------------------------------
// Ray order: row-major, or 8x4-pixel tiles (one warp batch per tile, for
// coherent traversal) when the image divides into tiles.
__device__ __forceinline__ uint32_t pixel_of(uint32_t i, uint32_t w, bool tiled) {
    if (!tiled) return i;
    uint32_t tile = i >> 5, j = i & 31u, tiles_x = w >> 3;
    uint32_t x = (tile % tiles_x) * 8u + (j & 7u), y = (tile / tiles_x) * 4u + (j >> 3);
    return y * w + x;
}

// The rays of rows row0 .. row0 + h - 1 of a w x full_h image (the whole
// image when row0 = 0 and full_h = h); ray i belongs to pixel pixel_of(i) of
// that band.
__global__ void k_camera_rays(const float *__restrict__ cam, uint32_t w, uint32_t h, float4 *__restrict__ rays,
                              bool tiled, uint32_t row0, uint32_t full_h) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    uint32_t pix = pixel_of(i, w, tiled);
    uint32_t x = pix % w, y = pix / w + row0;
    float u = __fdiv_rn((float)x, (float)w), v = __fdiv_rn((float)y, (float)full_h);
    float4 from = make_float4(cam[0], cam[1], cam[2], cam[3]);
    float d[4];
    for (int k = 0; k < 4; k++) {
        float b = __fadd_rn(cam[12 + k], __fmul_rn(cam[4 + k], u));
        float c = __fadd_rn(b, __fmul_rn(cam[8 + k], v));
        d[k] = __fsub_rn(c, cam[k]);
    }
    float4 dir = normalize4(make_float4(d[0], d[1], d[2], d[3]));
    rays[2 * (size_t)i] = from;
    rays[2 * (size_t)i + 1] = dir;
}

cudaError_t launch_camera_rays(const float *cam16_dev, uint32_t w, uint32_t h, float4 *rays, cudaStream_t s,
                               bool tiled, uint32_t row0, uint32_t full_h) {
    uint32_t n = w * h;
    if (n) k_camera_rays<<<blocks_for(n, 256), 256, 0, s>>>(cam16_dev, w, h, rays, tiled, row0, full_h ? full_h : h);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// shadow rays and CPU-tracer shading (GLVisitorCPUTrace.cpp:165-194)
// ---------------------------------------------------------------------------
struct PointLightSetup {
    float4 tl;      // normalised direction to the light (w = 0)
    float dist;     // distance to the light
    float4 org;     // shadow-ray origin pos + tl * 0.001
};

__device__ __forceinline__ PointLightSetup point_light(const float *L, float4 pos) {
    PointLightSetup r;
    float4 tl = make_float4(__fsub_rn(L[4], pos.x), __fsub_rn(L[5], pos.y), __fsub_rn(L[6], pos.z), 0.0f);
    r.dist = __fsqrt_rn(dot4(tl.x, tl.y, tl.z, tl.w, tl.x, tl.y, tl.z, tl.w));
    tl = normalize4(tl);
    r.tl = tl;
    r.org = make_float4(__fadd_rn(pos.x, __fmul_rn(tl.x, 0.001f)), __fadd_rn(pos.y, __fmul_rn(tl.y, 0.001f)),
                        __fadd_rn(pos.z, __fmul_rn(tl.z, 0.001f)), __fadd_rn(pos.w, __fmul_rn(tl.w, 0.001f)));
    return r;
}

__device__ __forceinline__ float4 hit_pos(float4 o, float4 d, float t) {
    return make_float4(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)),
                       __fadd_rn(o.z, __fmul_rn(d.z, t)), __fadd_rn(o.w, __fmul_rn(d.w, t)));
}

// Writes one shadow ray per (hit pixel, point light) into a compacted list
// (warp-aggregated atomics); slot[l * npix + p] = list index or 0xffffffff.
// leaf_hint (optional): per pixel, the leaf the pixel's ropes traversal ended
// in, passed in the direction's w lane as where the shadow ray may start.
__global__ void k_shadow_rays(const float4 *__restrict__ rays, const hk_hit *__restrict__ hits,
                              uint32_t npix, const float *__restrict__ lights, uint32_t nl,
                              const uint32_t *__restrict__ leaf_hint, float4 *__restrict__ srays,
                              uint32_t *__restrict__ slot, uint32_t *__restrict__ spix, uint32_t *scount) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    hk_hit h = p < npix ? hits[p] : hk_hit{kInf, -1};
    float4 o = make_float4(0, 0, 0, 0), d = o;
    if (p < npix) {
        o = rays[2 * (size_t)p];
        d = rays[2 * (size_t)p + 1];
    }
    float4 pos = hit_pos(o, d, h.t);
    pos.w = 0.0f;
    const float hint = (leaf_hint && p < npix) ? __uint_as_float(leaf_hint[p]) : 0.0f;
    for (uint32_t l = 0; l < nl; l++) {
        const float *L = lights + 8 * l;
        bool want = (p < npix) && h.tri >= 0 && L[3] == 1.0f;
        uint32_t m = __ballot_sync(0xffffffffu, want);
        uint32_t base = 0;
        if ((threadIdx.x & 31u) == 0 && m) base = atomicAdd(scount, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (p < npix) slot[(size_t)l * npix + p] = 0xffffffffu;
        if (want) {
            uint32_t k = base + __popc(m & ((1u << (threadIdx.x & 31u)) - 1u));
            PointLightSetup s = point_light(L, pos);
            // the origin's w lane (0 here) carries the light distance to the
            // occlusion trace, which stops at the first hit closer than it
            float4 org = s.org;
            org.w = s.dist;
            srays[2 * (size_t)k] = org;
            float4 dir = s.tl;
            dir.w = hint;
            srays[2 * (size_t)k + 1] = dir;
            spix[k] = p;
            slot[(size_t)l * npix + p] = k;
        }
    }
}

cudaError_t launch_shadow_rays(const float4 *rays, const hk_hit *hits, const TriRec *, uint32_t npix,
                               const float *lights_dev, uint32_t nl, const uint32_t *leaf_hint, float4 *srays,
                               uint32_t *slot, uint32_t *spix, uint32_t *scount, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(scount, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (npix)
        k_shadow_rays<<<blocks_for(npix, 256), 256, 0, s>>>(rays, hits, npix, lights_dev, nl, leaf_hint, srays, slot,
                                                            spix, scount);
    return cudaGetLastError();
}

// FrameBuffer::replacePixel (FrameBuffer.hpp:196-217)
__device__ __forceinline__ uint32_t pack_pixel(float4 c) {
    float v[3] = {c.x, c.y, c.z};
    uint32_t out = 0;
    for (int k = 0; k < 3; k++) {
        float x = (1.0f < v[k]) ? 1.0f : v[k];
        x = __fmul_rn(x, 255.0f);
        out |= (uint32_t)__float2int_rn(x) << (8 * k);
    }
    return out;
}

__global__ void k_shade_cpu(const float4 *__restrict__ rays, const hk_hit *__restrict__ hits,
                            const TriRec *__restrict__ tris, uint32_t npix, const float *__restrict__ lights,
                            uint32_t nl, const uint32_t *__restrict__ slot, const hk_hit *__restrict__ shits,
                            uint32_t *__restrict__ rgba, uint32_t w, bool tiled) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    hk_hit h = hits[p];
    uint32_t pix = pixel_of(p, w, tiled);
    if (h.tri < 0) {
        rgba[pix] = 0u;
        return;
    }
    float4 o = rays[2 * (size_t)p], d = rays[2 * (size_t)p + 1];
    float4 na = tris[h.tri].a;
    float4 pos = hit_pos(o, d, h.t);
    pos.w = 0.0f;
    float4 col = make_float4(0.1f, 0.1f, 0.1f, 1.0f);
    for (uint32_t l = 0; l < nl; l++) {
        const float *L = lights + 8 * l;
        float I = 0.0f;
        bool any = false;
        if (L[3] == 0.0f) {
            I = dot4(na.x, na.y, na.z, 0.0f, L[4], L[5], L[6], L[7]);
            any = true;
        }
        if (L[3] == 1.0f) {
            PointLightSetup s = point_light(L, pos);
            I = dot4(na.x, na.y, na.z, 0.0f, s.tl.x, s.tl.y, s.tl.z, s.tl.w);
            uint32_t k = slot[(size_t)l * npix + p];
            hk_hit sh = shits[k];
            if (sh.tri >= 0 && s.dist > sh.t) I = __fmul_rn(I, 0.5f);
            any = true;
        }
        if (any) {
            float sc = I > 0.0f ? I : 0.0f;
            col.x = __fadd_rn(col.x, __fmul_rn(L[0], sc));
            col.y = __fadd_rn(col.y, __fmul_rn(L[1], sc));
            col.z = __fadd_rn(col.z, __fmul_rn(L[2], sc));
            col.w = __fadd_rn(col.w, __fmul_rn(L[3], sc));
        }
    }
    rgba[pix] = pack_pixel(col);
}

cudaError_t launch_shade_cpu(const float4 *rays, const hk_hit *hits, const TriRec *tris, uint32_t npix,
                             const float *lights_dev, uint32_t nl, const uint32_t *slot, const hk_hit *shits,
                             uint32_t *rgba, cudaStream_t s, uint32_t w, bool tiled) {
    if (npix)
        k_shade_cpu<<<blocks_for(npix, 256), 256, 0, s>>>(rays, hits, tris, npix, lights_dev, nl, slot, shits, rgba,
                                                         w, tiled);
    return cudaGetLastError();
}

// loads the camera-ray, shadow-ray and CPU-shading kernels into the current
// device's context (the driver loads a kernel lazily, allocating module
// memory, at its first launch otherwise)
cudaError_t preload_render_kernels() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_camera_rays);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_shadow_rays);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_shade_cpu);
    return e;
}

// ---------------------------------------------------------------------------
// ShadePicture (shadePicture.cl:7-55): float4(normal, t) per pixel, misses
// t = FLT_MAX (SetInitialValues, GPU_setValues.cl:4-11)
// ---------------------------------------------------------------------------
__global__ void k_hit4(const hk_hit *__restrict__ hits, const TriRec *__restrict__ tris, uint32_t n,
                       float4 *__restrict__ out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    hk_hit h = hits[i];
    if (h.tri < 0) {
        out[i] = make_float4(0.0f, 0.0f, 0.0f, FLT_MAX);
    } else {
        float4 a = tris[h.tri].a;
        out[i] = make_float4(a.x, a.y, a.z, h.t);
    }
}

cudaError_t launch_hit4(const hk_hit *hits, const TriRec *tris, uint32_t n, float4 *hit4, cudaStream_t s) {
    if (n) k_hit4<<<blocks_for(n, 256), 256, 0, s>>>(hits, tris, n, hit4);
    return cudaGetLastError();
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

__device__ __forceinline__ uint32_t unorm8(float x) {
    x = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
    return (uint32_t)__float2int_rn(__fmul_rn(x, 255.0f));
}

__global__ void k_shade_picture(const float4 *__restrict__ rays, const float4 *__restrict__ hit4, uint32_t n,
                                const float *__restrict__ lights, uint32_t nl, uint32_t *__restrict__ rgba,
                                uint32_t w, bool tiled) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 col = make_float4(0.1f, 0.1f, 0.1f, 0.0f);
    float4 h = hit4[i];
    if (h.w != FLT_MAX && h.w > 0.0f) {
        float4 o = rays[2 * (size_t)i], d = rays[2 * (size_t)i + 1];
        float px = __fadd_rn(o.x, __fmul_rn(h.w, d.x)), py = __fadd_rn(o.y, __fmul_rn(h.w, d.y)),
              pz = __fadd_rn(o.z, __fmul_rn(h.w, d.z));
        for (uint32_t l = 0; l < nl; l++) {
            const float *L = lights + 8 * l;
            float I = 0.0f;
            if (L[3] == 1.0f) {
                float tx = __fsub_rn(L[4], px), ty = __fsub_rn(L[5], py), tz = __fsub_rn(L[6], pz);
                float inv = __fdiv_rn(1.0f, __fsqrt_rn(dot3(tx, ty, tz, tx, ty, tz)));
                tx = __fmul_rn(tx, inv);
                ty = __fmul_rn(ty, inv);
                tz = __fmul_rn(tz, inv);
                I = __fdiv_rn(dot3(h.x, h.y, h.z, tx, ty, tz), 2.0f);
            }
            if (L[3] == 0.0f) I = dot3(h.x, h.y, h.z, L[4], L[5], L[6]);
            float sc = I > 0.0f ? I : 0.0f;
            col.x = __fadd_rn(col.x, __fmul_rn(L[0], sc));
            col.y = __fadd_rn(col.y, __fmul_rn(L[1], sc));
            col.z = __fadd_rn(col.z, __fmul_rn(L[2], sc));
            col.w = __fadd_rn(col.w, __fmul_rn(L[3], sc));
        }
    }
    rgba[pixel_of(i, w, tiled)] = unorm8(col.x) | (unorm8(col.y) << 8) | (unorm8(col.z) << 16) | (unorm8(col.w) << 24);
}

cudaError_t launch_shade_picture(const float4 *rays, const float4 *hit4, uint32_t n, const float *lights_dev,
                                 uint32_t nl, uint32_t *rgba, cudaStream_t s, uint32_t w, bool tiled) {
    if (n) k_shade_picture<<<blocks_for(n, 256), 256, 0, s>>>(rays, hit4, n, lights_dev, nl, rgba, w ? w : n, tiled);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// one mirror bounce (no reference counterpart): reflected rays of primary
// hits on mirror triangles, then the per-pixel shading ray / hit
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reflect_ray(float4 o, float4 d, float t, float4 na, float4 &ro, float4 &rd) {
    float4 pos = hit_pos(o, d, t);
    pos.w = 0.0f;
    float dn = dot4(d.x, d.y, d.z, d.w, na.x, na.y, na.z, 0.0f);
    float k = __fmul_rn(2.0f, dn);
    rd = make_float4(__fsub_rn(d.x, __fmul_rn(na.x, k)), __fsub_rn(d.y, __fmul_rn(na.y, k)),
                     __fsub_rn(d.z, __fmul_rn(na.z, k)), 0.0f);
    ro = make_float4(__fadd_rn(pos.x, __fmul_rn(rd.x, 0.001f)), __fadd_rn(pos.y, __fmul_rn(rd.y, 0.001f)),
                     __fadd_rn(pos.z, __fmul_rn(rd.z, 0.001f)), 0.0f);
}

__global__ void k_mirror_rays(const float4 *__restrict__ rays, const hk_hit *__restrict__ hits,
                              const TriRec *__restrict__ tris, const uint8_t *__restrict__ mirror, uint32_t npix,
                              float4 *__restrict__ mrays, uint32_t *__restrict__ mslot, uint32_t *mcount) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    hk_hit h = p < npix ? hits[p] : hk_hit{kInf, -1};
    bool want = p < npix && h.tri >= 0 && mirror[h.tri];
    uint32_t m = __ballot_sync(0xffffffffu, want);
    uint32_t base = 0;
    if ((threadIdx.x & 31u) == 0 && m) base = atomicAdd(mcount, (uint32_t)__popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (p >= npix) return;
    mslot[p] = 0xffffffffu;
    if (!want) return;
    uint32_t k = base + __popc(m & ((1u << (threadIdx.x & 31u)) - 1u));
    float4 ro, rd;
    reflect_ray(rays[2 * (size_t)p], rays[2 * (size_t)p + 1], h.t, tris[h.tri].a, ro, rd);
    mrays[2 * (size_t)k] = ro;
    mrays[2 * (size_t)k + 1] = rd;
    mslot[p] = k;
}

// shading ray / hit per pixel: the reflected one on mirrors, else the primary
__global__ void k_mirror_merge(const float4 *__restrict__ rays, const hk_hit *__restrict__ hits,
                               const uint32_t *__restrict__ mslot, const float4 *__restrict__ mrays,
                               const hk_hit *__restrict__ mhits, uint32_t npix, float4 *__restrict__ srays,
                               hk_hit *__restrict__ shits) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    uint32_t k = mslot[p];
    if (k == 0xffffffffu) {
        srays[2 * (size_t)p] = rays[2 * (size_t)p];
        srays[2 * (size_t)p + 1] = rays[2 * (size_t)p + 1];
        shits[p] = hits[p];
    } else {
        srays[2 * (size_t)p] = mrays[2 * (size_t)k];
        srays[2 * (size_t)p + 1] = mrays[2 * (size_t)k + 1];
        shits[p] = mhits[k];
    }
}

cudaError_t launch_mirror_rays(const float4 *rays, const hk_hit *hits, const TriRec *tris, const uint8_t *mirror,
                               uint32_t npix, float4 *mrays, uint32_t *mslot, uint32_t *mcount, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(mcount, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (npix) k_mirror_rays<<<blocks_for(npix, 256), 256, 0, s>>>(rays, hits, tris, mirror, npix, mrays, mslot, mcount);
    return cudaGetLastError();
}

cudaError_t launch_mirror_merge(const float4 *rays, const hk_hit *hits, const uint32_t *mslot, const float4 *mrays,
                                const hk_hit *mhits, uint32_t npix, float4 *srays, hk_hit *shits, cudaStream_t s) {
    if (npix) k_mirror_merge<<<blocks_for(npix, 256), 256, 0, s>>>(rays, hits, mslot, mrays, mhits, npix, srays, shits);
    return cudaGetLastError();
}

}  // namespace hk
