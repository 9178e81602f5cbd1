// hk_internal.h -- launch descriptors shared between the host API and the
// kernel translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/hulkcuda.h"

namespace hk {

struct TriRec;

// one scene of a batched launch (device table entry)
struct SceneDesc {
    const uint2 *nodes;
    const uint32_t *refs;
    const TriRec *tris;
    const uint32_t *ropes;
    const float4 *cbox;
    float box[8];
    uint32_t nn;        // compact nodes (ropes legs bound)
    uint32_t ntris;
    uint32_t pad[2];
};

struct TraceLaunch {
    const uint2 *nodes;
    const uint32_t *refs;
    const TriRec *tris;
    const float4 *rays;
    hk_hit *hits;
    uint32_t n;                 // ray count (ignored when n_dev != nullptr)
    const uint32_t *n_dev;      // device-side ray count, or nullptr
    uint32_t ntris;
    const float *box;           // device pointer, 8 floats
    uint32_t *fetch;            // ray-batch counter
    unsigned long long *counters;
    uint32_t *err;
    uint32_t stack_depth;
    uint32_t max_steps;
    int variant;
    bool count;
    bool occlusion;             // shadow rays: origin w = light distance, stop at the first hit closer than it
    uint32_t *leaf_out;         // ropes: per ray, the leaf its traversal ended in (a start hint), or nullptr
    int grid, block;
    // ropes
    const uint32_t *ropes;      // 6 per node
    const float4 *cbox;         // 2 per node (min, max)
    uint32_t rope_nn;           // compact node count
    const uint32_t *rope_nn_dev;
    // batch mode (scenes != nullptr)
    const SceneDesc *scenes;
    const uint32_t *ray_offsets;
    uint32_t nscenes;
    uint32_t *remaining;
    unsigned long long *done_ns;
    unsigned long long *start_ns;
};

// The trace kernel is compiled for at most kTraceMaxBlock threads per block
// (its __launch_bounds__) and launched without opting in to more than the
// default 48 KB of dynamic shared memory.
constexpr uint32_t kTraceMaxBlock = 256;
constexpr size_t kTraceMaxSmem = 48 * 1024;

// Whether an instantiation shares its warp's leaf tests (coop_leaf, one
// 8-byte slot per thread): the closest-hit single-scene kernels of every
// variant but brute force. Counting launches of occlusion rays take the
// closest-hit kernel. The kernel and the launcher both use this.
__host__ __device__ constexpr bool trace_coop_slots(int variant, bool batch, bool any) {
    return variant != HK_TRACE_BRUTE && !batch && !any;
}

// dynamic shared memory of one trace launch: the shared-memory ring of
// SMEMSTACK (12 bytes per thread and ring entry) plus the coop_leaf slots
__host__ __device__ constexpr size_t trace_smem_bytes(int variant, uint32_t block, uint32_t stack_depth, bool batch,
                                                      bool occlusion, bool count) {
    return (variant == HK_TRACE_SMEMSTACK ? (size_t)stack_depth * block * 12 : 0) +
           (trace_coop_slots(variant, batch, occlusion && !count) ? (size_t)block * 8 : 0);
}

cudaError_t launch_trace(const TraceLaunch &L, cudaStream_t s);
// load the closest-hit and occlusion kernels of one variant (single scene, not
// counting) into the current device's context without launching them
cudaError_t preload_trace_kernels(int variant);

// hk_shade.cu
cudaError_t launch_precompute(const float4 *verts, const uint4 *tris, uint32_t nt, TriRec *out,
                              cudaStream_t s);
cudaError_t launch_cache_to_rec(const float *cache16, const float4 *verts, const uint4 *tris, uint32_t nt,
                                TriRec *out, cudaStream_t s);
cudaError_t launch_rec_to_cache(const TriRec *rec, uint32_t nt, float *cache16, cudaStream_t s);
cudaError_t launch_transform(const float4 *rest, const uint32_t *part, uint32_t nv, const float *mats12,
                             float4 *out, uint32_t *box_ord, cudaStream_t s);
cudaError_t launch_box_finish(const uint32_t *box_ord, float *box, cudaStream_t s);
cudaError_t launch_box(const float4 *verts, uint32_t nv, uint32_t *box_ord, float *box, cudaStream_t s);
// rays of rows row0 .. row0 + h - 1 of a w x full_h image (full_h 0: h)
cudaError_t launch_camera_rays(const float *cam16_dev, uint32_t w, uint32_t h, float4 *rays, cudaStream_t s,
                               bool tiled = false, uint32_t row0 = 0, uint32_t full_h = 0);
cudaError_t launch_shadow_rays(const float4 *rays, const hk_hit *hits, const TriRec *tris, uint32_t npix,
                               const float *lights_dev, uint32_t nl, const uint32_t *leaf_hint, float4 *srays,
                               uint32_t *slot, uint32_t *spix, uint32_t *scount, cudaStream_t s);
cudaError_t launch_shade_cpu(const float4 *rays, const hk_hit *hits, const TriRec *tris, uint32_t npix,
                             const float *lights_dev, uint32_t nl, const uint32_t *slot, const hk_hit *shits,
                             uint32_t *rgba, cudaStream_t s, uint32_t w = 0, bool tiled = false);
cudaError_t launch_hit4(const hk_hit *hits, const TriRec *tris, uint32_t n, float4 *hit4, cudaStream_t s);
// load the kernels of the trace + shadow + CPU-shading pipeline's shading side
cudaError_t preload_render_kernels();
cudaError_t launch_shade_picture(const float4 *rays, const float4 *hit4, uint32_t n, const float *lights_dev,
                                 uint32_t nl, uint32_t *rgba, cudaStream_t s, uint32_t w = 0, bool tiled = false);

cudaError_t launch_mirror_rays(const float4 *rays, const hk_hit *hits, const TriRec *tris, const uint8_t *mirror,
                               uint32_t npix, float4 *mrays, uint32_t *mslot, uint32_t *mcount, cudaStream_t s);
cudaError_t launch_mirror_merge(const float4 *rays, const hk_hit *hits, const uint32_t *mslot, const float4 *mrays,
                                const hk_hit *mhits, uint32_t npix, float4 *srays, hk_hit *shits, cudaStream_t s);

}  // namespace hk
