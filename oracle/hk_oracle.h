/*
 * hk_oracle -- CPU restatement of the reference HulkTracer ray-tracing hot
 * path, used ONLY as a parity checker by tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg. The product never links it.
 *
 * Layouts follow the reference (HulkEngine/public/SharedStructs.hpp):
 *   vertex   float[4]  (w = 1)
 *   triangle uint32[4] (TriangleIndices, 4th = padding)
 *   node     uint32[4] (KDTreeNode: m_flags, then leaf{start,count,leafID} or
 *                       junction{above,below,plane-bits})
 *   cache    float[16] (PolyToRayCache: normal4, e0_4, e1_4, e00, e01, e11, det)
 *   ray      float[8]  (origin4, dir4; w = 0)
 *   hit      float[8]  (t, normal.xyz, position.xyz, 0); id int32 (-1 = miss)
 */
#ifndef HK_ORACLE_H
#define HK_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HKO_LEAF 4u
#define HKO_JUNCTION 8u

/* normalisation used for the per-triangle normal, ray directions and the
 * to-light vector: the reference's SSE rsqrt + one Newton step (CPU-model
 * dependent), or IEEE 1/sqrtf (what the CUDA path computes). */
enum { HKO_NORM_SSE = 0, HKO_NORM_IEEE = 1 };

/* traversal variants */
enum {
    HKO_SHORTSTACK = 0,   /* ring stack (depth D), restart at root when empty */
    HKO_FULLSTACK = 1,    /* full stack */
    HKO_RESTART = 2,      /* kd-restart, no early exit (all leaves resident) */
    HKO_RESTART_EARLY = 3,/* kd-restart with exit once hit.t < tmax */
    HKO_ROPES = 4,        /* leaf ropes (needs hko_build_ropes) */
    HKO_BRUTE = 5         /* all triangles, index order */
};

typedef struct {
    const float *verts;      /* [nv][4] */
    const uint32_t *tris;    /* [nt][4] */
    uint32_t nt;
    const float *cache;      /* [nt][16] */
    const uint32_t *nodes;   /* [nn][4] */
    uint32_t nn;
    const uint32_t *refs;    /* leaf polygon list */
    const float *box;        /* scene box min4, max4 */
    /* compact form (ropes variant only): 2 x uint32 per node, see
     * hko_ref_to_compact; per compact node 6 ropes (-x,+x,-y,+y,-z,+z;
     * 0xffffffff = leaves the scene) and a box min4,max4 */
    const uint32_t *cnodes;
    uint32_t cnn;
    const uint32_t *cropes;
    const float *cbox;
} hko_tree;

typedef struct {
    uint64_t nodes;   /* node visits (junction + leaf) */
    uint64_t refs;    /* leaf references read */
    uint64_t tests;   /* triangle tests */
} hko_counters;

typedef struct {
    float ct, ci;          /* traversal / intersection cost */
    uint32_t max_depth;    /* c_maxKDTreeDepth */
    uint32_t leaf_below;   /* leaf if polygon count < leaf_below */
    uint32_t reduction;    /* c_reductionFactor (every k-th triangle sampled) */
} hko_sah_params;

/* intersection form of every traversal: 0 checkRayToPolyACC over the tree's
 * cache (SharedFunctions.hpp:105-150, the CPU path; default), 1
 * checkRayToPoly from the vertices (SharedFunctions.hpp:47-103, the form the
 * reference's OpenCL kernels call) */
void hko_set_isect_form(int form);

/* ---- vector helpers (exposed for tests) ---- */
float hko_dot4(const float *a, const float *b);
void hko_normalize(float *v, int mode);
float hko_box_surface(const float *box);
float hko_box_half_surface(const float *box);
float hko_box_volume(const float *box);

/* ---- per-triangle cache (KDTreeCPU::buildPolygonCache) ---- */
void hko_build_cache(const float *verts, const uint32_t *tris, uint32_t nt, int norm_mode,
                     float *cache_out);

/* ---- rigid per-part transform: v' = M[part] * (x,y,z,1) ---- */
void hko_transform(const float *rest, const uint32_t *part_of_vertex, uint32_t nv,
                   const float *mats12, float *out);
void hko_scene_box(const float *verts, uint32_t nv, float *box_out);

/* ---- primary rays (castRay), pixel (x,y) at index y*w + x ---- */
void hko_camera_rays(const float *cam16, uint32_t w, uint32_t h, int norm_mode, float *rays_out);

/* ---- SAH NlogN build (KDTreeCPU::buildKDTreeSAH_NlogN) ----
 * returns 0 on success; *nodes_out / *refs_out are malloc'ed (free with hko_free) */
int hko_build_sah_nlogn(const float *verts, const uint32_t *tris, uint32_t nt, const float *box,
                        const hko_sah_params *p, uint32_t **nodes_out, uint32_t *nn_out,
                        uint32_t **refs_out, uint32_t *nr_out);
/* KDTreeCPU::buildKDTreeSAH / buildNodeSAH (KDTreeSAH.cpp:9-244, the
 * --treeType=SAH builder): the same outputs; node 1 is the unlinked default
 * node the reference leaves there */
int hko_build_sah_resort(const float *verts, const uint32_t *tris, uint32_t nt, const float *box,
                         const hko_sah_params *p, uint32_t **nodes_out, uint32_t *nn_out,
                         uint32_t **refs_out, uint32_t *nr_out);
void hko_free(void *p);

/* ---- tree SAH cost with full surface areas ----
 * C = sum_inner ct*A(n)/A(root) + sum_leaf ci*|refs|*A(n)/A(root) */
double hko_tree_cost(const uint32_t *nodes, uint32_t nn, const float *box, double ct, double ci);
/* per-node boxes from the root box and the split planes: [nn][8] */
void hko_node_boxes(const uint32_t *nodes, uint32_t nn, const float *box, float *out);
/* Compact node format (2 x uint32 per node), the layout the CUDA kernels use:
 *   junction: w0 = (pair << 2) | axis, w1 = plane bits; children: below = pair,
 *             above = pair + 1 (pairs start at index 2; index 1 is padding)
 *   leaf:     w0 = (ref_start << 2) | 3, w1 = ref count (0 = empty cell, the
 *             reference's child index 0)
 * Returns the number of compact nodes written (capacity 2*nn + 2). */
uint32_t hko_ref_to_compact(const uint32_t *nodes, uint32_t nn, uint32_t *cnodes_out);
/* compact -> reference 16-byte nodes (same indices; leaf IDs in index order) */
void hko_compact_to_ref(const uint32_t *cnodes, uint32_t cnn, uint32_t *nodes_out);
/* ropes + boxes of every compact node */
void hko_build_ropes(const uint32_t *cnodes, uint32_t cnn, const float *box, uint32_t *ropes_out,
                     float *cbox_out);

/* ---- traversal ---- */
int hko_trace_one(const hko_tree *t, int variant, int stack_depth, const float *ray, float *hit,
                  hko_counters *cnt);
void hko_trace(const hko_tree *t, int variant, int stack_depth, const float *rays, uint32_t n,
               float *hits, int32_t *ids, uint64_t *counters /* n x 3 or NULL */, int nthreads);

/* ---- shading ----
 * CPU-tracer semantics (GLVisitorCPUTrace::traceScene + FrameBuffer::replacePixel):
 * ambient 0.1, Lambert, one shadow ray per point light (traced with the given
 * variant), misses = 0. Output R | G<<8 | B<<16. */
void hko_render_cpu(const hko_tree *t, int variant, int stack_depth, const float *rays,
                    uint32_t w, uint32_t h, const float *lights, uint32_t nl, int norm_mode,
                    uint32_t *rgba_out, int nthreads);
/* one mirror bounce before shading (mirror: per-triangle flags) */
void hko_render_mirror(const hko_tree *t, int variant, int stack_depth, const float *rays, uint32_t w,
                       uint32_t h, const float *lights, uint32_t nl, const uint8_t *mirror, int norm_mode,
                       uint32_t *rgba_out, int nthreads);
/* ShadePicture semantics (shadePicture.cl:7-55) from float4(normal, t) hits:
 * colour starts at 0.1 for every pixel, point lights /2, no shadow rays.
 * Output RGBA8 (alpha from colour.w). */
void hko_shade_picture(const float *rays, const float *hit4, uint32_t n, const float *lights,
                       uint32_t nl, uint32_t *rgba_out);

/* ---- binned SAH build (the GPU builder's algorithm, restated on the CPU) ---- */
typedef struct {
    float ct, ci;
    uint32_t max_depth;
    uint32_t leaf_size;     /* leaf when refs <= leaf_size */
    uint32_t bins;          /* 32 */
    uint32_t max_refs;      /* capacity of the reference arena (and of the leaf list) */
    uint32_t max_nodes;     /* capacity of the compact node array */
    uint32_t exact_max;     /* nodes with at most this many refs cost the event planes */
    /* learned mode (exact_max is then 32): nodes of 33..1024 refs take the
     * binned search plus the exact search restricted to their proposed bins */
    uint32_t learned;
    uint32_t topk;           /* proposals per node (list capacity depends on it) */
    float fallback_ratio;
    const int32_t *proposals; /* per compact node, 8 bins (axis * 32 + bin, -1: none) */
    /* T > 0: a decidable node of 2..T refs (T <= 32) is a deferred subtree
     * root: its subtree is built depth first after the levels and numbered
     * after every level's nodes (the CUDA builder's layout, hk_config
     * subtree_max); 0: every node level by level */
    uint32_t defer;
    /* M > 0: only nodes at depth >= max_depth - M are deferred (hk_config
     * subtree_depth); 0: any depth */
    uint32_t defer_margin;
} hko_binned_params;
int hko_build_binned(const float *verts, const uint32_t *tris, uint32_t nt, const float *box,
                     const hko_binned_params *p, uint32_t **nodes_out, uint32_t *nn_out,
                     uint32_t **refs_out, uint32_t *nr_out);

#ifdef __cplusplus
}
#endif
#endif
