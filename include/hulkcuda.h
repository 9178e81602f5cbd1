/*
 * hulkcuda.h -- C ABI of the B200 (sm_100a) ray-tracing hot path.
 *
 * Drop-in boundary for HulkEngine's OpenCL render path: the calls below take
 * the place of KDTreeCPU's build / collision API and of GLVisitorGPUTrace's
 * per-frame OpenCL driver. Plain pointers and sizes only; host arrays are
 * copied at call time; the context owns all device memory.
 *
 * Layouts are the reference's (HulkEngine/public/SharedStructs.hpp):
 *   vertex    float[4], w = 1                       (Scene::m_vertices)
 *   triangle  uint32[4] (3 indices + padding)       (TriangleIndices, :37-41)
 *   KD node   uint32[4] (KDTreeNode, :113-137)      flags | {above, below, plane}
 *                                                   or {start, count, leafID}
 *   cache     float[16] (PolyToRayCache, :80-90)    normal4, e0_4, e1_4,
 *                                                   e00, e01, e11, det
 *   ray       float[8]  (Ray, :71-76)               origin4, dir4, w = 0
 *   camera    float[16] (CameraPos, :99-105)        from, vertical, horizontal,
 *                                                   lowerLeft
 *   light     float[8]  (Light, :53-63)             color.xyz + type in .w,
 *                                                   pos-or-dir
 *   box       float[8]  (Box, :65-69)               min4, max4
 *
 * Every call returns hk_status and never aborts the process.
 */
#ifndef HULKCUDA_H
#define HULKCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The first six keep the values of the reference's EHulkResult
 * (HulkEngine/public/hulk_assert.h:42-50). */
typedef enum hk_status {
    HK_OK = 0,
    HK_E_ALLOC = 1,
    HK_E_FILE_OPEN = 2,
    HK_E_FILE_CLOSE = 3,
    HK_E_ILLEGAL_INPUT = 4,
    HK_E_NODE_NOT_FOUND = 5,
    HK_E_CUDA = 16,           /* a CUDA runtime call failed (see hk_last_error) */
    HK_E_DEVICE_TIMEOUT = 17, /* a bounded device-side wait expired */
    HK_E_CAPACITY = 18,       /* a fixed-capacity arena is too small */
    HK_E_BOUNDS = 19,         /* a device-side bound check fired */
    HK_E_STATE = 20           /* call order violated (e.g. trace before a tree exists) */
} hk_status;

/* Traversal variants. FULLSTACK follows KDTreeCPU::searchKDTree
 * (HulkEngine/src/KDTreeCPU.cpp:285-361, GPUTrace.cl:6-90); SHORTSTACK and
 * SMEMSTACK the ring stack of KDTreeCPU::searchKDTreeStackless
 * (KDTreeCPU.cpp:363-447; GPUTrace_shortStack.cl, GPUTrace_LDSshortStack.cl)
 * with the ring in registers or in shared memory; RESTART is kd-restart as in
 * GPUTrace_stackless.cl:53-117 with every leaf resident (no early exit);
 * RESTART_EARLY exits once the closest hit lies before the current segment's
 * end; ROPES follows leaf ropes (no reference counterpart); BRUTE tests every
 * triangle (GPUTrace_bruteforce.cl:30-42). */
typedef enum hk_variant {
    HK_TRACE_FULLSTACK = 0,
    HK_TRACE_SHORTSTACK = 1,
    HK_TRACE_SMEMSTACK = 2,
    HK_TRACE_RESTART = 3,
    HK_TRACE_RESTART_EARLY = 4,
    HK_TRACE_ROPES = 5,
    HK_TRACE_BRUTE = 6
} hk_variant;

typedef enum hk_build_mode {
    HK_BUILD_BINNED = 0,   /* exact binned SAH, every (axis, bin) plane costed */
    HK_BUILD_LEARNED = 1,  /* MLP proposes top-k bins, searched exactly; binned fallback */
    HK_BUILD_SAH_RESORT = 2 /* the reference's --treeType=SAH builder (KDTreeCPU::
                               buildKDTreeSAH / buildNodeSAH, HulkEngine/src/
                               KDTreeSAH.cpp:9-244): every node re-samples every
                               sah_sample-th polygon of its list and sweeps the
                               sorted candidates; leaf at max_depth or at most
                               leaf_size polygons. Ct, Ci, max_depth, leaf_size and
                               sah_sample come from hk_config (the reference's own
                               constants: 1, 5, 20, 9, 5). The tree equals the
                               reference's in the compact layout of hk_tree_import */
} hk_build_mode;

/* Shading semantics for hk_render */
enum {
    HK_SHADE_CPU = 0,          /* GLVisitorCPUTrace::traceScene: shadow rays, misses 0
                                  (shadow rays are traced as occlusion queries that stop
                                  at the first hit closer than the light: the same
                                  shading as the reference's closest-hit test) */
    HK_SHADE_PICTURE = 1,      /* ShadePicture (shadePicture.cl:7-55): no shadow rays */
    HK_SHADE_MIRROR = 2        /* HK_SHADE_CPU plus one mirror bounce (no reference
                                  counterpart): a primary hit on a mirror triangle
                                  (hk_scene_set_mirrors) is replaced by the hit of the
                                  reflected ray r = d - n*(2 d.n) leaving pos + r*0.001,
                                  which is then shaded (shadow rays included); a
                                  reflected ray that misses gives 0 */
};

typedef struct hk_config {
    int device;               /* CUDA device ordinal */
    float traverse_cost;      /* Ct (KDTreeCPU.cpp:17) */
    float intersect_cost;     /* Ci (KDTreeCPU.cpp:18) */
    uint32_t max_depth;       /* c_maxKDTreeDepth (SharedStructs.hpp:16) */
    uint32_t leaf_size;       /* a node with <= leaf_size refs becomes a leaf */
    uint32_t bins;            /* SAH bins per axis (32) */
    uint32_t short_stack;     /* ring depth of SHORTSTACK / SMEMSTACK (4..16) */
    uint32_t block_size;      /* trace kernel block size (multiple of 32, 32..256: the
                                 kernel's launch bound). A trace whose shared memory
                                 (SMEMSTACK: short_stack x block_size x 12 bytes, plus
                                 block_size x 8 bytes for the warp-shared leaf test of
                                 every closest-hit variant but BRUTE) exceeds 48 KB is
                                 refused with HK_E_ILLEGAL_INPUT */
    uint32_t blocks_per_sm;   /* persistent trace grid = SMs * blocks_per_sm */
    uint32_t max_refs;        /* builder reference arena capacity (0 = 16 x tris) */
    uint32_t topk;            /* learned builder: proposed bins refined per node (1..8, 4) */
    float fallback_ratio;     /* learned builder: the binned SAH's plane splits a node
                                 when the proposals' best costs more than ratio x the
                                 binned optimum (default 1: the cheaper of the two;
                                 1.02 lets a proposal up to 2% dearer stand; 0 = the
                                 binned plane always) */
    uint32_t exact_max;       /* builder: nodes with at most this many references take
                                 the exact SAH over their references' bounds (the
                                 reference's candidate set) instead of 32 bins; 0 =
                                 binned everywhere (default), else 32..1024 */
    uint32_t spin_limit;      /* builder: polls before a bounded device-side wait (a
                                 scan look-back, a reference tile waiting for its
                                 plan tile) gives up; the build then stops and
                                 returns HK_E_DEVICE_TIMEOUT (0 = 4M polls) */
    uint32_t max_steps;       /* traversal: node steps per ray before the trace stops
                                 the ray and returns HK_E_BOUNDS (0 = 2^26) */
    uint32_t sah_sample;      /* HK_BUILD_SAH_RESORT: every sah_sample-th polygon of a
                                 node makes candidates (c_reductionFactor,
                                 KDTreeCPU.hpp; 0 = 5) */
    uint32_t subtree_max;     /* HK_BUILD_BINNED / LEARNED: a node of 2..subtree_max
                                 references is not split by the level-synchronous
                                 passes; one warp builds its whole subtree after the
                                 last level (same splits, nodes numbered after the
                                 levels'). 0 = none, at most 32; default 32 */
    uint32_t subtree_depth;   /* only nodes within subtree_depth levels of max_depth are
                                 deferred that way (a deferred subtree is one warp's
                                 serial work, so its depth is bounded); 0 = any depth;
                                 default 8 */
    uint32_t level_streams;   /* HK_BUILD_BINNED without exact_max: 1 = one launch per
                                 level decides the large and the small nodes; 2 = the
                                 large nodes on a second stream beside the small ones
                                 (0 = 1) */
} hk_config;

typedef struct hk_tree_stats {
    uint32_t nodes;           /* compact nodes, including padding/empty cells */
    uint32_t leaves;
    uint32_t refs;            /* leaf references */
    uint32_t depth;
    float build_ms;           /* device time of the last build */
    uint32_t capacity_hit;    /* 1 if a level stopped splitting for lack of arena */
    uint32_t learned_nodes;   /* proposer rows decided by a proposed bin's plane */
    uint32_t fallback_nodes;  /* proposer rows decided by the binned SAH's plane */
} hk_tree_stats;

/* one hit: t (+inf on a miss) and the triangle index (-1 on a miss) */
typedef struct hk_hit {
    float t;
    int32_t tri;
} hk_hit;

typedef struct hk_ctx hk_ctx;

/* defaults: Ct 1, Ci 1.5, depth 24, leaf 4, 32 bins, stack 6, block 128 */
hk_status hk_config_default(hk_config *cfg);

/* Create a context on cfg->device. Replaces GLVisitorGPUTrace::initializeVisitor
 * (HulkEngine/src/GLVisitorGPUTrace.cpp:94-161) minus the GL interop. */
hk_status hk_create(hk_ctx **ctx, const hk_config *cfg);
hk_status hk_destroy(hk_ctx *ctx);
const char *hk_last_error(const hk_ctx *ctx);
/* run subsequent work on this cudaStream_t (NULL = the context's own stream) */
hk_status hk_set_stream(hk_ctx *ctx, void *cuda_stream);
/* Test aid for failure detection: bit 0 makes every later build withhold the
 * done flag of the first plan tile of tree level 1, so the reference tiles
 * that wait for it run out of polls (hk_config.spin_limit) and the build
 * returns HK_E_DEVICE_TIMEOUT without hanging; 0 restores normal builds. */
hk_status hk_set_debug_flags(hk_ctx *ctx, uint32_t flags);
/* The builder layout of the next builds (hk_config subtree_max <= 32,
 * subtree_depth, level_streams 0..2), as hk_autotune_build sets it. */
hk_status hk_set_build_layout(hk_ctx *ctx, uint32_t subtree_max, uint32_t subtree_depth, uint32_t level_streams);
/* The traversal launch configuration of the next traces (hk_config
 * block_size, a multiple of 32 up to 256, and short_stack 1..16), as
 * hk_autotune sets it; batches of the context take it too. */
hk_status hk_set_trace_config(hk_ctx *ctx, uint32_t block_size, uint32_t short_stack);
hk_status hk_synchronize(hk_ctx *ctx);

/* ---- scene (Scene::m_vertices / m_vertexIndices / m_sceneBox) ---- */
/* Copy the triangle soup to the device. Vertices must have w == 1 and every
 * index must be < nv (HK_E_ILLEGAL_INPUT otherwise). The scene box becomes the
 * vertices' bounds unless hk_scene_set_box overrides it. */
hk_status hk_scene_upload(hk_ctx *ctx, const float *verts4, uint32_t nv, const uint32_t *tris4,
                          uint32_t nt);
hk_status hk_scene_set_box(hk_ctx *ctx, const float *box8);
hk_status hk_scene_get_box(hk_ctx *ctx, float *box8);
/* Rigid animation: one part index per vertex; the uploaded vertices are the
 * rest pose. hk_scene_transform then writes M[part] * (x, y, z, 1) into the
 * current vertices on the device, recomputes the scene box and the triangle
 * cache (the per-frame Intersectable::update of HulkEngine/src/
 * Intersectable.cpp:116-141). mats12: nparts x 3x4 row-major. */
hk_status hk_scene_set_parts(hk_ctx *ctx, const uint32_t *part_of_vertex, uint32_t nparts);
hk_status hk_scene_transform(hk_ctx *ctx, const float *mats12);
hk_status hk_scene_get_vertices(hk_ctx *ctx, float *verts4);
/* vertex and triangle counts of the current scene */
hk_status hk_scene_get_counts(hk_ctx *ctx, uint32_t *nv, uint32_t *nt);
/* Per-triangle material flag (1 = mirror) for HK_SHADE_MIRROR. */
hk_status hk_scene_set_mirrors(hk_ctx *ctx, const uint8_t *mirror, uint32_t nt);

/* ---- per-triangle cache (KDTreeCPU::buildPolygonCache, KDTreeCPU.cpp:479-507;
 *      build_cache, GPUTrace_buildCache.cl:5-37) ---- */
/* Compute the cache on the device (normal normalised with IEEE 1/sqrt). */
hk_status hk_precompute(hk_ctx *ctx);
/* Use a cache computed elsewhere (e.g. the reference's, whose normals come
 * from the CPU's rsqrt). Normal / edge w lanes must be 0. */
hk_status hk_cache_import(hk_ctx *ctx, const float *cache16, uint32_t nt);
hk_status hk_cache_export(hk_ctx *ctx, float *cache16);

/* ---- KD tree ---- */
/* KDTreeCPU::buildKDTree (KDTreeCPU.cpp:61-94) on the GPU: exact binned SAH
 * or the learned split proposer. stats may be NULL. */
hk_status hk_build(hk_ctx *ctx, hk_build_mode mode, hk_tree_stats *stats);
/* Import a tree in the reference layout (KDTreeCPU::getNodeArray /
 * getPolygonArray, KDTreeCPU.hpp:62-72). */
hk_status hk_tree_import(hk_ctx *ctx, const uint32_t *nodes4, uint32_t nn, const uint32_t *refs,
                         uint32_t nr);
/* Export the current tree in the reference layout. With nodes4 == NULL only
 * the sizes are returned. */
hk_status hk_tree_export(hk_ctx *ctx, uint32_t *nodes4, uint32_t cap_nodes, uint32_t *refs,
                         uint32_t cap_refs, uint32_t *nn, uint32_t *nr);
/* Export the device's compact layout: 2 x uint32 per node (junction:
 * (pair << 2) | axis, plane bits; leaf: (start << 2) | 3, count). */
hk_status hk_tree_export_compact(hk_ctx *ctx, uint32_t *cnodes2, uint32_t cap_nodes,
                                 uint32_t *refs, uint32_t cap_refs, uint32_t *cnn, uint32_t *nr);
hk_status hk_tree_stats_get(hk_ctx *ctx, hk_tree_stats *stats);
/* Per level of the last HK_BUILD_BINNED / HK_BUILD_LEARNED build: the level's
 * nodes and the references they hold (what the builder reads and writes per
 * level); *nlevels levels, the first min(cap, *nlevels) written. */
hk_status hk_build_level_counts(hk_ctx *ctx, uint32_t *nodes, uint32_t *refs, uint32_t cap, uint32_t *nlevels);
/* The same build's deferred subtrees (nodes of 2..32 references whose
 * subtrees one warp each builds after the levels, numbered after the levels'
 * nodes): their roots and the references the roots hold, and the nodes and
 * leaf references the subtrees added (0, 0 when they did not fit and the
 * roots stayed leaves). Any pointer may be null. */
hk_status hk_build_subtree_counts(hk_ctx *ctx, uint32_t *roots, uint32_t *root_refs, uint32_t *nodes,
                                  uint32_t *leaf_refs);
/* SAH cost of the current tree (no reference counterpart; the tree-quality
 * measure of both builders): sum over junctions of ct * A(n) / A(root) plus
 * over leaves of ci * |refs(n)| * A(n) / A(root), A the full surface area of the
 * node's cell within the scene box, in double precision. An imported reference
 * tree and a GPU-built one are costed by the same function. */
hk_status hk_tree_cost(hk_ctx *ctx, double ct, double ci, double *cost);

/* ---- tracing (KDTreeCPU::checkCollision, KDTreeCPU.cpp:230-253; gpu_trace,
 *      GPUTrace_stackless.cl:122-168) ---- */
/* Host rays in, host hits out (copies included). Ray w lanes must be 0. */
hk_status hk_trace(hk_ctx *ctx, const float *rays8, uint32_t n, hk_variant variant, hk_hit *hits);
/* Device pointers (rays8: n x 8 floats, hits: n x hk_hit), stream-ordered on
 * the context's stream; no host synchronisation. */
hk_status hk_trace_device(hk_ctx *ctx, const float *d_rays8, uint32_t n, hk_variant variant,
                          hk_hit *d_hits);
/* Per-ray counters (node visits, refs read, triangle tests) of the last
 * hk_trace / hk_trace_device call when counting is enabled. */
hk_status hk_set_counting(hk_ctx *ctx, int enable);
hk_status hk_get_counters(hk_ctx *ctx, uint64_t *totals3);

/* ---- primary rays (castRay, GLVisitorCPUTrace.cpp:201-216) ---- */
hk_status hk_camera_rays(hk_ctx *ctx, const float *cam16, uint32_t w, uint32_t h, float *rays8);

/* ---- rendering: trace + shade (GLVisitorGPUTrace::traceScene,
 *      GLVisitorGPUTrace.cpp:296-410, headless) ----
 * rgba: w*h pixels, index y*w + x. HK_SHADE_CPU packs R | G<<8 | B<<16
 * (FrameBuffer::replacePixel, HulkEngine/public/FrameBuffer.hpp:196-217);
 * HK_SHADE_PICTURE writes RGBA8. */
hk_status hk_render(hk_ctx *ctx, const float *cam16, const float *lights8, uint32_t nl, uint32_t w,
                    uint32_t h, hk_variant variant, int shade, uint32_t *rgba);
hk_status hk_render_device(hk_ctx *ctx, const float *cam16, const float *lights8, uint32_t nl,
                           uint32_t w, uint32_t h, hk_variant variant, int shade, uint32_t *d_rgba);
/* Rows y0 .. y1 - 1 of the w x h frame (ray-tile sharding of one frame over
 * GPUs: every rank renders its band of rows of the same frame on its own
 * replica of the scene and tree). d_rgba holds w x (y1 - y0) pixels, index
 * (y - y0) * w + x; every pixel equals the one hk_render_device writes for
 * the whole frame. No reference counterpart (the reference renders on one
 * device). */
hk_status hk_render_rows_device(hk_ctx *ctx, const float *cam16, const float *lights8, uint32_t nl, uint32_t w,
                                uint32_t h, uint32_t y0, uint32_t y1, hk_variant variant, int shade,
                                uint32_t *d_rgba);
/* ShadePicture over caller hits: hit4 = float4(normal.xyz, t) per pixel as the
 * reference's pHitDataArray, t == FLT_MAX for a miss. */
hk_status hk_shade_picture(hk_ctx *ctx, const float *rays8, const float *hit4, uint32_t n,
                           const float *lights8, uint32_t nl, uint32_t *rgba);

/* ---- one animated frame: transform -> build -> trace -> shade ----
 * mats12 may be NULL for a static scene. With use_graph != 0 the frame's
 * device work is captured once into a CUDA graph and replayed (the graph is
 * re-captured when sizes or modes change). d_rgba is a device pointer. */
hk_status hk_frame(hk_ctx *ctx, const float *mats12, const float *cam16, const float *lights8,
                   uint32_t nl, uint32_t w, uint32_t h, hk_build_mode mode, hk_variant variant,
                   int use_graph, uint32_t *d_rgba, hk_tree_stats *stats);
/* shading of hk_frame (HK_SHADE_CPU by default; HK_SHADE_MIRROR needs
 * hk_scene_set_mirrors first) */
hk_status hk_set_frame_shading(hk_ctx *ctx, int shade);

/* Rays of the last hk_render / hk_render_device / hk_frame: primary rays and
 * shadow rays actually traced (synchronises the context's stream). */
hk_status hk_get_ray_counts(hk_ctx *ctx, uint64_t *primary, uint64_t *shadow);
/* Kernel nodes and all nodes of the captured frame graph (0 before capture). */
hk_status hk_frame_graph_info(hk_ctx *ctx, uint32_t *kernel_nodes, uint32_t *all_nodes);

/* ---- OBJ ingest ----
 * The reference's Wavefront OBJ loader (OBJLoader::viParseFile,
 * OBJLoader/OBJLoader.cpp:15-136): vertices "v x y z" (w = 1), triangles "f a b c"
 * (1-based vertex index before the first '/' of each token; only the first
 * three tokens of a face are read), comments, groups and normals skipped.
 * hk_obj_parse fills host arrays (pass null arrays first to get the counts);
 * hk_scene_load_obj parses and uploads the scene (hk_scene_upload). */
hk_status hk_obj_parse(const char *path, float *verts4, uint32_t cap_verts, uint32_t *tris4, uint32_t cap_tris,
                       uint32_t *nv, uint32_t *nt);
hk_status hk_scene_load_obj(hk_ctx *ctx, const char *path, uint32_t *nv, uint32_t *nt);

/* ---- AFF (BART animated scene) ingest ----
 * The reference's AFFParser (BartLoader/src/AFFParser.cpp; the interface is
 * LoaderInterface, HulkEngine/public/LoaderInterface.hpp:18-27, and
 * BartLoader/public/AFFParser.hpp:37-84) with its keyframe animation
 * (BartLoader/src/animation.cpp, kbsplpos.cpp, kbsplrot.cpp, quat.cpp) and
 * per-frame transform (AFFTransformVisitor::preAct, BartLoader/src/
 * AFFTransformVisitor.cpp:25-88). Host-side calls, no GPU needed except for
 * hk_scene_load_aff / hk_scene_animate_aff.
 *
 * Geometry comes from the triangle meshes ("m"), concatenated in file order
 * (includes "i" expanded in place, relative to the top file's directory, and
 * skipped above the "d" detail level, which starts at 0 on every open). Each
 * mesh is one part; its matrix is the product of the enclosing static ("xs":
 * T*R*S) and keyframed ("x" + "k": Kochanek-Bartels splines for translation
 * and scale, squad for rotation, clamped outside the keys) transforms. Lights
 * ("l", "la") keep the reference's Light layout; the viewpoint ("v") gives the
 * field of view and resolution; the "camera" animation places the camera
 * (GLVisitorCPUTrace::updateCamera, HulkEngine/src/GLVisitorCPUTrace.cpp:
 * 105-146). Materials, spheres, cones, polygons and textured triangles are
 * parsed and dropped, as by the reference. Results are bit-identical to the
 * reference's Scene::m_vertices at the same time. A syntax error returns
 * HK_E_ILLEGAL_INPUT, a missing file HK_E_FILE_OPEN; hk_aff_last_error (per
 * thread) names the cause. */
typedef struct hk_aff hk_aff;
typedef struct hk_aff_info {
    uint32_t nv, nt;          /* vertices and triangles of all meshes */
    uint32_t nmeshes;         /* parts: one per mesh */
    uint32_t ndynamic;        /* meshes under at least one keyframed transform */
    uint32_t ntransforms;     /* "xs" and "x" blocks */
    uint32_t nanimations;     /* "k" blocks */
    uint32_t nlights;
    int32_t has_view;         /* a "v" block was read (else the reference's defaults) */
    float from[3], at[3], up[3];
    float fov_deg, hither;    /* fov 45 without "v" */
    int32_t resx, resy;       /* 800 x 600 without "v" */
    int32_t has_anim_params;  /* an "a start end frames" line was read */
    float anim_start, anim_end;
    int32_t anim_frames;
    int32_t has_camera_anim;  /* a "k camera" block exists */
} hk_aff_info;

hk_status hk_aff_open(const char *path, hk_aff **out);
hk_status hk_aff_close(hk_aff *aff);
const char *hk_aff_last_error(void);
hk_status hk_aff_get_info(const hk_aff *aff, hk_aff_info *info);
/* Rest-pose vertices (float4, w = 1), triangles (uint4, global vertex indices)
 * and the mesh index of every vertex; each array may be null. Sizes from
 * hk_aff_get_info: nv x 4 floats, nt x 4 uints, nv uints. */
hk_status hk_aff_geometry(const hk_aff *aff, float *verts4, uint32_t *tris4, uint32_t *part_of_vertex);
/* nmeshes x 3x4 row-major matrices at `time` (the reference's Scene::m_time),
 * in the layout of hk_scene_transform. */
hk_status hk_aff_part_matrices(const hk_aff *aff, float time, float *mats12);
/* nlights x float[8] (Light layout: color.xyz, 1 = point light, position.xyzw). */
hk_status hk_aff_lights(const hk_aff *aff, float *lights8);
/* CameraPos (float[16], the hk_camera_rays layout) at `time`. */
hk_status hk_aff_camera(const hk_aff *aff, float time, float *cam16);
/* Upload the rest pose, one part per mesh, and transform it to `time`. */
hk_status hk_scene_load_aff(hk_ctx *ctx, const hk_aff *aff, float time);
/* Re-transform the loaded AFF scene to `time` (hk_scene_transform). */
hk_status hk_scene_animate_aff(hk_ctx *ctx, const hk_aff *aff, float time);

/* ---- tree interchange file ----
 * The reference's dataset dump (GLVisitorGPUTrace::saveDataSetToFile,
 * HulkEngine/src/GLVisitorGPUTrace.cpp:638-674, read back by
 * GLVisitorGPUTraceSSD::buildTree, GLVisitorGPUTraceSSD.cpp:43-107): a
 * KdFileHeader (9 x uint64 sizes / offsets, GLVisitorGPUTrace.hpp:52-63), the
 * KDTreeNode array, one LeafExtData {indexOffset, vertexOffset, vertxSize,
 * indexSize} per leaf node in node order, then at a 512-byte boundary the
 * per-leaf TriangleIndices (leaf-local vertex indices) and the per-leaf
 * vertices, each leaf's blocks padded to a multiple of 32 entries
 * (buildPerLeafData, GLVisitorGPUTrace.cpp:163-228). After the vertex block
 * this library appends a trailer the reference does not read: "HKLEAFPL",
 * uint64 triangle count, uint64 reference count, the scene box (8 floats),
 * then the leaf polygon list (global triangle ids), so a file written here
 * reloads onto its own scene.
 *
 * hk_tree_save_file writes the current tree and the current vertices.
 * hk_tree_load_file with load_scene = 0 needs the trailer and an uploaded
 * scene of the same triangle count and imports the tree as it was; with
 * load_scene = 1 it uploads the per-leaf triangles as the scene (triangle id =
 * position in the per-leaf lists, leaf by leaf) with a tree over them, as the
 * reference's SSD path renders such a file. */
hk_status hk_tree_save_file(hk_ctx *ctx, const char *path);
hk_status hk_tree_load_file(hk_ctx *ctx, const char *path, int load_scene);

/* ---- learned split proposer (no reference counterpart) ----
 * A 200 -> 256 -> 256 -> 256 -> 96 MLP (ReLU). Features of a node, from its
 * 32-bin binned-SAH histogram: per axis the counts of the references' clipped
 * lower bounds and upper bounds per bin as fractions of the node's references
 * (192), extents over the largest extent (3), depth / max_depth, refs / 1024,
 * 3 zeros. Output: one logit per (axis, bin 0..31) -- the bin expected
 * to hold the node's exact-SAH plane. In HK_BUILD_LEARNED, nodes of up to 32
 * references take the exact SAH in one warp, nodes of 33..1024 references are
 * the proposer's rows and larger nodes take the binned SAH (exact_max is not
 * used). A row gets the full binned SAH (every bin boundary costed exactly)
 * and the network's top-k bins (hk_config.topk); every clipped reference
 * bound inside a proposed bin -- the exact SAH's candidates there -- is
 * costed exactly, and the cheapest of them splits the node unless it costs
 * more than hk_config.fallback_ratio x the binned optimum, which is then the
 * fallback (stats: learned_nodes / fallback_nodes). Inference runs on the
 * tensor cores in BF16 with FP32 accumulation; training uses FP32 master
 * weights and Adam. */
hk_status hk_mlp_init(hk_ctx *ctx, uint64_t seed);
hk_status hk_mlp_save(hk_ctx *ctx, const char *path);
hk_status hk_mlp_load(hk_ctx *ctx, const char *path);
/* flat FP32 parameters: W1 (200x256) b1 W2 (256x256) b2 W3 b3 W4 (256x96) b4,
 * W stored in x out row-major; n = 207712 */
hk_status hk_mlp_get_params(hk_ctx *ctx, float *params, uint32_t n);
hk_status hk_mlp_set_params(hk_ctx *ctx, const float *params, uint32_t n);
/* tensor-core inference: logits[n][96] of X[n][200] (host arrays) */
hk_status hk_mlp_forward(hk_ctx *ctx, const float *X, uint32_t n, float *logits);
/* FP32 training kernels: mean softmax cross-entropy of labels y and its
 * gradient with respect to every parameter (flat layout above) */
hk_status hk_mlp_grad(hk_ctx *ctx, const float *X, const int32_t *y, uint32_t n, float *grads, float *loss);
/* record (features, label) rows during HK_BUILD_BINNED builds with
 * exact_max >= 33: one row per node of 33..exact_max references the exact SAH
 * splits, label = axis * 32 + the bin holding the exact plane; capacity 0
 * stops recording. Restarting recording empties the dataset. */
hk_status hk_mlp_record(hk_ctx *ctx, uint32_t capacity_rows);
hk_status hk_mlp_dataset(hk_ctx *ctx, float *X, int32_t *y, uint32_t cap_rows, uint32_t *rows);
/* train on the recorded rows (shuffled per epoch from seed); epoch_loss
 * (optional, host, epochs) receives the mean loss of every epoch */
hk_status hk_mlp_train(hk_ctx *ctx, uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float *epoch_loss);
/* Verification aid: with the log on, every HK_BUILD_LEARNED build records
 * the bins proposed for each proposer row, 8 int32 per compact node (axis * 32
 * + bin in proposal order, -1 past the last proposal and for nodes that were
 * not proposer rows); hk_get_proposal_log copies the log of the last build
 * (nn = the tree's compact node count; pass bins8 = NULL for it). */
hk_status hk_set_proposal_log(hk_ctx *ctx, int enable);
hk_status hk_get_proposal_log(hk_ctx *ctx, int32_t *bins8, uint32_t cap_nodes, uint32_t *nn);

/* ---- out-of-core leaf geometry ----
 * The reference's leaf residency (GPUTrace_stackless.cl:6-120 with
 * GLVisitorGPUTrace::launchTraceIterations, GLVisitorGPUTrace.cpp:412-502):
 * a kd-restart traversal that tests a leaf only when its triangles are
 * resident in a device pool; otherwise it requests the leaf, keeps its resume
 * point and stops; the leaves requested by a launch are paged in (the oldest
 * resident leaves evicted first, at most half the pool per round except for
 * the round's first leaf) and the traversal relaunched until no ray waits.
 * The leaves' records stay in pinned host memory and the device copies them
 * itself. Hits equal HK_TRACE_RESTART's for any pool size that holds the
 * largest leaf. hk_stream_setup snapshots the current tree and triangle
 * records (call it again after a rebuild or hk_precompute; hk_trace_streamed
 * returns HK_E_STATE until then) and empties the pool; the pool stays warm
 * across hk_trace_streamed calls. A pool smaller than a requested leaf, or
 * rounds that stop making progress, give HK_E_CAPACITY. */
typedef struct hk_stream_stats {
    uint32_t launches;        /* traversal launches (rounds) */
    uint32_t leaves_loaded;   /* page-ins */
    uint32_t leaves_evicted;
    uint32_t resident;        /* leaves resident at the end */
    uint64_t bytes_paged;     /* triangle-record bytes copied from host memory */
    float ms;                 /* device time of the whole call */
} hk_stream_stats;
hk_status hk_stream_setup(hk_ctx *ctx, uint32_t pool_tris);
hk_status hk_trace_streamed(hk_ctx *ctx, const float *rays8, uint32_t n, hk_hit *hits, hk_stream_stats *stats);

/* ---- autotuner (no reference counterpart) ----
 * Times the persistent traversal on n device rays of the current scene for
 * every candidate: traversal layout (ropes: compact nodes + per-node cells and
 * ropes; stack / restart variants: compact nodes only), block size
 * (64, 128, 256) and short-stack depth (4, 6, 8, 12, 16), picks the fastest
 * and writes it into the context's configuration. With cache_path non-NULL
 * the choice is stored per device and scene-size class in that text file and
 * reused on later calls (no timing then). */
typedef struct hk_tune_result {
    int variant;
    uint32_t block_size;
    uint32_t short_stack;
    float best_ms;          /* median launch time of the winner */
    float default_ms;       /* the default configuration (ropes, 128, stack 6) */
    uint32_t tried;         /* candidates timed (0 = taken from the cache) */
} hk_tune_result;
hk_status hk_autotune(hk_ctx *ctx, const float *d_rays8, uint32_t n, const char *cache_path,
                      hk_tune_result *result);
/* The builder's layout for the current scene: times builds of `mode`
 * (HK_BUILD_BINNED or HK_BUILD_LEARNED) with each candidate (subtree_max,
 * subtree_depth): (0, 0) every node level by level; (32, 0), (32, 10),
 * (32, 8), (32, 6) deferred subtrees; each with level_streams 1 and 2; takes
 * the fastest (median of `reps`
 * builds after one warm-up build; 0 = 5) and writes it into the context's
 * configuration. The candidates' trees differ only in node numbering: deferred
 * subtrees pay off on scenes whose small nodes would otherwise add tree
 * levels, and cost a serial chain on scenes whose small nodes sit in deep
 * regions. The current tree afterwards is a valid tree of the last
 * candidate. */
typedef struct hk_build_tune_result {
    uint32_t subtree_max;
    uint32_t subtree_depth;
    uint32_t level_streams;
    float best_ms;          /* median build time of the winner */
    float default_ms;       /* the configuration the context had */
    uint32_t tried;
} hk_build_tune_result;
hk_status hk_autotune_build(hk_ctx *ctx, hk_build_mode mode, uint32_t reps, hk_build_tune_result *result);

/* ---- batching: many scenes, uneven ray batches, one persistent launch ----
 * No reference counterpart (the reference renders one scene per frame). A
 * batch keeps its own copy of each scene's triangle records and GPU-built tree
 * (ropes included). hk_batch_trace_device traces the rays of every scene in a
 * single launch of the persistent traversal kernel: rays of scene s are
 * d_rays8[ray_offsets[s] .. ray_offsets[s+1]) and warps take 32 rays at a time
 * from one counter across all scenes. scene_ms (optional, host, nscenes)
 * receives the time from the launch's start until each scene's last ray
 * finished (device %globaltimer). */
typedef struct hk_batch hk_batch;
hk_status hk_batch_create(hk_ctx *ctx, hk_batch **batch);
/* A batch may outlive its context: hk_destroy frees the device memory of the
 * context's batches, later calls on them return HK_E_STATE, and
 * hk_batch_destroy then frees only the host side. */
hk_status hk_batch_destroy(hk_batch *batch);
/* upload + triangle records + GPU build (the context's settings), then keep a
 * copy; uses the context's scene slot as working space */
hk_status hk_batch_add_scene(hk_batch *batch, const float *verts4, uint32_t nv, const uint32_t *tris4,
                             uint32_t nt, uint32_t *scene_id);
hk_status hk_batch_trace_device(hk_batch *batch, const float *d_rays8, const uint32_t *ray_offsets,
                                uint32_t nscenes, hk_variant variant, hk_hit *d_hits, float *scene_ms);

/* ---- rendering without any device allocation ----
 * No counterpart in the reference: an addition for callers that cannot let
 * the library call cudaMalloc (hosts with their own pooled allocator, code
 * running while a graph capture is open elsewhere, fixed memory budgets).
 * The caller passes the tree, the triangle records and the image in its own
 * device memory:
 *   d_nodes2     compact nodes, 2 x uint32 each (hk_tree_export_compact layout)
 *   d_refs       leaf references (uint32)
 *   d_records16  16 floats per triangle: {n.xyz, e00} {p1.xyz, e01}
 *                {e0.xyz, e11} {e1.xyz, det} (the PolyToRayCache of
 *                hk_cache_export with vertex p1 in the free lanes)
 *   d_rgba       w*h pixels, HK_SHADE_CPU packing
 * and host box8 / cam16 / lights8. Everything else -- rays, hits, shadow rays,
 * counters -- lives in one static device array of HK_NOALLOC_SCRATCH_BYTES
 * that every GPU loading the library holds until the process exits. A call
 * needing more scratch than that (roughly w*h*(40 + 44*point_lights +
 * 4*lights) bytes; 512x512 with one point light fits) returns HK_E_CAPACITY
 * before doing anything. Traversal: FULLSTACK, SHORTSTACK, SMEMSTACK, RESTART,
 * RESTART_EARLY or BRUTE at a fixed block of 128 threads and a ring of 6
 * entries; ROPES needs per-node cells and ropes that this call does not take
 * and is refused with HK_E_ILLEGAL_INPUT. The first call on a device looks up
 * the array's device address and loads every kernel this call can launch
 * (with lazy module loading the driver would otherwise allocate module memory
 * at a variant's first launch); make that first call before any stream
 * capture starts. Calls share the array and keep the last call's contents
 * (counters are cleared per call); calls whose GPU work overlaps race on it.
 * The call synchronises cuda_stream before returning (to read the device
 * error word). */
#define HK_NOALLOC_SCRATCH_BYTES (24u << 20)
hk_status hk_render_noalloc(const uint32_t *d_nodes2, const uint32_t *d_refs, const float *d_records16,
                            uint32_t ntris, const float *box8, const float *cam16, const float *lights8,
                            uint32_t nl, uint32_t w, uint32_t h, hk_variant variant, uint32_t *d_rgba,
                            void *cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* HULKCUDA_H */
