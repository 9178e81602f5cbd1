// hk_api.cu -- the extern "C" boundary (include/hulkcuda.h): context,
// device arena, input validation, tree import/export and the per-call
// drivers around the kernels.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hk_build.h"
#include "hk_resort.h"
#include "hk_stream.h"
#include "hk_common.cuh"
#include "hk_internal.h"
#include "hk_mlp.h"
#include <random>
#include <unordered_map>

using namespace hk;

namespace {

template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n) {
        if (n <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        cudaError_t e = cudaMalloc((void **)&p, bytes);
        if (e == cudaSuccess) cap = std::max<size_t>(n, 1);
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

}  // namespace

static void batch_detach(hk_batch *b);

struct hk_ctx {
    hk_config cfg;
    int device = 0;
    int sm_count = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    // scene
    uint32_t nv = 0, nt = 0, nparts = 0;
    DevBuf<float4> verts, rest;
    DevBuf<uint4> tris;
    DevBuf<uint32_t> part;
    DevBuf<float> mats;
    DevBuf<float> box;          // 8 floats
    DevBuf<uint32_t> box_ord;   // 8 words
    float hbox[8] = {0};
    bool box_user = false;
    // triangle records
    DevBuf<TriRec> rec;
    DevBuf<float> cache_tmp;
    bool rec_valid = false;
    // tree (compact)
    DevBuf<uint2> nodes;
    DevBuf<uint32_t> refs;
    uint32_t nn = 0, nr = 0;
    bool tree_valid = false;
    bool tree_built = false;             // current tree = the GPU builder's output
    bool tree_on_device_counts = false;  // its sizes still live in device memory
    hk_tree_stats stats{};
    BuildState build;
    ResortState resort;   // HK_BUILD_SAH_RESORT
    StreamState ooc;      // out-of-core leaf geometry
    uint64_t tree_epoch = 0, rec_epoch = 0;   // bumped whenever the tree / the records change
    // ropes of an imported tree (computed on the host when first needed)
    std::vector<uint2> host_nodes;
    DevBuf<uint32_t> imp_ropes;
    DevBuf<float4> imp_cbox;
    bool imp_ropes_valid = false;
    // trace scratch
    DevBuf<uint32_t> fetch;
    DevBuf<unsigned long long> counters;
    DevBuf<uint32_t> errw;
    bool counting = false;
    DevBuf<float4> rays;
    DevBuf<hk_hit> hits;
    DevBuf<float> cam, lights;
    // shadow rays
    DevBuf<float4> srays;
    DevBuf<hk_hit> shits;
    DevBuf<uint32_t> slot, spix, scount;
    DevBuf<uint32_t> hleaf;     // per pixel: the leaf its primary ropes traversal ended in
    DevBuf<float4> hit4;
    DevBuf<uint32_t> rgba;
    // mirror bounce
    DevBuf<uint8_t> mirror;
    bool has_mirrors = false;
    DevBuf<float4> mrays, prays;
    DevBuf<hk_hit> mhits, phits;
    DevBuf<uint32_t> mslot, mcount;
    // frame graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t graph_key = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t last_primary = 0;
    int last_shade = HK_SHADE_CPU;
    int frame_shade = HK_SHADE_CPU;   // shading of hk_frame
    // learned split proposer
    LearnBuffers learn;
    DevBuf<float> mlp_params, mlp_grads, mlp_m, mlp_v;
    DevBuf<uint32_t> mlp_w1p, mlp_w2p, mlp_w3p, mlp_w4p;
    DevBuf<unsigned char> mlp_tcw;   // tcgen05 weight chunks
    int mlp_step = 0;
    DevBuf<float> rec_X;
    DevBuf<int32_t> rec_y;
    DevBuf<uint32_t> rec_rows;
    uint32_t rec_cap = 0;
    bool recording = false;
    bool prop_log = false;
    std::vector<hk_batch *> batches;     // live batches (detached when the context goes first)
    uint32_t debug_flags = 0;
};

// current tree arrays (imported or built)
static const uint2 *tree_nodes(hk_ctx *c) { return c->tree_built ? c->build.out_nodes : c->nodes.p; }
static const uint32_t *tree_refs(hk_ctx *c) { return c->tree_built ? c->build.out_refs : c->refs.p; }

#define HK_CUDA(ctx, call)                                                       \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess) {                                                 \
            (ctx)->err = std::string(#call) + ": " + cudaGetErrorString(e_);     \
            return HK_E_CUDA;                                                    \
        }                                                                        \
    } while (0)

static hk_status fail(hk_ctx *c, hk_status s, const char *msg) {
    if (c) c->err = msg;
    return s;
}

static hk_status check_err_word(hk_ctx *c) {
    uint32_t w = 0;
    HK_CUDA(c, cudaMemcpyAsync(&w, c->errw.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    if (w) {
        HK_CUDA(c, cudaMemsetAsync(c->errw.p, 0, 4, c->stream));
        if (w & 2u) return fail(c, HK_E_CAPACITY, "device: arena capacity exceeded");
        return fail(c, HK_E_BOUNDS, "device: traversal step bound exceeded (malformed tree?)");
    }
    return HK_OK;
}

extern "C" {

hk_status hk_config_default(hk_config *cfg) {
    if (!cfg) return HK_E_ILLEGAL_INPUT;
    memset(cfg, 0, sizeof(*cfg));
    cfg->device = 0;
    cfg->traverse_cost = 1.0f;
    cfg->intersect_cost = 1.5f;
    cfg->max_depth = 24;
    cfg->leaf_size = 4;
    cfg->bins = 32;
    cfg->short_stack = 6;
    cfg->block_size = 128;
    cfg->blocks_per_sm = 0;
    cfg->max_refs = 0;
    cfg->topk = 4;
    cfg->fallback_ratio = 1.0f;
    cfg->exact_max = 0;
    cfg->sah_sample = 5;
    cfg->subtree_max = 32;
    cfg->subtree_depth = 8;
    cfg->level_streams = 1;
    return HK_OK;
}

static hk_status validate_config(const hk_config *c) {
    if (c->short_stack < 1 || c->short_stack > 16) return HK_E_ILLEGAL_INPUT;
    if (c->block_size < 32 || c->block_size > kTraceMaxBlock || (c->block_size % 32)) return HK_E_ILLEGAL_INPUT;
    if (c->bins != 32) return HK_E_ILLEGAL_INPUT;
    if (c->max_depth < 1 || c->max_depth > 48) return HK_E_ILLEGAL_INPUT;
    if (!(c->intersect_cost > 0) || !(c->traverse_cost >= 0)) return HK_E_ILLEGAL_INPUT;
    if (c->topk < 1 || c->topk > 8 || !(c->fallback_ratio >= 0)) return HK_E_ILLEGAL_INPUT;
    if (c->exact_max != 0 && (c->exact_max < 32 || c->exact_max > 1024)) return HK_E_ILLEGAL_INPUT;
    if (c->subtree_max > 32 || c->level_streams > 2) return HK_E_ILLEGAL_INPUT;
    return HK_OK;
}

hk_status hk_create(hk_ctx **out, const hk_config *cfg) {
    if (!out) return HK_E_ILLEGAL_INPUT;
    *out = nullptr;
    hk_config c;
    if (cfg) c = *cfg;
    else hk_config_default(&c);
    if (validate_config(&c) != HK_OK) return HK_E_ILLEGAL_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || c.device < 0 || c.device >= ndev) return HK_E_CUDA;
    hk_ctx *x = new hk_ctx();
    x->cfg = c;
    x->device = c.device;
    if (cudaSetDevice(c.device) != cudaSuccess) {
        delete x;
        return HK_E_CUDA;
    }
    cudaDeviceGetAttribute(&x->sm_count, cudaDevAttrMultiProcessorCount, c.device);
    if (cudaStreamCreateWithFlags(&x->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete x;
        return HK_E_CUDA;
    }
    x->stream = x->own_stream;
    cudaEventCreate(&x->ev0);
    cudaEventCreate(&x->ev1);
    if (x->fetch.ensure(4) || x->counters.ensure(3) || x->errw.ensure(1) || x->box.ensure(8) ||
        x->box_ord.ensure(8) || x->scount.ensure(1)) {
        hk_destroy(x);
        return HK_E_ALLOC;
    }
    cudaMemset(x->errw.p, 0, 4);
    cudaMemset(x->counters.p, 0, 24);
    *out = x;
    return HK_OK;
}

hk_status hk_destroy(hk_ctx *c) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    // batches still alive lose their device memory and their context; a
    // later hk_batch_destroy only frees the host side
    for (hk_batch *b : c->batches) batch_detach(b);
    c->batches.clear();
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->verts.release(); c->rest.release(); c->tris.release(); c->part.release(); c->mats.release();
    c->box.release(); c->box_ord.release(); c->rec.release(); c->cache_tmp.release();
    c->nodes.release(); c->refs.release(); c->imp_ropes.release(); c->imp_cbox.release(); c->fetch.release(); c->counters.release(); c->errw.release();
    c->rays.release(); c->hits.release(); c->cam.release(); c->lights.release();
    c->srays.release(); c->shits.release(); c->slot.release(); c->spix.release(); c->scount.release();
    c->hleaf.release();
    c->hit4.release(); c->rgba.release();
    c->mirror.release(); c->mrays.release(); c->prays.release(); c->mhits.release(); c->phits.release();
    c->mslot.release(); c->mcount.release();
    build_release(c->build);
    c->resort.release();
    c->ooc.release();
    c->mlp_params.release(); c->mlp_grads.release(); c->mlp_m.release(); c->mlp_v.release();
    c->mlp_w1p.release(); c->mlp_w2p.release(); c->mlp_w3p.release(); c->mlp_w4p.release(); c->mlp_tcw.release();
    c->rec_X.release(); c->rec_y.release(); c->rec_rows.release();
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return HK_OK;
}

const char *hk_last_error(const hk_ctx *c) { return c ? c->err.c_str() : "null context"; }

hk_status hk_set_stream(hk_ctx *c, void *s) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    c->stream = s ? (cudaStream_t)s : c->own_stream;
    return HK_OK;
}

hk_status hk_synchronize(hk_ctx *c) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_err_word(c);
}

// ---------------------------------------------------------------------------
// scene
// ---------------------------------------------------------------------------
static void host_box(const float *v, uint32_t nv, float *box) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            float x = v[4 * (size_t)i + k];
            lo[k] = std::fmin(lo[k], x);
            hi[k] = std::fmax(hi[k], x);
        }
    for (int k = 0; k < 3; k++) {
        box[k] = lo[k];
        box[4 + k] = hi[k];
    }
    box[3] = box[7] = 1.0f;
}

static void invalidate_graph(hk_ctx *c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    c->graph_key = 0;
}

hk_status hk_scene_upload(hk_ctx *c, const float *verts4, uint32_t nv, const uint32_t *tris4, uint32_t nt) {
    if (!c || (nv && !verts4) || (nt && !tris4)) return fail(c, HK_E_ILLEGAL_INPUT, "null scene array");
    if (nt > (1u << 28)) return fail(c, HK_E_ILLEGAL_INPUT, "too many triangles");
    for (uint32_t i = 0; i < nv; i++) {
        const float *v = verts4 + 4 * (size_t)i;
        if (v[3] != 1.0f || !std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]))
            return fail(c, HK_E_ILLEGAL_INPUT, "vertices must be finite with w == 1");
    }
    for (size_t i = 0; i < (size_t)nt * 4; i++)
        if ((i & 3) != 3 && tris4[i] >= nv) return fail(c, HK_E_ILLEGAL_INPUT, "triangle index out of range");
    cudaSetDevice(c->device);
    invalidate_graph(c);
    HK_CUDA(c, c->verts.ensure(nv));
    HK_CUDA(c, c->tris.ensure(nt));
    HK_CUDA(c, c->rec.ensure(nt));
    HK_CUDA(c, cudaMemcpyAsync(c->verts.p, verts4, (size_t)nv * 16, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->tris.p, tris4, (size_t)nt * 16, cudaMemcpyHostToDevice, c->stream));
    c->nv = nv;
    c->nt = nt;
    c->nparts = 0;
    c->rec_valid = false;
    c->tree_valid = false;
    c->box_user = false;
    host_box(verts4, nv, c->hbox);
    HK_CUDA(c, cudaMemcpyAsync(c->box.p, c->hbox, 32, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_scene_set_box(hk_ctx *c, const float *box8) {
    if (!c || !box8) return HK_E_ILLEGAL_INPUT;
    for (int k = 0; k < 3; k++)
        if (!(box8[k] <= box8[4 + k])) return fail(c, HK_E_ILLEGAL_INPUT, "box min > max");
    cudaSetDevice(c->device);
    memcpy(c->hbox, box8, 32);
    c->box_user = true;
    c->imp_ropes_valid = false;
    HK_CUDA(c, cudaMemcpyAsync(c->box.p, c->hbox, 32, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_scene_get_box(hk_ctx *c, float *box8) {
    if (!c || !box8) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaMemcpyAsync(box8, c->box.p, 32, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_scene_set_parts(hk_ctx *c, const uint32_t *part, uint32_t nparts) {
    if (!c || !part || nparts == 0) return fail(c, HK_E_ILLEGAL_INPUT, "parts");
    if (c->nv == 0) return fail(c, HK_E_STATE, "upload the scene first");
    for (uint32_t i = 0; i < c->nv; i++)
        if (part[i] >= nparts) return fail(c, HK_E_ILLEGAL_INPUT, "part index out of range");
    cudaSetDevice(c->device);
    invalidate_graph(c);
    HK_CUDA(c, c->part.ensure(c->nv));
    HK_CUDA(c, c->rest.ensure(c->nv));
    HK_CUDA(c, c->mats.ensure((size_t)nparts * 12));
    HK_CUDA(c, cudaMemcpyAsync(c->part.p, part, (size_t)c->nv * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->rest.p, c->verts.p, (size_t)c->nv * 16, cudaMemcpyDeviceToDevice, c->stream));
    c->nparts = nparts;
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

// device part of a frame's transform: mats already in c->mats
static hk_status transform_device(hk_ctx *c) {
    HK_CUDA(c, launch_transform(c->rest.p, c->part.p, c->nv, c->mats.p, c->verts.p, c->box_ord.p, c->stream));
    if (!c->box_user) HK_CUDA(c, launch_box_finish(c->box_ord.p, c->box.p, c->stream));
    HK_CUDA(c, launch_precompute(c->verts.p, c->tris.p, c->nt, c->rec.p, c->stream));
    c->rec_valid = true;
    c->rec_epoch++;
    return HK_OK;
}

hk_status hk_scene_transform(hk_ctx *c, const float *mats12) {
    if (!c || !mats12) return HK_E_ILLEGAL_INPUT;
    if (c->nparts == 0) return fail(c, HK_E_STATE, "hk_scene_set_parts first");
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaMemcpyAsync(c->mats.p, mats12, (size_t)c->nparts * 48, cudaMemcpyHostToDevice, c->stream));
    hk_status s = transform_device(c);
    if (s != HK_OK) return s;
    c->tree_valid = false;
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_scene_set_mirrors(hk_ctx *c, const uint8_t *mirror, uint32_t nt) {
    if (!c || (nt && !mirror)) return HK_E_ILLEGAL_INPUT;
    if (nt != c->nt) return fail(c, HK_E_ILLEGAL_INPUT, "mirror flags size != triangle count");
    cudaSetDevice(c->device);
    invalidate_graph(c);
    HK_CUDA(c, c->mirror.ensure(std::max<uint32_t>(nt, 1)));
    HK_CUDA(c, cudaMemcpyAsync(c->mirror.p, mirror, nt, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->has_mirrors = true;
    return HK_OK;
}

hk_status hk_scene_get_counts(hk_ctx *c, uint32_t *nv, uint32_t *nt) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (nv) *nv = c->nv;
    if (nt) *nt = c->nt;
    return HK_OK;
}

hk_status hk_scene_get_vertices(hk_ctx *c, float *verts4) {
    if (!c || !verts4) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaMemcpyAsync(verts4, c->verts.p, (size_t)c->nv * 16, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

// ---------------------------------------------------------------------------
// triangle cache
// ---------------------------------------------------------------------------
hk_status hk_precompute(hk_ctx *c) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (c->nt == 0 && c->nv == 0) return fail(c, HK_E_STATE, "no scene");
    cudaSetDevice(c->device);
    HK_CUDA(c, launch_precompute(c->verts.p, c->tris.p, c->nt, c->rec.p, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->rec_valid = true;
    c->rec_epoch++;
    return HK_OK;
}

hk_status hk_cache_import(hk_ctx *c, const float *cache16, uint32_t nt) {
    if (!c || (nt && !cache16)) return HK_E_ILLEGAL_INPUT;
    if (nt != c->nt) return fail(c, HK_E_ILLEGAL_INPUT, "cache size != triangle count");
    for (uint32_t i = 0; i < nt; i++) {
        const float *q = cache16 + 16 * (size_t)i;
        // w lanes of normal / e0 / e1 are 0 for w == 1 vertices (NaN normal of a
        // zero-area triangle included: it never produces a hit)
        bool nan_n = std::isnan(q[0]) || std::isnan(q[1]) || std::isnan(q[2]);
        if (!(q[7] == 0.0f && q[11] == 0.0f && (q[3] == 0.0f || nan_n)))
            return fail(c, HK_E_ILLEGAL_INPUT, "cache w lanes must be 0");
    }
    cudaSetDevice(c->device);
    HK_CUDA(c, c->cache_tmp.ensure((size_t)nt * 16));
    HK_CUDA(c, cudaMemcpyAsync(c->cache_tmp.p, cache16, (size_t)nt * 64, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, launch_cache_to_rec(c->cache_tmp.p, c->verts.p, c->tris.p, nt, c->rec.p, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->rec_valid = true;
    c->rec_epoch++;
    return HK_OK;
}

hk_status hk_cache_export(hk_ctx *c, float *cache16) {
    if (!c || !cache16) return HK_E_ILLEGAL_INPUT;
    if (!c->rec_valid) return fail(c, HK_E_STATE, "no cache");
    cudaSetDevice(c->device);
    HK_CUDA(c, c->cache_tmp.ensure((size_t)c->nt * 16));
    HK_CUDA(c, launch_rec_to_cache(c->rec.p, c->nt, c->cache_tmp.p, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(cache16, c->cache_tmp.p, (size_t)c->nt * 64, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

// ---------------------------------------------------------------------------
// tree import / export
// ---------------------------------------------------------------------------
hk_status hk_tree_import(hk_ctx *c, const uint32_t *nodes4, uint32_t nn, const uint32_t *refs, uint32_t nr) {
    if (!c || !nodes4 || nn == 0 || (nr && !refs)) return fail(c, HK_E_ILLEGAL_INPUT, "tree arrays");
    if (c->nt == 0) return fail(c, HK_E_STATE, "upload the scene first");
    if (nn >= (1u << 29) || nr >= (1u << 30)) return fail(c, HK_E_ILLEGAL_INPUT, "tree too large");
    for (uint32_t i = 0; i < nr; i++)
        if (refs[i] >= c->nt) return fail(c, HK_E_ILLEGAL_INPUT, "leaf reference out of range");
    // breadth-first relayout into child pairs; reference child 0 -> empty cell
    std::vector<uint2> out;
    out.reserve(2 * (size_t)nn + 2);
    std::vector<uint32_t> src;
    src.reserve(2 * (size_t)nn + 2);
    std::vector<uint8_t> seen(nn, 0);
    const uint32_t kEmpty = 0xffffffffu, kPad = 0xfffffffeu;
    src.push_back(0);
    src.push_back(kPad);
    seen[0] = 1;
    for (size_t h = 0; h < src.size(); h++) {
        uint32_t s = src[h];
        uint2 cn;
        if (s == kEmpty || s == kPad) {
            cn = make_uint2(kLeafTag, 0);
        } else {
            const uint32_t *n = nodes4 + 4 * (size_t)s;
            if (n[0] == 4u) {
                if ((uint64_t)n[1] + n[2] > nr) return fail(c, HK_E_ILLEGAL_INPUT, "leaf range out of bounds");
                cn = make_uint2((n[1] << 2) | kLeafTag, n[2]);
            } else if ((n[0] & ~3u) == 8u && (n[0] & 3u) < 3u) {
                uint32_t above = n[1], below = n[2];
                if (above >= nn || below >= nn) return fail(c, HK_E_ILLEGAL_INPUT, "child index out of range");
                for (uint32_t ch : {below, above}) {
                    if (ch == 0) continue;
                    if (seen[ch]) return fail(c, HK_E_ILLEGAL_INPUT, "tree is not a tree (shared or cyclic child)");
                    seen[ch] = 1;
                }
                uint32_t pair = (uint32_t)src.size();
                src.push_back(below ? below : kEmpty);
                src.push_back(above ? above : kEmpty);
                cn = make_uint2((pair << 2) | (n[0] & 3u), n[3]);
            } else {
                return fail(c, HK_E_ILLEGAL_INPUT, "bad node flags");
            }
        }
        out.push_back(cn);
    }
    cudaSetDevice(c->device);
    invalidate_graph(c);
    HK_CUDA(c, c->nodes.ensure(out.size()));
    HK_CUDA(c, c->refs.ensure(std::max<uint32_t>(nr, 1)));
    HK_CUDA(c, cudaMemcpyAsync(c->nodes.p, out.data(), out.size() * 8, cudaMemcpyHostToDevice, c->stream));
    if (nr) HK_CUDA(c, cudaMemcpyAsync(c->refs.p, refs, (size_t)nr * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->nn = (uint32_t)out.size();
    c->nr = nr;
    c->tree_valid = true;
    c->tree_epoch++;
    c->tree_built = false;
    c->host_nodes.swap(out);
    c->imp_ropes_valid = false;
    c->tree_on_device_counts = false;
    memset(&c->stats, 0, sizeof(c->stats));
    c->stats.nodes = c->nn;
    c->stats.refs = nr;
    return HK_OK;
}

static hk_status sync_tree_sizes(hk_ctx *c) {
    if (c->tree_on_device_counts) {
        hk_status s = build_read_stats(c->build, c->stream, &c->stats);
        if (s != HK_OK) {
            // the builder's output is not a tree: nothing may trace or export it
            c->tree_valid = false;
            c->tree_built = false;
            c->tree_on_device_counts = false;
            char msg[96];
            snprintf(msg, sizeof msg, "build failed (error bits 0x%x)", c->build.last_err);
            return fail(c, s, msg);
        }
        c->nn = c->stats.nodes;
        c->nr = c->stats.refs;
        c->tree_on_device_counts = false;
    }
    return HK_OK;
}

hk_status hk_tree_export_compact(hk_ctx *c, uint32_t *cn, uint32_t cap_nodes, uint32_t *refs, uint32_t cap_refs,
                                 uint32_t *nn, uint32_t *nr) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid) return fail(c, HK_E_STATE, "no tree");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    if (nn) *nn = c->nn;
    if (nr) *nr = c->nr;
    if (!cn) return HK_OK;
    if (cap_nodes < c->nn || cap_refs < c->nr) return fail(c, HK_E_CAPACITY, "export buffers too small");
    HK_CUDA(c, cudaMemcpyAsync(cn, tree_nodes(c), (size_t)c->nn * 8, cudaMemcpyDeviceToHost, c->stream));
    if (c->nr && refs) HK_CUDA(c, cudaMemcpyAsync(refs, tree_refs(c), (size_t)c->nr * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_tree_export(hk_ctx *c, uint32_t *nodes4, uint32_t cap_nodes, uint32_t *refs, uint32_t cap_refs,
                         uint32_t *nn, uint32_t *nr) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid) return fail(c, HK_E_STATE, "no tree");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    if (nn) *nn = c->nn;
    if (nr) *nr = c->nr;
    if (!nodes4) return HK_OK;
    if (cap_nodes < c->nn || cap_refs < c->nr) return fail(c, HK_E_CAPACITY, "export buffers too small");
    std::vector<uint2> cn(c->nn);
    HK_CUDA(c, cudaMemcpyAsync(cn.data(), tree_nodes(c), (size_t)c->nn * 8, cudaMemcpyDeviceToHost, c->stream));
    if (c->nr && refs) HK_CUDA(c, cudaMemcpyAsync(refs, tree_refs(c), (size_t)c->nr * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    // same indices; empty cells become the reference's child 0
    uint32_t leaf = 0;
    auto empty = [&](uint32_t i) { return (cn[i].x & 3u) == kLeafTag && cn[i].y == 0; };
    for (uint32_t i = 0; i < c->nn; i++) {
        uint32_t *n = nodes4 + 4 * (size_t)i;
        if ((cn[i].x & 3u) == kLeafTag) {
            n[0] = 4u;
            n[1] = cn[i].x >> 2;
            n[2] = cn[i].y;
            n[3] = leaf++;
        } else {
            uint32_t pair = cn[i].x >> 2;
            n[0] = (cn[i].x & 3u) | 8u;
            n[2] = empty(pair) ? 0u : pair;
            n[1] = empty(pair + 1) ? 0u : pair + 1;
            n[3] = cn[i].y;
        }
    }
    return HK_OK;
}

hk_status hk_tree_stats_get(hk_ctx *c, hk_tree_stats *st) {
    if (!c || !st) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    *st = c->stats;
    return HK_OK;
}

hk_status hk_build_level_counts(hk_ctx *c, uint32_t *nodes, uint32_t *refs, uint32_t cap, uint32_t *nlevels) {
    if (!c || !nlevels) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid || !c->tree_built) return fail(c, HK_E_STATE, "no tree from hk_build's level-synchronous builder");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    BuildCounters bc;
    HK_CUDA(c, cudaMemcpyAsync(&bc, c->build.ctr, sizeof bc, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    uint32_t n = 0;
    while (n < (uint32_t)kMaxLevels && bc.lvl[n].nodes) n++;
    *nlevels = n;
    for (uint32_t l = 0; l < n && l < cap; l++) {
        if (nodes) nodes[l] = bc.lvl[l].nodes;
        if (refs) refs[l] = bc.lvl[l].refs;
    }
    return HK_OK;
}

hk_status hk_build_subtree_counts(hk_ctx *c, uint32_t *roots, uint32_t *root_refs, uint32_t *nodes,
                                  uint32_t *leaf_refs) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid || !c->tree_built) return fail(c, HK_E_STATE, "no tree from hk_build's level-synchronous builder");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    BuildCounters bc;
    HK_CUDA(c, cudaMemcpyAsync(&bc, c->build.ctr, sizeof bc, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    const LevelCounters &fin = bc.lvl[c->build.last_level];
    if (roots) *roots = fin.defer_nodes_total;
    if (root_refs) *root_refs = fin.defer_refs_total;
    if (nodes) *nodes = bc.sub_fits ? bc.sub_nodes : 0u;
    if (leaf_refs) *leaf_refs = bc.sub_fits ? bc.sub_refs : 0u;
    return HK_OK;
}

hk_status hk_set_build_layout(hk_ctx *c, uint32_t subtree_max, uint32_t subtree_depth, uint32_t level_streams) {
    if (!c || subtree_max > 32 || level_streams > 2) return HK_E_ILLEGAL_INPUT;
    c->cfg.subtree_max = subtree_max;
    c->cfg.subtree_depth = subtree_depth;
    c->cfg.level_streams = level_streams;
    invalidate_graph(c);
    return HK_OK;
}

hk_status hk_set_trace_config(hk_ctx *c, uint32_t block_size, uint32_t short_stack) {
    if (!c || block_size < 32 || block_size > kTraceMaxBlock || (block_size % 32) || short_stack < 1 ||
        short_stack > 16)
        return HK_E_ILLEGAL_INPUT;
    c->cfg.block_size = block_size;
    c->cfg.short_stack = short_stack;
    invalidate_graph(c);
    return HK_OK;
}

hk_status hk_set_debug_flags(hk_ctx *c, uint32_t flags) {
    if (!c || (flags & ~1u)) return HK_E_ILLEGAL_INPUT;
    c->debug_flags = flags;
    invalidate_graph(c);
    return HK_OK;
}

hk_status hk_set_proposal_log(hk_ctx *c, int enable) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    c->prop_log = enable != 0;
    invalidate_graph(c);
    return HK_OK;
}

hk_status hk_get_proposal_log(hk_ctx *c, int32_t *bins8, uint32_t cap_nodes, uint32_t *nn) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid || !c->tree_built || !c->build.prop_log || !c->prop_log)
        return fail(c, HK_E_STATE, "no logged learned build");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    if (nn) *nn = c->nn;
    if (!bins8) return HK_OK;
    if (cap_nodes < c->nn) return fail(c, HK_E_CAPACITY, "log buffer too small");
    HK_CUDA(c, cudaMemcpyAsync(bins8, c->build.prop_log, (size_t)c->nn * 8 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                               c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

// SAH cost of the current tree: sum over reachable junctions of ct A(n) / A(root)
// plus over leaves of ci |refs(n)| A(n) / A(root), A the full surface area of
// the node's cell (the scene box split by the planes above it), in double
// precision. Cells follow the compact layout: pair = below child, pair + 1 =
// above child; an empty cell (count 0) adds nothing.
hk_status hk_tree_cost(hk_ctx *c, double ct, double ci, double *cost) {
    if (!c || !cost) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid) return fail(c, HK_E_STATE, "no tree");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    std::vector<uint2> cn(c->nn);
    float box[8];
    HK_CUDA(c, cudaMemcpyAsync(cn.data(), tree_nodes(c), (size_t)c->nn * 8, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(box, c->box.p, 32, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    auto area = [](const float *lo, const float *hi) {
        const double sx = (double)hi[0] - lo[0], sy = (double)hi[1] - lo[1], sz = (double)hi[2] - lo[2];
        return 2.0 * (sx * sy + sy * sz + sx * sz);
    };
    const double aroot = area(box, box + 4);
    struct Item {
        uint32_t i;
        float lo[3], hi[3];
    };
    std::vector<Item> todo;
    todo.push_back(Item{0, {box[0], box[1], box[2]}, {box[4], box[5], box[6]}});
    double sum = 0.0;
    size_t visited = 0;
    while (!todo.empty()) {
        const Item it = todo.back();
        todo.pop_back();
        if (it.i >= c->nn || ++visited > c->nn) return fail(c, HK_E_BOUNDS, "tree cost: malformed tree");
        const uint2 n = cn[it.i];
        const double a = area(it.lo, it.hi);
        if ((n.x & 3u) == kLeafTag) {
            sum += ci * (double)n.y * a / aroot;
            continue;
        }
        sum += ct * a / aroot;
        const uint32_t ax = n.x & 3u, pair = n.x >> 2;
        float p;
        memcpy(&p, &n.y, 4);
        Item b = it, u = it;
        b.i = pair;
        b.hi[ax] = p;
        u.i = pair + 1;
        u.lo[ax] = p;
        todo.push_back(u);
        todo.push_back(b);
    }
    *cost = sum;
    return HK_OK;
}

// ---------------------------------------------------------------------------
// build
// ---------------------------------------------------------------------------
static BuildParams build_params(hk_ctx *c, hk_build_mode mode) {
    BuildParams p;
    p.ct = c->cfg.traverse_cost;
    p.ci = c->cfg.intersect_cost;
    p.max_depth = c->cfg.max_depth;
    p.leaf_size = c->cfg.leaf_size;
    p.max_refs = c->cfg.max_refs ? c->cfg.max_refs : std::max<uint32_t>(16u * c->nt, 1024u);
    p.mode = (int)mode;
    p.topk = c->cfg.topk;
    p.fallback_ratio = c->cfg.fallback_ratio;
    p.exact_max = c->cfg.exact_max;
    p.record = c->recording ? 1 : 0;
    p.prop_log = c->prop_log ? 1 : 0;
    p.spin_limit = c->cfg.spin_limit;
    p.debug_flags = c->debug_flags;
    p.defer = c->cfg.subtree_max;
    p.defer_margin = c->cfg.subtree_depth;
    p.level_streams = c->cfg.level_streams;
    c->build.learn = &c->learn;
    return p;
}

// enqueue a build on c->stream (no host synchronisation)
static hk_status build_enqueue(hk_ctx *c, hk_build_mode mode) {
    BuildParams p = build_params(c, mode);
    hk_status s = build_prepare(c->build, p, c->nt, c->sm_count);
    if (s != HK_OK) return fail(c, s, "builder arena allocation failed");
    BuildOutputs o;
    s = build_ensure_outputs(c->build, &o);
    if (s != HK_OK) return fail(c, s, "builder output allocation failed");
    cudaError_t e = build_launch(c->build, c->verts.p, c->tris.p, c->nt, c->box.p, c->stream);
    if (e != cudaSuccess) {
        c->err = std::string("build launch: ") + cudaGetErrorString(e);
        return HK_E_CUDA;
    }
    // the device tree lives in the builder's output buffers
    c->tree_valid = true;
    c->tree_epoch++;
    c->tree_built = true;
    c->tree_on_device_counts = true;
    return HK_OK;
}

}  // extern "C"


extern "C" {

// HK_BUILD_SAH_RESORT: the reference's --treeType=SAH builder on the GPU
// (hk_build_resort.cu); its tree takes the place of an imported one
static hk_status build_resort(hk_ctx *c, hk_tree_stats *stats) {
    const ResortParams p{c->cfg.traverse_cost, c->cfg.intersect_cost, c->cfg.max_depth, c->cfg.leaf_size,
                         c->cfg.sah_sample ? c->cfg.sah_sample : 5u};
    float hb[8];
    HK_CUDA(c, cudaMemcpyAsync(hb, c->box.p, 32, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    invalidate_graph(c);
    c->tree_valid = false;
    c->tree_built = false;
    HK_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    std::string err;
    hk_status s = resort_build(c->resort, p, c->verts.p, c->tris.p, c->nt, hb, c->stream, &err);
    if (s != HK_OK) return fail(c, s, err.c_str());
    HK_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    const ResortState &R = c->resort;
    HK_CUDA(c, c->nodes.ensure(R.nn));
    HK_CUDA(c, c->refs.ensure(std::max<uint32_t>(R.nr, 1)));
    HK_CUDA(c, c->imp_ropes.ensure(6 * (size_t)R.nn));
    HK_CUDA(c, c->imp_cbox.ensure(2 * (size_t)R.nn));
    HK_CUDA(c, cudaMemcpyAsync(c->nodes.p, R.nodes.p, (size_t)R.nn * 8, cudaMemcpyDeviceToDevice, c->stream));
    if (R.nr)
        HK_CUDA(c, cudaMemcpyAsync(c->refs.p, R.out_refs.p, (size_t)R.nr * 4, cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->imp_ropes.p, R.out_ropes.p, (size_t)R.nn * 24, cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->imp_cbox.p, R.out_cbox.p, (size_t)R.nn * 32, cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->nn = R.nn;
    c->nr = R.nr;
    c->tree_valid = true;
    c->tree_epoch++;
    c->tree_built = false;
    c->tree_on_device_counts = false;
    c->imp_ropes_valid = true;
    c->host_nodes.clear();
    memset(&c->stats, 0, sizeof(c->stats));
    c->stats.nodes = R.nn;
    c->stats.refs = R.nr;
    c->stats.depth = R.depth;
    c->stats.build_ms = ms;
    if (stats) *stats = c->stats;
    return HK_OK;
}

hk_status hk_build(hk_ctx *c, hk_build_mode mode, hk_tree_stats *stats) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (c->nt == 0) return fail(c, HK_E_STATE, "no scene");
    if (mode == HK_BUILD_SAH_RESORT) {
        cudaSetDevice(c->device);
        return build_resort(c, stats);
    }
    if (mode != HK_BUILD_BINNED && mode != HK_BUILD_LEARNED) return fail(c, HK_E_ILLEGAL_INPUT, "mode");
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    hk_status s = build_enqueue(c, mode);
    if (s != HK_OK) return s;
    HK_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    s = check_err_word(c);
    if (s != HK_OK) return s;
    s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->stats.build_ms = ms;
    if (stats) *stats = c->stats;
    return HK_OK;
}

// ---------------------------------------------------------------------------
// tracing
// ---------------------------------------------------------------------------
// Ropes and cells of an imported tree: each face of a node's cell points to
// the node across it (the sibling across the parent's split plane, the
// parent's rope otherwise); children always follow their parent in the
// compact order, so one forward pass suffices.
static hk_status ensure_imported_ropes(hk_ctx *c) {
    if (c->imp_ropes_valid) return HK_OK;
    const std::vector<uint2> &N = c->host_nodes;
    size_t nn = N.size();
    std::vector<uint32_t> ropes(6 * nn, 0xffffffffu);
    std::vector<float4> cbox(2 * nn, make_float4(0, 0, 0, 0));
    cbox[0] = make_float4(c->hbox[0], c->hbox[1], c->hbox[2], 0.0f);
    cbox[1] = make_float4(c->hbox[4], c->hbox[5], c->hbox[6], 0.0f);
    auto set = [](float4 &v, uint32_t a, float x) {
        if (a == 0) v.x = x;
        else if (a == 1) v.y = x;
        else v.z = x;
    };
    for (size_t i = 0; i < nn; i++) {
        if (i == 1 || (N[i].x & 3u) == kLeafTag) continue;
        uint32_t axis = N[i].x & 3u, pair = N[i].x >> 2;
        float plane;
        memcpy(&plane, &N[i].y, 4);
        for (uint32_t ch = 0; ch < 2; ch++) {
            size_t k = pair + ch;
            cbox[2 * k] = cbox[2 * i];
            cbox[2 * k + 1] = cbox[2 * i + 1];
            for (int f = 0; f < 6; f++) ropes[6 * k + f] = ropes[6 * i + f];
            if (ch == 0) {
                set(cbox[2 * k + 1], axis, plane);
                ropes[6 * k + 2 * axis + 1] = pair + 1;
            } else {
                set(cbox[2 * k], axis, plane);
                ropes[6 * k + 2 * axis] = pair;
            }
        }
    }
    HK_CUDA(c, c->imp_ropes.ensure(ropes.size()));
    HK_CUDA(c, c->imp_cbox.ensure(cbox.size()));
    HK_CUDA(c, cudaMemcpyAsync(c->imp_ropes.p, ropes.data(), ropes.size() * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->imp_cbox.p, cbox.data(), cbox.size() * 16, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->imp_ropes_valid = true;
    return HK_OK;
}

static hk_status trace_enqueue(hk_ctx *c, const float4 *d_rays, uint32_t n, const uint32_t *n_dev, hk_variant v,
                               hk_hit *d_hits, bool occlusion = false, uint32_t *leaf_out = nullptr) {
    if ((int)v < HK_TRACE_FULLSTACK || (int)v > HK_TRACE_BRUTE) return fail(c, HK_E_ILLEGAL_INPUT, "variant");
    if (!c->rec_valid) return fail(c, HK_E_STATE, "no triangle cache (hk_precompute or hk_cache_import)");
    if (v != HK_TRACE_BRUTE && !c->tree_valid) return fail(c, HK_E_STATE, "no tree");
    TraceLaunch L;
    memset(&L, 0, sizeof(L));
    if (v == HK_TRACE_ROPES) {
        if (c->tree_built) {
            L.ropes = c->build.out_ropes;
            L.cbox = c->build.out_cbox;
            L.rope_nn_dev = build_nodes_total_ptr(c->build);
        } else {
            hk_status s = ensure_imported_ropes(c);
            if (s != HK_OK) return s;
            L.ropes = c->imp_ropes.p;
            L.cbox = c->imp_cbox.p;
            L.rope_nn = c->nn;
        }
    }
    L.nodes = tree_nodes(c);
    L.refs = tree_refs(c);
    L.tris = c->rec.p;
    L.rays = d_rays;
    L.hits = d_hits;
    L.n = n;
    L.n_dev = n_dev;
    L.ntris = c->nt;
    L.box = c->box.p;
    L.fetch = c->fetch.p;
    L.counters = c->counters.p;
    L.err = c->errw.p;
    L.stack_depth = c->cfg.short_stack;
    L.max_steps = c->cfg.max_steps ? c->cfg.max_steps : (1u << 26);
    L.variant = (int)v;
    L.count = c->counting;
    L.occlusion = occlusion;
    L.leaf_out = v == HK_TRACE_ROPES ? leaf_out : nullptr;
    L.block = (int)c->cfg.block_size;
    if (trace_smem_bytes(L.variant, c->cfg.block_size, L.stack_depth, false, occlusion, L.count) > kTraceMaxSmem)
        return fail(c, HK_E_ILLEGAL_INPUT,
                    "shared memory of this traversal exceeds 48 KB (short_stack x block_size x 12 + block_size x 8)");
    int per_sm = c->cfg.blocks_per_sm ? (int)c->cfg.blocks_per_sm : std::max(1, 2048 / L.block);
    L.grid = c->sm_count * per_sm;
    if (c->counting) HK_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 24, c->stream));
    HK_CUDA(c, launch_trace(L, c->stream));
    return HK_OK;
}

hk_status hk_trace_device(hk_ctx *c, const float *d_rays8, uint32_t n, hk_variant v, hk_hit *d_hits) {
    if (!c || (n && (!d_rays8 || !d_hits))) return HK_E_ILLEGAL_INPUT;
    if ((reinterpret_cast<uintptr_t>(d_rays8) & 15u) || (reinterpret_cast<uintptr_t>(d_hits) & 7u))
        return fail(c, HK_E_ILLEGAL_INPUT, "device arrays must be 16-byte (rays) / 8-byte (hits) aligned");
    cudaSetDevice(c->device);
    return trace_enqueue(c, reinterpret_cast<const float4 *>(d_rays8), n, nullptr, v, d_hits);
}

hk_status hk_trace(hk_ctx *c, const float *rays8, uint32_t n, hk_variant v, hk_hit *hits) {
    if (!c || (n && (!rays8 || !hits))) return HK_E_ILLEGAL_INPUT;
    for (size_t i = 0; i < n; i++)
        if (rays8[8 * i + 3] != 0.0f || rays8[8 * i + 7] != 0.0f)
            return fail(c, HK_E_ILLEGAL_INPUT, "ray w lanes must be 0");
    cudaSetDevice(c->device);
    HK_CUDA(c, c->rays.ensure(2 * (size_t)std::max<uint32_t>(n, 1)));
    HK_CUDA(c, c->hits.ensure(std::max<uint32_t>(n, 1)));
    HK_CUDA(c, cudaMemcpyAsync(c->rays.p, rays8, (size_t)n * 32, cudaMemcpyHostToDevice, c->stream));
    hk_status s = trace_enqueue(c, c->rays.p, n, nullptr, v, c->hits.p);
    if (s != HK_OK) return s;
    HK_CUDA(c, cudaMemcpyAsync(hits, c->hits.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_err_word(c);
}

hk_status hk_stream_setup(hk_ctx *c, uint32_t pool_tris) {
    if (!c || pool_tris == 0) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid || !c->rec_valid) return fail(c, HK_E_STATE, "streaming needs a tree and triangle records");
    cudaSetDevice(c->device);
    hk_status s = sync_tree_sizes(c);
    if (s != HK_OK) return s;
    std::string err;
    s = stream_setup(c->ooc, tree_nodes(c), c->nn, tree_refs(c), c->nr, c->rec.p, pool_tris, c->stream, &err);
    if (s != HK_OK) return fail(c, s, err.c_str());
    c->ooc.tree_epoch = c->tree_epoch;
    c->ooc.rec_epoch = c->rec_epoch;
    return HK_OK;
}

hk_status hk_trace_streamed(hk_ctx *c, const float *rays8, uint32_t n, hk_hit *hits, hk_stream_stats *stats) {
    if (!c || (n && (!rays8 || !hits))) return HK_E_ILLEGAL_INPUT;
    if (!c->ooc.ready) return fail(c, HK_E_STATE, "hk_stream_setup first");
    if (c->ooc.tree_epoch != c->tree_epoch || c->ooc.rec_epoch != c->rec_epoch)
        return fail(c, HK_E_STATE, "the tree or the records changed since hk_stream_setup");
    for (size_t i = 0; i < n; i++)
        if (rays8[8 * i + 3] != 0.0f || rays8[8 * i + 7] != 0.0f)
            return fail(c, HK_E_ILLEGAL_INPUT, "ray w lanes must be 0");
    cudaSetDevice(c->device);
    HK_CUDA(c, c->rays.ensure(2 * (size_t)std::max<uint32_t>(n, 1)));
    HK_CUDA(c, c->hits.ensure(std::max<uint32_t>(n, 1)));
    HK_CUDA(c, cudaMemcpyAsync(c->rays.p, rays8, (size_t)n * 32, cudaMemcpyHostToDevice, c->stream));
    StreamTraceArgs a;
    a.nodes = tree_nodes(c);
    a.refs = tree_refs(c);
    a.rays = c->rays.p;
    a.hits = c->hits.p;
    a.n = n;
    a.box = c->box.p;
    a.max_steps = c->cfg.max_steps ? c->cfg.max_steps : (1u << 26);
    a.err = c->errw.p;
    std::string err;
    hk_status s = stream_trace(c->ooc, a, c->stream, stats, &err);
    if (s != HK_OK) return fail(c, s, err.c_str());
    HK_CUDA(c, cudaMemcpyAsync(hits, c->hits.p, (size_t)n * 8, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_err_word(c);
}

hk_status hk_set_counting(hk_ctx *c, int enable) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    c->counting = enable != 0;
    return HK_OK;
}

hk_status hk_get_counters(hk_ctx *c, uint64_t *tot) {
    if (!c || !tot) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaMemcpyAsync(tot, c->counters.p, 24, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_camera_rays(hk_ctx *c, const float *cam16, uint32_t w, uint32_t h, float *rays8) {
    if (!c || !cam16 || !rays8) return HK_E_ILLEGAL_INPUT;
    size_t n = (size_t)w * h;
    if (n == 0 || n > (1u << 30)) return fail(c, HK_E_ILLEGAL_INPUT, "image size");
    cudaSetDevice(c->device);
    HK_CUDA(c, c->cam.ensure(16));
    HK_CUDA(c, c->rays.ensure(2 * n));
    HK_CUDA(c, cudaMemcpyAsync(c->cam.p, cam16, 64, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, launch_camera_rays(c->cam.p, w, h, c->rays.p, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(rays8, c->rays.p, n * 32, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

// ---------------------------------------------------------------------------
// rendering
// ---------------------------------------------------------------------------
static hk_status validate_lights(hk_ctx *c, const float *lights8, uint32_t nl) {
    if (nl && !lights8) return fail(c, HK_E_ILLEGAL_INPUT, "lights");
    if (nl > 64) return fail(c, HK_E_ILLEGAL_INPUT, "at most 64 lights");
    return HK_OK;
}

static hk_status render_buffers(hk_ctx *c, uint32_t npix, uint32_t nl) {
    size_t ns = (size_t)npix * std::max<uint32_t>(nl, 1);
    HK_CUDA(c, c->rays.ensure(2 * (size_t)npix));
    HK_CUDA(c, c->hits.ensure(npix));
    HK_CUDA(c, c->srays.ensure(2 * ns));
    HK_CUDA(c, c->shits.ensure(ns));
    HK_CUDA(c, c->slot.ensure(ns));
    HK_CUDA(c, c->spix.ensure(ns));
    HK_CUDA(c, c->hleaf.ensure(npix));
    HK_CUDA(c, c->hit4.ensure(npix));
    HK_CUDA(c, c->rgba.ensure(npix));
    HK_CUDA(c, c->cam.ensure(16));
    HK_CUDA(c, c->lights.ensure(8 * (size_t)std::max<uint32_t>(nl, 1)));
    if (c->has_mirrors) {
        HK_CUDA(c, c->mrays.ensure(2 * (size_t)npix));
        HK_CUDA(c, c->prays.ensure(2 * (size_t)npix));
        HK_CUDA(c, c->mhits.ensure(npix));
        HK_CUDA(c, c->phits.ensure(npix));
        HK_CUDA(c, c->mslot.ensure(npix));
        HK_CUDA(c, c->mcount.ensure(1));
    }
    return HK_OK;
}

// camera + lights already in c->cam / c->lights
// rows row0 .. row0 + h - 1 of a w x full_h frame (full_h 0: the frame is
// w x h) into d_rgba, w x h pixels
static hk_status render_enqueue(hk_ctx *c, uint32_t nl, uint32_t w, uint32_t h, hk_variant v, int shade,
                                uint32_t *d_rgba, uint32_t row0 = 0, uint32_t full_h = 0) {
    uint32_t npix = w * h;
    c->last_primary = npix;
    c->last_shade = shade;
    const bool tiled = (w % 8u == 0) && (h % 4u == 0);
    HK_CUDA(c, launch_camera_rays(c->cam.p, w, h, c->rays.p, c->stream, tiled, row0, full_h));
    // ropes: each pixel's last leaf, where its shadow rays may start
    const bool hint = v == HK_TRACE_ROPES && shade != HK_SHADE_PICTURE;
    hk_status s = trace_enqueue(c, c->rays.p, npix, nullptr, v, c->hits.p, false, hint ? c->hleaf.p : nullptr);
    if (s != HK_OK) return s;
    if (shade == HK_SHADE_PICTURE) {
        HK_CUDA(c, launch_hit4(c->hits.p, c->rec.p, npix, c->hit4.p, c->stream));
        HK_CUDA(c, launch_shade_picture(c->rays.p, c->hit4.p, npix, c->lights.p, nl, d_rgba, c->stream, w, tiled));
        return HK_OK;
    }
    const float4 *shade_rays = c->rays.p;
    const hk_hit *shade_hits = c->hits.p;
    if (shade == HK_SHADE_MIRROR) {
        // one mirror bounce: reflected rays, traced, merged into the shading rays
        HK_CUDA(c, launch_mirror_rays(c->rays.p, c->hits.p, c->rec.p, c->mirror.p, npix, c->mrays.p, c->mslot.p,
                                      c->mcount.p, c->stream));
        s = trace_enqueue(c, c->mrays.p, 0, c->mcount.p, v, c->mhits.p);
        if (s != HK_OK) return s;
        HK_CUDA(c, launch_mirror_merge(c->rays.p, c->hits.p, c->mslot.p, c->mrays.p, c->mhits.p, npix, c->prays.p,
                                       c->phits.p, c->stream));
        shade_rays = c->prays.p;
        shade_hits = c->phits.p;
    }
    HK_CUDA(c, launch_shadow_rays(shade_rays, shade_hits, c->rec.p, npix, c->lights.p, nl,
                                  hint ? c->hleaf.p : nullptr, c->srays.p, c->slot.p, c->spix.p, c->scount.p,
                                  c->stream));
    s = trace_enqueue(c, c->srays.p, 0, c->scount.p, v, c->shits.p, true);
    if (s != HK_OK) return s;
    HK_CUDA(c, launch_shade_cpu(shade_rays, shade_hits, c->rec.p, npix, c->lights.p, nl, c->slot.p, c->shits.p,
                                d_rgba, c->stream, w, tiled));
    return HK_OK;
}

hk_status hk_render_device(hk_ctx *c, const float *cam16, const float *lights8, uint32_t nl, uint32_t w, uint32_t h,
                           hk_variant v, int shade, uint32_t *d_rgba) {
    if (!c || !cam16 || !d_rgba) return HK_E_ILLEGAL_INPUT;
    if ((size_t)w * h == 0 || (size_t)w * h > (1u << 28)) return fail(c, HK_E_ILLEGAL_INPUT, "image size");
    if (shade != HK_SHADE_CPU && shade != HK_SHADE_PICTURE && shade != HK_SHADE_MIRROR)
        return fail(c, HK_E_ILLEGAL_INPUT, "shade mode");
    if (shade == HK_SHADE_MIRROR && !c->has_mirrors) return fail(c, HK_E_STATE, "hk_scene_set_mirrors first");
    hk_status s = validate_lights(c, lights8, nl);
    if (s != HK_OK) return s;
    cudaSetDevice(c->device);
    s = render_buffers(c, w * h, nl);
    if (s != HK_OK) return s;
    HK_CUDA(c, cudaMemcpyAsync(c->cam.p, cam16, 64, cudaMemcpyHostToDevice, c->stream));
    if (nl) HK_CUDA(c, cudaMemcpyAsync(c->lights.p, lights8, (size_t)nl * 32, cudaMemcpyHostToDevice, c->stream));
    return render_enqueue(c, nl, w, h, v, shade, d_rgba);
}

hk_status hk_render_rows_device(hk_ctx *c, const float *cam16, const float *lights8, uint32_t nl, uint32_t w,
                                uint32_t h, uint32_t y0, uint32_t y1, hk_variant v, int shade, uint32_t *d_rgba) {
    if (!c || !cam16 || !d_rgba) return HK_E_ILLEGAL_INPUT;
    if (y0 >= y1 || y1 > h) return fail(c, HK_E_ILLEGAL_INPUT, "row range");
    if ((size_t)w * h == 0 || (size_t)w * h > (1u << 28)) return fail(c, HK_E_ILLEGAL_INPUT, "image size");
    if (shade != HK_SHADE_CPU && shade != HK_SHADE_PICTURE && shade != HK_SHADE_MIRROR)
        return fail(c, HK_E_ILLEGAL_INPUT, "shade mode");
    if (shade == HK_SHADE_MIRROR && !c->has_mirrors) return fail(c, HK_E_STATE, "hk_scene_set_mirrors first");
    hk_status s = validate_lights(c, lights8, nl);
    if (s != HK_OK) return s;
    cudaSetDevice(c->device);
    const uint32_t rows = y1 - y0;
    s = render_buffers(c, w * rows, nl);
    if (s != HK_OK) return s;
    HK_CUDA(c, cudaMemcpyAsync(c->cam.p, cam16, 64, cudaMemcpyHostToDevice, c->stream));
    if (nl) HK_CUDA(c, cudaMemcpyAsync(c->lights.p, lights8, (size_t)nl * 32, cudaMemcpyHostToDevice, c->stream));
    return render_enqueue(c, nl, w, rows, v, shade, d_rgba, y0, h);
}

hk_status hk_render(hk_ctx *c, const float *cam16, const float *lights8, uint32_t nl, uint32_t w, uint32_t h,
                    hk_variant v, int shade, uint32_t *rgba) {
    if (!c || !rgba) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    if ((size_t)w * h == 0 || (size_t)w * h > (1u << 28)) return fail(c, HK_E_ILLEGAL_INPUT, "image size");
    hk_status s = render_buffers(c, w * h, nl);
    if (s != HK_OK) return s;
    s = hk_render_device(c, cam16, lights8, nl, w, h, v, shade, c->rgba.p);
    if (s != HK_OK) return s;
    HK_CUDA(c, cudaMemcpyAsync(rgba, c->rgba.p, (size_t)w * h * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_err_word(c);
}

hk_status hk_shade_picture(hk_ctx *c, const float *rays8, const float *hit4, uint32_t n, const float *lights8,
                           uint32_t nl, uint32_t *rgba) {
    if (!c || (n && (!rays8 || !hit4 || !rgba))) return HK_E_ILLEGAL_INPUT;
    hk_status s = validate_lights(c, lights8, nl);
    if (s != HK_OK) return s;
    cudaSetDevice(c->device);
    HK_CUDA(c, c->rays.ensure(2 * (size_t)std::max<uint32_t>(n, 1)));
    HK_CUDA(c, c->hit4.ensure(std::max<uint32_t>(n, 1)));
    HK_CUDA(c, c->rgba.ensure(std::max<uint32_t>(n, 1)));
    HK_CUDA(c, c->lights.ensure(8 * (size_t)std::max<uint32_t>(nl, 1)));
    HK_CUDA(c, cudaMemcpyAsync(c->rays.p, rays8, (size_t)n * 32, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->hit4.p, hit4, (size_t)n * 16, cudaMemcpyHostToDevice, c->stream));
    if (nl) HK_CUDA(c, cudaMemcpyAsync(c->lights.p, lights8, (size_t)nl * 32, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, launch_shade_picture(c->rays.p, c->hit4.p, n, c->lights.p, nl, c->rgba.p, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(rgba, c->rgba.p, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

// ---------------------------------------------------------------------------
// frame: transform -> build -> trace -> shade, optionally as a CUDA graph
// ---------------------------------------------------------------------------
static hk_status frame_enqueue(hk_ctx *c, bool animated, uint32_t nl, uint32_t w, uint32_t h, hk_build_mode mode,
                               hk_variant v, uint32_t *d_rgba) {
    hk_status s;
    if (animated) {
        s = transform_device(c);
        if (s != HK_OK) return s;
    } else if (!c->rec_valid) {
        HK_CUDA(c, launch_precompute(c->verts.p, c->tris.p, c->nt, c->rec.p, c->stream));
        c->rec_valid = true;
    c->rec_epoch++;
    }
    s = build_enqueue(c, mode);
    if (s != HK_OK) return s;
    return render_enqueue(c, nl, w, h, v, c->frame_shade, d_rgba);
}

hk_status hk_set_frame_shading(hk_ctx *c, int shade) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (shade != HK_SHADE_CPU && shade != HK_SHADE_PICTURE && shade != HK_SHADE_MIRROR)
        return fail(c, HK_E_ILLEGAL_INPUT, "shade mode");
    if (shade == HK_SHADE_MIRROR && !c->has_mirrors) return fail(c, HK_E_STATE, "hk_scene_set_mirrors first");
    if (shade != c->frame_shade) invalidate_graph(c);
    c->frame_shade = shade;
    return HK_OK;
}

hk_status hk_frame(hk_ctx *c, const float *mats12, const float *cam16, const float *lights8, uint32_t nl, uint32_t w,
                   uint32_t h, hk_build_mode mode, hk_variant v, int use_graph, uint32_t *d_rgba,
                   hk_tree_stats *stats) {
    if (!c || !cam16 || !d_rgba) return HK_E_ILLEGAL_INPUT;
    if (c->nt == 0) return fail(c, HK_E_STATE, "no scene");
    if (mats12 && c->nparts == 0) return fail(c, HK_E_STATE, "hk_scene_set_parts first");
    if ((size_t)w * h == 0 || (size_t)w * h > (1u << 28)) return fail(c, HK_E_ILLEGAL_INPUT, "image size");
    hk_status s = validate_lights(c, lights8, nl);
    if (s != HK_OK) return s;
    cudaSetDevice(c->device);
    s = render_buffers(c, w * h, nl);
    if (s != HK_OK) return s;
    // size every arena before any capture so that the graph never allocates
    BuildParams bp = build_params(c, mode);
    s = build_prepare(c->build, bp, c->nt, c->sm_count);
    if (s != HK_OK) return fail(c, s, "builder arena allocation failed");
    BuildOutputs bo;
    s = build_ensure_outputs(c->build, &bo);
    if (s != HK_OK) return fail(c, s, "builder output allocation failed");
    // inputs of this frame
    if (mats12) HK_CUDA(c, cudaMemcpyAsync(c->mats.p, mats12, (size_t)c->nparts * 48, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(c->cam.p, cam16, 64, cudaMemcpyHostToDevice, c->stream));
    if (nl) HK_CUDA(c, cudaMemcpyAsync(c->lights.p, lights8, (size_t)nl * 32, cudaMemcpyHostToDevice, c->stream));
    bool animated = mats12 != nullptr;
    if (!use_graph) {
        s = frame_enqueue(c, animated, nl, w, h, mode, v, d_rgba);
        if (s != HK_OK) return s;
    } else {
        uint64_t key = ((uint64_t)w << 40) ^ ((uint64_t)h << 20) ^ ((uint64_t)nl << 12) ^ ((uint64_t)mode << 8) ^
                       ((uint64_t)v << 4) ^ (animated ? 1u : 0u) ^ ((uint64_t)(uintptr_t)d_rgba << 1) ^
                       ((uint64_t)c->nt << 44) ^ ((uint64_t)c->frame_shade << 2);
        if (!c->graph_exec || c->graph_key != key) {
            invalidate_graph(c);
            HK_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            s = frame_enqueue(c, animated, nl, w, h, mode, v, d_rgba);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (s != HK_OK) {
                if (g) cudaGraphDestroy(g);
                return s;
            }
            if (e != cudaSuccess) {
                c->err = std::string("graph capture: ") + cudaGetErrorString(e);
                return HK_E_CUDA;
            }
            c->graph = g;
            HK_CUDA(c, cudaGraphInstantiate(&c->graph_exec, g, 0));
            c->graph_key = key;
        }
        HK_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
        c->tree_valid = true;
    c->tree_epoch++;
        c->tree_built = true;
        c->tree_on_device_counts = true;
    }
    if (stats) {
        HK_CUDA(c, cudaStreamSynchronize(c->stream));
        s = check_err_word(c);
        if (s != HK_OK) return s;
        s = sync_tree_sizes(c);
        if (s != HK_OK) return s;
        *stats = c->stats;
    }
    return HK_OK;
}

hk_status hk_get_ray_counts(hk_ctx *c, uint64_t *primary, uint64_t *shadow) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    uint32_t ns = 0, nm = 0;
    if (c->last_shade != HK_SHADE_PICTURE && c->last_primary)
        HK_CUDA(c, cudaMemcpyAsync(&ns, c->scount.p, 4, cudaMemcpyDeviceToHost, c->stream));
    if (c->last_shade == HK_SHADE_MIRROR && c->last_primary)
        HK_CUDA(c, cudaMemcpyAsync(&nm, c->mcount.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    if (primary) *primary = c->last_primary;
    if (shadow) *shadow = (uint64_t)ns + nm;   /* secondary rays: shadow + mirror */
    return HK_OK;
}

hk_status hk_frame_graph_info(hk_ctx *c, uint32_t *kernel_nodes, uint32_t *all_nodes) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    uint32_t k = 0, a = 0;
    if (c->graph) {
        size_t n = 0;
        HK_CUDA(c, cudaGraphGetNodes(c->graph, nullptr, &n));
        std::vector<cudaGraphNode_t> nodes(n);
        HK_CUDA(c, cudaGraphGetNodes(c->graph, nodes.data(), &n));
        for (size_t i = 0; i < n; i++) {
            cudaGraphNodeType t;
            HK_CUDA(c, cudaGraphNodeGetType(nodes[i], &t));
            if (t == cudaGraphNodeTypeKernel) k++;
        }
        a = (uint32_t)n;
    }
    if (kernel_nodes) *kernel_nodes = k;
    if (all_nodes) *all_nodes = a;
    return HK_OK;
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
}  // extern "C"

struct hk_batch {
    hk_ctx *ctx;
    struct Scene {
        DevBuf<TriRec> rec;
        DevBuf<uint2> nodes;
        DevBuf<uint32_t> refs, ropes;
        DevBuf<float4> cbox;
        float box[8];
        uint32_t nn, nr, nt;
    };
    std::vector<Scene *> scenes;
    DevBuf<SceneDesc> table;
    DevBuf<uint32_t> offsets, remaining;
    DevBuf<unsigned long long> times;   // [0] start, [1..] per-scene done
};

extern "C" {

hk_status hk_batch_create(hk_ctx *c, hk_batch **out) {
    if (!c || !out) return HK_E_ILLEGAL_INPUT;
    hk_batch *b = new hk_batch();
    b->ctx = c;
    c->batches.push_back(b);
    *out = b;
    return HK_OK;
}

}  // extern "C"

// frees the batch's device memory (its context's device current, its stream
// idle) and cuts it from the context
static void batch_detach(hk_batch *b) {
    for (auto *s : b->scenes) {
        s->rec.release(); s->nodes.release(); s->refs.release(); s->ropes.release(); s->cbox.release();
        delete s;
    }
    b->scenes.clear();
    b->table.release(); b->offsets.release(); b->remaining.release(); b->times.release();
    b->ctx = nullptr;
}

extern "C" {

hk_status hk_batch_destroy(hk_batch *b) {
    if (!b) return HK_E_ILLEGAL_INPUT;
    if (hk_ctx *c = b->ctx) {
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        for (size_t i = 0; i < c->batches.size(); i++)
            if (c->batches[i] == b) {
                c->batches.erase(c->batches.begin() + (long)i);
                break;
            }
        batch_detach(b);
    }
    delete b;
    return HK_OK;
}

hk_status hk_batch_add_scene(hk_batch *b, const float *verts4, uint32_t nv, const uint32_t *tris4, uint32_t nt,
                             uint32_t *scene_id) {
    if (!b || nt == 0) return HK_E_ILLEGAL_INPUT;
    if (!b->ctx) return HK_E_STATE;   // its context was destroyed
    hk_ctx *c = b->ctx;
    hk_status st = hk_scene_upload(c, verts4, nv, tris4, nt);
    if (st != HK_OK) return st;
    st = hk_precompute(c);
    if (st != HK_OK) return st;
    hk_tree_stats ts;
    st = hk_build(c, HK_BUILD_BINNED, &ts);
    if (st != HK_OK) return st;
    auto *s = new hk_batch::Scene();
    s->nn = ts.nodes;
    s->nr = ts.refs;
    s->nt = nt;
    memcpy(s->box, c->hbox, 32);
    HK_CUDA(c, s->rec.ensure(nt));
    HK_CUDA(c, s->nodes.ensure(s->nn));
    HK_CUDA(c, s->refs.ensure(std::max<uint32_t>(s->nr, 1)));
    HK_CUDA(c, s->ropes.ensure((size_t)s->nn * 6));
    HK_CUDA(c, s->cbox.ensure((size_t)s->nn * 2));
    HK_CUDA(c, cudaMemcpyAsync(s->rec.p, c->rec.p, (size_t)nt * sizeof(TriRec), cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(s->nodes.p, c->build.out_nodes, (size_t)s->nn * 8, cudaMemcpyDeviceToDevice, c->stream));
    if (s->nr)
        HK_CUDA(c, cudaMemcpyAsync(s->refs.p, c->build.out_refs, (size_t)s->nr * 4, cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(s->ropes.p, c->build.out_ropes, (size_t)s->nn * 24, cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(s->cbox.p, c->build.out_cbox, (size_t)s->nn * 32, cudaMemcpyDeviceToDevice, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    if (scene_id) *scene_id = (uint32_t)b->scenes.size();
    b->scenes.push_back(s);
    return HK_OK;
}

hk_status hk_batch_trace_device(hk_batch *b, const float *d_rays8, const uint32_t *ray_offsets, uint32_t nscenes,
                                hk_variant v, hk_hit *d_hits, float *scene_ms) {
    if (!b || !ray_offsets || !d_rays8 || !d_hits) return HK_E_ILLEGAL_INPUT;
    if (!b->ctx) return HK_E_STATE;   // its context was destroyed
    hk_ctx *c = b->ctx;
    if (nscenes == 0 || nscenes != b->scenes.size()) return fail(c, HK_E_ILLEGAL_INPUT, "nscenes != scenes in batch");
    if ((int)v < HK_TRACE_FULLSTACK || (int)v > HK_TRACE_BRUTE) return fail(c, HK_E_ILLEGAL_INPUT, "variant");
    if (trace_smem_bytes(v, c->cfg.block_size, c->cfg.short_stack, true, false, c->counting) > kTraceMaxSmem)
        return fail(c, HK_E_ILLEGAL_INPUT, "shared ring too large (short_stack x block_size x 12 > 48 KB)");
    if (ray_offsets[0] != 0) return fail(c, HK_E_ILLEGAL_INPUT, "ray_offsets[0] must be 0");
    std::vector<uint32_t> rem(nscenes);
    for (uint32_t i = 0; i < nscenes; i++) {
        if (ray_offsets[i + 1] < ray_offsets[i]) return fail(c, HK_E_ILLEGAL_INPUT, "ray_offsets must ascend");
        rem[i] = ray_offsets[i + 1] - ray_offsets[i];
    }
    uint32_t n = ray_offsets[nscenes];
    cudaSetDevice(c->device);
    std::vector<SceneDesc> table(nscenes);
    for (uint32_t i = 0; i < nscenes; i++) {
        auto *s = b->scenes[i];
        SceneDesc &d = table[i];
        memset(&d, 0, sizeof(d));
        d.nodes = s->nodes.p;
        d.refs = s->refs.p;
        d.tris = s->rec.p;
        d.ropes = s->ropes.p;
        d.cbox = s->cbox.p;
        memcpy(d.box, s->box, 32);
        d.nn = s->nn;
        d.ntris = s->nt;
    }
    HK_CUDA(c, b->table.ensure(nscenes));
    HK_CUDA(c, b->offsets.ensure(nscenes + 1));
    HK_CUDA(c, b->remaining.ensure(nscenes));
    HK_CUDA(c, b->times.ensure(nscenes + 1));
    HK_CUDA(c, cudaMemcpyAsync(b->table.p, table.data(), nscenes * sizeof(SceneDesc), cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(b->offsets.p, ray_offsets, (nscenes + 1) * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(b->remaining.p, rem.data(), nscenes * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemsetAsync(b->times.p, 0xff, 8, c->stream));
    HK_CUDA(c, cudaMemsetAsync(b->times.p + 1, 0, nscenes * 8, c->stream));
    TraceLaunch L;
    memset(&L, 0, sizeof(L));
    L.rays = reinterpret_cast<const float4 *>(d_rays8);
    L.hits = d_hits;
    L.n = n;
    L.fetch = c->fetch.p;
    L.counters = c->counters.p;
    L.err = c->errw.p;
    L.stack_depth = c->cfg.short_stack;
    L.max_steps = c->cfg.max_steps ? c->cfg.max_steps : (1u << 26);
    L.variant = (int)v;
    L.count = c->counting;
    L.block = (int)c->cfg.block_size;
    int per_sm = c->cfg.blocks_per_sm ? (int)c->cfg.blocks_per_sm : std::max(1, 2048 / L.block);
    L.grid = c->sm_count * per_sm;
    L.scenes = b->table.p;
    L.ray_offsets = b->offsets.p;
    L.nscenes = nscenes;
    L.remaining = b->remaining.p;
    L.start_ns = b->times.p;
    L.done_ns = b->times.p + 1;
    if (c->counting) HK_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 24, c->stream));
    HK_CUDA(c, launch_trace(L, c->stream));
    if (scene_ms) {
        std::vector<unsigned long long> t(nscenes + 1);
        HK_CUDA(c, cudaMemcpyAsync(t.data(), b->times.p, (nscenes + 1) * 8, cudaMemcpyDeviceToHost, c->stream));
        HK_CUDA(c, cudaStreamSynchronize(c->stream));
        for (uint32_t i = 0; i < nscenes; i++)
            scene_ms[i] = (t[i + 1] >= t[0]) ? (float)((double)(t[i + 1] - t[0]) * 1e-6) : 0.0f;
        return check_err_word(c);
    }
    return HK_OK;
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
static float time_trace(hk_ctx *c, const float4 *d_rays, uint32_t n, hk_variant v, hk_hit *d_hits, int reps) {
    std::vector<float> ts;
    for (int r = 0; r < reps + 2; r++) {
        cudaEventRecord(c->ev0, c->stream);
        if (trace_enqueue(c, d_rays, n, nullptr, v, d_hits) != HK_OK) return -1.0f;
        cudaEventRecord(c->ev1, c->stream);
        if (cudaEventSynchronize(c->ev1) != cudaSuccess) return -1.0f;
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        if (r >= 2) ts.push_back(ms);
    }
    std::sort(ts.begin(), ts.end());
    return ts[ts.size() / 2];
}

static std::string tune_key(hk_ctx *c) {
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, c->device);
    uint32_t cls = 0;
    while ((1u << (cls + 1)) <= std::max<uint32_t>(c->nt, 1)) cls++;
    char buf[256];
    snprintf(buf, sizeof buf, "%s|sm%d|tris2^%u", prop.name, c->sm_count, cls);
    return buf;
}

// median device time of reps builds after one warm-up build (-1: a build failed)
static float time_build(hk_ctx *c, hk_build_mode mode, uint32_t reps) {
    std::vector<float> ts;
    for (uint32_t r = 0; r < reps + 1; r++) {
        hk_tree_stats st;
        if (hk_build(c, mode, &st) != HK_OK) return -1.0f;
        if (r >= 1) ts.push_back(st.build_ms);
    }
    std::sort(ts.begin(), ts.end());
    return ts[ts.size() / 2];
}

hk_status hk_autotune_build(hk_ctx *c, hk_build_mode mode, uint32_t reps, hk_build_tune_result *res) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    if (mode != HK_BUILD_BINNED && mode != HK_BUILD_LEARNED) return fail(c, HK_E_ILLEGAL_INPUT, "mode");
    if (c->nt == 0) return fail(c, HK_E_STATE, "no scene");
    if (reps == 0) reps = 5;
    cudaSetDevice(c->device);
    hk_build_tune_result r;
    memset(&r, 0, sizeof r);
    r.default_ms = time_build(c, mode, reps);
    if (r.default_ms < 0) return HK_E_CUDA;
    r.subtree_max = c->cfg.subtree_max;
    r.subtree_depth = c->cfg.subtree_depth;
    r.level_streams = c->cfg.level_streams ? c->cfg.level_streams : 1u;
    r.best_ms = r.default_ms;
    const uint32_t cand[][2] = {{0, 0}, {32, 0}, {32, 10}, {32, 8}, {32, 6}};
    for (const auto &k : cand) {
        for (uint32_t ls = 1; ls <= 2; ls++) {
            c->cfg.subtree_max = k[0];
            c->cfg.subtree_depth = k[1];
            c->cfg.level_streams = ls;
            invalidate_graph(c);
            const float ms = time_build(c, mode, reps);
            r.tried++;
            if (ms < 0) return HK_E_CUDA;
            if (ms < r.best_ms) {
                r.best_ms = ms;
                r.subtree_max = k[0];
                r.subtree_depth = k[1];
                r.level_streams = ls;
            }
        }
    }
    c->cfg.subtree_max = r.subtree_max;
    c->cfg.subtree_depth = r.subtree_depth;
    c->cfg.level_streams = r.level_streams;
    invalidate_graph(c);
    if (res) *res = r;
    return HK_OK;
}

hk_status hk_autotune(hk_ctx *c, const float *d_rays8, uint32_t n, const char *cache_path, hk_tune_result *res) {
    if (!c || !d_rays8 || n == 0) return HK_E_ILLEGAL_INPUT;
    if (!c->tree_valid || !c->rec_valid) return fail(c, HK_E_STATE, "autotune needs a scene and a tree");
    cudaSetDevice(c->device);
    hk_tune_result r;
    memset(&r, 0, sizeof r);
    std::string key = tune_key(c);
    if (cache_path) {
        FILE *f = fopen(cache_path, "r");
        if (f) {
            char line[512];
            while (fgets(line, sizeof line, f)) {
                char k[300];
                int var;
                unsigned bs, ss;
                float ms;
                if (sscanf(line, "%299[^,],%d,%u,%u,%f", k, &var, &bs, &ss, &ms) == 5 && key == k) {
                    r.variant = var;
                    r.block_size = bs;
                    r.short_stack = ss;
                    r.best_ms = ms;
                }
            }
            fclose(f);
            if (r.block_size) {
                c->cfg.block_size = r.block_size;
                c->cfg.short_stack = r.short_stack;
                if (res) *res = r;
                return HK_OK;
            }
        }
    }
    hk_config saved = c->cfg;
    DevBuf<hk_hit> hits;
    HK_CUDA(c, hits.ensure(n));
    const float4 *rays = reinterpret_cast<const float4 *>(d_rays8);
    c->cfg.block_size = 128;
    c->cfg.short_stack = 6;
    c->cfg.blocks_per_sm = 0;
    r.default_ms = time_trace(c, rays, n, HK_TRACE_ROPES, hits.p, 3);
    float best = 1e30f;
    const hk_variant vs[] = {HK_TRACE_ROPES, HK_TRACE_SHORTSTACK, HK_TRACE_SMEMSTACK, HK_TRACE_FULLSTACK,
                             HK_TRACE_RESTART_EARLY};
    const uint32_t blocks[] = {64, 128, 256};
    const uint32_t stacks[] = {4, 6, 8, 12, 16};
    for (hk_variant v : vs) {
        bool uses_stack = (v == HK_TRACE_SHORTSTACK || v == HK_TRACE_SMEMSTACK);
        for (uint32_t bs : blocks) {
            for (uint32_t ss : stacks) {
                if (!uses_stack && ss != 6) continue;
                // the shared ring (12 B per level and thread) plus the leaf-test slots (8 B per thread)
                if (trace_smem_bytes(v, bs, ss, false, false, false) > kTraceMaxSmem) continue;
                c->cfg.block_size = bs;
                c->cfg.short_stack = ss;
                float ms = time_trace(c, rays, n, v, hits.p, 3);
                r.tried++;
                if (ms > 0 && ms < best) {
                    best = ms;
                    r.variant = (int)v;
                    r.block_size = bs;
                    r.short_stack = ss;
                }
            }
        }
    }
    hits.release();
    c->cfg = saved;
    if (r.tried == 0 || best >= 1e30f) return fail(c, HK_E_CUDA, "autotune: no candidate ran");
    r.best_ms = best;
    c->cfg.block_size = r.block_size;
    c->cfg.short_stack = r.short_stack;
    if (cache_path) {
        FILE *f = fopen(cache_path, "a");
        if (!f) return fail(c, HK_E_FILE_OPEN, "autotune cache not writable");
        fprintf(f, "%s,%d,%u,%u,%.6f\n", key.c_str(), r.variant, r.block_size, r.short_stack, r.best_ms);
        if (fclose(f) != 0) return fail(c, HK_E_FILE_CLOSE, "autotune cache close failed");
    }
    if (res) *res = r;
    return check_err_word(c);
}

// ---------------------------------------------------------------------------
// learned split proposer: parameters, inference, training
// ---------------------------------------------------------------------------
static hk_status mlp_alloc(hk_ctx *c) {
    HK_CUDA(c, c->mlp_params.ensure(kMlpParams));
    HK_CUDA(c, c->mlp_grads.ensure(kMlpParams));
    HK_CUDA(c, c->mlp_m.ensure(kMlpParams));
    HK_CUDA(c, c->mlp_v.ensure(kMlpParams));
    HK_CUDA(c, c->mlp_w1p.ensure(packed_words(kMlpIn, kMlpHid)));
    HK_CUDA(c, c->mlp_w2p.ensure(packed_words(kMlpHid, kMlpHid)));
    HK_CUDA(c, c->mlp_w3p.ensure(packed_words(kMlpHid, kMlpHid)));
    HK_CUDA(c, c->mlp_w4p.ensure(packed_words(kMlpHid, kMlpOut)));
    HK_CUDA(c, c->mlp_tcw.ensure(tc_packed_bytes()));
    return HK_OK;
}

// BF16 fragment copies of the current FP32 weights
static hk_status mlp_pack(hk_ctx *c) {
    const float *P = c->mlp_params.p;
    HK_CUDA(c, mlp_setup());
    HK_CUDA(c, build_learn_setup());
    HK_CUDA(c, pack_b(P + kOffW1, kMlpIn, kMlpHid, c->mlp_w1p.p, c->stream));
    HK_CUDA(c, pack_b(P + kOffW2, kMlpHid, kMlpHid, c->mlp_w2p.p, c->stream));
    HK_CUDA(c, pack_b(P + kOffW3, kMlpHid, kMlpHid, c->mlp_w3p.p, c->stream));
    HK_CUDA(c, pack_b(P + kOffW4, kMlpHid, kMlpOut, c->mlp_w4p.p, c->stream));
    HK_CUDA(c, pack_umma(P, c->mlp_tcw.p, c->stream));
    MlpDevice &M = c->learn.mlp;
    M.tcw = c->mlp_tcw.p;
    M.w1p = c->mlp_w1p.p;
    M.w2p = c->mlp_w2p.p;
    M.w3p = c->mlp_w3p.p;
    M.w4p = c->mlp_w4p.p;
    M.b1 = P + kOffB1;
    M.b2 = P + kOffB2;
    M.b3 = P + kOffB3;
    M.b4 = P + kOffB4;
    c->learn.have_mlp = true;
    invalidate_graph(c);
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

static hk_status mlp_upload(hk_ctx *c, const float *params) {
    hk_status s = mlp_alloc(c);
    if (s != HK_OK) return s;
    HK_CUDA(c, cudaMemcpyAsync(c->mlp_params.p, params, kMlpParams * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemsetAsync(c->mlp_m.p, 0, kMlpParams * 4, c->stream));
    HK_CUDA(c, cudaMemsetAsync(c->mlp_v.p, 0, kMlpParams * 4, c->stream));
    c->mlp_step = 0;
    return mlp_pack(c);
}

hk_status hk_mlp_init(hk_ctx *c, uint64_t seed) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    std::vector<float> P(kMlpParams, 0.0f);
    std::mt19937_64 rng(seed);
    auto he = [&](size_t off, int fan_in, size_t n) {
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)fan_in));
        for (size_t i = 0; i < n; i++) P[off + i] = nd(rng);
    };
    he(kOffW1, kMlpIn, (size_t)kMlpIn * kMlpHid);
    he(kOffW2, kMlpHid, (size_t)kMlpHid * kMlpHid);
    he(kOffW3, kMlpHid, (size_t)kMlpHid * kMlpHid);
    he(kOffW4, kMlpHid, (size_t)kMlpHid * kMlpOut);
    return mlp_upload(c, P.data());
}

static const char kMlpMagic[8] = {'H', 'K', 'M', 'L', 'P', '1', 0, 0};

hk_status hk_mlp_save(hk_ctx *c, const char *path) {
    if (!c || !path) return HK_E_ILLEGAL_INPUT;
    if (!c->learn.have_mlp) return fail(c, HK_E_STATE, "no network");
    cudaSetDevice(c->device);
    std::vector<float> P(kMlpParams);
    HK_CUDA(c, cudaMemcpyAsync(P.data(), c->mlp_params.p, kMlpParams * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    FILE *f = fopen(path, "wb");
    if (!f) return fail(c, HK_E_FILE_OPEN, "cannot open weights file for writing");
    uint32_t hdr[4] = {1u, (uint32_t)kMlpIn, (uint32_t)kMlpHid, (uint32_t)kMlpOut};
    uint32_t n = (uint32_t)kMlpParams;
    bool ok = fwrite(kMlpMagic, 1, 8, f) == 8 && fwrite(hdr, 4, 4, f) == 4 && fwrite(&n, 4, 1, f) == 1 &&
              fwrite(P.data(), 4, kMlpParams, f) == kMlpParams;
    if (fclose(f) != 0 || !ok) return fail(c, HK_E_FILE_CLOSE, "weights file write failed");
    return HK_OK;
}

hk_status hk_mlp_load(hk_ctx *c, const char *path) {
    if (!c || !path) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    FILE *f = fopen(path, "rb");
    if (!f) return fail(c, HK_E_FILE_OPEN, "cannot open weights file");
    char magic[8];
    uint32_t hdr[4], n = 0;
    std::vector<float> P(kMlpParams);
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, kMlpMagic, 8) == 0 && fread(hdr, 4, 4, f) == 4 &&
              hdr[0] == 1u && hdr[1] == (uint32_t)kMlpIn && hdr[2] == (uint32_t)kMlpHid &&
              hdr[3] == (uint32_t)kMlpOut && fread(&n, 4, 1, f) == 1 && n == kMlpParams &&
              fread(P.data(), 4, kMlpParams, f) == kMlpParams;
    fclose(f);
    if (!ok) return fail(c, HK_E_ILLEGAL_INPUT, "not a proposer weights file of this network");
    return mlp_upload(c, P.data());
}

hk_status hk_mlp_get_params(hk_ctx *c, float *params, uint32_t n) {
    if (!c || !params || n != kMlpParams) return HK_E_ILLEGAL_INPUT;
    if (!c->learn.have_mlp) return fail(c, HK_E_STATE, "no network");
    cudaSetDevice(c->device);
    HK_CUDA(c, cudaMemcpyAsync(params, c->mlp_params.p, kMlpParams * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_mlp_set_params(hk_ctx *c, const float *params, uint32_t n) {
    if (!c || !params || n != kMlpParams) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    return mlp_upload(c, params);
}

hk_status hk_mlp_forward(hk_ctx *c, const float *X, uint32_t n, float *logits) {
    if (!c || (n && (!X || !logits))) return HK_E_ILLEGAL_INPUT;
    if (!c->learn.have_mlp) return fail(c, HK_E_STATE, "no network");
    cudaSetDevice(c->device);
    DevBuf<float> dx, dl;
    HK_CUDA(c, dx.ensure((size_t)n * kMlpIn));
    HK_CUDA(c, dl.ensure((size_t)n * kMlpOut));
    HK_CUDA(c, cudaMemcpyAsync(dx.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, mlp_infer(c->learn.mlp, dx.p, nullptr, n, dl.p, c->sm_count, c->stream, c->errw.p));
    HK_CUDA(c, cudaMemcpyAsync(logits, dl.p, (size_t)n * kMlpOut * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    dx.release();
    dl.release();
    uint32_t w = 0;
    HK_CUDA(c, cudaMemcpy(&w, c->errw.p, 4, cudaMemcpyDeviceToHost));
    if (w) {
        HK_CUDA(c, cudaMemset(c->errw.p, 0, 4));
        return fail(c, HK_E_DEVICE_TIMEOUT, "tensor-core pipeline wait ran out");
    }
    return HK_OK;
}

// FP32 forward + backward of rows Xb (device) with labels yb; gradients into
// c->mlp_grads, summed loss into *dloss (device)
struct MlpWork {
    DevBuf<float> H1, H2, H3, Z4, d1, d2, d3, d4, loss;
    cudaError_t ensure(uint32_t B) {
        cudaError_t e;
        if ((e = H1.ensure((size_t)B * kMlpHid)) || (e = H2.ensure((size_t)B * kMlpHid)) ||
            (e = H3.ensure((size_t)B * kMlpHid)) || (e = Z4.ensure((size_t)B * kMlpOut)) ||
            (e = d1.ensure((size_t)B * kMlpHid)) || (e = d2.ensure((size_t)B * kMlpHid)) ||
            (e = d3.ensure((size_t)B * kMlpHid)) || (e = d4.ensure((size_t)B * kMlpOut)) || (e = loss.ensure(1)))
            return e;
        return cudaSuccess;
    }
    void release() {
        H1.release(); H2.release(); H3.release(); Z4.release();
        d1.release(); d2.release(); d3.release(); d4.release(); loss.release();
    }
};

static hk_status mlp_fwd_bwd(hk_ctx *c, MlpWork &W, const float *Xb, const int32_t *yb, int B) {
    const float *P = c->mlp_params.p;
    float *G = c->mlp_grads.p;
    cudaStream_t s = c->stream;
    const int I = kMlpIn, Hd = kMlpHid, O = kMlpOut;
    HK_CUDA(c, sgemm(false, false, Xb, P + kOffW1, W.H1.p, P + kOffB1, B, Hd, I, I, Hd, Hd, true, false, s));
    HK_CUDA(c, sgemm(false, false, W.H1.p, P + kOffW2, W.H2.p, P + kOffB2, B, Hd, Hd, Hd, Hd, Hd, true, false, s));
    HK_CUDA(c, sgemm(false, false, W.H2.p, P + kOffW3, W.H3.p, P + kOffB3, B, Hd, Hd, Hd, Hd, Hd, true, false, s));
    HK_CUDA(c, sgemm(false, false, W.H3.p, P + kOffW4, W.Z4.p, P + kOffB4, B, O, Hd, Hd, O, O, false, false, s));
    HK_CUDA(c, softmax_xent(W.Z4.p, yb, B, W.d4.p, W.loss.p, s));
    // layer 4
    HK_CUDA(c, sgemm(true, false, W.H3.p, W.d4.p, G + kOffW4, nullptr, Hd, O, B, Hd, O, O, false, false, s));
    HK_CUDA(c, colsum(W.d4.p, B, O, G + kOffB4, s));
    HK_CUDA(c, sgemm(false, true, W.d4.p, P + kOffW4, W.d3.p, nullptr, B, Hd, O, O, O, Hd, false, false, s));
    HK_CUDA(c, relu_back(W.d3.p, W.H3.p, (size_t)B * Hd, s));
    // layer 3
    HK_CUDA(c, sgemm(true, false, W.H2.p, W.d3.p, G + kOffW3, nullptr, Hd, Hd, B, Hd, Hd, Hd, false, false, s));
    HK_CUDA(c, colsum(W.d3.p, B, Hd, G + kOffB3, s));
    HK_CUDA(c, sgemm(false, true, W.d3.p, P + kOffW3, W.d2.p, nullptr, B, Hd, Hd, Hd, Hd, Hd, false, false, s));
    HK_CUDA(c, relu_back(W.d2.p, W.H2.p, (size_t)B * Hd, s));
    // layer 2
    HK_CUDA(c, sgemm(true, false, W.H1.p, W.d2.p, G + kOffW2, nullptr, Hd, Hd, B, Hd, Hd, Hd, false, false, s));
    HK_CUDA(c, colsum(W.d2.p, B, Hd, G + kOffB2, s));
    HK_CUDA(c, sgemm(false, true, W.d2.p, P + kOffW2, W.d1.p, nullptr, B, Hd, Hd, Hd, Hd, Hd, false, false, s));
    HK_CUDA(c, relu_back(W.d1.p, W.H1.p, (size_t)B * Hd, s));
    // layer 1
    HK_CUDA(c, sgemm(true, false, Xb, W.d1.p, G + kOffW1, nullptr, I, Hd, B, I, Hd, Hd, false, false, s));
    HK_CUDA(c, colsum(W.d1.p, B, Hd, G + kOffB1, s));
    return HK_OK;
}

hk_status hk_mlp_grad(hk_ctx *c, const float *X, const int32_t *y, uint32_t n, float *grads, float *loss) {
    if (!c || !X || !y || n == 0 || !grads) return HK_E_ILLEGAL_INPUT;
    if (!c->learn.have_mlp) return fail(c, HK_E_STATE, "no network");
    for (uint32_t i = 0; i < n; i++)
        if (y[i] < 0 || y[i] >= kMlpOut) return fail(c, HK_E_ILLEGAL_INPUT, "label out of range");
    cudaSetDevice(c->device);
    DevBuf<float> dx;
    DevBuf<int32_t> dy;
    MlpWork W;
    HK_CUDA(c, dx.ensure((size_t)n * kMlpIn));
    HK_CUDA(c, dy.ensure(n));
    HK_CUDA(c, W.ensure(n));
    HK_CUDA(c, cudaMemcpyAsync(dx.p, X, (size_t)n * kMlpIn * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(dy.p, y, (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
    HK_CUDA(c, cudaMemsetAsync(W.loss.p, 0, 4, c->stream));
    hk_status st = mlp_fwd_bwd(c, W, dx.p, dy.p, (int)n);
    if (st != HK_OK) return st;
    float ls = 0;
    HK_CUDA(c, cudaMemcpyAsync(grads, c->mlp_grads.p, kMlpParams * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(&ls, W.loss.p, 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    if (loss) *loss = ls / (float)n;
    dx.release();
    dy.release();
    W.release();
    return HK_OK;
}

hk_status hk_mlp_record(hk_ctx *c, uint32_t cap) {
    if (!c) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    invalidate_graph(c);
    if (cap == 0) {
        c->recording = false;
        return HK_OK;
    }
    HK_CUDA(c, c->rec_X.ensure((size_t)cap * kMlpIn));
    HK_CUDA(c, c->rec_y.ensure(cap));
    HK_CUDA(c, c->rec_rows.ensure(1));
    HK_CUDA(c, cudaMemsetAsync(c->rec_rows.p, 0, 4, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    c->rec_cap = cap;
    c->learn.rec_X = c->rec_X.p;
    c->learn.rec_y = c->rec_y.p;
    c->learn.rec_rows = c->rec_rows.p;
    c->learn.rec_cap = cap;
    c->recording = true;
    return HK_OK;
}

static hk_status dataset_rows(hk_ctx *c, uint32_t *rows) {
    uint32_t r = 0;
    if (c->rec_rows.p) {
        HK_CUDA(c, cudaMemcpyAsync(&r, c->rec_rows.p, 4, cudaMemcpyDeviceToHost, c->stream));
        HK_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    *rows = std::min(r, c->rec_cap);
    return HK_OK;
}

hk_status hk_mlp_dataset(hk_ctx *c, float *X, int32_t *y, uint32_t cap, uint32_t *rows) {
    if (!c || !rows) return HK_E_ILLEGAL_INPUT;
    cudaSetDevice(c->device);
    uint32_t r;
    hk_status st = dataset_rows(c, &r);
    if (st != HK_OK) return st;
    *rows = r;
    if (!X && !y) return HK_OK;
    if (cap < r) return fail(c, HK_E_CAPACITY, "dataset buffers too small");
    if (X && r) HK_CUDA(c, cudaMemcpyAsync(X, c->rec_X.p, (size_t)r * kMlpIn * 4, cudaMemcpyDeviceToHost, c->stream));
    if (y && r) HK_CUDA(c, cudaMemcpyAsync(y, c->rec_y.p, (size_t)r * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    return HK_OK;
}

hk_status hk_mlp_train(hk_ctx *c, uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float *epoch_loss) {
    if (!c || epochs == 0 || batch == 0 || batch > 65536 || !(lr > 0)) return HK_E_ILLEGAL_INPUT;
    if (!c->learn.have_mlp) return fail(c, HK_E_STATE, "hk_mlp_init or hk_mlp_load first");
    cudaSetDevice(c->device);
    uint32_t rows;
    hk_status st = dataset_rows(c, &rows);
    if (st != HK_OK) return st;
    if (rows < batch) return fail(c, HK_E_STATE, "fewer recorded rows than one batch");
    DevBuf<uint32_t> perm;
    DevBuf<float> Xb;
    DevBuf<int32_t> yb;
    MlpWork W;
    HK_CUDA(c, perm.ensure(rows));
    HK_CUDA(c, Xb.ensure((size_t)batch * kMlpIn));
    HK_CUDA(c, yb.ensure(batch));
    HK_CUDA(c, W.ensure(batch));
    std::vector<uint32_t> idx(rows);
    std::mt19937_64 rng(seed);
    for (uint32_t e = 0; e < epochs; e++) {
        for (uint32_t i = 0; i < rows; i++) idx[i] = i;
        std::shuffle(idx.begin(), idx.end(), rng);
        HK_CUDA(c, cudaMemcpyAsync(perm.p, idx.data(), (size_t)rows * 4, cudaMemcpyHostToDevice, c->stream));
        HK_CUDA(c, cudaMemsetAsync(W.loss.p, 0, 4, c->stream));
        uint32_t nb = rows / batch;
        for (uint32_t b = 0; b < nb; b++) {
            HK_CUDA(c, gather_rows(c->rec_X.p, c->rec_y.p, perm.p + (size_t)b * batch, (int)batch, Xb.p, yb.p,
                                   c->stream));
            st = mlp_fwd_bwd(c, W, Xb.p, yb.p, (int)batch);
            if (st != HK_OK) return st;
            c->mlp_step++;
            HK_CUDA(c, adam(c->mlp_params.p, c->mlp_grads.p, c->mlp_m.p, c->mlp_v.p, kMlpParams, lr, c->mlp_step,
                            c->stream));
        }
        float ls = 0;
        HK_CUDA(c, cudaMemcpyAsync(&ls, W.loss.p, 4, cudaMemcpyDeviceToHost, c->stream));
        HK_CUDA(c, cudaStreamSynchronize(c->stream));
        if (epoch_loss) epoch_loss[e] = ls / (float)(nb * batch);
    }
    perm.release();
    Xb.release();
    yb.release();
    W.release();
    return mlp_pack(c);
}

// ---------------------------------------------------------------------------
// tree interchange file (the reference's KdFileHeader dataset layout)
// ---------------------------------------------------------------------------
struct KdFileHeader {
    uint64_t headerSize, KDTreeSize, KDTreeOffset, leafExtDataSize, leafExtDataOffset, indexPerLeafSize,
        indexPerLeafOffset, vertexPerLeafSize, vertexPerLeafOffset;
};
struct LeafExtData {
    uint32_t indexOffset, vertexOffset, vertxSize, indexSize;
};
static const char kLeafTrailer[8] = {'H', 'K', 'L', 'E', 'A', 'F', 'P', 'L'};
constexpr uint32_t kObjectPerLeafMult = 32;   // per-leaf blocks padded to 32 entries
constexpr uint32_t kRefLeaf = 4u;             // KDTreeNode::m_flags of a leaf

hk_status hk_tree_save_file(hk_ctx *c, const char *path) {
    if (!c || !path) return HK_E_ILLEGAL_INPUT;
    uint32_t nn = 0, nr = 0;
    hk_status st = hk_tree_export(c, nullptr, 0, nullptr, 0, &nn, &nr);
    if (st != HK_OK) return st;
    std::vector<uint32_t> nodes((size_t)nn * 4), refs(std::max<uint32_t>(nr, 1));
    st = hk_tree_export(c, nodes.data(), nn, refs.data(), nr, &nn, &nr);
    if (st != HK_OK) return st;
    std::vector<float> verts((size_t)c->nv * 4);
    std::vector<uint32_t> tris((size_t)c->nt * 4);
    HK_CUDA(c, cudaMemcpyAsync(verts.data(), c->verts.p, verts.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaMemcpyAsync(tris.data(), c->tris.p, tris.size() * 4, cudaMemcpyDeviceToHost, c->stream));
    HK_CUDA(c, cudaStreamSynchronize(c->stream));
    float box[8];
    if ((st = hk_scene_get_box(c, box)) != HK_OK) return st;
    // per-leaf data: leaf-local vertex numbering in first-use order
    std::vector<LeafExtData> ext;
    std::vector<uint32_t> idx;      // 4 per entry
    std::vector<float> lverts;      // 4 per entry
    std::unordered_map<uint32_t, uint32_t> vmap;
    for (uint32_t i = 0; i < nn; i++) {
        const uint32_t *n = &nodes[4 * (size_t)i];
        if (n[0] != kRefLeaf) continue;
        vmap.clear();
        LeafExtData e{(uint32_t)(idx.size() / 4), (uint32_t)(lverts.size() / 4), 0, 0};
        uint32_t nloc = 0;
        for (uint32_t k = 0; k < n[2]; k++) {
            const uint32_t t = refs[n[1] + k];
            uint32_t loc[4] = {0, 0, 0, 0};
            for (int v = 0; v < 3; v++) {
                const uint32_t g = tris[4 * (size_t)t + v];
                auto it = vmap.find(g);
                if (it != vmap.end()) {
                    loc[v] = it->second;
                } else {
                    loc[v] = nloc;
                    vmap.emplace(g, nloc++);
                    lverts.insert(lverts.end(), &verts[4 * (size_t)g], &verts[4 * (size_t)g] + 4);
                }
            }
            idx.insert(idx.end(), loc, loc + 4);
        }
        uint32_t ni = (uint32_t)(idx.size() / 4) - e.indexOffset, nv = (uint32_t)(lverts.size() / 4) - e.vertexOffset;
        const uint32_t ri = (ni + kObjectPerLeafMult - 1) & ~(kObjectPerLeafMult - 1);
        const uint32_t rv = (nv + kObjectPerLeafMult - 1) & ~(kObjectPerLeafMult - 1);
        idx.resize(idx.size() + 4 * (size_t)(ri - ni), 0u);
        lverts.resize(lverts.size() + 4 * (size_t)(rv - nv), 0.0f);
        e.indexSize = ri;
        e.vertxSize = rv;
        ext.push_back(e);
    }
    KdFileHeader h{};
    h.headerSize = sizeof(KdFileHeader);
    h.KDTreeOffset = h.headerSize;
    h.KDTreeSize = (uint64_t)nn * 16;
    h.leafExtDataOffset = h.KDTreeOffset + h.KDTreeSize;
    h.leafExtDataSize = ext.size() * sizeof(LeafExtData);
    h.indexPerLeafOffset = (h.leafExtDataOffset + h.leafExtDataSize + 511) & ~(uint64_t)511;
    h.indexPerLeafSize = idx.size() * 4;
    h.vertexPerLeafOffset = h.indexPerLeafOffset + h.indexPerLeafSize;
    h.vertexPerLeafSize = lverts.size() * 4;
    FILE *f = fopen(path, "wb");
    if (!f) return fail(c, HK_E_FILE_OPEN, "cannot open tree file for writing");
    const uint64_t gap = h.indexPerLeafOffset - (h.leafExtDataOffset + h.leafExtDataSize);
    std::vector<char> zeros(gap, 0);
    const uint64_t counts[2] = {c->nt, nr};
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(nodes.data(), 16, nn, f) == nn &&
              (ext.empty() || fwrite(ext.data(), sizeof(LeafExtData), ext.size(), f) == ext.size()) &&
              (gap == 0 || fwrite(zeros.data(), 1, gap, f) == gap) &&
              (idx.empty() || fwrite(idx.data(), 4, idx.size(), f) == idx.size()) &&
              (lverts.empty() || fwrite(lverts.data(), 4, lverts.size(), f) == lverts.size()) &&
              fwrite(kLeafTrailer, 1, 8, f) == 8 && fwrite(counts, 8, 2, f) == 2 && fwrite(box, 4, 8, f) == 8 &&
              (nr == 0 || fwrite(refs.data(), 4, nr, f) == nr);
    if (fclose(f) != 0 || !ok) return fail(c, HK_E_FILE_CLOSE, "tree file write failed");
    return HK_OK;
}

hk_status hk_tree_load_file(hk_ctx *c, const char *path, int load_scene) {
    if (!c || !path) return HK_E_ILLEGAL_INPUT;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(c, HK_E_FILE_OPEN, "cannot open tree file");
    fseek(f, 0, SEEK_END);
    const uint64_t fsize = (uint64_t)ftell(f);
    fseek(f, 0, SEEK_SET);
    KdFileHeader h{};
    auto bad = [&](const char *m) {
        fclose(f);
        return fail(c, HK_E_ILLEGAL_INPUT, m);
    };
    if (fread(&h, sizeof(h), 1, f) != 1 || h.headerSize != sizeof(KdFileHeader)) return bad("not a tree file");
    auto in_file = [&](uint64_t off, uint64_t size) { return off <= fsize && size <= fsize - off; };
    if (h.KDTreeSize % 16 || h.leafExtDataSize % sizeof(LeafExtData) || h.indexPerLeafSize % 16 ||
        h.vertexPerLeafSize % 16 || !in_file(h.KDTreeOffset, h.KDTreeSize) ||
        !in_file(h.leafExtDataOffset, h.leafExtDataSize) || !in_file(h.indexPerLeafOffset, h.indexPerLeafSize) ||
        !in_file(h.vertexPerLeafOffset, h.vertexPerLeafSize) || h.KDTreeSize / 16 >= (1u << 29))
        return bad("tree file sizes or offsets out of range");
    const uint32_t nn = (uint32_t)(h.KDTreeSize / 16);
    const size_t nleaf = h.leafExtDataSize / sizeof(LeafExtData);
    std::vector<uint32_t> nodes((size_t)nn * 4);
    std::vector<LeafExtData> ext(nleaf);
    std::vector<uint32_t> idx(h.indexPerLeafSize / 4);
    std::vector<float> lverts(h.vertexPerLeafSize / 4);
    bool ok = fseek(f, (long)h.KDTreeOffset, SEEK_SET) == 0 && fread(nodes.data(), 16, nn, f) == nn &&
              fseek(f, (long)h.leafExtDataOffset, SEEK_SET) == 0 &&
              (nleaf == 0 || fread(ext.data(), sizeof(LeafExtData), nleaf, f) == nleaf) &&
              fseek(f, (long)h.indexPerLeafOffset, SEEK_SET) == 0 &&
              (idx.empty() || fread(idx.data(), 4, idx.size(), f) == idx.size()) &&
              fseek(f, (long)h.vertexPerLeafOffset, SEEK_SET) == 0 &&
              (lverts.empty() || fread(lverts.data(), 4, lverts.size(), f) == lverts.size());
    if (!ok) return bad("tree file truncated");
    // the trailer (written by this library)
    std::vector<uint32_t> refs;
    uint64_t counts[2] = {0, 0};
    float box[8];
    bool have_trailer = false;
    {
        char m[8];
        const uint64_t toff = h.vertexPerLeafOffset + h.vertexPerLeafSize;
        if (toff + 56 <= fsize && fseek(f, (long)toff, SEEK_SET) == 0 && fread(m, 1, 8, f) == 8 &&
            memcmp(m, kLeafTrailer, 8) == 0 && fread(counts, 8, 2, f) == 2 && fread(box, 4, 8, f) == 8 &&
            counts[1] < (1ull << 30) && toff + 56 + counts[1] * 4 <= fsize) {
            refs.resize(counts[1]);
            have_trailer = counts[1] == 0 || fread(refs.data(), 4, counts[1], f) == counts[1];
        }
    }
    fclose(f);
    if (!load_scene) {
        if (!have_trailer) return fail(c, HK_E_ILLEGAL_INPUT, "no leaf polygon list in the file (load_scene = 1)");
        if (counts[0] != c->nt) return fail(c, HK_E_STATE, "the uploaded scene does not match the file");
        return hk_tree_import(c, nodes.data(), nn, refs.data(), (uint32_t)refs.size());
    }
    // the per-leaf triangles become the scene; leaves take consecutive ids
    std::vector<float> verts;
    std::vector<uint32_t> tris, lrefs;
    size_t leaf = 0;
    for (uint32_t i = 0; i < nn; i++) {
        uint32_t *n = &nodes[4 * (size_t)i];
        if (n[0] != kRefLeaf) continue;
        if (leaf >= nleaf) return fail(c, HK_E_ILLEGAL_INPUT, "fewer leaf records than leaves");
        const LeafExtData &e = ext[leaf++];
        const uint32_t cnt = n[2];
        if (cnt > e.indexSize || (uint64_t)e.indexOffset + e.indexSize > idx.size() / 4 ||
            (uint64_t)e.vertexOffset + e.vertxSize > lverts.size() / 4)
            return fail(c, HK_E_ILLEGAL_INPUT, "leaf record out of range");
        const uint32_t vbase = (uint32_t)(verts.size() / 4);
        for (uint32_t k = 0; k < e.vertxSize; k++) {
            const float *v = &lverts[4 * ((size_t)e.vertexOffset + k)];
            verts.insert(verts.end(), {v[0], v[1], v[2], 1.0f});
        }
        n[1] = (uint32_t)lrefs.size();
        for (uint32_t k = 0; k < cnt; k++) {
            const uint32_t *t = &idx[4 * ((size_t)e.indexOffset + k)];
            if (t[0] >= e.vertxSize || t[1] >= e.vertxSize || t[2] >= e.vertxSize)
                return fail(c, HK_E_ILLEGAL_INPUT, "leaf vertex index out of range");
            lrefs.push_back((uint32_t)(tris.size() / 4));
            tris.insert(tris.end(), {vbase + t[0], vbase + t[1], vbase + t[2], 0u});
        }
    }
    if (tris.empty()) return fail(c, HK_E_ILLEGAL_INPUT, "the file holds no triangles");
    hk_status st = hk_scene_upload(c, verts.data(), (uint32_t)(verts.size() / 4), tris.data(), (uint32_t)(tris.size() / 4));
    if (st != HK_OK) return st;
    if (!have_trailer) {
        // bounds of the vertices the triangles use (the padding entries are not)
        for (int k = 0; k < 3; k++) {
            box[k] = INFINITY;
            box[4 + k] = -INFINITY;
        }
        box[3] = box[7] = 0.0f;
        for (size_t i = 0; i < tris.size(); i++) {
            if ((i & 3) == 3) continue;
            const float *v = &verts[4 * (size_t)tris[i]];
            for (int k = 0; k < 3; k++) {
                box[k] = std::min(box[k], v[k]);
                box[4 + k] = std::max(box[4 + k], v[k]);
            }
        }
    }
    if ((st = hk_scene_set_box(c, box)) != HK_OK) return st;
    if ((st = hk_precompute(c)) != HK_OK) return st;
    return hk_tree_import(c, nodes.data(), nn, lrefs.data(), (uint32_t)lrefs.size());
}

}  // extern "C"
