/*
 * hk_oracle.c -- CPU restatement of the reference HulkTracer hot path.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use this library, always as the checker.
 *
 * Every function cites the reference file:line it restates (paths relative to
 * the HulkTracer project root). Float arithmetic keeps the reference's
 * operation order; the 4-lane SSE vector ops of HulkEngine/public/SPMatrix.hpp
 * are restated lane by lane. Compile with -ffp-contract=off (no FMA
 * contraction) and without -ffast-math.
 */
#include "hk_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* SPVector lane arithmetic (HulkEngine/public/SPMatrix.hpp)                 */
/* ------------------------------------------------------------------------ */

/* dot product, SPMatrix.hpp:284-289: r = a*b; r = movehl(r,r) + r;
 * t = shuffle(r,1) + r  ->  (p3 + p1) + (p2 + p0) */
float hko_dot4(const float *a, const float *b) {
    float p0 = a[0] * b[0], p1 = a[1] * b[1], p2 = a[2] * b[2], p3 = a[3] * b[3];
    float r0 = p2 + p0;
    float r1 = p3 + p1;
    return r1 + r0;
}

/* cross product, SPMatrix.hpp:269-278 (w = A.w*B.w) */
static void cross4(const float *A, const float *B, float *o) {
    float m2_0 = A[2] * B[1], m2_1 = A[0] * B[2], m2_2 = A[1] * B[0];
    float m1_0 = A[1] * B[2], m1_1 = A[2] * B[0], m1_2 = A[0] * B[1], m1_3 = A[3] * B[3];
    o[0] = m1_0 - m2_0;
    o[1] = m1_1 - m2_1;
    o[2] = m1_2 - m2_2;
    o[3] = m1_3 - 0.0f;
}

static void sub4(const float *a, const float *b, float *o) {
    for (int k = 0; k < 4; k++) o[k] = a[k] - b[k];
}
static void add4(const float *a, const float *b, float *o) {
    for (int k = 0; k < 4; k++) o[k] = a[k] + b[k];
}
static void scale4(const float *a, float s, float *o) {
    for (int k = 0; k < 4; k++) o[k] = a[k] * s;
}

/* SPVector::normalize, SPMatrix.hpp:302-323: rsqrtps + one Newton step
 * 0.5*r0*(3 - (x*r0)*r0); or IEEE 1/sqrtf for the CUDA path. */
void hko_normalize(float *v, int mode) {
    float len2 = hko_dot4(v, v);
    float t;
    if (mode == HKO_NORM_SSE) {
        __m128 a = _mm_set1_ps(len2);
        __m128 r0 = _mm_rsqrt_ps(a);
        __m128 res = _mm_mul_ps(_mm_mul_ps(_mm_set1_ps(0.5f), r0),
                                _mm_sub_ps(_mm_set1_ps(3.0f), _mm_mul_ps(_mm_mul_ps(a, r0), r0)));
        t = _mm_cvtss_f32(res);
    } else {
        t = 1.0f / sqrtf(len2);
    }
    scale4(v, t, v);
}

/* _mm_min_ps / _mm_max_ps lane semantics: (a < b) ? a : b */
static inline float mn(float a, float b) { return a < b ? a : b; }
static inline float mx(float a, float b) { return a > b ? a : b; }

/* getBoxSurface / getHalfBoxSurface / getBoxVolume, SharedFunctions.hpp:24-44 */
float hko_box_surface(const float *box) {
    float sx = box[4] - box[0], sy = box[5] - box[1], sz = box[6] - box[2];
    return 2.0f * (sx * sy + sz * sy + sx * sz);
}
float hko_box_half_surface(const float *box) {
    float sx = box[4] - box[0], sy = box[5] - box[1], sz = box[6] - box[2];
    return (sx * sy + sz * sy + sx * sz);
}
float hko_box_volume(const float *box) {
    float sx = box[4] - box[0], sy = box[5] - box[1], sz = box[6] - box[2];
    return sx * sy * sz;
}

void hko_free(void *p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Per-triangle cache: KDTreeCPU::buildPolygonCache (KDTreeCPU.cpp:479-507)  */
/* ------------------------------------------------------------------------ */
void hko_build_cache(const float *verts, const uint32_t *tris, uint32_t nt, int norm_mode,
                     float *cache) {
    for (uint32_t i = 0; i < nt; i++) {
        const float *p1 = verts + 4 * (size_t)tris[4 * i];
        const float *p2 = verts + 4 * (size_t)tris[4 * i + 1];
        const float *p3 = verts + 4 * (size_t)tris[4 * i + 2];
        float a1[4], a2[4], a3[4], c1[4], c2[4], c3[4], n[4], s[4];
        sub4(p2, p1, a1);
        sub4(p3, p2, a2);
        sub4(p1, p3, a3);
        cross4(a1, a2, c1);
        cross4(a2, a3, c2);
        cross4(a3, a1, c3);
        add4(c1, c2, s);
        add4(s, c3, n);
        hko_normalize(n, norm_mode);
        float *o = cache + 16 * (size_t)i;
        float e0[4], e1[4];
        sub4(p2, p1, e0);
        sub4(p3, p1, e1);
        memcpy(o, n, 16);
        memcpy(o + 4, e0, 16);
        memcpy(o + 8, e1, 16);
        float e00 = hko_dot4(e0, e0), e01 = hko_dot4(e0, e1), e11 = hko_dot4(e1, e1);
        o[12] = e00;
        o[13] = e01;
        o[14] = e11;
        /* (m_e00 * m_e11) - pow(m_e01, 2): float product, then double pow */
        o[15] = (float)((double)(e00 * e11) - (double)e01 * (double)e01);
    }
}

/* ------------------------------------------------------------------------ */
/* rigid per-part transform (the per-frame update of Intersectable.cpp:      */
/* 116-141, here with one 3x4 matrix per part)                               */
/* ------------------------------------------------------------------------ */
void hko_transform(const float *rest, const uint32_t *part, uint32_t nv, const float *m,
                   float *out) {
    for (uint32_t i = 0; i < nv; i++) {
        const float *M = m + 12 * (size_t)part[i];
        const float *v = rest + 4 * (size_t)i;
        for (int r = 0; r < 3; r++)
            out[4 * i + r] = ((M[4 * r] * v[0] + M[4 * r + 1] * v[1]) + M[4 * r + 2] * v[2]) + M[4 * r + 3];
        out[4 * i + 3] = 1.0f;
    }
}

void hko_scene_box(const float *verts, uint32_t nv, float *box) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = 0; i < nv; i++)
        for (int k = 0; k < 3; k++) {
            lo[k] = fminf(lo[k], verts[4 * i + k]);
            hi[k] = fmaxf(hi[k], verts[4 * i + k]);
        }
    for (int k = 0; k < 3; k++) {
        box[k] = lo[k];
        box[4 + k] = hi[k];
    }
    box[3] = 1.0f;
    box[7] = 1.0f;
}

/* castRay (GLVisitorCPUTrace.cpp:201-216): dir = (lowerLeft + vf*(x/W) + hf*(y/H)) - from */
void hko_camera_rays(const float *cam, uint32_t w, uint32_t h, int mode, float *rays) {
    const float *from = cam, *vf = cam + 4, *hf = cam + 8, *ll = cam + 12;
    for (uint32_t y = 0; y < h; y++)
        for (uint32_t x = 0; x < w; x++) {
            float u = (float)x / (float)w, v = (float)y / (float)h;
            float a[4], b[4], c[4], d[4];
            scale4(vf, u, a);
            add4(ll, a, b);
            scale4(hf, v, a);
            add4(b, a, c);
            sub4(c, from, d);
            hko_normalize(d, mode);
            float *r = rays + 8 * ((size_t)y * w + x);
            memcpy(r, from, 16);
            memcpy(r + 4, d, 16);
        }
}

/* ------------------------------------------------------------------------ */
/* SAH NlogN build (KDTreeSAH.cpp:247-521, KDTreeCPU.cpp:46-57,450-477)       */
/* ------------------------------------------------------------------------ */
enum { EV_BEGIN = 0, EV_COPLANAR = 1, EV_END = 2 };
enum { REL_ABOVE = 0, REL_BELOW = 1, REL_INTERSECT = 2, REL_COPLANAR = 3 };

typedef struct {
    float value;
    uint32_t marker;
    uint32_t poly;
} cand_t;

typedef struct {
    uint32_t *a;
    size_t n, cap;
} uvec;
typedef struct {
    cand_t *a;
    size_t n, cap;
} cvec;

static void uv_push(uvec *v, uint32_t x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 16;
        v->a = (uint32_t *)realloc(v->a, v->cap * sizeof(uint32_t));
    }
    v->a[v->n++] = x;
}
static void cv_push(cvec *v, cand_t x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 16;
        v->a = (cand_t *)realloc(v->a, v->cap * sizeof(cand_t));
    }
    v->a[v->n++] = x;
}
static void cv_reserve(cvec *v, size_t cap) {
    if (cap > v->cap) {
        v->cap = cap;
        v->a = (cand_t *)realloc(v->a, v->cap * sizeof(cand_t));
    }
}

typedef struct {
    float box[8];
    float surface;
    uint32_t depth;
    uint32_t node;
    size_t eval;
    uvec polys;
    cvec cands[3];
} split_iter;

typedef struct {
    const float *verts;
    const uint32_t *tris;
    hko_sah_params p;
    uvec nodes;     /* 4 words per node */
    uvec leafpolys;
    uint32_t leaf_count;
    uint8_t *rel;   /* m_pPolyRelations */
} sah_ctx;

static uint32_t new_node(sah_ctx *c) {
    uint32_t idx = (uint32_t)(c->nodes.n / 4);
    for (int k = 0; k < 4; k++) uv_push(&c->nodes, 0);
    return idx;
}

static int cmp_cand(const void *x, const void *y) {
    float a = ((const cand_t *)x)->value, b = ((const cand_t *)y)->value;
    return (a < b) ? -1 : (b < a) ? 1 : 0;
}

/* KDTreeCPU::checkPolygonToAAPlane, KDTreeCPU.cpp:450-477 */
static int poly_to_plane(const sah_ctx *c, uint32_t axis, float value, uint32_t poly) {
    float c1 = c->verts[4 * (size_t)c->tris[4 * poly] + axis];
    float c2 = c->verts[4 * (size_t)c->tris[4 * poly + 1] + axis];
    float c3 = c->verts[4 * (size_t)c->tris[4 * poly + 2] + axis];
    if ((c1 == value) & (c2 == value) & (c3 == value)) return REL_COPLANAR;
    if ((c1 >= value) & (c2 >= value) & (c3 >= value)) return REL_ABOVE;
    if ((c1 <= value) & (c2 <= value) & (c3 <= value)) return REL_BELOW;
    return REL_INTERSECT;
}

/* KDTreeCPU::makeLeafNode, KDTreeCPU.cpp:46-57 */
static void make_leaf(sah_ctx *c, split_iter *it) {
    uint32_t *n = c->nodes.a + 4 * (size_t)it->node;
    n[0] = HKO_LEAF;
    n[3] = c->leaf_count++;
    n[2] = (uint32_t)it->polys.n;
    n[1] = (uint32_t)c->leafpolys.n;
    for (size_t i = 0; i < it->polys.n; i++) uv_push(&c->leafpolys, it->polys.a[i]);
}

static void free_iter(split_iter *it) {
    free(it->polys.a);
    for (int j = 0; j < 3; j++) free(it->cands[j].a);
    memset(it, 0, sizeof(*it));
}

/* KDTreeCPU::buildNodeSAHNlogN, KDTreeSAH.cpp:313-521 */
static void build_node_nlogn(sah_ctx *c, split_iter *it) {
    const float Ct = c->p.ct, Ci = c->p.ci;
    if (it->depth >= c->p.max_depth || it->polys.n < c->p.leaf_below) { /* :316-321 */
        make_leaf(c, it);
        return;
    }
    float bestScore = FLT_MAX, bestUpper = 0, bestLower = 0, bestValue = 0;
    uint32_t bestDim = 0;
    float dim[4];
    sub4(it->box + 4, it->box, dim);
    float invBoxSurface = 1.0f / it->surface;
    for (uint32_t j = 0; j < 3; j++) { /* :338-405 */
        uint32_t below = 0, coplanar = 0, above = 0;
        uint32_t counters[3] = {0, 0, 0};
        uint32_t plusPrev = 0, copPrev = 0;
        float x = dim[(j + 1) % 3], y = dim[(j + 2) % 3];
        float XplusY = x + y;
        float planeArea = x * y;
        cvec *cv = &it->cands[j];
        size_t i = 0;
        int first = 1;
        while (i < cv->n) {
            float cur = cv->a[i].value;
            while (i < cv->n && cv->a[i].value == cur) {
                counters[cv->a[i].marker]++;
                i++;
            }
            below = below + copPrev + plusPrev;
            coplanar = copPrev;
            above = above - counters[EV_COPLANAR] - counters[EV_END];
            if (first) {
                below = 0;
                coplanar = counters[EV_COPLANAR];
                above = ((uint32_t)it->eval) - counters[EV_COPLANAR];
                first = 0;
            }
            plusPrev = counters[EV_BEGIN];
            copPrev = counters[EV_COPLANAR];
            counters[0] = counters[1] = counters[2] = 0;
            float upper = planeArea + (it->box[4 + j] - cur) * (XplusY);
            float lower = planeArea + (cur - it->box[j]) * (XplusY);
            float costBelow = lower * (float)below;
            float costAbove = upper * (float)above;
            float costIntersect = planeArea * (float)coplanar;
            float score = Ct + Ci * ((costIntersect + costBelow + costAbove) * invBoxSurface);
            if (score < bestScore) {
                bestScore = score;
                bestValue = cur;
                bestDim = j;
                bestUpper = upper;
                bestLower = lower;
            }
        }
    }
    float leafcost = Ci * (float)it->eval; /* :407-413 */
    if (bestScore >= leafcost) {
        make_leaf(c, it);
        return;
    }
    uint32_t *nd = c->nodes.a + 4 * (size_t)it->node;
    memcpy(&nd[3], &bestValue, 4);
    nd[0] = bestDim | HKO_JUNCTION;

    split_iter A, B; /* above, below */
    memset(&A, 0, sizeof A);
    memset(&B, 0, sizeof B);
    for (size_t i = 0; i < it->polys.n; i++) { /* :426-447 */
        uint32_t poly = it->polys.a[i];
        int r = poly_to_plane(c, bestDim, bestValue, poly);
        c->rel[poly] = (uint8_t)r;
        if (r == REL_ABOVE) uv_push(&A.polys, poly);
        else if (r == REL_BELOW) uv_push(&B.polys, poly);
        else {
            uv_push(&A.polys, poly);
            uv_push(&B.polys, poly);
        }
    }
    for (uint32_t j = 0; j < 3; j++) { /* :456-489 */
        cv_reserve(&A.cands[j], it->cands[j].n);
        cv_reserve(&B.cands[j], it->cands[j].n);
        for (size_t i = 0; i < it->cands[j].n; i++) {
            cand_t e = it->cands[j].a[i];
            switch (c->rel[e.poly]) {
            case REL_ABOVE: cv_push(&A.cands[j], e); break;
            case REL_BELOW: cv_push(&B.cands[j], e); break;
            case REL_INTERSECT:
                if (j == bestDim) {
                    cand_t t = e;
                    t.value = (bestValue > e.value) ? bestValue : e.value; /* MAX */
                    cv_push(&A.cands[j], t);
                    t.value = (bestValue < e.value) ? bestValue : e.value; /* MIN */
                    cv_push(&B.cands[j], t);
                } else {
                    cv_push(&A.cands[j], e);
                    cv_push(&B.cands[j], e);
                }
                break;
            default: break; /* co-planar polygons leave the candidate lists */
            }
        }
        A.eval += A.cands[j].n;
        B.eval += B.cands[j].n;
    }
    A.eval /= 6;
    B.eval /= 6;
    /* the parent's lists are no longer needed */
    uint32_t depth = it->depth, node = it->node;
    float box[8];
    memcpy(box, it->box, sizeof box);
    free_iter(it);

    if (A.polys.n > 0) { /* :494-507 */
        A.depth = depth + 1;
        memcpy(A.box, box, sizeof box);
        A.surface = bestUpper;
        A.box[bestDim] = bestValue;
        uint32_t idx = new_node(c);
        A.node = idx;
        c->nodes.a[4 * (size_t)node + 1] = idx;
        build_node_nlogn(c, &A);
    }
    free_iter(&A);
    if (B.polys.n > 0) { /* :508-520 */
        B.depth = depth + 1;
        memcpy(B.box, box, sizeof box);
        B.surface = bestLower;
        B.box[4 + bestDim] = bestValue;
        uint32_t idx = new_node(c);
        B.node = idx;
        c->nodes.a[4 * (size_t)node + 2] = idx;
        build_node_nlogn(c, &B);
    }
    free_iter(&B);
}

/* KDTreeCPU::buildKDTree + buildKDTreeSAH_NlogN, KDTreeCPU.cpp:61-94,
 * KDTreeSAH.cpp:247-311 */
int hko_build_sah_nlogn(const float *verts, const uint32_t *tris, uint32_t nt, const float *box,
                        const hko_sah_params *p, uint32_t **nodes_out, uint32_t *nn_out,
                        uint32_t **refs_out, uint32_t *nr_out) {
    sah_ctx c;
    memset(&c, 0, sizeof c);
    c.verts = verts;
    c.tris = tris;
    c.p = *p;
    c.rel = (uint8_t *)calloc(nt ? nt : 1, 1);
    new_node(&c); /* root (buildKDTree pushes it, KDTreeCPU.cpp:74-75) */
    split_iter root;
    memset(&root, 0, sizeof root);
    for (uint32_t i = 0; i < nt; i++) uv_push(&root.polys, i);
    memcpy(root.box, box, 8 * sizeof(float));
    root.surface = hko_box_surface(box);
    for (uint32_t i = 0; i < nt; i += p->reduction) {
        root.eval++;
        const float *p1 = verts + 4 * (size_t)tris[4 * i];
        const float *p2 = verts + 4 * (size_t)tris[4 * i + 1];
        const float *p3 = verts + 4 * (size_t)tris[4 * i + 2];
        for (uint32_t j = 0; j < 3; j++) {
            float lo = mn(mn(p1[j], p2[j]), p3[j]);
            float hi = mx(mx(p1[j], p2[j]), p3[j]);
            cand_t e;
            e.poly = i;
            e.marker = EV_BEGIN;
            e.value = lo;
            cv_push(&root.cands[j], e);
            e.marker = EV_END;
            e.value = hi;
            cv_push(&root.cands[j], e);
        }
    }
    for (int j = 0; j < 3; j++)
        if (root.cands[j].n) qsort(root.cands[j].a, root.cands[j].n, sizeof(cand_t), cmp_cand);
    build_node_nlogn(&c, &root);
    free_iter(&root);
    free(c.rel);
    *nodes_out = c.nodes.a;
    *nn_out = (uint32_t)(c.nodes.n / 4);
    *refs_out = c.leafpolys.a ? c.leafpolys.a : (uint32_t *)malloc(4);
    *nr_out = (uint32_t)c.leafpolys.n;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* SAH with per-node re-sampling (--treeType=SAH): KDTreeCPU::buildKDTreeSAH  */
/* + buildNodeSAH, KDTreeSAH.cpp:9-244                                        */
/* ------------------------------------------------------------------------ */
/* KDTreeCPU::buildNodeSAH, KDTreeSAH.cpp:35-244. Every node re-samples its
 * own polygon list (every reduction-th entry, in list order), clips each
 * sampled triangle's bounds to the node box, makes a co-planar candidate
 * where the clipped extent is at most FLT_EPSILON and begin / end candidates
 * otherwise, sorts by value and sweeps with the same counters as the NlogN
 * build; the counts start from list size / reduction (integer division) and
 * run in unsigned 32-bit arithmetic, as there. */
static void build_node_resort(sah_ctx *c, split_iter *it) {
    const float Ct = c->p.ct, Ci = c->p.ci;
    if (it->depth >= c->p.max_depth || it->polys.n < c->p.leaf_below) { /* :38-43 */
        make_leaf(c, it);
        return;
    }
    for (size_t i = 0; i < it->polys.n; i += c->p.reduction) { /* :51-82 */
        uint32_t poly = it->polys.a[i];
        const float *p1 = c->verts + 4 * (size_t)c->tris[4 * poly];
        const float *p2 = c->verts + 4 * (size_t)c->tris[4 * poly + 1];
        const float *p3 = c->verts + 4 * (size_t)c->tris[4 * poly + 2];
        for (uint32_t j = 0; j < 3; j++) {
            float lo = mn(mn(p1[j], p2[j]), p3[j]);
            float hi = mx(mx(p1[j], p2[j]), p3[j]);
            lo = mx(lo, it->box[j]);
            hi = mn(hi, it->box[4 + j]);
            cand_t e;
            e.poly = poly;
            if (fabsf(lo - hi) <= FLT_EPSILON) {
                e.marker = EV_COPLANAR;
                e.value = lo;
                cv_push(&it->cands[j], e);
            } else {
                e.marker = EV_BEGIN;
                e.value = lo;
                cv_push(&it->cands[j], e);
                e.marker = EV_END;
                e.value = hi;
                cv_push(&it->cands[j], e);
            }
        }
    }
    const uint32_t sampled_count = (uint32_t)(it->polys.n / c->p.reduction);
    float bestScore = FLT_MAX, bestUpper = 0, bestLower = 0, bestValue = 0;
    uint32_t bestDim = 0;
    float dim[4];
    sub4(it->box + 4, it->box, dim);
    float invBoxSurface = 1.0f / it->surface;
    for (uint32_t j = 0; j < 3; j++) { /* :96-183 */
        cvec *cv = &it->cands[j];
        if (cv->n) qsort(cv->a, cv->n, sizeof(cand_t), cmp_cand);
        uint32_t below = 0, coplanar = 0, above = 0;
        uint32_t counters[3] = {0, 0, 0};
        uint32_t plusPrev = 0, copPrev = 0;
        float x = dim[(j + 1) % 3], y = dim[(j + 2) % 3];
        float XplusY = x + y;
        float planeArea = x * y;
        size_t i = 0;
        int first = 1;
        while (i < cv->n) {
            float cur = cv->a[i].value;
            while (i < cv->n && cv->a[i].value == cur) {
                counters[cv->a[i].marker]++;
                i++;
            }
            below = below + copPrev + plusPrev;
            coplanar = copPrev;
            above = above - counters[EV_COPLANAR] - counters[EV_END];
            if (first) {
                below = 0;
                coplanar = counters[EV_COPLANAR];
                above = sampled_count - counters[EV_COPLANAR];
                first = 0;
            }
            plusPrev = counters[EV_BEGIN];
            copPrev = counters[EV_COPLANAR];
            counters[0] = counters[1] = counters[2] = 0;
            float upper = planeArea + (it->box[4 + j] - cur) * (XplusY);
            float lower = planeArea + (cur - it->box[j]) * (XplusY);
            float costBelow = lower * (float)below;
            float costAbove = upper * (float)above;
            float costIntersect = planeArea * (float)coplanar;
            float score = Ct + Ci * ((costIntersect + costBelow + costAbove) * invBoxSurface);
            if (score < bestScore) {
                bestScore = score;
                bestValue = cur;
                bestDim = j;
                bestUpper = upper;
                bestLower = lower;
            }
        }
    }
    for (int j = 0; j < 3; j++) {
        free(it->cands[j].a);
        memset(&it->cands[j], 0, sizeof it->cands[j]);
    }
    float leafcost = Ci * (float)sampled_count; /* :186-191 */
    if (bestScore >= leafcost) {
        make_leaf(c, it);
        return;
    }
    uint32_t *nd = c->nodes.a + 4 * (size_t)it->node;
    memcpy(&nd[3], &bestValue, 4);
    nd[0] = bestDim | HKO_JUNCTION;
    split_iter A, B; /* above, below */
    memset(&A, 0, sizeof A);
    memset(&B, 0, sizeof B);
    for (size_t i = 0; i < it->polys.n; i++) { /* :203-222 */
        uint32_t poly = it->polys.a[i];
        int r = poly_to_plane(c, bestDim, bestValue, poly);
        if (r == REL_ABOVE) uv_push(&A.polys, poly);
        else if (r == REL_BELOW) uv_push(&B.polys, poly);
        else {
            uv_push(&A.polys, poly);
            uv_push(&B.polys, poly);
        }
    }
    uint32_t depth = it->depth, node = it->node;
    float box[8];
    memcpy(box, it->box, sizeof box);
    free_iter(it);
    if (A.polys.n > 0) { /* :226-238 */
        A.depth = depth + 1;
        memcpy(A.box, box, sizeof box);
        A.surface = bestUpper;
        A.box[bestDim] = bestValue;
        uint32_t idx = new_node(c);
        A.node = idx;
        c->nodes.a[4 * (size_t)node + 1] = idx;
        build_node_resort(c, &A);
    }
    free_iter(&A);
    if (B.polys.n > 0) { /* :239-251 */
        B.depth = depth + 1;
        memcpy(B.box, box, sizeof box);
        B.surface = bestLower;
        B.box[4 + bestDim] = bestValue;
        uint32_t idx = new_node(c);
        B.node = idx;
        c->nodes.a[4 * (size_t)node + 2] = idx;
        build_node_resort(c, &B);
    }
    free_iter(&B);
}

/* KDTreeCPU::buildKDTree + buildKDTreeSAH, KDTreeCPU.cpp:61-94,
 * KDTreeSAH.cpp:9-32. buildKDTree has pushed the root and buildKDTreeSAH
 * pushes a second default node that nothing links to (index 1); the root's
 * box surface is the half surface here (getHalfBoxSurface). */
int hko_build_sah_resort(const float *verts, const uint32_t *tris, uint32_t nt, const float *box,
                         const hko_sah_params *p, uint32_t **nodes_out, uint32_t *nn_out,
                         uint32_t **refs_out, uint32_t *nr_out) {
    sah_ctx c;
    memset(&c, 0, sizeof c);
    c.verts = verts;
    c.tris = tris;
    c.p = *p;
    new_node(&c);
    new_node(&c);
    split_iter root;
    memset(&root, 0, sizeof root);
    for (uint32_t i = 0; i < nt; i++) uv_push(&root.polys, i);
    memcpy(root.box, box, 8 * sizeof(float));
    root.surface = hko_box_half_surface(box);
    build_node_resort(&c, &root);
    free_iter(&root);
    *nodes_out = c.nodes.a;
    *nn_out = (uint32_t)(c.nodes.n / 4);
    *refs_out = c.leafpolys.a ? c.leafpolys.a : (uint32_t *)malloc(4);
    *nr_out = (uint32_t)c.leafpolys.n;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* tree cost and node boxes                                                  */
/* ------------------------------------------------------------------------ */
void hko_node_boxes(const uint32_t *nodes, uint32_t nn, const float *box, float *out) {
    /* parents precede children in both the reference DFS order and the BFS
     * order of the GPU builder, so one forward pass suffices */
    memset(out, 0, (size_t)nn * 8 * sizeof(float));
    memcpy(out, box, 8 * sizeof(float));
    uint8_t *seen = (uint8_t *)calloc(nn ? nn : 1, 1);
    seen[0] = 1;
    for (uint32_t i = 0; i < nn; i++) {
        const uint32_t *n = nodes + 4 * (size_t)i;
        if (!seen[i] || !(n[0] & HKO_JUNCTION)) continue;
        uint32_t axis = n[0] & 3;
        float plane;
        memcpy(&plane, &n[3], 4);
        uint32_t above = n[1], below = n[2];
        if (above && above < nn) {
            memcpy(out + 8 * (size_t)above, out + 8 * (size_t)i, 32);
            out[8 * (size_t)above + axis] = plane;
            seen[above] = 1;
        }
        if (below && below < nn) {
            memcpy(out + 8 * (size_t)below, out + 8 * (size_t)i, 32);
            out[8 * (size_t)below + 4 + axis] = plane;
            seen[below] = 1;
        }
    }
    free(seen);
}

double hko_tree_cost(const uint32_t *nodes, uint32_t nn, const float *box, double ct, double ci) {
    float *b = (float *)malloc((size_t)(nn ? nn : 1) * 8 * sizeof(float));
    hko_node_boxes(nodes, nn, box, b);
    /* reachability from the root */
    uint8_t *reach = (uint8_t *)calloc(nn ? nn : 1, 1);
    reach[0] = 1;
    double aroot = 0.0, cost = 0.0;
    {
        double sx = (double)box[4] - box[0], sy = (double)box[5] - box[1], sz = (double)box[6] - box[2];
        aroot = 2.0 * (sx * sy + sy * sz + sx * sz);
    }
    for (uint32_t i = 0; i < nn; i++) {
        if (!reach[i]) continue;
        const uint32_t *n = nodes + 4 * (size_t)i;
        const float *q = b + 8 * (size_t)i;
        double sx = (double)q[4] - q[0], sy = (double)q[5] - q[1], sz = (double)q[6] - q[2];
        double a = 2.0 * (sx * sy + sy * sz + sx * sz);
        if (n[0] & HKO_JUNCTION) {
            cost += ct * a / aroot;
            if (n[1] && n[1] < nn) reach[n[1]] = 1;
            if (n[2] && n[2] < nn) reach[n[2]] = 1;
        } else {
            cost += ci * (double)n[2] * a / aroot;
        }
    }
    free(reach);
    free(b);
    return cost;
}

/* ------------------------------------------------------------------------ */
/* ray traversal                                                              */
/* ------------------------------------------------------------------------ */

/* isRayToAbovePlane / isRayToBelowPlane, SharedFunctions.hpp:154-220 */
static int above_plane(float p0, float d0, float e0, float *t0, float *t1) {
    if (d0 > 0) {
        float ti = (e0 - p0) / d0;
        if (ti > *t1) return 0;
        if (ti > *t0) *t0 = ti;
        return 1;
    } else if (d0 < 0) {
        float ti = (e0 - p0) / d0;
        if (ti < *t0) return 0;
        if (ti < *t1) *t1 = ti;
        return 1;
    }
    return e0 < p0;
}
static int below_plane(float p0, float d0, float e0, float *t0, float *t1) {
    if (d0 < 0) {
        float ti = (e0 - p0) / d0;
        if (ti > *t1) return 0;
        if (ti > *t0) *t0 = ti;
        return 1;
    } else if (d0 > 0) {
        float ti = (e0 - p0) / d0;
        if (ti < *t0) return 0;
        if (ti < *t1) *t1 = ti;
        return 1;
    }
    return e0 > p0;
}
/* checkRayToBoundingBoxGPU, SharedFunctions.hpp:245-264 (non short-circuit &) */
static int ray_box(const float *box, const float *o, const float *d, float *ts, float *te) {
    float t0 = 0.0f, t1 = FLT_MAX;
    int r = above_plane(o[0], d[0], box[0], &t0, &t1);
    r &= below_plane(o[0], d[0], box[4], &t0, &t1);
    r &= above_plane(o[1], d[1], box[1], &t0, &t1);
    r &= below_plane(o[1], d[1], box[5], &t0, &t1);
    r &= above_plane(o[2], d[2], box[2], &t0, &t1);
    r &= below_plane(o[2], d[2], box[6], &t0, &t1);
    if (r) {
        *te = t1;
        *ts = t0;
    }
    return r;
}

typedef struct {
    float t;
    float n[4];
    float pos[4];
    int32_t id;
} hit_t;

/* checkRayToPolyACC, SharedFunctions.hpp:105-150 */
static int isect_acc(const float *o, const float *d, const float *p1, const float *cache, float *t_out,
                     float *pos_out) {
    float denum = hko_dot4(cache, d);
    if (fabsf(denum) < FLT_EPSILON) return 0;
    denum = 1.0f / denum;
    float v[4];
    sub4(p1, o, v);
    float time = hko_dot4(cache, v) * denum;
    if (time < 0) return 0;
    float hp[4], hq[4];
    for (int k = 0; k < 4; k++) hp[k] = o[k] + d[k] * time;
    sub4(hp, p1, hq);
    float q0 = hko_dot4(cache + 4, hq), q1 = hko_dot4(cache + 8, hq);
    float e00 = cache[12], e01 = cache[13], e11 = cache[14], det = cache[15];
    float s1 = (e11 * q0) - (e01 * q1);
    float s2 = (e00 * q1) - (e01 * q0);
    if (s1 >= 0 && s2 >= 0 && (s1 + s2) <= det) {
        *t_out = time;
        memcpy(pos_out, hp, 16);
        return 1;
    }
    return 0;
}

/* checkRayToPoly, SharedFunctions.hpp:47-103 -- the form the reference's
 * OpenCL kernels call (GPU_common.cl:46-72, GPUTrace_bruteforce.cl:30-42):
 * the normal recomputed per test, normalize(e0 x e1 + e1 x e2 + e2 x e0), and
 * det, s1, s2 by fused multiply-add. Restated with IEEE single precision in
 * the source's order (OpenCL lets an implementation relax division, sqrt and
 * dot; this is the correctly rounded reading): dot over four lanes as
 * ((x0 y0 + x1 y1) + x2 y2) + x3 y3, cross with w = 0, normalize as
 * v * (1 / sqrt(v . v)), pow(e01, 2) as the rounded square. */
static float dot4_seq(const float *a, const float *b) {
    return ((a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]) + a[3] * b[3];
}

static void cross_w0(const float *a, const float *b, float *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
    o[3] = 0.0f;
}

static int isect_poly(const float *o, const float *d, const float *p1, const float *p2, const float *p3,
                      float *t_out, float *pos_out) {
    float e0[4], e1[4], e2[4], c0[4], c1[4], c2[4], n[4];
    sub4(p2, p1, e0);
    sub4(p3, p1, e1);
    sub4(p3, p2, e2);
    cross_w0(e0, e1, c0);
    cross_w0(e1, e2, c1);
    cross_w0(e2, e0, c2);
    for (int k = 0; k < 4; k++) n[k] = (c0[k] + c1[k]) + c2[k];
    const float inv = 1.0f / sqrtf(dot4_seq(n, n));
    for (int k = 0; k < 4; k++) n[k] = n[k] * inv;
    float denum = dot4_seq(n, d);
    if (fabsf(denum) < FLT_EPSILON) return 0;
    denum = 1.0f / denum;
    float v[4];
    sub4(p1, o, v);
    float time = dot4_seq(n, v) * denum;
    if (time < 0) return 0;
    float hp[4], hq[4];
    for (int k = 0; k < 4; k++) hp[k] = o[k] + d[k] * time;
    sub4(hp, p1, hq);
    float q0 = dot4_seq(e0, hq), q1 = dot4_seq(e1, hq);
    float e00 = dot4_seq(e0, e0), e01 = dot4_seq(e0, e1), e11 = dot4_seq(e1, e1);
    float det = fmaf(e00, e11, -(e01 * e01));
    float s1 = fmaf(e11, q0, -(e01 * q1));
    float s2 = fmaf(e00, q1, -(e01 * q0));
    if (s1 >= 0 && s2 >= 0 && (s1 + s2) <= det) {
        *t_out = time;
        memcpy(pos_out, hp, 16);
        return 1;
    }
    return 0;
}

/* which intersection form the traversals use: 0 checkRayToPolyACC over the
 * tree's cache (the CPU path), 1 checkRayToPoly from the vertices */
static int g_isect_form = 0;
void hko_set_isect_form(int form) { g_isect_form = form; }

static int isect_tri_form(const hko_tree *t, uint32_t poly, const float *o, const float *d, float *tt, float *pos) {
    const float *p1 = t->verts + 4 * (size_t)t->tris[4 * poly];
    if (g_isect_form == 1) {
        const float *p2 = t->verts + 4 * (size_t)t->tris[4 * poly + 1];
        const float *p3 = t->verts + 4 * (size_t)t->tris[4 * poly + 2];
        return isect_poly(o, d, p1, p2, p3, tt, pos);
    }
    return isect_acc(o, d, p1, t->cache + 16 * (size_t)poly, tt, pos);
}

/* KDTreeCPU::testNodePolygons, KDTreeCPU.cpp:255-283 */
static int test_leaf(const hko_tree *t, const uint32_t *node, const float *o, const float *d, hit_t *hit,
                     hko_counters *cnt) {
    int ret = 0;
    uint32_t end = node[2] + node[1];
    for (uint32_t i = node[1]; i < end; i++) {
        uint32_t poly = t->refs[i];
        cnt->refs++;
        cnt->tests++;
        float tt, pos[4];
        if (isect_tri_form(t, poly, o, d, &tt, pos)) {
            if (tt < hit->t) {
                ret = 1;
                hit->t = tt;
                memcpy(hit->pos, pos, 16);
                memcpy(hit->n, t->cache + 16 * (size_t)poly, 16);
                hit->id = (int32_t)poly;
            }
        }
    }
    return ret;
}

static inline float node_plane(const uint32_t *n) {
    float f;
    memcpy(&f, &n[3], 4);
    return f;
}

/* KDTreeCPU::searchKDTreeStackless, KDTreeCPU.cpp:363-447 (ring of depth D;
 * the reference CPU uses 5, the OpenCL short-stack kernels 6) */
static int search_shortstack(const hko_tree *t, const float *o, const float *d, float ts, float te,
                             int D, hit_t *hit, hko_counters *cnt) {
    struct { float s, e; uint32_t node; } frame[64];
    memset(frame, 0, sizeof frame);
    int size = 0, idx = 0;
    float tmin = ts, tmax = ts;
    int ret = 0;
    float inv[4];
    for (int k = 0; k < 4; k++) inv[k] = 1.0f / d[k];
    const uint32_t *N = t->nodes;
    uint32_t cur = 0;
    while (tmax < te) {
        if (size == 0) {
            cur = 0;
            tmin = tmax;
            tmax = te;
        } else {
            --size;
            --idx;
            if (idx == -1) idx += D;
            tmin = frame[idx].s;
            tmax = frame[idx].e;
            cur = frame[idx].node;
        }
        while (N[4 * (size_t)cur] & HKO_JUNCTION) {
            cnt->nodes++;
            const uint32_t *n = N + 4 * (size_t)cur;
            uint32_t axis = n[0] & 3;
            float dc = d[axis], rs = o[axis], pl = node_plane(n);
            float split = (pl - rs) * inv[axis];
            uint32_t first = n[1], second = n[2];
            if (rs < pl || (rs == pl && dc <= 0)) {
                first = n[2];
                second = n[1];
            }
            if (split >= tmax || split <= 0) {
                cur = first;
            } else if (split <= tmin) {
                cur = second;
            } else {
                frame[idx].s = split;
                frame[idx].e = tmax;
                frame[idx].node = second;
                idx = (idx + 1) % D;
                size++;
                size = size > D ? D : size;
                cur = first;
                tmax = split;
            }
            if (cur == 0) break;
        }
        if (N[4 * (size_t)cur] & HKO_LEAF) {
            cnt->nodes++;
            ret |= test_leaf(t, N + 4 * (size_t)cur, o, d, hit, cnt);
            if (hit->t < tmax) break;
        }
    }
    return ret;
}

/* KDTreeCPU::searchKDTree, KDTreeCPU.cpp:285-361 (== GPUTrace.cl:6-90) */
static int search_fullstack(const hko_tree *t, const float *o, const float *d, float ts, float te,
                            hit_t *hit, hko_counters *cnt) {
    struct { float s, e; uint32_t node; } todo[64];
    int ret = 0;
    float tmin = ts, tmax = te;
    uint32_t todoCount = 0;
    float inv[4];
    for (int k = 0; k < 4; k++) inv[k] = 1.0f / d[k];
    const uint32_t *N = t->nodes;
    uint32_t cur = 0;
    do {
        if (hit->t < tmin) break;
        const uint32_t *n = N + 4 * (size_t)cur;
        cnt->nodes++;
        if (n[0] & HKO_LEAF) {
            ret |= test_leaf(t, n, o, d, hit, cnt);
            cur = 0;
        } else {
            uint32_t axis = n[0] & 3;
            float dc = d[axis], rs = o[axis], pl = node_plane(n);
            float split = (pl - rs) * inv[axis];
            uint32_t first = n[1], second = n[2];
            if (rs < pl || (rs == pl && dc <= 0)) {
                first = n[2];
                second = n[1];
            }
            if (split > tmax || split <= 0) {
                cur = first;
            } else if (split < tmin) {
                cur = second;
            } else {
                if (second != 0 && todoCount < 64) {
                    todo[todoCount].node = second;
                    todo[todoCount].s = split;
                    todo[todoCount].e = tmax;
                    todoCount++;
                }
                cur = first;
                tmax = split;
            }
        }
        if (cur == 0 && todoCount > 0) {
            todoCount--;
            tmin = todo[todoCount].s;
            tmax = todo[todoCount].e;
            cur = todo[todoCount].node;
        }
    } while (cur != 0);
    return ret;
}

/* kd-restart, GPUTrace_stackless.cl:53-117 with every leaf resident: the
 * ThreadContext starts zeroed, so the first descent uses tmin = tmax = 0;
 * there is no early exit after a leaf unless `early` is set. */
static int search_restart(const hko_tree *t, const float *o, const float *d, float ts, float te,
                          int early, hit_t *hit, hko_counters *cnt) {
    (void)ts;
    int ret = 0;
    float inv[4];
    for (int k = 0; k < 4; k++) inv[k] = 1.0f / d[k];
    const uint32_t *N = t->nodes;
    float tmax = 0.0f, tmin = 0.0f;
    if (hit->t < tmax) return 0;
    while (tmax < te) {
        tmin = tmax;
        tmax = te;
        uint32_t cur = 0;
        while (N[4 * (size_t)cur] & HKO_JUNCTION) {
            cnt->nodes++;
            const uint32_t *n = N + 4 * (size_t)cur;
            uint32_t axis = n[0] & 3;
            float rs = o[axis], dc = d[axis], iv = inv[axis], pl = node_plane(n);
            float split = (pl - rs) * (iv);
            uint32_t first = n[1], second = n[2];
            if (rs < pl || (rs == pl && dc <= 0)) {
                first = n[2];
                second = n[1];
            }
            if (split >= tmax || split <= 0) {
                cur = first;
            } else if (split <= tmin) {
                cur = second;
            } else {
                cur = first;
                tmax = split;
            }
            if (cur == 0) break;
        }
        if (N[4 * (size_t)cur] & HKO_LEAF) {
            cnt->nodes++;
            ret |= test_leaf(t, N + 4 * (size_t)cur, o, d, hit, cnt);
            if (early && hit->t < tmax) break;
        }
    }
    return ret;
}

static int search_ropes(const hko_tree *t, const float *o, const float *d, float ts, float te,
                        hit_t *hit, hko_counters *cnt);

int hko_trace_one(const hko_tree *t, int variant, int D, const float *ray, float *out,
                  hko_counters *cnt) {
    const float *o = ray, *d = ray + 4;
    hit_t hit;
    hit.t = INFINITY;
    hit.id = -1;
    memset(hit.n, 0, sizeof hit.n);
    memset(hit.pos, 0, sizeof hit.pos);
    int r = 0;
    if (variant == HKO_BRUTE) {
        /* GPUTrace_bruteforce.cl:30-42 over the cached intersection form */
        for (uint32_t i = 0; i < t->nt; i++) {
            float tt, pos[4];
            cnt->tests++;
            if (isect_tri_form(t, i, o, d, &tt, pos)) {
                r = 1;
                if (tt < hit.t) {
                    hit.t = tt;
                    memcpy(hit.pos, pos, 16);
                    memcpy(hit.n, t->cache + 16 * (size_t)i, 16);
                    hit.id = (int32_t)i;
                }
            }
        }
    } else {
        /* KDTreeCPU::checkCollision, KDTreeCPU.cpp:230-253 */
        float ts = 0.0f, te = INFINITY;
        if (ray_box(t->box, o, d, &ts, &te)) {
            switch (variant) {
            case HKO_SHORTSTACK: r = search_shortstack(t, o, d, ts, te, D, &hit, cnt); break;
            case HKO_FULLSTACK: r = search_fullstack(t, o, d, ts, te, &hit, cnt); break;
            case HKO_RESTART: r = search_restart(t, o, d, ts, te, 0, &hit, cnt); break;
            case HKO_RESTART_EARLY: r = search_restart(t, o, d, ts, te, 1, &hit, cnt); break;
            case HKO_ROPES: r = search_ropes(t, o, d, ts, te, &hit, cnt); break;
            default: r = 0;
            }
        }
    }
    if (r) {
        out[0] = hit.t;
        out[1] = hit.n[0];
        out[2] = hit.n[1];
        out[3] = hit.n[2];
        out[4] = hit.pos[0];
        out[5] = hit.pos[1];
        out[6] = hit.pos[2];
        out[7] = (float)hit.id;
        return hit.id;
    }
    memset(out, 0, 8 * sizeof(float));
    out[0] = INFINITY;
    out[7] = -1.0f;
    return -1;
}

void hko_trace(const hko_tree *t, int variant, int D, const float *rays, uint32_t n, float *hits,
               int32_t *ids, uint64_t *counters, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (long i = 0; i < (long)n; i++) {
        hko_counters c = {0, 0, 0};
        ids[i] = hko_trace_one(t, variant, D, rays + 8 * (size_t)i, hits + 8 * (size_t)i, &c);
        if (counters) {
            counters[3 * i] = c.nodes;
            counters[3 * i + 1] = c.refs;
            counters[3 * i + 2] = c.tests;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* shading                                                                    */
/* ------------------------------------------------------------------------ */

/* FrameBuffer::replacePixel, FrameBuffer.hpp:196-217: min(1, c) * 255 then
 * cvtps2dq (round to nearest even) and pack R | G<<8 | B<<16 */
static uint32_t pack_pixel(const float *c) {
    uint32_t v = 0;
    for (int k = 0; k < 3; k++) {
        float x = (1.0f < c[k]) ? 1.0f : c[k];
        x = x * 255.0f;
        int32_t q = (int32_t)nearbyintf(x);
        v |= (uint32_t)q << (8 * k);
    }
    return v;
}

/* GLVisitorCPUTrace::traceScene, GLVisitorCPUTrace.cpp:149-200 */
void hko_render_cpu(const hko_tree *t, int variant, int D, const float *rays, uint32_t w, uint32_t h,
                    const float *lights, uint32_t nl, int mode, uint32_t *rgba, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (long y = 0; y < (long)h; y++) {
        for (uint32_t x = 0; x < w; x++) {
            size_t pix = (size_t)y * w + x;
            const float *ray = rays + 8 * pix;
            float hit[8];
            hko_counters c = {0, 0, 0};
            int id = hko_trace_one(t, variant, D, ray, hit, &c);
            if (id < 0) {
                rgba[pix] = 0;
                continue;
            }
            float color[4] = {0.1f, 0.1f, 0.1f, 1.0f};
            float n4[4] = {hit[1], hit[2], hit[3], 0.0f};
            float pos[4] = {hit[4], hit[5], hit[6], 0.0f};
            for (uint32_t k = 0; k < nl; k++) {
                const float *L = lights + 8 * (size_t)k;
                if (L[3] == 0.0f) { /* directional */
                    float I = hko_dot4(n4, L + 4);
                    float s = (I > 0) ? I : 0.0f;
                    for (int q = 0; q < 4; q++) color[q] = color[q] + L[q] * s;
                }
                if (L[3] == 1.0f) { /* point */
                    float tl[4];
                    sub4(L + 4, pos, tl);
                    tl[3] = 0.0f;
                    float dist = sqrtf(hko_dot4(tl, tl));
                    hko_normalize(tl, mode);
                    float sray[8];
                    for (int q = 0; q < 4; q++) {
                        sray[q] = pos[q] + tl[q] * 0.001f;
                        sray[4 + q] = tl[q];
                    }
                    float sh[8];
                    hko_counters c2 = {0, 0, 0};
                    int sid = hko_trace_one(t, variant, D, sray, sh, &c2);
                    float I = hko_dot4(n4, tl);
                    if (sid >= 0 && dist > sh[0]) I *= 0.5f;
                    float s = (I > 0) ? I : 0.0f;
                    for (int q = 0; q < 4; q++) color[q] = color[q] + L[q] * s;
                }
            }
            rgba[pix] = pack_pixel(color);
        }
    }
}

/* One mirror bounce (no reference counterpart; the CUDA path's HK_SHADE_MIRROR):
 * a primary hit on a mirror triangle is replaced by the hit of the reflected ray
 * r = d - n*(2 d.n) leaving pos + r*0.001, which is shaded like a primary hit
 * (GLVisitorCPUTrace.cpp:165-194 semantics, shadow rays included); a reflected
 * ray that misses gives 0. */
void hko_render_mirror(const hko_tree *t, int variant, int D, const float *rays, uint32_t w, uint32_t h,
                       const float *lights, uint32_t nl, const uint8_t *mirror, int mode, uint32_t *rgba,
                       int nthreads) {
    size_t n = (size_t)w * h;
    float *srays = (float *)malloc(n * 8 * sizeof(float));
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (long i = 0; i < (long)n; i++) {
        const float *ray = rays + 8 * (size_t)i;
        float *out = srays + 8 * (size_t)i;
        memcpy(out, ray, 32);
        float hit[8];
        hko_counters c = {0, 0, 0};
        int id = hko_trace_one(t, variant, D, ray, hit, &c);
        if (id < 0 || !mirror[id]) continue;
        const float *o = ray, *d = ray + 4;
        const float *nrm = t->cache + 16 * (size_t)id;
        float n4[4] = {nrm[0], nrm[1], nrm[2], 0.0f};
        float pos[4];
        for (int k = 0; k < 4; k++) pos[k] = o[k] + d[k] * hit[0];
        pos[3] = 0.0f;
        float k2 = 2.0f * hko_dot4(d, n4);
        float r[4];
        for (int q = 0; q < 3; q++) r[q] = d[q] - n4[q] * k2;
        r[3] = 0.0f;
        for (int q = 0; q < 3; q++) out[q] = pos[q] + r[q] * 0.001f;
        out[3] = 0.0f;
        memcpy(out + 4, r, 16);
    }
    hko_render_cpu(t, variant, D, srays, w, h, lights, nl, mode, rgba, nthreads);
    free(srays);
}

/* ShadePicture, shadePicture.cl:7-55 (float3 dot as (x*x + y*y) + z*z) */
static float dot3(const float *a, const float *b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

static uint32_t unorm8(float x) {
    x = x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x);
    return (uint32_t)nearbyintf(x * 255.0f);
}

void hko_shade_picture(const float *rays, const float *hit4, uint32_t n, const float *lights,
                       uint32_t nl, uint32_t *rgba) {
    for (uint32_t i = 0; i < n; i++) {
        float color[4] = {0.1f, 0.1f, 0.1f, 0.0f};
        const float *h = hit4 + 4 * (size_t)i;
        if (h[3] != FLT_MAX && h[3] > 0) {
            const float *o = rays + 8 * (size_t)i, *d = o + 4;
            float pos[3];
            for (int k = 0; k < 3; k++) pos[k] = o[k] + h[3] * d[k];
            for (uint32_t l = 0; l < nl; l++) {
                const float *L = lights + 8 * (size_t)l;
                float I = 0.0f;
                if (L[3] == 1.0f) {
                    float tl[3] = {L[4] - pos[0], L[5] - pos[1], L[6] - pos[2]};
                    float inv = 1.0f / sqrtf(dot3(tl, tl));
                    for (int k = 0; k < 3; k++) tl[k] = tl[k] * inv;
                    I = dot3(h, tl) / 2.0f;
                }
                if (L[3] == 0.0f) I = dot3(h, L + 4);
                float s = I > 0.0f ? I : 0.0f;
                for (int q = 0; q < 4; q++) color[q] = color[q] + L[q] * s;
            }
        }
        rgba[i] = unorm8(color[0]) | (unorm8(color[1]) << 8) | (unorm8(color[2]) << 16) |
                  (unorm8(color[3]) << 24);
    }
}

/* ------------------------------------------------------------------------ */
/* compact node format                                                       */
/* ------------------------------------------------------------------------ */
#define CLEAF 3u

uint32_t hko_ref_to_compact(const uint32_t *nodes, uint32_t nn, uint32_t *c) {
    /* breadth-first: the compact node at position q holds reference node src[q] */
    uint32_t cap = 2 * nn + 2;
    uint32_t *src = (uint32_t *)malloc((size_t)cap * sizeof(uint32_t));
    uint32_t head = 0, cnt = 2;
    src[0] = 0;
    src[1] = 0xffffffffu; /* padding */
    c[2] = CLEAF; c[3] = 0;
    for (head = 0; head < cnt; head++) {
        if (head == 1) continue;
        uint32_t s = src[head];
        if (s == 0xffffffffu) { /* empty cell */
            c[2 * head] = CLEAF;
            c[2 * head + 1] = 0;
            continue;
        }
        const uint32_t *n = nodes + 4 * (size_t)s;
        if (n[0] & HKO_JUNCTION) {
            uint32_t pair = cnt;
            cnt += 2;
            src[pair] = n[2] ? n[2] : 0xffffffffu;      /* below */
            src[pair + 1] = n[1] ? n[1] : 0xffffffffu;  /* above */
            c[2 * head] = (pair << 2) | (n[0] & 3);
            c[2 * head + 1] = n[3];
        } else {
            c[2 * head] = (n[1] << 2) | CLEAF;
            c[2 * head + 1] = n[2];
        }
    }
    free(src);
    return cnt;
}

void hko_compact_to_ref(const uint32_t *c, uint32_t cnn, uint32_t *nodes) {
    uint32_t leaf = 0;
    for (uint32_t i = 0; i < cnn; i++) {
        uint32_t w0 = c[2 * i], w1 = c[2 * i + 1];
        uint32_t *n = nodes + 4 * (size_t)i;
        if ((w0 & 3) == CLEAF) {
            n[0] = HKO_LEAF;
            n[1] = w0 >> 2;
            n[2] = w1;
            n[3] = leaf++;
        } else {
            uint32_t pair = w0 >> 2;
            n[0] = (w0 & 3) | HKO_JUNCTION;
            /* empty children become the reference's "no child" index 0 */
            n[2] = (c[2 * pair] & 3) == CLEAF && c[2 * pair + 1] == 0 ? 0 : pair;
            n[1] = (c[2 * (pair + 1)] & 3) == CLEAF && c[2 * (pair + 1) + 1] == 0 ? 0 : pair + 1;
            n[3] = w1;
        }
    }
}

/* Ropes: each face of a node's cell points to the node on the other side of
 * that face, the sibling for the face on the parent's split plane and the
 * parent's rope otherwise (so a rope may name a junction, from which the
 * traversal descends by point location). */
void hko_build_ropes(const uint32_t *c, uint32_t cnn, const float *box, uint32_t *ropes,
                     float *cbox) {
    for (uint32_t i = 0; i < cnn; i++)
        for (int f = 0; f < 6; f++) ropes[6 * (size_t)i + f] = 0xffffffffu;
    memset(cbox, 0, (size_t)cnn * 8 * sizeof(float));
    memcpy(cbox, box, 8 * sizeof(float));
    /* children always follow their parent in the compact order */
    for (uint32_t i = 0; i < cnn; i++) {
        uint32_t w0 = c[2 * i];
        if (i == 1 || (w0 & 3) == CLEAF) continue;
        uint32_t axis = w0 & 3, pair = w0 >> 2;
        float plane;
        memcpy(&plane, &c[2 * i + 1], 4);
        for (uint32_t ch = 0; ch < 2; ch++) {
            uint32_t k = pair + ch;
            memcpy(cbox + 8 * (size_t)k, cbox + 8 * (size_t)i, 32);
            memcpy(ropes + 6 * (size_t)k, ropes + 6 * (size_t)i, 6 * sizeof(uint32_t));
            if (ch == 0) { /* below: its +axis face touches the above child */
                cbox[8 * (size_t)k + 4 + axis] = plane;
                ropes[6 * (size_t)k + 2 * axis + 1] = pair + 1;
            } else {
                cbox[8 * (size_t)k + axis] = plane;
                ropes[6 * (size_t)k + 2 * axis] = pair;
            }
        }
    }
}

/* Ropes traversal on the compact tree (new; no reference counterpart).
 * Starting at the root with t = ts, locate the leaf cell holding the point
 * o + d*t (ties on a plane follow the reference's near-side rule: below when
 * the coordinate is smaller, or equal with a non-positive direction
 * component), test it, stop when the closest hit lies before the cell's exit,
 * else follow the rope of the exit face. */
static int search_ropes(const hko_tree *t, const float *o, const float *d, float ts, float te,
                        hit_t *hit, hko_counters *cnt) {
    const uint32_t *C = t->cnodes;
    float inv[4];
    for (int k = 0; k < 4; k++) inv[k] = 1.0f / d[k];
    float tentry = ts;
    uint32_t cur = 0;
    int ret = 0;
    for (uint32_t guard = 0; guard < 4u * t->cnn + 8u; guard++) {
        float p[3];
        for (int k = 0; k < 3; k++) p[k] = o[k] + d[k] * tentry;
        while ((C[2 * cur] & 3) != CLEAF) {
            cnt->nodes++;
            uint32_t axis = C[2 * cur] & 3, pair = C[2 * cur] >> 2;
            float pl;
            memcpy(&pl, &C[2 * cur + 1], 4);
            int below = (p[axis] < pl) || (p[axis] == pl && d[axis] <= 0);
            cur = below ? pair : pair + 1;
        }
        const float *b = t->cbox + 8 * (size_t)cur;
        float texit = te;
        int face = -1;
        for (int k = 0; k < 3; k++) {
            if (d[k] > 0) {
                float tt = (b[4 + k] - o[k]) * inv[k];
                if (tt < texit) { texit = tt; face = 2 * k + 1; }
            } else if (d[k] < 0) {
                float tt = (b[k] - o[k]) * inv[k];
                if (tt < texit) { texit = tt; face = 2 * k; }
            }
        }
        uint32_t count = C[2 * cur + 1];
        cnt->nodes++;
        if (count) {
            uint32_t ref[4] = {HKO_LEAF, C[2 * cur] >> 2, count, 0};
            ret |= test_leaf(t, ref, o, d, hit, cnt);
            if (hit->t < texit) break;
        }
        if (face < 0) break;
        uint32_t r = t->cropes[6 * (size_t)cur + face];
        if (r == 0xffffffffu) break;
        /* guarantee progress when the exit distance does not advance */
        tentry = texit > tentry ? texit : tentry;
        cur = r;
    }
    return ret;
}

/* ------------------------------------------------------------------------ */
/* binned SAH build: the algorithm of the CUDA builder, restated serially     */
/* (no reference counterpart; the reference builds with the exact event      */
/* sweep above). Breadth-first, level by level:                              */
/*  - a node is a leaf when refs <= leaf_size or depth >= max_depth;         */
/*  - a node with at most exact_max refs costs every clipped bound of its     */
/*    refs on every axis with a positive extent (the exact SAH candidates),   */
/*    ties going to the lower axis, then the lower plane;                     */
/*  - otherwise every axis with a positive extent gets bins planes            */
/*    p_k = min + ext*(k/bins), k = 1..bins-1, and exact counts of the refs   */
/*    below / above each plane from two histograms of the refs' clipped       */
/*    bounds (bins are corrected so that p_b <= lo < p_{b+1} and              */
/*    p_c < hi <= p_{c+1} hold exactly) plus the refs lying flat on a plane;  */
/*  - cost(k) = ct + ci*(A_below*N_below + A_above*N_above)/A_node with full  */
/*    surface areas; the first minimum over (axis, k) wins; the node stays a  */
/*    leaf when no plane is valid or the best cost >= ci*N;                   */
/*  - a ref goes below if lo < p or lo == hi == p, above if hi > p or         */
/*    lo == hi == p (checkPolygonToAAPlane, KDTreeCPU.cpp:450-477, on the      */
/*    clipped bounds); ref order is kept;                                     */
/*  - children are numbered as pairs (below, above) in the order their        */
/*    parents appear in the level; an empty child is an empty leaf.           */
/* Learned mode (the CUDA builder's k_learn, restated with the bins the GPU  */
/* proposed, taken from its proposal log): nodes of at most 32 refs take the  */
/* exact search; a node of 33..1024 refs takes the binned search and, for    */
/* each proposed bin (axis a, bin b, closed interval [P0, P1] = [p_b,        */
/* p_{b+1}], p_0 = node min, p_32 = node max), the exact search over the      */
/* clipped bounds inside the interval (a bin whose in-interval lower bounds,  */
/* upper bounds or flat refs exceed the list capacity (the largest power of  */
/* two c with 3 topk c <= 2048) is skipped); the best of those by          */
/* (cost, axis, plane) replaces the binned plane unless it costs more than    */
/* fallback_ratio x the binned optimum.                                       */
/* ------------------------------------------------------------------------ */
typedef struct {
    float box[8];
    uint32_t start, count, depth, cidx;
} bnode_t;

static float bplane(const float *box, uint32_t a, uint32_t k, uint32_t bins) {
    float ext = box[4 + a] - box[a];
    return box[a] + ext * ((float)k * (1.0f / (float)bins));
}

static float surf(const float *b) {
    float sx = b[4] - b[0], sy = b[5] - b[1], sz = b[6] - b[2];
    return 2.0f * (sx * sy + sz * sy + sx * sz);
}

typedef struct {
    const hko_binned_params *p;
    const float *tb;            /* per triangle: min xyz, max xyz */
    uint32_t *hlo, *hhi, *hon;  /* bins counters */
    float *pl;                  /* bins + 1 planes */
} bin_ctx;

/* the split of one decidable node whose references are refs[n->start ..
 * n->start + n->count): the axis (-1: leaf), its plane and the below / above
 * counts of the chosen plane */
static int32_t decide_binned(bin_ctx *c, const bnode_t *n, const uint32_t *refs, float *plane_out,
                             uint32_t *nb_out, uint32_t *na_out) {
    const hko_binned_params *p = c->p;
    const float *tb = c->tb;
    const uint32_t B = p->bins;
    uint32_t *hlo = c->hlo, *hhi = c->hhi, *hon = c->hon;
    float *pl = c->pl;
    int32_t axis = -1;
    float plane = 0.0f;
    float A = surf(n->box);
    float best = INFINITY;
    uint32_t bnb = 0, bna = 0;
    if (n->count <= (p->learned ? 32u : p->exact_max)) {
        /* small node: every clipped reference bound is a candidate
         * (+0.0f makes a -0 bound the plane +0) */
        for (uint32_t a = 0; a < 3; a++) {
            float lo_b = n->box[a], hi_b = n->box[4 + a];
            if (!(hi_b - lo_b > 0)) continue;
            for (uint32_t q = 0; q < 2 * n->count; q++) {
                const float *tq = tb + 6 * (size_t)refs[n->start + q / 2];
                float pk = ((q & 1) ? mn(tq[3 + a], hi_b) : mx(tq[a], lo_b)) + 0.0f;
                if (!(pk > lo_b && pk < hi_b)) continue;
                uint32_t nb = 0, na = 0;
                for (uint32_t r = 0; r < n->count; r++) {
                    const float *t6 = tb + 6 * (size_t)refs[n->start + r];
                    float lo = mx(t6[a], lo_b), hi = mn(t6[3 + a], hi_b);
                    int on = lo == hi && lo == pk;
                    nb += (lo < pk || on) ? 1u : 0u;
                    na += (hi > pk || on) ? 1u : 0u;
                }
                float bb[8], ba[8];
                memcpy(bb, n->box, 32);
                memcpy(ba, n->box, 32);
                bb[4 + a] = pk;
                ba[a] = pk;
                float cost = p->ct + p->ci * ((surf(bb) * (float)nb + surf(ba) * (float)na) / A);
                /* first minimum in (axis, plane) order */
                if (cost < best || (cost == best && (int32_t)a == axis && pk < plane)) {
                    best = cost;
                    axis = (int32_t)a;
                    plane = pk;
                    bnb = nb;
                    bna = na;
                }
            }
        }
    } else
    for (uint32_t a = 0; a < 3; a++) {
        float lo_b = n->box[a], hi_b = n->box[4 + a];
        float ext = hi_b - lo_b;
        if (!(ext > 0)) continue;
        float inv = (float)B / ext;
        for (uint32_t k = 1; k < B; k++) pl[k] = bplane(n->box, a, k, B);
        memset(hlo, 0, B * 4);
        memset(hhi, 0, B * 4);
        memset(hon, 0, B * 4);
        for (uint32_t r = 0; r < n->count; r++) {
            const float *t6 = tb + 6 * (size_t)refs[n->start + r];
            float lo = mx(t6[a], lo_b), hi = mn(t6[3 + a], hi_b);
            int b = (int)((lo - lo_b) * inv);
            b = b < 0 ? 0 : (b > (int)B - 1 ? (int)B - 1 : b);
            while (b > 0 && lo < pl[b]) b--;
            while (b < (int)B - 1 && lo >= pl[b + 1]) b++;
            int c2 = (int)((hi - lo_b) * inv);
            c2 = c2 < 0 ? 0 : (c2 > (int)B - 1 ? (int)B - 1 : c2);
            while (c2 > 0 && hi <= pl[c2]) c2--;
            while (c2 < (int)B - 1 && hi > pl[c2 + 1]) c2++;
            hlo[b]++;
            hhi[c2]++;
            if (lo == hi && b >= 1 && lo == pl[b]) hon[b]++;
        }
        uint32_t below = 0, above = n->count;
        for (uint32_t k = 1; k < B; k++) {
            below += hlo[k - 1];
            above -= hhi[k - 1];
            float pk = pl[k];
            if (!(pk > lo_b && pk < hi_b)) continue;
            if (k < B - 1 && !(pk < pl[k + 1])) continue;
            uint32_t nb = below + hon[k], na = above + hon[k];
            float bb[8], ba[8];
            memcpy(bb, n->box, 32);
            memcpy(ba, n->box, 32);
            bb[4 + a] = pk;
            ba[a] = pk;
            float cost = p->ct + p->ci * ((surf(bb) * (float)nb + surf(ba) * (float)na) / A);
            if (cost < best) {
                best = cost;
                axis = (int32_t)a;
                plane = pk;
                bnb = nb;
                bna = na;
            }
        }
    }
    if (p->learned && n->count > 32 && n->count <= 1024 && p->proposals) {
        const int32_t *prop = p->proposals + 8 * (size_t)n->cidx;
        uint32_t K = p->topk < 8 ? (p->topk ? p->topk : 1) : 8;
        uint32_t cap = 1;
        while (2u * cap * 3u * K <= 2048u) cap *= 2u;
        float rbest = INFINITY, rpk = 0.0f;
        int32_t rax = 3;
        uint32_t rnb = 0, rna = 0;
        for (uint32_t i = 0; i < 8 && prop[i] >= 0; i++) {
            uint32_t a = (uint32_t)prop[i] / 32u, b = (uint32_t)prop[i] % 32u;
            float lo_b = n->box[a], hi_b = n->box[4 + a];
            float P0 = b == 0 ? lo_b : bplane(n->box, a, b, 32);
            float P1 = b == 31 ? hi_b : bplane(n->box, a, b + 1, 32);
            uint32_t nl = 0, nh = 0, nf = 0;
            for (uint32_t r = 0; r < n->count; r++) {
                const float *t6 = tb + 6 * (size_t)refs[n->start + r];
                float lo = mx(t6[a], lo_b), hi = mn(t6[3 + a], hi_b);
                int inl = P0 <= lo && lo <= P1, inh = P0 <= hi && hi <= P1;
                nl += inl;
                nh += inh;
                nf += inl && lo == hi;
            }
            if (nl > cap || nh > cap || nf > cap) continue;
            for (uint32_t q = 0; q < 2 * n->count; q++) {
                const float *tq = tb + 6 * (size_t)refs[n->start + q / 2];
                float v = (q & 1) ? mn(tq[3 + a], hi_b) : mx(tq[a], lo_b);
                if (!(P0 <= v && v <= P1)) continue;
                if (!(v > lo_b && v < hi_b)) continue;
                float pk = v + 0.0f;
                uint32_t nb = 0, na = 0;
                for (uint32_t r = 0; r < n->count; r++) {
                    const float *t6 = tb + 6 * (size_t)refs[n->start + r];
                    float lo = mx(t6[a], lo_b), hi = mn(t6[3 + a], hi_b);
                    int on = lo == hi && lo == pk;
                    nb += (lo < pk || on) ? 1u : 0u;
                    na += (hi > pk || on) ? 1u : 0u;
                }
                float bb[8], ba[8];
                memcpy(bb, n->box, 32);
                memcpy(ba, n->box, 32);
                bb[4 + a] = pk;
                ba[a] = pk;
                float cost = p->ct + p->ci * ((surf(bb) * (float)nb + surf(ba) * (float)na) / A);
                if (cost < rbest || (cost == rbest && ((int32_t)a < rax || ((int32_t)a == rax && pk < rpk)))) {
                    rbest = cost;
                    rax = (int32_t)a;
                    rpk = pk;
                    rnb = nb;
                    rna = na;
                }
            }
        }
        if (rbest < INFINITY && rbest <= p->fallback_ratio * best) {
            best = rbest;
            axis = rax;
            plane = rpk;
            bnb = rnb;
            bna = rna;
        }
    }
    if (axis >= 0 && !(best < p->ci * (float)n->count)) axis = -1;
    *plane_out = plane;
    *nb_out = bnb;
    *na_out = bna;
    return axis;
}

/* the stable partition of a split node's references: below ones to
 * out[0 .. *nb), above ones after them (*na) */
static void partition_refs(const float *tb, const bnode_t *n, const uint32_t *refs, uint32_t a, float pk,
                           uint32_t *out, uint32_t *nb, uint32_t *na) {
    uint32_t k = 0;
    for (uint32_t r = 0; r < n->count; r++) {
        uint32_t tri = refs[n->start + r];
        const float *t6 = tb + 6 * (size_t)tri;
        float lo = mx(t6[a], n->box[a]), hi = mn(t6[3 + a], n->box[4 + a]);
        if (lo < pk || (lo == hi && lo == pk)) out[k++] = tri;
    }
    *nb = k;
    for (uint32_t r = 0; r < n->count; r++) {
        uint32_t tri = refs[n->start + r];
        const float *t6 = tb + 6 * (size_t)tri;
        float lo = mx(t6[a], n->box[a]), hi = mn(t6[3 + a], n->box[4 + a]);
        if (hi > pk || (lo == hi && lo == pk)) out[k++] = tri;
    }
    *na = k - *nb;
}

/* One deferred subtree, depth first (the CUDA builder's k_subtree): the node
 * on top of the stack is decided; a leaf appends its references; a split
 * takes the next pair of node indices (below, above), pushes the above child
 * and then the below child (so the below child is taken next); an empty
 * child is an empty leaf. Returns 0, or -1 when out of memory. */
typedef struct {
    bnode_t n;
    uint32_t *refs;   /* the node's references (n.start = 0) */
} snode_t;

static int expand_subtree(bin_ctx *c, uvec *cn, uvec *leafrefs, const bnode_t *root, const uint32_t *root_refs) {
    const hko_binned_params *p = c->p;
    size_t cap = 2u * (p->max_depth + 2u), sp = 0;
    snode_t *st = (snode_t *)malloc(cap * sizeof(snode_t));
    if (!st) return -1;
    st[0].n = *root;
    st[0].n.start = 0;
    st[0].refs = (uint32_t *)malloc((root->count ? root->count : 1) * sizeof(uint32_t));
    memcpy(st[0].refs, root_refs, root->count * sizeof(uint32_t));
    sp = 1;
    while (sp > 0) {
        snode_t e = st[--sp];
        bnode_t *n = &e.n;
        float pk = 0.0f;
        uint32_t nb = 0, na = 0;
        int32_t a = -1;
        if (n->count > p->leaf_size && n->depth < p->max_depth) a = decide_binned(c, n, e.refs, &pk, &nb, &na);
        if (a < 0) {
            cn->a[2 * n->cidx] = ((uint32_t)leafrefs->n << 2) | CLEAF;
            cn->a[2 * n->cidx + 1] = n->count;
            for (uint32_t r = 0; r < n->count; r++) uv_push(leafrefs, e.refs[r]);
            free(e.refs);
            continue;
        }
        uint32_t pair = (uint32_t)(cn->n / 2);
        for (int k = 0; k < 4; k++) uv_push(cn, 0);
        cn->a[2 * n->cidx] = (pair << 2) | (uint32_t)a;
        memcpy(&cn->a[2 * n->cidx + 1], &pk, 4);
        uint32_t *part = (uint32_t *)malloc((n->count ? 2 * n->count : 1) * sizeof(uint32_t));
        uint32_t cb = 0, ca = 0;
        partition_refs(c->tb, n, e.refs, (uint32_t)a, pk, part, &cb, &ca);
        for (int ch = 1; ch >= 0; ch--) {
            uint32_t cnt2 = ch ? ca : cb;
            uint32_t idx = pair + (uint32_t)ch;
            if (cnt2 == 0) {
                cn->a[2 * idx] = CLEAF;
                cn->a[2 * idx + 1] = 0;
                continue;
            }
            if (sp == cap) {
                cap *= 2;
                st = (snode_t *)realloc(st, cap * sizeof(snode_t));
            }
            snode_t *d = &st[sp++];
            memcpy(d->n.box, n->box, 32);
            if (ch == 0) d->n.box[4 + a] = pk; else d->n.box[a] = pk;
            d->n.start = 0;
            d->n.count = cnt2;
            d->n.depth = n->depth + 1;
            d->n.cidx = idx;
            d->refs = (uint32_t *)malloc(cnt2 * sizeof(uint32_t));
            memcpy(d->refs, part + (ch ? cb : 0), cnt2 * sizeof(uint32_t));
        }
        free(part);
        free(e.refs);
    }
    free(st);
    return 0;
}

int hko_build_binned(const float *verts, const uint32_t *tris, uint32_t nt, const float *box,
                     const hko_binned_params *p, uint32_t **nodes_out, uint32_t *nn_out,
                     uint32_t **refs_out, uint32_t *nr_out) {
    const uint32_t B = p->bins;
    float *tb = (float *)malloc((size_t)(nt ? nt : 1) * 6 * sizeof(float));
    for (uint32_t i = 0; i < nt; i++) {
        const float *p1 = verts + 4 * (size_t)tris[4 * i];
        const float *p2 = verts + 4 * (size_t)tris[4 * i + 1];
        const float *p3 = verts + 4 * (size_t)tris[4 * i + 2];
        for (int a = 0; a < 3; a++) {
            tb[6 * i + a] = mn(mn(p1[a], p2[a]), p3[a]);
            tb[6 * i + 3 + a] = mx(mx(p1[a], p2[a]), p3[a]);
        }
    }
    bin_ctx bc;
    bc.p = p;
    bc.tb = tb;
    bc.hlo = (uint32_t *)malloc(B * sizeof(uint32_t));
    bc.hhi = (uint32_t *)malloc(B * sizeof(uint32_t));
    bc.hon = (uint32_t *)malloc(B * sizeof(uint32_t));
    bc.pl = (float *)malloc((B + 1) * sizeof(float));
    uvec cn = {0, 0, 0}, leafrefs = {0, 0, 0};
    for (int k = 0; k < 4; k++) uv_push(&cn, 0);
    cn.a[2] = CLEAF; /* padding node */
    bnode_t *cur = (bnode_t *)malloc(sizeof(bnode_t));
    uint32_t ncur = 1;
    memcpy(cur[0].box, box, 32);
    cur[0].start = 0;
    cur[0].count = nt;
    cur[0].depth = 0;
    cur[0].cidx = 0;
    uint32_t *refs = (uint32_t *)malloc((size_t)(nt ? nt : 1) * sizeof(uint32_t));
    for (uint32_t i = 0; i < nt; i++) refs[i] = i;
    /* deferred subtree roots, in the order the levels meet them */
    bnode_t *droot = NULL;
    uvec drefs = {0, 0, 0};
    uint32_t nd = 0, dcap = 0;
    while (ncur > 0) {
        /* 1) decisions; -2: a deferred subtree root */
        int32_t *axis = (int32_t *)malloc(ncur * sizeof(int32_t));
        float *plane = (float *)malloc(ncur * sizeof(float));
        uint64_t child_refs = 0;
        for (uint32_t s = 0; s < ncur; s++) {
            bnode_t *n = &cur[s];
            axis[s] = -1;
            plane[s] = 0.0f;
            if (n->count <= p->leaf_size || n->depth >= p->max_depth) continue;
            if (n->count >= 2u && n->count <= p->defer &&
                (p->defer_margin == 0 || p->defer_margin >= p->max_depth || n->depth >= p->max_depth - p->defer_margin)) {
                axis[s] = -2;
                continue;
            }
            uint32_t bnb = 0, bna = 0;
            axis[s] = decide_binned(&bc, n, refs, &plane[s], &bnb, &bna);
            if (axis[s] >= 0) child_refs += (uint64_t)bnb + bna;
        }
        /* capacity guard: a level whose children would overflow the reference
         * arena, the leaf-reference array (deferred references count as leaf
         * references) or the node array stops splitting (every node of the
         * level becomes a leaf) */
        {
            uint64_t leaf_refs_level = 0, splits = 0;
            for (uint32_t s = 0; s < ncur; s++) {
                if (axis[s] >= 0) splits++;
                else leaf_refs_level += cur[s].count;
            }
            if (child_refs > p->max_refs ||
                (uint64_t)leafrefs.n + drefs.n + leaf_refs_level + child_refs > p->max_refs ||
                (uint64_t)(cn.n / 2) + 2 * splits > p->max_nodes)
                for (uint32_t s = 0; s < ncur; s++) axis[s] = -1;
        }
        /* 2) emit leaves, deferred roots and partition */
        bnode_t *nxt = (bnode_t *)malloc((size_t)2 * ncur * sizeof(bnode_t) + sizeof(bnode_t));
        uint32_t nnxt = 0;
        uint32_t *nrefs = (uint32_t *)malloc((size_t)(child_refs ? child_refs : 1) * sizeof(uint32_t));
        uint32_t nr = 0;
        for (uint32_t s = 0; s < ncur; s++) {
            bnode_t *n = &cur[s];
            if (axis[s] == -2) {
                if (nd == dcap) {
                    dcap = dcap ? 2 * dcap : 64;
                    droot = (bnode_t *)realloc(droot, dcap * sizeof(bnode_t));
                }
                droot[nd] = *n;
                droot[nd].start = (uint32_t)drefs.n;
                nd++;
                for (uint32_t r = 0; r < n->count; r++) uv_push(&drefs, refs[n->start + r]);
                continue;
            }
            if (axis[s] < 0) {
                cn.a[2 * n->cidx] = ((uint32_t)leafrefs.n << 2) | CLEAF;
                cn.a[2 * n->cidx + 1] = n->count;
                for (uint32_t r = 0; r < n->count; r++) uv_push(&leafrefs, refs[n->start + r]);
                continue;
            }
            uint32_t a = (uint32_t)axis[s];
            float pk = plane[s];
            uint32_t pair = (uint32_t)(cn.n / 2);
            for (int k = 0; k < 4; k++) uv_push(&cn, 0);
            cn.a[2 * n->cidx] = (pair << 2) | a;
            memcpy(&cn.a[2 * n->cidx + 1], &pk, 4);
            uint32_t bcount = 0, acount = 0, bstart = nr;
            partition_refs(tb, n, refs, a, pk, nrefs + nr, &bcount, &acount);
            nr += bcount + acount;
            for (uint32_t ch = 0; ch < 2; ch++) {
                uint32_t cnt2 = ch ? acount : bcount;
                uint32_t idx = pair + ch;
                if (cnt2 == 0) {
                    cn.a[2 * idx] = CLEAF;
                    cn.a[2 * idx + 1] = 0;
                    continue;
                }
                bnode_t *c2 = &nxt[nnxt++];
                memcpy(c2->box, n->box, 32);
                if (ch == 0) c2->box[4 + a] = pk; else c2->box[a] = pk;
                c2->start = ch ? bstart + bcount : bstart;
                c2->count = cnt2;
                c2->depth = n->depth + 1;
                c2->cidx = idx;
            }
        }
        free(axis);
        free(plane);
        free(cur);
        free(refs);
        cur = nxt;
        ncur = nnxt;
        refs = nrefs;
    }
    /* 3) the deferred subtrees, in order, after every level's nodes and leaf
     * references; when they do not all fit the node and reference capacities
     * every deferred root stays a leaf instead */
    {
        size_t n0 = cn.n, r0 = leafrefs.n;
        for (uint32_t i = 0; i < nd; i++) expand_subtree(&bc, &cn, &leafrefs, &droot[i], drefs.a + droot[i].start);
        if ((uint64_t)(cn.n / 2) > p->max_nodes || (uint64_t)leafrefs.n > p->max_refs) {
            cn.n = n0;
            leafrefs.n = r0;
            for (uint32_t i = 0; i < nd; i++) {
                cn.a[2 * droot[i].cidx] = ((uint32_t)leafrefs.n << 2) | CLEAF;
                cn.a[2 * droot[i].cidx + 1] = droot[i].count;
                for (uint32_t r = 0; r < droot[i].count; r++) uv_push(&leafrefs, drefs.a[droot[i].start + r]);
            }
        }
    }
    free(droot);
    free(drefs.a);
    free(cur);
    free(refs);
    free(bc.hlo);
    free(bc.hhi);
    free(bc.hon);
    free(bc.pl);
    free(tb);
    *nodes_out = cn.a;
    *nn_out = (uint32_t)(cn.n / 2);
    *refs_out = leafrefs.a ? leafrefs.a : (uint32_t *)malloc(4);
    *nr_out = (uint32_t)leafrefs.n;
    return 0;
}
