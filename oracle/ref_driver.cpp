// C entry points over the compiled reference HulkEngine CPU path.
//
// Test infrastructure only (built by oracle/build_ref.py into oracle/_ref).
// It fills a reference Scene directly (or through the reference's own AFF
// loader, at the end of this file), runs the reference's own
// KDTreeCPU::buildKDTree / checkCollision, and restates the per-pixel shading
// loop of GLVisitorCPUTrace::traceScene (HulkEngine/src/GLVisitorCPUTrace.cpp:
// 149-200) on top of the reference's checkCollision and
// FrameBuffer::replacePixel (HulkEngine/public/FrameBuffer.hpp:196-217).
#include <vector>
#include <cstring>
#include <omp.h>
#include "KDTreeCPU.hpp"
#include "Scene.hpp"
#include "Settings.hpp"
#include "SharedFunctions.hpp"
#include "AFFParser.hpp"
#include "BoundingBoxVisitor.hpp"
#include "util.hpp"

thread_local unsigned hkref_last_poly = 0;
thread_local unsigned long long hkref_nodes = 0;
thread_local unsigned long long hkref_tests = 0;
int hkref_aff_rearm = 0;

namespace {
struct RefCtx {
    Scene scene;
    KDTreeCPU tree;
    RefCtx() : scene("hkref") {}
};

void set_settings() {
    static bool done = false;
    if (done) return;
    // Settings::parseStrings (HulkEngine/src/Settings.cpp:11-28) skips argv[0..1]
    wchar_t a0[] = L"hk", a1[] = L"scene", a2[] = L"--renderType=CPUTrace",
            a3[] = L"--treeType=SAHNlogN";
    wchar_t *argv[] = {a0, a1, a2, a3};
    Settings::getInstance().parseStrings(4, argv);
    done = true;
}
}  // namespace

extern "C" {

// verts: nv x float4 (w = 1), tris: nt x uint4, box: min.xyzw, max.xyzw
void *hkref_create(const float *verts, unsigned nv, const unsigned *tris, unsigned nt,
                   const float *box) {
    set_settings();
    RefCtx *c = new RefCtx();
    for (unsigned i = 0; i < nv; i++) {
        SPVector v(verts[4 * i], verts[4 * i + 1], verts[4 * i + 2], verts[4 * i + 3]);
        c->scene.m_vertices.push_back(v);
    }
    for (unsigned i = 0; i < nt; i++) {
        TriangleIndices t;
        for (int k = 0; k < 4; k++) t.indices[k] = tris[4 * i + k];
        c->scene.m_vertexIndices.push_back(t);
    }
    c->scene.m_sceneBox.m_min = SPVector(box[0], box[1], box[2], box[3]);
    c->scene.m_sceneBox.m_max = SPVector(box[4], box[5], box[6], box[7]);
    return c;
}

void hkref_destroy(void *h) { delete (RefCtx *)h; }

// --treeType: 1 selects buildKDTreeSAH (KDTreeSAH.cpp:9-244), 0 the default
// buildKDTreeSAH_NlogN (Settings::parseStrings, HulkEngine/src/Settings.cpp:8-23)
void hkref_set_tree_type(int sah) {
    set_settings();
    wchar_t a0[] = L"hk", a1[] = L"scene", a2[] = L"--treeType=SAH", a3[] = L"--treeType=SAHNlogN";
    wchar_t *argv[] = {a0, a1, sah ? a2 : a3};
    Settings::getInstance().parseStrings(3, argv);
}

int hkref_build(void *h) {
    RefCtx *c = (RefCtx *)h;
    return (int)c->tree.buildKDTree(c->scene);
}

// Replace the vertex positions (same topology) before a rebuild: the
// per-frame path of the CPU visitor (GLWindow.cpp:129 then buildKDTree).
void hkref_set_vertices(void *h, const float *verts, const float *box) {
    RefCtx *c = (RefCtx *)h;
    for (unsigned i = 0; i < c->scene.m_vertices.size(); i++)
        c->scene.m_vertices[i] = SPVector(verts[4 * i], verts[4 * i + 1], verts[4 * i + 2], verts[4 * i + 3]);
    c->scene.m_sceneBox.m_min = SPVector(box[0], box[1], box[2], box[3]);
    c->scene.m_sceneBox.m_max = SPVector(box[4], box[5], box[6], box[7]);
}

unsigned hkref_node_count(void *h) {
    uint n;
    ((RefCtx *)h)->tree.getNodeArray(n);
    return n;
}
unsigned hkref_ref_count(void *h) {
    uint n;
    ((RefCtx *)h)->tree.getPolygonArray(n);
    return n;
}
// nodes as 4 x u32 each (flags, data words) -- the 16-byte KDTreeNode layout
void hkref_get_nodes(void *h, unsigned *out) {
    uint n;
    const KDTreeNode *p = ((RefCtx *)h)->tree.getNodeArray(n);
    std::memcpy(out, p, sizeof(KDTreeNode) * n);
}
void hkref_get_refs(void *h, unsigned *out) {
    uint n;
    const uint *p = ((RefCtx *)h)->tree.getPolygonArray(n);
    std::memcpy(out, p, sizeof(uint) * n);
}
// PolyToRayCache per triangle as 16 floats: normal4, e0_4, e1_4, e00, e01, e11, det
void hkref_get_cache(void *h, float *out) {
    RefCtx *c = (RefCtx *)h;
    for (unsigned i = 0; i < c->tree.m_polygonCache.size(); i++) {
        const PolyToRayCache &pc = c->tree.m_polygonCache[i];
        float *o = out + 16 * i;
        for (int k = 0; k < 4; k++) {
            o[k] = pc.m_normal.vector[k];
            o[4 + k] = pc.m_e0.vector[k];
            o[8 + k] = pc.m_e1.vector[k];
        }
        o[12] = pc.m_e00; o[13] = pc.m_e01; o[14] = pc.m_e11; o[15] = pc.m_det;
    }
}

// rays: n x (origin float4, dir float4). hits: n x 8 floats
// (t, nx, ny, nz, px, py, pz, 0); ids: winning polygon or -1;
// counters (optional): n x 2 (node visits, triangle tests).
void hkref_trace(void *h, const float *rays, unsigned n, float *hits, int *ids,
                 unsigned long long *counters, int nthreads) {
    RefCtx *c = (RefCtx *)h;
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < (long)n; i++) {
        Ray ray;
        const float *r = rays + 8 * i;
        ray.m_rayStart = SPVector(r[0], r[1], r[2], r[3]);
        ray.m_rayDir = SPVector(r[4], r[5], r[6], r[7]);
        HitData hd;
        hkref_last_poly = 0xFFFFFFFFu;
        hkref_nodes = 0;
        hkref_tests = 0;
        bool hit = c->tree.checkCollision(ray, hd);
        float *o = hits + 8 * i;
        if (hit) {
            o[0] = hd.time;
            o[1] = hd.normal.x; o[2] = hd.normal.y; o[3] = hd.normal.z;
            o[4] = hd.position.x; o[5] = hd.position.y; o[6] = hd.position.z;
            ids[i] = (int)hkref_last_poly;
        } else {
            for (int k = 0; k < 7; k++) o[k] = 0.0f;
            o[0] = INFINITY;
            ids[i] = -1;
        }
        o[7] = 0.0f;
        if (counters) {
            counters[2 * i] = hkref_nodes;
            counters[2 * i + 1] = hkref_tests;
        }
    }
}

// Restated GLVisitorCPUTrace::traceScene (GLVisitorCPUTrace.cpp:149-200):
// rays come precomputed (w x h, row-major by image row), lights are
// (color float4 with type in .w, pos-or-dir float4). Output pixels follow
// FrameBuffer::getPixel indexing (column*width + row), i.e. y*w + x.
void hkref_render(void *h, const float *rays, unsigned w, unsigned hgt, const float *lights,
                  unsigned nl, unsigned *rgba, int nthreads) {
    RefCtx *c = (RefCtx *)h;
    Scene &sc = c->scene;
    sc.m_lights.clear();
    for (unsigned k = 0; k < nl; k++) {
        Light L;
        L.color = SPVector(lights[8 * k], lights[8 * k + 1], lights[8 * k + 2], lights[8 * k + 3]);
        L.data.pos = _mm_set_ps(lights[8 * k + 7], lights[8 * k + 6], lights[8 * k + 5], lights[8 * k + 4]);
        sc.m_lights.push_back(L);
    }
    sc.m_frameBuffer.initialize(w, hgt, 0);
    sc.m_frameBuffer.clearBuffer();
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for
    for (int i = 0; i < (int)hgt; i++) {
        HitData hitData;
        SPVector color(0.0f, 0.0f, 0.0f);
        Ray ray;
        for (uint j = 0; j < w; j++) {
            const float *r = rays + 8 * ((size_t)i * w + j);
            ray.m_rayStart = SPVector(r[0], r[1], r[2], r[3]);
            ray.m_rayDir = SPVector(r[4], r[5], r[6], r[7]);
            if (c->tree.checkCollision(ray, hitData)) {
                static const SPVector ambiant(0.1, 0.1, 0.1);
                color = ambiant;
                for (uint k = 0; k < sc.m_lights.size(); k++) {
                    if (E_directionalLight == sc.m_lights[k].color.w) {
                        float intensity = hitData.normal * sc.m_lights[k].data.dir;
                        color += sc.m_lights[k].color * MAX(intensity, 0);
                    }
                    if (E_pointLight == sc.m_lights[k].color.w) {
                        SPVector toLight = sc.m_lights[k].data.pos - hitData.position;
                        toLight.w = 0;
                        float distToLight = sqrt(toLight * toLight);
                        toLight.normalize();
                        HitData shadowHit;
                        ray.m_rayDir = toLight;
                        ray.m_rayStart = hitData.position + toLight * 0.001;
                        bool hit = c->tree.checkCollision(ray, shadowHit);
                        float intensity = hitData.normal * toLight;
                        if (hit && distToLight > shadowHit.time) {
                            intensity *= 0.5;
                        }
                        color += sc.m_lights[k].color * MAX(intensity, 0);
                    }
                }
                sc.m_frameBuffer.replacePixel(j, i, color);
            }
        }
    }
    std::memcpy(rgba, sc.m_frameBuffer.getBufferBits(), sizeof(unsigned) * w * hgt);
}

// The reference's SSE normalize (SPMatrix.hpp:314-323) applied to n float4s.
void hkref_normalize(float *v, unsigned n) {
    for (unsigned i = 0; i < n; i++) {
        SPVector s(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
        s.normalize();
        for (int k = 0; k < 4; k++) v[4 * i + k] = s.vector[k];
    }
}

// Box helpers pinned by the reference unit tests (test/sharedFunctionTest.cpp:7-33).
float hkref_box_surface(const float *box) {
    Box b;
    b.m_min = SPVector(box[0], box[1], box[2], box[3]);
    b.m_max = SPVector(box[4], box[5], box[6], box[7]);
    return getBoxSurface(b);
}
float hkref_box_volume(const float *box) {
    Box b;
    b.m_min = SPVector(box[0], box[1], box[2], box[3]);
    b.m_max = SPVector(box[4], box[5], box[6], box[7]);
    return getBoxVolume(b);
}

// ---- AFF (BART) scenes through the reference's own loader ----
// AFFParser::viParseFile (BartLoader/src/AFFParser.cpp:1462-1539) fills a
// Scene; AFFTransformVisitor (BartLoader/src/AFFTransformVisitor.cpp) and
// BoundingBoxVisitor run per frame as GLWindow::display does
// (HulkEngine/src/GLWindow.cpp:111-133).
struct RefAff {
    Scene scene;
    AFFParser parser;
    Visitor *xf = nullptr;
    RefAff() : scene("hkaff") {}
    ~RefAff() {
        if (xf) parser.freeTransformVisitor(xf);
    }
};

void *hkref_aff_open(const char *path) {
    FILE *f = fopen(path, "r");
    if (!f) return nullptr;
    std::string p(path);
    RefAff *a = new RefAff();
    a->parser.viParseFile(f, p.substr(0, p.rfind('/') + 1), a->scene);
    fclose(f);
    a->xf = a->parser.getTransformVisitor(a->scene);
    hkref_aff_rearm = 1;
    return a;
}

void hkref_aff_close(void *h) { delete (RefAff *)h; }

// vertices, triangles, lights; fov, resolution, aspect
void hkref_aff_counts(void *h, unsigned *nv, unsigned *nt, unsigned *nl) {
    RefAff *a = (RefAff *)h;
    *nv = a->scene.m_vertices.size();
    *nt = a->scene.m_vertexIndices.size();
    *nl = a->scene.m_lights.size();
}

void hkref_aff_view(void *h, float *fov, int *res, float *aspect) {
    RefAff *a = (RefAff *)h;
    *fov = a->scene.m_fov;
    res[0] = a->scene.m_resx;
    res[1] = a->scene.m_resy;
    *aspect = a->scene.m_aspect;
}

void hkref_aff_tris(void *h, unsigned *tris4) {
    RefAff *a = (RefAff *)h;
    for (unsigned i = 0; i < a->scene.m_vertexIndices.size(); i++)
        for (int k = 0; k < 3; k++) tris4[4 * i + k] = a->scene.m_vertexIndices[i].indices[k];
    for (unsigned i = 0; i < a->scene.m_vertexIndices.size(); i++) tris4[4 * i + 3] = 0;
}

void hkref_aff_lights(void *h, float *l8) {
    RefAff *a = (RefAff *)h;
    for (unsigned i = 0; i < a->scene.m_lights.size(); i++) {
        Light &L = a->scene.m_lights[i];
        SPVector pos(L.data.pos);
        for (int k = 0; k < 4; k++) {
            l8[8 * i + k] = L.color.vector[k];
            l8[8 * i + 4 + k] = pos.vector[k];
        }
    }
}

// one frame at `time`: transformed vertices (float4) and the scene box
void hkref_aff_frame(void *h, float time, float *verts4, float *box8) {
    RefAff *a = (RefAff *)h;
    a->scene.setTime(time);
    a->xf->traverse(a->scene.m_pRoot);
    BoundingBoxVisitor bb(a->scene);
    bb.traverse(a->scene.m_pRoot);
    for (unsigned i = 0; i < a->scene.m_vertices.size(); i++)
        for (int k = 0; k < 4; k++) verts4[4 * i + k] = a->scene.m_vertices[i].vector[k];
    for (int k = 0; k < 4; k++) {
        box8[k] = a->scene.m_sceneBox.m_min.vector[k];
        box8[4 + k] = a->scene.m_sceneBox.m_max.vector[k];
    }
}

// GLVisitorCPUTrace::updateCamera (HulkEngine/src/GLVisitorCPUTrace.cpp:
// 105-146), which needs GL headers to compile, restated over the reference's
// SPVector / SPMatrix and its loader's getTransformation.
void hkref_aff_camera(void *h, float time, float *cam16) {
    RefAff *a = (RefAff *)h;
    a->scene.setTime(time);
    SPMatrix rotMat, transMat;
    double trans[3] = {0}, rot[4] = {0};
    a->parser.getTransformation(a->scene, "camera", rot, trans);
    transMat.TranslateMatrix((float)trans[0], (float)trans[1], (float)trans[2]);
    rotMat.rotateMatrix((float)rot[0], (float)rot[1], (float)rot[2], -(float)rot[3]);
    SPVector from(0, 0, 0), down(0, -1, 0), left(-1, 0, 0), to(0, 0, -1);
    SPVector f = from * transMat;
    down = down * rotMat;
    left = left * rotMat;
    to = to * rotMat;
    down.w = 0;
    left.w = 0;
    to.w = 0;
    f.w = 0;
    float verticalFactor = tan(DEG_TO_RAD(a->scene.m_fov) / 2);
    float horizontalFactor = verticalFactor * a->scene.m_aspect;
    down = down * verticalFactor;
    left = left * horizontalFactor;
    SPVector lowerLeft = f + to + down + left;
    SPVector vert = left * -2.0;
    SPVector horiz = down * -2.0;
    for (int k = 0; k < 4; k++) {
        cam16[k] = f.vector[k];
        cam16[4 + k] = vert.vector[k];
        cam16[8 + k] = horiz.vector[k];
        cam16[12 + k] = lowerLeft.vector[k];
    }
}

}  // extern "C"
