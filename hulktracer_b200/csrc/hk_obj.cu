// hk_obj.cu -- Wavefront OBJ ingest (host code only).
//
// Restates the reference's loader, OBJLoader::viParseFile
// (OBJLoader/OBJLoader.cpp:15-136): whitespace-separated tokens; "v x y z" is
// a vertex (w = 1, SPVector's default, HulkEngine/public/SPMatrix.hpp:78); "f"
// takes the next three tokens as one triangle, each "v[/t[/n]]" giving the
// 1-based vertex index before the first '/' (a fourth token of a quad is then
// read as an ordinary token and ignored, as in the reference); "vn" consumes
// three numbers; "g" consumes one name; "#" drops the rest of the line (at most
// 99 characters, the reference's fgets); every other token is ignored. Indices
// that fall outside the vertex list are an error here (the reference would
// read past its array).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/hulkcuda.h"

namespace {

struct ObjData {
    std::vector<float> verts;      // 4 per vertex
    std::vector<uint32_t> tris;    // 4 per triangle (4th = 0)
};

// 1-based index before the first '/' of a face token (atoi semantics)
long face_vertex(const char *tok) {
    char buf[128];
    size_t k = 0;
    while (tok[k] && tok[k] != '/' && k + 1 < sizeof buf) {
        buf[k] = tok[k];
        k++;
    }
    buf[k] = '\0';
    return atol(buf);
}

hk_status parse(const char *path, ObjData &out) {
    FILE *f = fopen(path, "r");
    if (!f) return HK_E_FILE_OPEN;
    char token[256];
    char face[3][128];
    std::vector<long> idx;
    while (!feof(f)) {
        token[0] = '\0';
        if (fscanf(f, "%255s", token) != 1) break;
        if (!strcmp(token, "g")) {
            if (fscanf(f, "%255s", token) != 1) break;
        } else if (!strcmp(token, "v")) {
            float x = 0, y = 0, z = 0;
            if (fscanf(f, "%f %f %f", &x, &y, &z) != 3) {
                fclose(f);
                return HK_E_ILLEGAL_INPUT;
            }
            out.verts.insert(out.verts.end(), {x, y, z, 1.0f});
        } else if (!strcmp(token, "vn")) {
            float x, y, z;
            if (fscanf(f, "%f %f %f", &x, &y, &z) != 3) {
                fclose(f);
                return HK_E_ILLEGAL_INPUT;
            }
        } else if (!strcmp(token, "f")) {
            for (int i = 0; i < 3; i++)
                if (fscanf(f, "%127s", face[i]) != 1) {
                    fclose(f);
                    return HK_E_ILLEGAL_INPUT;
                }
            for (int i = 0; i < 3; i++) idx.push_back(face_vertex(face[i]) - 1);
        } else if (!strcmp(token, "#")) {
            if (!fgets(token, 100, f)) break;
        }
    }
    if (fclose(f) != 0) return HK_E_FILE_CLOSE;
    const long nv = (long)(out.verts.size() / 4);
    for (long v : idx)
        if (v < 0 || v >= nv) return HK_E_ILLEGAL_INPUT;
    out.tris.reserve(idx.size() / 3 * 4);
    for (size_t t = 0; t + 2 < idx.size(); t += 3)
        out.tris.insert(out.tris.end(), {(uint32_t)idx[t], (uint32_t)idx[t + 1], (uint32_t)idx[t + 2], 0u});
    return HK_OK;
}

}  // namespace

extern "C" {

hk_status hk_obj_parse(const char *path, float *verts4, uint32_t cap_verts, uint32_t *tris4, uint32_t cap_tris,
                       uint32_t *nv, uint32_t *nt) {
    if (!path || !nv || !nt) return HK_E_ILLEGAL_INPUT;
    ObjData d;
    hk_status s = parse(path, d);
    if (s != HK_OK) return s;
    *nv = (uint32_t)(d.verts.size() / 4);
    *nt = (uint32_t)(d.tris.size() / 4);
    if (!verts4 && !tris4) return HK_OK;
    if (!verts4 || !tris4 || cap_verts < *nv || cap_tris < *nt) return HK_E_CAPACITY;
    memcpy(verts4, d.verts.data(), d.verts.size() * sizeof(float));
    memcpy(tris4, d.tris.data(), d.tris.size() * sizeof(uint32_t));
    return HK_OK;
}

hk_status hk_scene_load_obj(hk_ctx *ctx, const char *path, uint32_t *nv, uint32_t *nt) {
    if (!ctx || !path) return HK_E_ILLEGAL_INPUT;
    ObjData d;
    hk_status s = parse(path, d);
    if (s != HK_OK) return s;
    if (d.tris.empty()) return HK_E_ILLEGAL_INPUT;
    if (nv) *nv = (uint32_t)(d.verts.size() / 4);
    if (nt) *nt = (uint32_t)(d.tris.size() / 4);
    return hk_scene_upload(ctx, d.verts.data(), (uint32_t)(d.verts.size() / 4), d.tris.data(),
                           (uint32_t)(d.tris.size() / 4));
}

}  // extern "C"
