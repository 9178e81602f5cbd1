// hk_aff.cu -- AFF (BART animated scene) ingest, host code only.
//
// The reference loads BART scenes with AFFParser (BartLoader/src/AFFParser.cpp)
// into a node tree of static transforms ("xs", RigidTransform), animated
// transforms ("x", AnimatedTransform) and triangle meshes ("m"), keeps the
// keyframe animations ("k") in a list, and every frame re-transforms the mesh
// vertices with AFFTransformVisitor (BartLoader/src/AFFTransformVisitor.cpp:
// 25-130). Here the parse produces flat arrays instead of a node tree:
//
//   * the meshes' rest-pose vertices (w = 1) and triangles, concatenated in
//     file order, which is the order of the reference's Scene::m_vertices and
//     Scene::m_vertexIndices (HulkEngine/src/Scene.cpp:110-121,155-166);
//   * one part per mesh (the vertex -> part map of hk_scene_set_parts);
//   * the transform nodes in creation order, each with its parent, so that a
//     single forward pass evaluates every world matrix.
//
// hk_aff_part_matrices then evaluates the keyframe splines at a time and
// writes one 3x4 matrix per mesh; hk_scene_transform applies them on the
// device. The arithmetic reproduces the reference's bit for bit: the splines
// in double precision in the reference's operation order, the matrices in
// single precision with the association of SPMatrix::operator*= (HulkEngine/
// public/SPMatrix.hpp:137-161), and the device transform rounds after every
// operation in VectorMult's order (SPMatrix.hpp:166-173).
//
// Commands that add nothing to the reference's scene ("f", "fm", "c", "s",
// "p", "pp", "tt", "ttp", "tpa", "b", "am") are parsed with the reference's
// syntax and dropped, as the reference drops them (AFFParser.cpp:286-530,
// 620-790). Where the reference calls exit(1) on a syntax error, a call here
// returns HK_E_ILLEGAL_INPUT (HK_E_FILE_OPEN for a missing file) and
// hk_aff_last_error names the cause.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/hulkcuda.h"

namespace {

thread_local std::string t_aff_error;

hk_status fail(hk_status s, const std::string &msg) {
    t_aff_error = msg;
    return s;
}

// ---------------------------------------------------------------- lexer ----
// A cursor over the whole file with the fscanf conversions the reference
// uses: %f (strtof: the same correctly rounded conversion as glibc's %f), %d,
// %s, literal words and whitespace directives.
struct Cursor {
    std::string text;
    size_t pos = 0;

    int get() { return pos < text.size() ? (unsigned char)text[pos++] : EOF; }
    void unget() {
        if (pos > 0) pos--;
    }
    static bool is_ws(int c) { return c == ' ' || c == '\t' || c == '\n' || c == '\f' || c == '\r' || c == '\v'; }
    void skip_ws() {
        while (pos < text.size() && is_ws((unsigned char)text[pos])) pos++;
    }
    bool read_float(float &v) {
        skip_ws();
        if (pos >= text.size()) return false;
        const char *b = text.c_str() + pos;
        char *e = nullptr;
        float f = strtof(b, &e);
        if (e == b) return false;
        pos += (size_t)(e - b);
        v = f;
        return true;
    }
    bool read_int(int &v) {
        skip_ws();
        if (pos >= text.size()) return false;
        const char *b = text.c_str() + pos;
        char *e = nullptr;
        long l = strtol(b, &e, 10);
        if (e == b) return false;
        pos += (size_t)(e - b);
        v = (int)l;
        return true;
    }
    bool read_word(std::string &w) {
        skip_ws();
        size_t b = pos;
        while (pos < text.size() && !is_ws((unsigned char)text[pos])) pos++;
        w.assign(text, b, pos - b);
        return pos > b;
    }
    // a literal word of a scanf format (" from %f" matches "from")
    bool expect(const char *word) {
        skip_ws();
        size_t n = strlen(word);
        if (text.compare(pos, n, word) != 0) return false;
        pos += n;
        return true;
    }
    bool floats(float *v, int n) {
        for (int i = 0; i < n; i++)
            if (!read_float(v[i])) return false;
        return true;
    }
    // parseComment's fgets(str, 1000, f): at most 999 characters, through '\n'
    void drop_line() {
        for (int k = 0; k < 999 && pos < text.size(); k++)
            if (text[pos++] == '\n') break;
    }
};

bool read_file(const std::string &path, std::string &out) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    char buf[1 << 16];
    size_t n;
    out.clear();
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, n);
    fclose(f);
    return true;
}

// ------------------------------------------------------- spline algebra ----
// Kochanek-Bartels splines (BartLoader/src/kbsplpos.cpp, kbsplrot.cpp; from
// Eberly's Magic Software). Positions and scales are cubic Hermite segments
// whose tangents come from the tension / continuity / bias of the keys; a
// rotation is a squad of quaternions whose inner control points come from the
// same multipliers applied to quaternion logarithms.
struct V3 {
    double x, y, z;
};

struct Cubic {  // P(u) = c0 + u (c1 + u (c2 + u c3)), u in [0, 1] over [t0, t1]
    V3 c0, c1, c2, c3;
    double t0, t1, span;
};

struct Quat {
    double w, x, y, z;
};

struct Squad {
    Quat p, a, b, q;
    double t0, t1, span;
};

struct PosKey {
    double t;
    V3 v;
    double tension, continuity, bias;
};

struct RotKey {
    double t;
    double ax, ay, az, angle;
    double tension, continuity, bias;
};

// the four Hermite multipliers of segment [k1, k2] (kbsplpos.cpp:40-72)
struct Tcb {
    double out0, out1, in0, in1;
};

Tcb tcb(double t0, double t1, double t2, double t3, double ten1, double con1, double bia1, double ten2,
        double con2, double bia2) {
    Tcb m;
    const double a0 = 2 * (t2 - t1) / (t2 - t0);
    m.out0 = 0.5 * a0 * (1 - ten1) * (1 + con1) * (1 + bia1);
    m.out1 = 0.5 * a0 * (1 - ten1) * (1 - con1) * (1 - bia1);
    const double a1 = 2 * (t2 - t1) / (t3 - t1);
    m.in0 = 0.5 * a1 * (1 - ten2) * (1 - con2) * (1 + bia2);
    m.in1 = 0.5 * a1 * (1 - ten2) * (1 + con2) * (1 - bia2);
    return m;
}

std::vector<Cubic> pos_spline(const std::vector<PosKey> &k) {
    std::vector<Cubic> segs;
    for (size_t i = 0; i + 3 < k.size(); i++) {
        const PosKey &k0 = k[i], &k1 = k[i + 1], &k2 = k[i + 2], &k3 = k[i + 3];
        const Tcb m = tcb(k0.t, k1.t, k2.t, k3.t, k1.tension, k1.continuity, k1.bias, k2.tension,
                          k2.continuity, k2.bias);
        const double *p0 = &k0.v.x, *p1 = &k1.v.x, *p2 = &k2.v.x, *p3 = &k3.v.x;
        Cubic c;
        double *c0 = &c.c0.x, *c1 = &c.c1.x, *c2 = &c.c2.x, *c3 = &c.c3.x;
        for (int a = 0; a < 3; a++) {
            const double d = p2[a] - p1[a];
            const double tout = m.out1 * d + m.out0 * (p1[a] - p0[a]);
            const double tin = m.in1 * (p3[a] - p2[a]) + m.in0 * d;
            c0[a] = p1[a];
            c1[a] = tout;
            c2[a] = 3 * d - 2 * tout - tin;
            c3[a] = -2 * d + tout + tin;
        }
        c.t0 = k1.t;
        c.t1 = k2.t;
        c.span = c.t1 - c.t0;
        segs.push_back(c);
    }
    return segs;
}

// segment and local parameter of time t, clamped to the first and last
// segment (ComputeIAndU, kbsplpos.cpp:118-150; the same rule in
// KB_RotInterpolate, kbsplrot.cpp:146-170)
template <class Seg>
void locate(const std::vector<Seg> &s, double t, size_t &i, double &u) {
    if (s[0].t0 < t) {
        if (t < s.back().t1) {
            for (i = 0; i < s.size(); i++)
                if (t < s[i].t1) break;
            u = (t - s[i].t0) / s[i].span;
        } else {
            i = s.size() - 1;
            u = 1.0;
        }
    } else {
        i = 0;
        u = 0.0;
    }
}

V3 pos_eval(const std::vector<Cubic> &s, double t) {
    size_t i;
    double u;
    locate(s, t, i, u);
    const Cubic &c = s[i];
    return {c.c0.x + u * (c.c1.x + u * (c.c2.x + u * c.c3.x)), c.c0.y + u * (c.c1.y + u * (c.c2.y + u * c.c3.y)),
            c.c0.z + u * (c.c1.z + u * (c.c2.z + u * c.c3.z))};
}

// quaternion algebra (BartLoader/src/quat.cpp); sin(angle) below 1e-3 takes
// the small-angle branch of Log / Exp / Slerp, as there
constexpr double kQuatEps = 1e-3;

Quat q_axis_angle(double angle, double x, double y, double z) {
    const double h = 0.5 * angle;
    const double s = sin(h);
    return {cos(h), s * x, s * y, s * z};
}

void q_to_axis_angle(const Quat &q, double &angle, double &x, double &y, double &z) {
    const double len2 = q.x * q.x + q.y * q.y + q.z * q.z;
    if (len2 > 0.0) {
        angle = 2.0 * acos(q.w);
        const double inv = 1.0 / sqrt(len2);
        x = q.x * inv;
        y = q.y * inv;
        z = q.z * inv;
    } else {
        angle = 0;
        x = 1.0;
        y = 0.0;
        z = 0.0;
    }
}

Quat q_mul(const Quat &a, const Quat &b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z, a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z, a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x};
}

Quat q_conj(const Quat &q) { return {q.w, -q.x, -q.y, -q.z}; }
double q_dot(const Quat &a, const Quat &b) { return a.w * b.w + a.x * b.x + a.y * b.y + a.z * b.z; }
Quat q_scale(const Quat &q, double c) { return {q.w * c, q.x * c, q.y * c, q.z * c}; }
Quat q_add(const Quat &a, const Quat &b) { return {a.w + b.w, a.x + b.x, a.y + b.y, a.z + b.z}; }
Quat q_sub(const Quat &a, const Quat &b) { return {a.w - b.w, a.x - b.x, a.y - b.y, a.z - b.z}; }

Quat q_log(const Quat &q) {
    if (fabs(q.w) < 1.0) {
        const double angle = acos(q.w);
        const double sn = sin(angle);
        if (fabs(sn) >= kQuatEps) {
            const double c = angle / sn;
            return {0.0, c * q.x, c * q.y, c * q.z};
        }
    }
    return {0.0, q.x, q.y, q.z};
}

Quat q_exp(const Quat &q) {
    const double angle = sqrt(q.x * q.x + q.y * q.y + q.z * q.z);
    const double sn = sin(angle);
    Quat r{cos(angle), q.x, q.y, q.z};
    if (fabs(sn) >= kQuatEps) {
        const double c = sn / angle;
        r.x = c * q.x;
        r.y = c * q.y;
        r.z = c * q.z;
    }
    return r;
}

Quat q_slerp(double t, const Quat &p, const Quat &q) {
    double c = q_dot(p, q);
    if (c < -1.0)
        c = -1.0;
    else if (c > 1.0)
        c = 1.0;
    const double angle = acos(c);
    const double sn = sin(angle);
    if (sn < kQuatEps) return p;
    const double inv = 1.0 / sn;
    const double c0 = sin((1.0 - t) * angle) * inv;
    const double c1 = sin(t * angle) * inv;
    return {c0 * p.w + c1 * q.w, c0 * p.x + c1 * q.x, c0 * p.y + c1 * q.y, c0 * p.z + c1 * q.z};
}

// KB_RotInitialize (kbsplrot.cpp:32-123). The keys are taken by value and,
// as there, a key whose quaternion is flipped to keep consecutive keys within
// 90 degrees is rewritten in axis-angle form, so the next segments rebuild
// their quaternions from the rewritten key.
std::vector<Squad> rot_spline(std::vector<RotKey> k) {
    std::vector<Squad> segs;
    for (size_t i = 0; i + 3 < k.size(); i++) {
        RotKey &k0 = k[i], &k1 = k[i + 1], &k2 = k[i + 2], &k3 = k[i + 3];
        const Quat q0 = q_axis_angle(k0.angle, k0.ax, k0.ay, k0.az);
        const Quat q1 = q_axis_angle(k1.angle, k1.ax, k1.ay, k1.az);
        Quat q2 = q_axis_angle(k2.angle, k2.ax, k2.ay, k2.az);
        const Quat q3 = q_axis_angle(k3.angle, k3.ax, k3.ay, k3.az);
        if (q_dot(q1, q2) < 0.0) {
            q2 = {-q2.w, -q2.x, -q2.y, -q2.z};
            q_to_axis_angle(q2, k2.angle, k2.ax, k2.ay, k2.az);
        }
        const Quat logdq = q_log(q_mul(q_conj(q1), q2));
        const Tcb m = tcb(k0.t, k1.t, k2.t, k3.t, k1.tension, k1.continuity, k1.bias, k2.tension,
                          k2.continuity, k2.bias);
        const Quat tout = q_add(q_scale(logdq, m.out1), q_scale(q_log(q_mul(q_conj(q0), q1)), m.out0));
        const Quat tin = q_add(q_scale(logdq, m.in0), q_scale(q_log(q_mul(q_conj(q2), q3)), m.in1));
        const Quat arg0 = q_scale(q_sub(tout, logdq), 0.5);
        const Quat arg1 = q_scale(q_sub(logdq, tin), 0.5);
        Squad s;
        s.p = q1;
        s.q = q2;
        s.a = q_mul(q1, q_exp(arg0));
        s.b = q_mul(q2, q_exp(arg1));
        s.t0 = k1.t;
        s.t1 = k2.t;
        s.span = s.t1 - s.t0;
        segs.push_back(s);
    }
    return segs;
}

// KB_RotInterpolate + ToAngleAxis: axis (x, y, z) and angle in radians
void rot_eval(const std::vector<Squad> &s, double t, double out[4]) {
    size_t i;
    double u;
    locate(s, t, i, u);
    const Squad &g = s[i];
    const Quat q = q_slerp(2 * u * (1 - u), q_slerp(u, g.p, g.q), q_slerp(u, g.a, g.b));
    q_to_axis_angle(q, out[3], out[0], out[1], out[2]);
}

// ------------------------------------------------------------ matrices ----
// SPMatrix: row-vector convention, v' = v * M, translation in row 3.
struct M44 {
    float m[4][4];
};

M44 m_identity() {
    M44 r{};
    for (int i = 0; i < 4; i++) r.m[i][i] = 1.0f;
    return r;
}

M44 m_translate(float x, float y, float z) {
    M44 r = m_identity();
    r.m[3][0] = x;
    r.m[3][1] = y;
    r.m[3][2] = z;
    return r;
}

M44 m_scale(float x, float y, float z) {
    M44 r = m_identity();
    r.m[0][0] = x;
    r.m[1][1] = y;
    r.m[2][2] = z;
    return r;
}

// SPMatrix::rotateMatrix (HulkEngine/src/SPMatrix.cpp:54-83); the axis is
// used as given (not normalised), as there
M44 m_rotate(float x, float y, float z, float angle) {
    const float c = cosf(angle), s = sinf(angle), k = 1 - c;
    const float xy = k * x * y, xz = k * x * z, yz = k * y * z;
    M44 r{};
    r.m[0][0] = c + k * x * x;
    r.m[0][1] = xy - s * z;
    r.m[0][2] = xz + s * y;
    r.m[1][0] = xy + s * z;
    r.m[1][1] = c + k * y * y;
    r.m[1][2] = yz - s * x;
    r.m[2][0] = xz - s * y;
    r.m[2][1] = yz + s * x;
    r.m[2][2] = c + k * z * z;
    r.m[3][3] = 1.0f;
    return r;
}

// a * b with each output row accumulated left to right over b's rows
M44 m_mul(const M44 &a, const M44 &b) {
    M44 r;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float acc = a.m[i][0] * b.m[0][j];
            acc = acc + a.m[i][1] * b.m[1][j];
            acc = acc + a.m[i][2] * b.m[2][j];
            acc = acc + a.m[i][3] * b.m[3][j];
            r.m[i][j] = acc;
        }
    return r;
}

// ---------------------------------------------------------------- scene ----
struct Animation {
    std::string name;
    std::vector<Cubic> transl, scale;
    std::vector<Squad> rot;
    std::vector<std::pair<float, int>> visibility;
};

struct Xform {
    int parent;        // index of the enclosing transform, -1 at the root
    bool animated;     // "x" (keyframed) or "xs" (static)
    std::string name;  // "x"
    float scale[3], axis[3], deg, trans[3];  // "xs"
    int anim = -1;     // first animation with this name, after the parse
};

struct Mesh {
    int parent;
    bool dynamic;  // under at least one animated transform
    uint32_t v0, nv, t0, nt;
};

}  // namespace

struct hk_aff {
    std::vector<float> verts;    // rest pose, 4 per vertex (w = 1)
    std::vector<uint32_t> tris;  // 4 per triangle, global vertex indices
    std::vector<uint32_t> part;  // mesh index per vertex
    std::vector<Xform> xf;
    std::vector<Mesh> mesh;
    std::vector<Animation> anims;
    std::vector<float> lights;   // 8 per light: color.xyz, type (1 = point), pos.xyzw
    hk_aff_info info{};
    int camera_anim = -1;

    // parse state
    std::string dir;             // includes resolve against the top file's directory
    std::vector<int> stack;      // open transforms
    int detail = 0;              // "d" level; "i" files above it are skipped
    int depth = 0;

    const Animation *find(const char *name) const {
        for (const Animation &a : anims)
            if (a.name == name) return &a;
        return nullptr;
    }
};

namespace {

hk_status parse_file(hk_aff &A, const std::string &path);

hk_status syntax(const char *what) { return fail(HK_E_ILLEGAL_INPUT, std::string("AFF syntax error: ") + what); }

// "v" from at up angle hither resolution (AFFParser.cpp:107-155)
hk_status parse_view(hk_aff &A, Cursor &c) {
    hk_aff_info &I = A.info;
    float hither;
    int rx, ry;
    if (!c.expect("from") || !c.floats(I.from, 3)) return syntax("viewpoint from");
    if (!c.expect("at") || !c.floats(I.at, 3)) return syntax("viewpoint at");
    if (!c.expect("up") || !c.floats(I.up, 3)) return syntax("viewpoint up");
    if (!c.expect("angle") || !c.read_float(I.fov_deg)) return syntax("viewpoint angle");
    if (!c.expect("hither") || !c.read_float(hither)) return syntax("viewpoint hither");
    if (hither < 0.0001) hither = 1.0f;
    if (!c.expect("resolution") || !c.read_int(rx) || !c.read_int(ry)) return syntax("viewpoint resolution");
    I.hither = hither;
    I.resx = rx;
    I.resy = ry;
    I.has_view = 1;
    return HK_OK;
}

// "l" / "la name": position and optional color (AFFParser.cpp:178-227)
hk_status parse_light(hk_aff &A, Cursor &c) {
    int ch = c.get();
    if (ch == 'a') {
        std::string name;
        if (!c.read_word(name)) return syntax("animated light name");
    } else {
        c.unget();
    }
    float p[3], col[3] = {1.0f, 1.0f, 1.0f};
    if (!c.floats(p, 3)) return syntax("light position");
    c.skip_ws();
    float first;
    if (c.read_float(first)) {
        col[0] = first;
        if (!c.read_float(col[1]) || !c.read_float(col[2])) return syntax("light color");
    }
    c.skip_ws();
    A.lights.insert(A.lights.end(), {col[0], col[1], col[2], 1.0f, p[0], p[1], p[2], 1.0f});
    return HK_OK;
}

// "f r g b kd ks shine t ior" or "fm" with 12 numbers (AFFParser.cpp:286-345)
hk_status parse_fill(Cursor &c) {
    float v[12];
    int ch = c.get();
    if (ch == 'm') return c.floats(v, 12) ? HK_OK : syntax("fill material");
    c.unget();
    return c.floats(v, 8) ? HK_OK : syntax("fill color");
}

// "p n" (n vertices) or "pp n" (n vertices with normals) (AFFParser.cpp:455-515)
hk_status parse_poly(Cursor &c) {
    int ch = c.get();
    const bool patch = ch == 'p';
    if (!patch) c.unget();
    int n;
    if (!c.read_int(n) || n < 0) return syntax("polygon");
    float v[6];
    for (int i = 0; i < n; i++)
        if (!c.floats(v, patch ? 6 : 3)) return syntax("polygon vertex");
    return HK_OK;
}

// "tt name" / "ttp name" textured triangles, "tpa n" animated triangles
// (AFFParser.cpp:620-790)
hk_status parse_t(Cursor &c) {
    int ch = c.get();
    float v[8];
    if (ch == 't') {
        int p = c.get();
        const bool patch = p == 'p';
        if (!patch) c.unget();
        std::string tex;
        if (!c.read_word(tex)) return syntax("textured triangle");
        for (int q = 0; q < 3; q++)
            if (!c.floats(v, patch ? 8 : 5)) return syntax("textured triangle");
        c.skip_ws();
        return HK_OK;
    }
    if (ch == 'p') {
        if (c.get() != 'a') return HK_OK;  // "tp" followed by anything else is ignored there too
        int n;
        if (!c.read_int(n) || n < 0) return syntax("animated triangle");
        for (int q = 0; q < n; q++) {
            if (!c.floats(v, 1)) return syntax("animated triangle time");
            for (int w = 0; w < 3; w++)
                if (!c.floats(v, 6)) return syntax("animated triangle vertex");
        }
        return HK_OK;
    }
    return syntax("tt, ttp and tpa are the valid t codes");
}

// "xs s3 axis3 deg t3 {" or "x name {" (AFFParser.cpp:1074-1145)
hk_status parse_xform(hk_aff &A, Cursor &c) {
    Xform x;
    x.parent = A.stack.empty() ? -1 : A.stack.back();
    int ch = c.get();
    x.animated = ch != 's';
    if (x.animated) {
        c.unget();
        if (!c.read_word(x.name)) return syntax("transform name");
    } else {
        if (!c.floats(x.scale, 3) || !c.floats(x.axis, 3) || !c.read_float(x.deg) || !c.floats(x.trans, 3))
            return syntax("static transform");
    }
    c.skip_ws();
    if (c.get() != '{') return syntax("{ expected after a transform");
    A.stack.push_back((int)A.xf.size());
    A.xf.push_back(x);
    return HK_OK;
}

// "k name { transl|rot|scale|visibility n rows... }" (AFFParser.cpp:894-1060)
hk_status parse_keys(hk_aff &A, Cursor &c) {
    Animation an;
    if (!c.read_word(an.name)) return syntax("animation name");
    c.skip_ws();
    if (c.get() != '{') return syntax("{ expected after an animation name");
    c.skip_ws();
    int ch;
    while ((ch = c.get()) != '}') {
        if (ch == EOF) return syntax("unterminated animation");
        c.unget();
        std::string motion;
        int n;
        if (!c.read_word(motion) || !c.read_int(n)) return syntax("keyframe motion and count");
        const bool vis = motion == "visibility";
        if (n < 4 && !vis) return syntax("at least 4 keyframes are needed");
        if (motion == "transl" || motion == "scale") {
            std::vector<PosKey> keys(n);
            for (PosKey &k : keys) {
                float f[7];
                if (!c.floats(f, 7)) return syntax("position keyframe");
                k = {f[0], {f[1], f[2], f[3]}, f[4], f[5], f[6]};
            }
            (motion == "transl" ? an.transl : an.scale) = pos_spline(keys);
        } else if (motion == "rot") {
            std::vector<RotKey> keys(n);
            for (RotKey &k : keys) {
                float f[8];
                if (!c.floats(f, 8)) return syntax("rotation keyframe");
                // degrees to radians in double, from the single-precision value read
                k = {f[0], f[1], f[2], f[3], f[4] * M_PI / 180.0, f[5], f[6], f[7]};
            }
            an.rot = rot_spline(keys);
        } else if (vis) {
            for (int i = 0; i < n; i++) {
                float t;
                int v;
                if (!c.read_float(t) || !c.read_int(v)) return syntax("visibility keyframe");
                an.visibility.push_back({t, v});
            }
        } else {
            return syntax("keyframe type must be transl, rot, scale or visibility");
        }
        c.skip_ws();
    }
    A.anims.push_back(std::move(an));
    return HK_OK;
}

// "m vertices n ... [normals n ...] [texturecoords n name ...] triangles n ..."
// (AFFParser.cpp:1215-1449). Indices are stored as the reference stores them,
// in 16 bits, and must then fall inside the mesh.
hk_status parse_mesh(hk_aff &A, Cursor &c) {
    std::string w;
    int nv = 0, nn = 0, nt = 0, ntx = 0;
    if (!c.read_word(w) || w != "vertices") return syntax("mesh: 'vertices' expected");
    if (!c.read_int(nv) || nv < 0) return syntax("mesh vertex count");
    const uint32_t v0 = (uint32_t)(A.verts.size() / 4);
    const uint32_t mesh_id = (uint32_t)A.mesh.size();
    for (int i = 0; i < nv; i++) {
        float p[3];
        if (!c.floats(p, 3)) return syntax("mesh vertex");
        A.verts.insert(A.verts.end(), {p[0], p[1], p[2], 1.0f});
        A.part.push_back(mesh_id);
    }
    c.skip_ws();
    c.read_word(w);
    const bool normals = w == "normals";
    if (normals) {
        if (!c.read_int(nn) || nn < 0) return syntax("mesh normal count");
        float p[3];
        for (int i = 0; i < nn; i++)
            if (!c.floats(p, 3)) return syntax("mesh normal");
        c.read_word(w);
    }
    // getTriangles reads normal (texture) indices whenever the mesh declared
    // a normals (texturecoords) section, even an empty one
    bool textures = false;
    if (w == "texturecoords") {
        std::string tex;
        if (!c.read_int(ntx) || ntx < 0) return syntax("mesh texture coordinate count");
        if (!c.read_word(tex)) return syntax("mesh texture name");
        float p[2];
        for (int i = 0; i < ntx; i++)
            if (!c.floats(p, 2)) return syntax("mesh texture coordinate");
        textures = true;
        c.read_word(w);
    }
    if (w != "triangles") return syntax("mesh: 'triangles' expected");
    if (!c.read_int(nt) || nt < 0) return syntax("mesh triangle count");
    const uint32_t t0 = (uint32_t)(A.tris.size() / 4);
    for (int i = 0; i < nt; i++) {
        int v[3], x[3];
        if (!c.read_int(v[0]) || !c.read_int(v[1]) || !c.read_int(v[2])) return syntax("mesh triangle");
        if (normals && (!c.read_int(x[0]) || !c.read_int(x[1]) || !c.read_int(x[2])))
            return syntax("mesh normal indices");
        if (textures && (!c.read_int(x[0]) || !c.read_int(x[1]) || !c.read_int(x[2])))
            return syntax("mesh texture indices");
        uint32_t g[3];
        for (int k = 0; k < 3; k++) {
            const uint32_t local = (uint16_t)v[k];
            if (local >= (uint32_t)nv) return syntax("mesh triangle index outside the mesh");
            g[k] = v0 + local;
        }
        A.tris.insert(A.tris.end(), {g[0], g[1], g[2], 0u});
    }
    Mesh m;
    m.parent = A.stack.empty() ? -1 : A.stack.back();
    m.dynamic = false;
    for (int s : A.stack)
        if (A.xf[s].animated) m.dynamic = true;
    m.v0 = v0;
    m.nv = (uint32_t)nv;
    m.t0 = t0;
    m.nt = (uint32_t)nt;
    A.mesh.push_back(m);
    return HK_OK;
}

// the command loop of AFFParser::viParseFile (AFFParser.cpp:1469-1539)
hk_status parse_text(hk_aff &A, Cursor &c) {
    int ch;
    while ((ch = c.get()) != EOF) {
        hk_status s = HK_OK;
        switch (ch) {
            case ' ': case '\t': case '\n': case '\f': case '\r':
                continue;
            case '#': case '%':
                c.drop_line();
                break;
            case 'v':
                s = parse_view(A, c);
                break;
            case 'l':
                s = parse_light(A, c);
                break;
            case 'b': {
                float v[3];
                if (!c.floats(v, 3)) s = syntax("background color");
                break;
            }
            case 'f':
                s = parse_fill(c);
                break;
            case 'c': {
                float v[8];
                if (!c.floats(v, 8)) s = syntax("cylinder or cone");
                break;
            }
            case 's': {
                float v[4];
                if (!c.floats(v, 4)) s = syntax("sphere");
                break;
            }
            case 'p':
                s = parse_poly(c);
                break;
            case 'i': {
                int level;
                std::string name;
                if (!c.read_int(level) || !c.read_word(name)) {
                    s = syntax("include");
                    break;
                }
                if (level <= A.detail) s = parse_file(A, A.dir + name);
                break;
            }
            case 'd':
                if (!c.read_int(A.detail)) s = syntax("detail level");
                break;
            case 't':
                s = parse_t(c);
                break;
            case 'x':
                s = parse_xform(A, c);
                break;
            case '}':
                if (A.stack.empty()) s = syntax("'}' without an open transform");
                else A.stack.pop_back();
                break;
            case 'a': {
                int m = c.get();
                if (m == 'm') {
                    float v[3];
                    if (!c.floats(v, 3)) s = syntax("ambient light");
                } else {
                    c.unget();
                    float st, en;
                    int nf;
                    if (!c.read_float(st) || !c.read_float(en) || !c.read_int(nf)) {
                        s = syntax("animation parameters");
                    } else {
                        A.info.has_anim_params = 1;
                        A.info.anim_start = st;
                        A.info.anim_end = en;
                        A.info.anim_frames = nf;
                    }
                }
                break;
            }
            case 'k':
                s = parse_keys(A, c);
                break;
            case 'm':
                s = parse_mesh(A, c);
                break;
            default: {
                char buf[64];
                snprintf(buf, sizeof buf, "unknown command code '%c'", (char)ch);
                s = syntax(buf);
            }
        }
        if (s != HK_OK) return s;
    }
    return HK_OK;
}

hk_status parse_file(hk_aff &A, const std::string &path) {
    if (++A.depth > 64) return syntax("includes nested deeper than 64 files");
    Cursor c;
    if (!read_file(path, c.text)) return fail(HK_E_FILE_OPEN, "cannot open AFF file " + path);
    hk_status s = parse_text(A, c);
    if (s != HK_OK && t_aff_error.find(" (in ") == std::string::npos) t_aff_error += " (in " + path + ")";
    A.depth--;
    return s;
}

// world matrices of every transform at time t (AFFTransformVisitor::preAct,
// AFFTransformVisitor.cpp:25-88). Parents precede children in A.xf.
void world_matrices(const hk_aff &A, float time, std::vector<M44> &W) {
    W.resize(A.xf.size());
    const double t = time;
    for (size_t i = 0; i < A.xf.size(); i++) {
        const Xform &x = A.xf[i];
        M44 m = x.parent < 0 ? m_identity() : W[x.parent];
        if (x.animated) {
            if (x.anim >= 0) {
                const Animation &an = A.anims[x.anim];
                if (!an.transl.empty()) {
                    const V3 p = pos_eval(an.transl, t);
                    m = m_mul(m_translate((float)p.x, (float)p.y, (float)p.z), m);
                }
                if (!an.rot.empty()) {
                    double r[4];
                    rot_eval(an.rot, t, r);
                    m = m_mul(m_rotate((float)r[0], (float)r[1], (float)r[2], (float)-r[3]), m);
                }
                if (!an.scale.empty()) {
                    const V3 s = pos_eval(an.scale, t);
                    m = m_mul(m_scale((float)s.x, (float)s.y, (float)s.z), m);
                }
            }
        } else {
            const M44 tp = m_mul(m_translate(x.trans[0], x.trans[1], x.trans[2]), m);
            const M44 sr = m_mul(m_scale(x.scale[0], x.scale[1], x.scale[2]),
                                 m_rotate(x.axis[0], x.axis[1], x.axis[2], (float)(x.deg * M_PI / 180.0)));
            m = m_mul(sr, tp);
        }
        W[i] = m;
    }
}

hk_status check(const hk_aff *a) { return a ? HK_OK : fail(HK_E_ILLEGAL_INPUT, "null AFF handle"); }

}  // namespace

extern "C" {

const char *hk_aff_last_error(void) { return t_aff_error.c_str(); }

hk_status hk_aff_open(const char *path, hk_aff **out) {
    if (!path || !out) return fail(HK_E_ILLEGAL_INPUT, "null argument");
    *out = nullptr;
    hk_aff *A = new (std::nothrow) hk_aff();
    if (!A) return fail(HK_E_ALLOC, "out of host memory");
    std::string p(path);
    const size_t slash = p.find_last_of('/');
    A->dir = slash == std::string::npos ? std::string() : p.substr(0, slash + 1);
    t_aff_error.clear();
    hk_status s = parse_file(*A, p);
    if (s == HK_OK && !A->stack.empty()) s = syntax("transform block not closed at the end of the file");
    if (s != HK_OK) {
        delete A;
        return s;
    }
    for (Xform &x : A->xf)
        if (x.animated)
            for (size_t k = 0; k < A->anims.size(); k++)
                if (A->anims[k].name == x.name) {
                    x.anim = (int)k;
                    break;
                }
    for (size_t k = 0; k < A->anims.size(); k++)
        if (A->anims[k].name == "camera") {
            A->camera_anim = (int)k;
            break;
        }
    hk_aff_info &I = A->info;
    I.nv = (uint32_t)(A->verts.size() / 4);
    I.nt = (uint32_t)(A->tris.size() / 4);
    I.nmeshes = (uint32_t)A->mesh.size();
    I.ntransforms = (uint32_t)A->xf.size();
    I.nanimations = (uint32_t)A->anims.size();
    I.nlights = (uint32_t)(A->lights.size() / 8);
    I.ndynamic = 0;
    for (const Mesh &m : A->mesh) I.ndynamic += m.dynamic ? 1u : 0u;
    I.has_camera_anim = A->camera_anim >= 0;
    if (!I.has_view) {  // the reference Scene's defaults (HulkEngine/src/Scene.cpp:21-27)
        I.fov_deg = 45.0f;
        I.resx = 800;
        I.resy = 600;
    }
    *out = A;
    return HK_OK;
}

hk_status hk_aff_close(hk_aff *aff) {
    delete aff;
    return HK_OK;
}

hk_status hk_aff_get_info(const hk_aff *aff, hk_aff_info *info) {
    if (check(aff) != HK_OK || !info) return fail(HK_E_ILLEGAL_INPUT, "null argument");
    *info = aff->info;
    return HK_OK;
}

hk_status hk_aff_geometry(const hk_aff *aff, float *verts4, uint32_t *tris4, uint32_t *part_of_vertex) {
    if (check(aff) != HK_OK) return HK_E_ILLEGAL_INPUT;
    if (verts4) memcpy(verts4, aff->verts.data(), aff->verts.size() * sizeof(float));
    if (tris4) memcpy(tris4, aff->tris.data(), aff->tris.size() * sizeof(uint32_t));
    if (part_of_vertex) memcpy(part_of_vertex, aff->part.data(), aff->part.size() * sizeof(uint32_t));
    return HK_OK;
}

hk_status hk_aff_part_matrices(const hk_aff *aff, float time, float *mats12) {
    if (check(aff) != HK_OK || !mats12) return fail(HK_E_ILLEGAL_INPUT, "null argument");
    std::vector<M44> W;
    world_matrices(*aff, time, W);
    for (size_t k = 0; k < aff->mesh.size(); k++) {
        const int p = aff->mesh[k].parent;
        const M44 m = p < 0 ? m_identity() : W[p];
        float *o = mats12 + 12 * k;
        // output component i = x M[0][i] + y M[1][i] + z M[2][i] + M[3][i]
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 4; j++) o[4 * i + j] = m.m[j][i];
    }
    return HK_OK;
}

hk_status hk_aff_lights(const hk_aff *aff, float *lights8) {
    if (check(aff) != HK_OK || !lights8) return fail(HK_E_ILLEGAL_INPUT, "null argument");
    memcpy(lights8, aff->lights.data(), aff->lights.size() * sizeof(float));
    return HK_OK;
}

// GLVisitorCPUTrace::updateCamera (HulkEngine/src/GLVisitorCPUTrace.cpp:
// 105-146): the "camera" animation's translation moves the eye from the
// origin, its rotation turns the -z view direction, and the image plane spans
// tan(fov / 2) vertically and that times the aspect ratio horizontally.
hk_status hk_aff_camera(const hk_aff *aff, float time, float *cam16) {
    if (check(aff) != HK_OK || !cam16) return fail(HK_E_ILLEGAL_INPUT, "null argument");
    double tr[3] = {0, 0, 0}, rot[4] = {0, 0, 0, 0};
    if (aff->camera_anim >= 0) {
        const Animation &an = aff->anims[aff->camera_anim];
        if (!an.rot.empty()) rot_eval(an.rot, (double)time, rot);
        if (!an.transl.empty()) {
            const V3 p = pos_eval(an.transl, (double)time);
            tr[0] = p.x;
            tr[1] = p.y;
            tr[2] = p.z;
        }
    }
    const M44 T = m_translate((float)tr[0], (float)tr[1], (float)tr[2]);
    const M44 R = m_rotate((float)rot[0], (float)rot[1], (float)rot[2], -(float)rot[3]);
    // (x, y, z, 1) * M, accumulated left to right
    auto apply = [](const float v[4], const M44 &m, float o[4]) {
        for (int j = 0; j < 4; j++) {
            float acc = v[0] * m.m[0][j];
            acc = acc + v[1] * m.m[1][j];
            acc = acc + v[2] * m.m[2][j];
            acc = acc + v[3] * m.m[3][j];
            o[j] = acc;
        }
    };
    const float o0[4] = {0, 0, 0, 1}, d0[4] = {0, -1, 0, 1}, l0[4] = {-1, 0, 0, 1}, t0[4] = {0, 0, -1, 1};
    float from[4], down[4], left[4], to[4];
    apply(o0, T, from);
    apply(d0, R, down);
    apply(l0, R, left);
    apply(t0, R, to);
    down[3] = left[3] = to[3] = from[3] = 0.0f;
    const hk_aff_info &I = aff->info;
    const float aspect = I.has_view ? (float)I.resx / (float)I.resy : 800.0f / 600.0f;
    const float vf = tanf(I.fov_deg * 0.017453292519943f / 2);
    const float hf = vf * aspect;
    for (int k = 0; k < 4; k++) {
        down[k] = down[k] * vf;
        left[k] = left[k] * hf;
    }
    for (int k = 0; k < 4; k++) {
        cam16[k] = from[k];
        cam16[4 + k] = left[k] * -2.0f;
        cam16[8 + k] = down[k] * -2.0f;
        cam16[12 + k] = from[k] + to[k] + down[k] + left[k];
    }
    return HK_OK;
}

hk_status hk_scene_load_aff(hk_ctx *ctx, const hk_aff *aff, float time) {
    if (!ctx || check(aff) != HK_OK) return HK_E_ILLEGAL_INPUT;
    const hk_aff_info &I = aff->info;
    if (I.nt == 0 || I.nmeshes == 0) return fail(HK_E_ILLEGAL_INPUT, "AFF scene has no triangles");
    hk_status s = hk_scene_upload(ctx, aff->verts.data(), I.nv, aff->tris.data(), I.nt);
    if (s != HK_OK) return s;
    s = hk_scene_set_parts(ctx, aff->part.data(), I.nmeshes);
    if (s != HK_OK) return s;
    return hk_scene_animate_aff(ctx, aff, time);
}

hk_status hk_scene_animate_aff(hk_ctx *ctx, const hk_aff *aff, float time) {
    if (!ctx || check(aff) != HK_OK) return HK_E_ILLEGAL_INPUT;
    std::vector<float> mats(12 * (size_t)aff->info.nmeshes);
    hk_status s = hk_aff_part_matrices(aff, time, mats.data());
    if (s != HK_OK) return s;
    return hk_scene_transform(ctx, mats.data());
}

}  // extern "C"
