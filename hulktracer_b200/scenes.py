"""Seeded procedural scenes and cameras for the ray-tracing hot path.

Every scene is an indexed triangle soup in the reference's scene-array layout
(``Scene::m_vertices`` / ``Scene::m_vertexIndices``, HulkEngine/public/Scene.hpp:
68-71): vertices as ``float32[V, 4]`` with ``w = 1`` (HulkEngine/src/
Intersectable.cpp:54) and triangles as ``uint32[T, 4]`` (``TriangleIndices``,
HulkEngine/public/SharedStructs.hpp:37-41; the 4th index is padding).

The reference only loads AFF/OBJ files; these generators stand in for them with
the shapes and sizes of the benchmark scenes:

* ``static_small``  -- 64x64 quad ground grid over [-10,10]^2 at y=0 (8,192 tris)
  plus 32 UV spheres of 16x16 segments (512 tris each), 24,576 triangles.
* ``static_large``  -- 200 Gaussian clusters of small randomly oriented
  triangles in a 100^3 box plus 24 axis-aligned wall quads of 2,048 tris.
* ``animated_parts`` -- 64 rigid parts (geodesic spheres, boxes, tori of about
  3,100 triangles each) with per-part rotation and drift, ~200k triangles.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Scene:
    verts: np.ndarray                     # float32 [V, 4], w = 1
    tris: np.ndarray                      # uint32 [T, 4]
    lights: np.ndarray                    # float32 [L, 8]: color.xyz,type | pos-or-dir.xyzw
    camera: np.ndarray                    # float32 [4, 4]: from, vertical, horizontal, lowerLeft
    width: int
    height: int
    name: str = ""
    # rigid animation (animated scenes only)
    part_of_vertex: np.ndarray | None = None   # uint32 [V]
    rest_verts: np.ndarray | None = None       # float32 [V, 4], untransformed
    part_center: np.ndarray | None = None      # float64 [P, 3]
    part_axis: np.ndarray | None = None        # float64 [P, 3]
    part_omega: np.ndarray | None = None       # float64 [P]
    part_drift: np.ndarray | None = None       # float64 [P, 3]
    extra: dict = field(default_factory=dict)

    @property
    def ntris(self) -> int:
        return int(self.tris.shape[0])

    def scene_box(self) -> np.ndarray:
        """Axis-aligned bounds of all vertices as float32[8] (min.xyzw, max.xyzw)."""
        return scene_box(self.verts)


E_DIRECTIONAL = 0.0
E_POINT = 1.0


def scene_box(verts: np.ndarray) -> np.ndarray:
    v = verts[:, :3]
    mn = v.min(axis=0)
    mx = v.max(axis=0)
    return np.array([mn[0], mn[1], mn[2], 1.0, mx[0], mx[1], mx[2], 1.0], dtype=np.float32)


def point_light(pos, color=(1.0, 1.0, 1.0)) -> np.ndarray:
    """Point light in the reference ``Light`` layout (SharedStructs.hpp:50-63):
    color.w holds the light type."""
    return np.array([color[0], color[1], color[2], E_POINT, pos[0], pos[1], pos[2], 0.0],
                    dtype=np.float32)


def directional_light(direction, color=(1.0, 1.0, 1.0)) -> np.ndarray:
    d = np.asarray(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    return np.array([color[0], color[1], color[2], E_DIRECTIONAL, d[0], d[1], d[2], 0.0],
                    dtype=np.float32)


def look_at_camera(eye, target, fov_deg: float, width: int, height: int) -> np.ndarray:
    """Pinhole camera in the reference ``CameraPos`` layout (SharedStructs.hpp:99-105).

    Mirrors ``GLVisitorCPUTrace::updateCamera`` (HulkEngine/src/GLVisitorCPUTrace.cpp:
    105-148): ``lowerLeft = from + to + down + left`` with ``|down| = tan(fov/2)``,
    ``|left| = |down| * aspect``; ``verticalFactor = -2 left`` spans the image
    left to right and ``horizontalFactor = -2 down`` spans it bottom to top.
    All w components are 0.
    """
    eye = np.asarray(eye, dtype=np.float64)
    fwd = np.asarray(target, dtype=np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    up = np.array([0.0, 1.0, 0.0])
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    true_up = np.cross(right, fwd)
    vfac = math.tan(math.radians(fov_deg) / 2.0)
    hfac = vfac * (width / height)
    down = -true_up * vfac
    left = -right * hfac
    lower_left = eye + fwd + down + left
    cam = np.zeros((4, 4), dtype=np.float32)
    cam[0, :3] = eye
    cam[1, :3] = left * -2.0
    cam[2, :3] = down * -2.0
    cam[3, :3] = lower_left
    return cam


# ----------------------------------------------------------------------------
# mesh primitives (float64, centred at the origin)
# ----------------------------------------------------------------------------

def _grid(n: int, lo: float, hi: float, y: float = 0.0):
    xs = np.linspace(lo, hi, n + 1)
    gx, gz = np.meshgrid(xs, xs, indexing="ij")
    v = np.stack([gx.ravel(), np.full(gx.size, y), gz.ravel()], axis=1)
    i = np.arange(n)
    a = (i[:, None] * (n + 1) + i[None, :]).ravel()
    b = a + 1
    c = a + (n + 1)
    d = c + 1
    t = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], axis=0)
    return v, t


def _uv_sphere(seg: int):
    """seg x seg quads -> 2*seg*seg triangles; pole quads keep their zero-area
    half so each sphere has exactly 2*seg^2 triangles."""
    th = np.linspace(0.0, math.pi, seg + 1)
    ph = np.linspace(0.0, 2.0 * math.pi, seg + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    v = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], axis=-1).reshape(-1, 3)
    i = np.arange(seg)
    a = (i[:, None] * (seg + 1) + i[None, :]).ravel()
    b = a + 1
    c = a + (seg + 1)
    d = c + 1
    t = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], axis=0)
    return v, t


def _geodesic_sphere(freq: int):
    """Icosahedron with each face split into freq^2 triangles, projected to the
    unit sphere (20 * freq^2 triangles)."""
    p = (1.0 + 5 ** 0.5) / 2.0
    iv = np.array([[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0], [0, -1, p], [0, 1, p],
                   [0, -1, -p], [0, 1, -p], [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], float)
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts, tris = [], []
    for (ia, ib, ic) in faces:
        A, B, C = iv[ia], iv[ib], iv[ic]
        base = len(verts)
        idx = {}
        for r in range(freq + 1):
            for s in range(freq + 1 - r):
                idx[(r, s)] = len(verts)
                w = freq - r - s
                verts.append((A * w + B * r + C * s) / freq)
        for r in range(freq):
            for s in range(freq - r):
                tris.append((idx[(r, s)], idx[(r + 1, s)], idx[(r, s + 1)]))
                if s + r + 1 < freq:
                    tris.append((idx[(r + 1, s)], idx[(r + 1, s + 1)], idx[(r, s + 1)]))
        del base
    v = np.asarray(verts)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v, np.asarray(tris, dtype=np.int64)


def _box(n: int):
    """Unit cube [-1,1]^3 with each face split into n x n quads (12 n^2 tris)."""
    vs, ts = [], []
    off = 0
    g = np.linspace(-1.0, 1.0, n + 1)
    U, V = np.meshgrid(g, g, indexing="ij")
    i = np.arange(n)
    a = (i[:, None] * (n + 1) + i[None, :]).ravel()
    b = a + 1
    c = a + (n + 1)
    d = c + 1
    quad = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], axis=0)
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            p = np.zeros((U.size, 3))
            p[:, axis] = sgn
            p[:, (axis + 1) % 3] = U.ravel()
            p[:, (axis + 2) % 3] = V.ravel()
            vs.append(p)
            ts.append(quad + off)
            off += p.shape[0]
    return np.concatenate(vs), np.concatenate(ts)


def _torus(nu: int, nv: int, R: float = 1.0, r: float = 0.35):
    u = np.linspace(0.0, 2 * math.pi, nu, endpoint=False)
    w = np.linspace(0.0, 2 * math.pi, nv, endpoint=False)
    U, W = np.meshgrid(u, w, indexing="ij")
    v = np.stack([(R + r * np.cos(W)) * np.cos(U), r * np.sin(W), (R + r * np.cos(W)) * np.sin(U)],
                 axis=-1).reshape(-1, 3)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = (i * nv + j).ravel()
    b = (i * nv + (j + 1) % nv).ravel()
    c = (((i + 1) % nu) * nv + j).ravel()
    d = (((i + 1) % nu) * nv + (j + 1) % nv).ravel()
    t = np.concatenate([np.stack([a, c, b], 1), np.stack([b, c, d], 1)], axis=0)
    return v, t


def _pack(vs, ts):
    """Concatenate float64 vertex / int triangle lists into the scene arrays."""
    verts, tris, off = [], [], 0
    for v, t in zip(vs, ts):
        verts.append(v)
        tris.append(t + off)
        off += v.shape[0]
    v = np.concatenate(verts)
    t = np.concatenate(tris)
    V = np.ones((v.shape[0], 4), dtype=np.float32)
    V[:, :3] = v.astype(np.float32)
    T = np.zeros((t.shape[0], 4), dtype=np.uint32)
    T[:, :3] = t.astype(np.uint32)
    return V, T


# ----------------------------------------------------------------------------
# benchmark scenes
# ----------------------------------------------------------------------------

def static_small(seed: int = 1, width: int = 512, height: int = 512) -> Scene:
    """24,576 triangles: ground grid + 32 UV spheres, one point light."""
    rng = np.random.default_rng(seed)
    vs, ts = [], []
    v, t = _grid(64, -10.0, 10.0, 0.0)
    vs.append(v)
    ts.append(t)
    sv, st = _uv_sphere(16)
    for _ in range(32):
        r = rng.uniform(0.3, 1.5)
        c = np.array([rng.uniform(-9, 9), rng.uniform(0.5, 4.0), rng.uniform(-9, 9)])
        vs.append(sv * r + c)
        ts.append(st)
    V, T = _pack(vs, ts)
    cam = look_at_camera((0.0, 6.0, 18.0), (0.0, 1.0, 0.0), 60.0, width, height)
    lights = np.stack([point_light((5.0, 12.0, 5.0))])
    return Scene(V, T, lights, cam, width, height, name="static_small_24k")


def _random_small_tris(rng, n, centers, sigmas, cluster_of):
    """n triangles with edge lengths U(0.01, 0.2) and uniformly random orientation."""
    c = centers[cluster_of] + rng.normal(size=(n, 3)) * sigmas[cluster_of, None]
    # random orthonormal frame per triangle
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)
    e1 = rng.uniform(0.01, 0.2, n)
    e2 = rng.uniform(0.01, 0.2, n)
    ang = rng.uniform(0.3, 2.8, n)
    p0 = np.zeros((n, 3))
    p1 = np.stack([e1, np.zeros(n), np.zeros(n)], 1)
    p2 = np.stack([e2 * np.cos(ang), e2 * np.sin(ang), np.zeros(n)], 1)
    cen = (p0 + p1 + p2) / 3.0
    pts = np.stack([p0 - cen, p1 - cen, p2 - cen], 1)             # [n,3,3]
    pts = np.einsum("nij,nkj->nki", R, pts) + c[:, None, :]
    v = pts.reshape(-1, 3)
    t = np.arange(3 * n).reshape(n, 3)
    return v, t


def static_large(seed: int = 2, width: int = 1920, height: int = 1080,
                 n_cluster_tris: int = 1_000_000) -> Scene:
    """1,000,000 clustered small triangles + 24 wall quads x 2,048 tris."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-50, 50, size=(200, 3))
    sigmas = rng.uniform(0.2, 2.0, size=200)
    cluster_of = rng.integers(0, 200, size=n_cluster_tris)
    vs, ts = [], []
    v, t = _random_small_tris(rng, n_cluster_tris, centers, sigmas, cluster_of)
    vs.append(v)
    ts.append(t)
    # 24 axis-aligned wall quads (32x32 quads = 2048 tris each) forming rooms
    g = np.linspace(-1.0, 1.0, 33)
    U, W = np.meshgrid(g, g, indexing="ij")
    i = np.arange(32)
    a = (i[:, None] * 33 + i[None, :]).ravel()
    quad = np.concatenate([np.stack([a, a + 33, a + 1], 1), np.stack([a + 1, a + 33, a + 34], 1)])
    for k in range(24):
        axis = k % 3
        pos = -50.0 + 100.0 * ((k // 3) + 0.5) / 8.0
        p = np.zeros((U.size, 3))
        p[:, axis] = pos
        p[:, (axis + 1) % 3] = U.ravel() * 50.0
        p[:, (axis + 2) % 3] = W.ravel() * 50.0
        vs.append(p)
        ts.append(quad)
    V, T = _pack(vs, ts)
    cam = look_at_camera((0.0, 10.0, 120.0), (0.0, 0.0, 0.0), 60.0, width, height)
    lights = np.stack([point_light((30.0, 80.0, 60.0))])
    sc = Scene(V, T, lights, cam, width, height, name="static_large_1M")
    # mirror material on 30% of triangles (hash of the triangle index)
    h = (np.arange(T.shape[0], dtype=np.uint64) * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    sc.extra["mirror"] = (h.astype(np.float64) / 4294967296.0 < 0.3).astype(np.uint8)
    return sc


def animated_parts(seed: int = 3, width: int = 1280, height: int = 720, n_parts: int = 64,
                   scale: float = 1.0) -> Scene:
    """64 rigid parts (~3,100 triangles each, ~200k total) with per-part rotation
    axis, angular speed U(0.1,1) rad/frame and linear drift U(-0.05,0.05)^3."""
    rng = np.random.default_rng(seed)
    prims = [_geodesic_sphere(12), _box(16), _torus(57, 30)]
    vs, ts, parts, centers = [], [], [], []
    for p in range(n_parts):
        v, t = prims[p % 3]
        size = rng.uniform(2.5, 4.0) * scale
        c = rng.uniform([-12, -6, -12], [12, 6, 12]) * scale
        vs.append(v * size + c)
        ts.append(t)
        parts.append(np.full(v.shape[0], p, dtype=np.uint32))
        centers.append(c)
    V, T = _pack(vs, ts)
    axis = rng.normal(size=(n_parts, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    omega = rng.uniform(0.1, 1.0, size=n_parts)
    drift = rng.uniform(-0.05, 0.05, size=(n_parts, 3))
    # parts fill about three quarters of the view
    cam = look_at_camera((0.0, 7.0 * scale, 20.0 * scale), (0.0, 0.0, 0.0), 60.0, width, height)
    lights = np.stack([point_light((20.0 * scale, 30.0 * scale, 25.0 * scale))])
    sc = Scene(V, T, lights, cam, width, height, name="animated_parts_200k",
               part_of_vertex=np.concatenate(parts), rest_verts=V.copy(),
               part_center=np.asarray(centers), part_axis=axis, part_omega=omega, part_drift=drift)
    return sc


def from_aff(path: str) -> Scene:
    """An AFF (BART) scene file as an animated scene: one part per mesh, the
    rest pose as vertices, the file's lights (one white point light above the
    scene when it has none), resolution and camera. Frame f is the reference's
    fixed-tick time f / 10 (engine.fixed_tick_time); its part matrices and
    camera come from the file's keyframes (``part_matrices``, ``frame_camera``)."""
    import os

    from .engine import Aff
    aff = Aff(path)
    i = aff.info
    verts, tris, part = aff.geometry()
    lights = aff.lights()
    if lights.shape[0] == 0:
        box = scene_box(verts)
        lights = np.array([[1, 1, 1, E_POINT, (box[0] + box[4]) / 2, box[5] + (box[5] - box[1]), (box[2] + box[6]) / 2,
                            1]], np.float32)
    w, h = max(8, i["resx"] // 8 * 8), max(4, i["resy"] // 4 * 4)
    return Scene(verts=verts, tris=tris, lights=lights, camera=aff.camera(0.0).reshape(4, 4), width=w, height=h,
                 name="aff_" + os.path.splitext(os.path.basename(path))[0], part_of_vertex=part, rest_verts=verts,
                 part_center=np.zeros((i["nmeshes"], 3)), extra={"aff": aff})


def frame_camera(sc: Scene, frame: int) -> np.ndarray:
    """The camera of ``frame``: an AFF scene's "camera" animation, else fixed."""
    if "aff" in sc.extra:
        from .engine import fixed_tick_time
        return sc.extra["aff"].camera(fixed_tick_time(frame)).reshape(4, 4)
    return sc.camera


def part_matrices(sc: Scene, frame: int) -> np.ndarray:
    """Per-part 3x4 row-major rigid transforms (float32[P, 12]) for ``frame``:
    rotate about the part centre by omega*frame around its axis, then drift
    (an AFF scene: its keyframed transforms at the frame's time)."""
    if "aff" in sc.extra:
        from .engine import fixed_tick_time
        return sc.extra["aff"].part_matrices(fixed_tick_time(frame))
    P = sc.part_center.shape[0]
    out = np.zeros((P, 12), dtype=np.float32)
    for p in range(P):
        a = sc.part_axis[p]
        th = sc.part_omega[p] * frame
        c, s = math.cos(th), math.sin(th)
        x, y, z = a
        R = np.array([[c + x * x * (1 - c), x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                      [y * x * (1 - c) + z * s, c + y * y * (1 - c), y * z * (1 - c) - x * s],
                      [z * x * (1 - c) - y * s, z * y * (1 - c) + x * s, c + z * z * (1 - c)]])
        ctr = sc.part_center[p]
        t = ctr - R @ ctr + sc.part_drift[p] * frame
        M = np.concatenate([R, t[:, None]], axis=1)
        out[p] = M.astype(np.float32).ravel()
    return out


def random_soup(n: int, seed: int = 0, extent: float = 10.0, size: float = 1.0) -> Scene:
    """Random triangle soup for small parity cases."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-extent, extent, size=(n, 3))
    d = rng.normal(size=(n, 3, 3)) * size
    v = (c[:, None, :] + d).reshape(-1, 3)
    t = np.arange(3 * n).reshape(n, 3)
    V, T = _pack([v], [t])
    cam = look_at_camera((0.0, 0.5 * extent, 2.2 * extent), (0.0, 0.0, 0.0), 60.0, 64, 64)
    lights = np.stack([point_light((extent, 2 * extent, extent))])
    return Scene(V, T, lights, cam, 64, 64, name="soup%d" % n)


# ----------------------------------------------------------------------------
# batched scenes and incoherent rays
# ----------------------------------------------------------------------------

def cluster_soup(n_tris: int, seed: int, n_clusters: int = 64, extent: float = 50.0) -> Scene:
    """Clustered small random triangles (the large static generator at any size)."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-extent, extent, size=(n_clusters, 3))
    sigmas = rng.uniform(0.05, 0.4, size=n_clusters) * extent
    cluster_of = rng.integers(0, n_clusters, size=n_tris)
    v, t = _random_small_tris(rng, n_tris, centers, sigmas, cluster_of)
    V, T = _pack([v], [t])
    cam = look_at_camera((0.0, 0.3 * extent, 2.2 * extent), (0.0, 0.0, 0.0), 60.0, 256, 256)
    lights = np.stack([point_light((0.6 * extent, 1.6 * extent, 1.2 * extent))])
    return Scene(V, T, lights, cam, 256, 256, name="soup%d" % n_tris)


def incoherent_rays(sc: Scene, n: int, seed: int) -> np.ndarray:
    """A quarter primary rays through random pixels; the rest leave random
    points of random triangles in cosine-weighted directions about the face
    normal (stand-ins for shadow rays and two diffuse bounces). float32
    [n, 8], directions normalised, w = 0."""
    rng = np.random.default_rng(seed)
    n_prim = n // 4
    out = np.zeros((n, 8), np.float32)
    cam = sc.camera.astype(np.float64)
    u = rng.random(n_prim)
    v = rng.random(n_prim)
    d = cam[3, :3] + cam[1, :3] * u[:, None] + cam[2, :3] * v[:, None] - cam[0, :3]
    out[:n_prim, :3] = cam[0, :3]
    out[:n_prim, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    m = n - n_prim
    tri = rng.integers(0, sc.ntris, size=m)
    p = sc.verts[sc.tris[tri, :3], :3].astype(np.float64)           # [m, 3, 3]
    a, b = rng.random(m), rng.random(m)
    flip = a + b > 1.0
    a[flip], b[flip] = 1.0 - a[flip], 1.0 - b[flip]
    pos = p[:, 0] + (p[:, 1] - p[:, 0]) * a[:, None] + (p[:, 2] - p[:, 0]) * b[:, None]
    nrm = np.cross(p[:, 1] - p[:, 0], p[:, 2] - p[:, 0])
    ln = np.linalg.norm(nrm, axis=1, keepdims=True)
    nrm = np.where(ln > 0, nrm / np.maximum(ln, 1e-30), np.array([0.0, 1.0, 0.0]))
    # cosine-weighted hemisphere sample in the normal's frame
    r1, r2 = rng.random(m), rng.random(m)
    phi = 2.0 * math.pi * r1
    sx, sy, sz = np.cos(phi) * np.sqrt(r2), np.sin(phi) * np.sqrt(r2), np.sqrt(1.0 - r2)
    helper = np.where(np.abs(nrm[:, :1]) > 0.9, np.array([0.0, 1.0, 0.0]), np.array([1.0, 0.0, 0.0]))
    t1 = np.cross(nrm, helper)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(nrm, t1)
    side = np.where(rng.random(m) < 0.5, 1.0, -1.0)[:, None]     # either face
    dirs = t1 * sx[:, None] + t2 * sy[:, None] + nrm * (sz[:, None] * side)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    out[n_prim:, :3] = pos + dirs * 1e-3
    out[n_prim:, 4:7] = dirs
    return out


def batch_scenes(n_scenes: int = 64, seed: int = 5, tris=(10_000, 2_000_000), rays=(65_536, 4_194_304)):
    """Scenes with log-uniform triangle counts and log-uniform ray counts."""
    rng = np.random.default_rng(seed)
    nt = np.exp(rng.uniform(math.log(tris[0]), math.log(tris[1]), n_scenes)).astype(np.int64)
    nr = np.exp(rng.uniform(math.log(rays[0]), math.log(rays[1]), n_scenes)).astype(np.int64)
    return [(cluster_soup(int(nt[i]), seed * 1000 + i), int(nr[i])) for i in range(n_scenes)]


def from_obj(path: str, width: int = 800, height: int = 600) -> Scene:
    """A scene from a Wavefront OBJ file (parsed by the library), with the
    reference OBJ loader's frame size and light (OBJLoader/OBJLoader.cpp:
    119-135: 800x600, one directional light along normalize(-1, 1, 1), colour
    0.9) and a camera that looks at the mesh's bounding box from its +z side."""
    from .engine import obj_parse
    V, T = obj_parse(path)
    lo, hi = V[:, :3].min(axis=0).astype(np.float64), V[:, :3].max(axis=0).astype(np.float64)
    c, r = (lo + hi) / 2.0, float(np.linalg.norm(hi - lo)) / 2.0
    cam = look_at_camera(tuple(c + np.array([0.25 * r, 0.35 * r, 2.2 * r])), tuple(c), 60.0, width, height)
    d = np.array([-1.0, 1.0, 1.0]) / math.sqrt(3.0)
    lights = np.stack([directional_light(tuple(d), (0.9, 0.9, 0.9))])
    return Scene(V, T, lights, cam, width, height, name=os.path.basename(path))

