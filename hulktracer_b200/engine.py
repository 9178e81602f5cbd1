"""Host-side mirror of HulkEngine's KD-tree and GPU-visitor surface over the C ABI.

* :class:`Context` -- one ``hk_ctx`` (device arena + stream), numpy in/out.
* :class:`KDTreeCUDA` -- the ``KDTreeCPU`` interface (HulkEngine/src/KDTreeCPU.hpp:
  53-72): ``buildKDTree``, ``checkCollision`` (batched), ``getNodeArray``,
  ``getPolygonArray``; the GPU builder fills the empty ``KDTreeGPU`` slot
  (HulkEngine/src/KDTreeGPU.hpp:12-22).
* :class:`TraceCUDA` -- a headless ``GLVisitorGPUTrace`` (HulkEngine/src/
  GLVisitorGPUTrace.hpp:26-72): ``initializeVisitor``, ``buildTree``,
  ``traceScene`` returning the framebuffer instead of a GL texture.

Every call goes to ``libhulkcuda.so``; failures raise :class:`HkError`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import HkError, ptr

EHulkResult_ok = 0


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def obj_parse(path: str):
    """Vertices float32[V, 4] (w = 1) and triangles uint32[T, 4] of an OBJ file,
    parsed by the library as the reference's OBJ loader reads it."""
    L = _lib.load()
    nv, nt = C.c_uint32(), C.c_uint32()
    st = L.hk_obj_parse(path.encode(), None, 0, None, 0, C.byref(nv), C.byref(nt))
    if st != 0:
        raise HkError(st, "hk_obj_parse(%s)" % path)
    v = np.zeros((nv.value, 4), np.float32)
    t = np.zeros((nt.value, 4), np.uint32)
    st = L.hk_obj_parse(path.encode(), ptr(v), nv.value, ptr(t), nt.value, C.byref(nv), C.byref(nt))
    if st != 0:
        raise HkError(st, "hk_obj_parse(%s)" % path)
    return v, t


def fixed_tick_time(frame: int) -> float:
    """Scene time of frame `frame` under the reference's --fixedTic=1 clock
    (GLWindow::display, HulkEngine/src/GLWindow.cpp:115-123): tick / 10 as a
    float, with ticks 59 and 421 skipped."""
    tick = 0
    for _ in range(frame):
        tick += 1
        if tick in (59, 421):
            tick += 1
    return float(np.float32(tick) / np.float32(10))


class Aff:
    """An AFF (BART) scene parsed by the library (hk_aff_*): rest-pose meshes,
    transforms and keyframe animations. Host-side; no GPU needed."""

    def __init__(self, path: str):
        self.L = _lib.load()
        self.h = C.c_void_p()
        st = self.L.hk_aff_open(path.encode(), C.byref(self.h))
        if st != 0:
            raise HkError(st, "hk_aff_open(%s): %s" % (path, self.L.hk_aff_last_error().decode()))
        info = _lib.AffInfo()
        self._check(self.L.hk_aff_get_info(self.h, C.byref(info)))
        self.info = info.as_dict()

    def _check(self, st):
        if st != 0:
            raise HkError(st, self.L.hk_aff_last_error().decode())

    def close(self):
        if self.h:
            self.L.hk_aff_close(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def geometry(self):
        """(verts float32[V, 4], tris uint32[T, 4], part uint32[V])"""
        i = self.info
        v = np.zeros((i["nv"], 4), np.float32)
        t = np.zeros((i["nt"], 4), np.uint32)
        p = np.zeros(i["nv"], np.uint32)
        self._check(self.L.hk_aff_geometry(self.h, ptr(v), ptr(t), ptr(p)))
        return v, t, p

    def part_matrices(self, time: float):
        m = np.zeros((self.info["nmeshes"], 12), np.float32)
        self._check(self.L.hk_aff_part_matrices(self.h, float(time), ptr(m)))
        return m

    def lights(self):
        out = np.zeros((self.info["nlights"], 8), np.float32)
        if out.size:
            self._check(self.L.hk_aff_lights(self.h, ptr(out)))
        return out

    def camera(self, time: float):
        cam = np.zeros(16, np.float32)
        self._check(self.L.hk_aff_camera(self.h, float(time), ptr(cam)))
        return cam


class Context:
    def __init__(self, device: int = 0, **cfg):
        self.L = _lib.load()
        c = _lib.Config()
        self._check(self.L.hk_config_default(C.byref(c)))
        for k, v in cfg.items():
            if not hasattr(c, k):
                raise KeyError(k)
            setattr(c, k, v)
        c.device = device
        self.cfg = c
        h = C.c_void_p()
        st = self.L.hk_create(C.byref(h), C.byref(c))
        if st != 0:
            raise HkError(st, "hk_create failed")
        self.h = h
        self.ntris = 0
        self.nverts = 0

    def _check(self, st):
        if st != 0:
            msg = self.L.hk_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise HkError(st, msg)

    def close(self):
        if getattr(self, "h", None):
            self.L.hk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- scene --
    def upload(self, verts, tris):
        v, t = _f32(verts), _u32(tris)
        self._check(self.L.hk_scene_upload(self.h, ptr(v), v.shape[0], ptr(t), t.shape[0]))
        self.ntris, self.nverts = t.shape[0], v.shape[0]

    def load_obj(self, path):
        """Parse an OBJ file and upload it as the scene."""
        nv, nt = C.c_uint32(), C.c_uint32()
        self._check(self.L.hk_scene_load_obj(self.h, path.encode(), C.byref(nv), C.byref(nt)))
        self.nverts, self.ntris = nv.value, nt.value

    def load_aff(self, aff: "Aff", time: float = 0.0):
        """Upload an AFF scene (one part per mesh) transformed to `time`."""
        self._check(self.L.hk_scene_load_aff(self.h, aff.h, float(time)))
        self.nverts, self.ntris = aff.info["nv"], aff.info["nt"]

    def animate_aff(self, aff: "Aff", time: float):
        self._check(self.L.hk_scene_animate_aff(self.h, aff.h, float(time)))

    def set_box(self, box):
        self._check(self.L.hk_scene_set_box(self.h, ptr(_f32(box))))

    def get_box(self):
        b = np.zeros(8, np.float32)
        self._check(self.L.hk_scene_get_box(self.h, ptr(b)))
        return b

    def set_parts(self, part_of_vertex, nparts):
        self._part = _u32(part_of_vertex)
        self._check(self.L.hk_scene_set_parts(self.h, ptr(self._part), int(nparts)))

    def set_mirrors(self, mirror):
        m = np.ascontiguousarray(mirror, dtype=np.uint8)
        self._check(self.L.hk_scene_set_mirrors(self.h, ptr(m), m.shape[0]))

    def transform(self, mats12):
        self._check(self.L.hk_scene_transform(self.h, ptr(_f32(mats12))))

    def get_vertices(self):
        v = np.zeros((self.nverts, 4), np.float32)
        self._check(self.L.hk_scene_get_vertices(self.h, ptr(v)))
        return v

    # -- cache --
    def precompute(self):
        self._check(self.L.hk_precompute(self.h))

    def import_cache(self, cache16):
        c = _f32(cache16)
        self._check(self.L.hk_cache_import(self.h, ptr(c), c.shape[0]))

    def export_cache(self):
        c = np.zeros((self.ntris, 16), np.float32)
        self._check(self.L.hk_cache_export(self.h, ptr(c)))
        return c

    # -- tree --
    def build(self, mode=_lib.BUILD_BINNED):
        st = _lib.TreeStats()
        self._check(self.L.hk_build(self.h, int(mode), C.byref(st)))
        return st.as_dict()

    def import_tree(self, nodes, refs):
        n, r = _u32(nodes).reshape(-1, 4), _u32(refs)
        self._check(self.L.hk_tree_import(self.h, ptr(n), n.shape[0], ptr(r), r.shape[0]))

    def level_counts(self):
        """(nodes, refs) per level of the last level-synchronous build."""
        n = C.c_uint32()
        cap = 64
        nodes = np.zeros(cap, np.uint32)
        refs = np.zeros(cap, np.uint32)
        self._check(self.L.hk_build_level_counts(self.h, ptr(nodes), ptr(refs), cap, C.byref(n)))
        k = min(n.value, cap)
        return nodes[:k].copy(), refs[:k].copy()

    def subtree_counts(self):
        """The last build's deferred subtrees: roots, the references they hold,
        and the nodes and leaf references the subtrees added."""
        v = [C.c_uint32() for _ in range(4)]
        self._check(self.L.hk_build_subtree_counts(self.h, *[C.byref(x) for x in v]))
        return dict(zip(("roots", "root_refs", "nodes", "leaf_refs"), (x.value for x in v)))

    def export_tree(self):
        nn, nr = C.c_uint32(), C.c_uint32()
        self._check(self.L.hk_tree_export(self.h, None, 0, None, 0, C.byref(nn), C.byref(nr)))
        nodes = np.zeros((nn.value, 4), np.uint32)
        refs = np.zeros(max(nr.value, 1), np.uint32)
        self._check(self.L.hk_tree_export(self.h, ptr(nodes), nn.value, ptr(refs), nr.value, C.byref(nn),
                                          C.byref(nr)))
        return nodes, refs[:nr.value]

    def export_compact(self):
        nn, nr = C.c_uint32(), C.c_uint32()
        self._check(self.L.hk_tree_export_compact(self.h, None, 0, None, 0, C.byref(nn), C.byref(nr)))
        nodes = np.zeros((nn.value, 2), np.uint32)
        refs = np.zeros(max(nr.value, 1), np.uint32)
        self._check(self.L.hk_tree_export_compact(self.h, ptr(nodes), nn.value, ptr(refs), nr.value,
                                                  C.byref(nn), C.byref(nr)))
        return nodes, refs[:nr.value]

    def save_tree_file(self, path):
        """The current tree + vertices in the reference's dataset file layout."""
        self._check(self.L.hk_tree_save_file(self.h, path.encode()))

    def load_tree_file(self, path, load_scene=False):
        """Import a tree file onto the uploaded scene, or (load_scene) upload
        the file's per-leaf triangles as the scene with the tree over them."""
        self._check(self.L.hk_tree_load_file(self.h, path.encode(), 1 if load_scene else 0))
        nv, nt = C.c_uint32(), C.c_uint32()
        self._check(self.L.hk_scene_get_counts(self.h, C.byref(nv), C.byref(nt)))
        self.nverts, self.ntris = nv.value, nt.value

    def tree_cost(self, ct=None, ci=None):
        """SAH cost of the current tree (full surface areas over the scene box;
        the context's Ct / Ci unless given)."""
        out = C.c_double()
        ct = self.cfg.traverse_cost if ct is None else ct
        ci = self.cfg.intersect_cost if ci is None else ci
        self._check(self.L.hk_tree_cost(self.h, float(ct), float(ci), C.byref(out)))
        return out.value

    def stats(self):
        st = _lib.TreeStats()
        self._check(self.L.hk_tree_stats_get(self.h, C.byref(st)))
        return st.as_dict()

    # -- trace --
    def trace(self, rays, variant=_lib.SHORTSTACK):
        r = _f32(rays).reshape(-1, 8)
        hits = np.zeros(r.shape[0], _lib.HIT_DTYPE)
        self._check(self.L.hk_trace(self.h, ptr(r), r.shape[0], int(variant), ptr(hits)))
        return hits

    def stream_setup(self, pool_tris: int):
        """Out-of-core leaf geometry: snapshot the tree's leaf records into pinned
        host memory and empty a device pool of pool_tris triangle records."""
        self._check(self.L.hk_stream_setup(self.h, int(pool_tris)))

    def trace_streamed(self, rays):
        """kd-restart with leaves paged into the pool on demand: (hits, stats)."""
        r = _f32(rays).reshape(-1, 8)
        hits = np.zeros(r.shape[0], _lib.HIT_DTYPE)
        st = _lib.StreamStats()
        self._check(self.L.hk_trace_streamed(self.h, ptr(r), r.shape[0], ptr(hits), C.byref(st)))
        return hits, st.as_dict()

    def trace_device(self, d_rays: int, n: int, d_hits: int, variant=_lib.SHORTSTACK):
        self._check(self.L.hk_trace_device(self.h, C.c_void_p(d_rays), n, int(variant), C.c_void_p(d_hits)))

    def set_counting(self, on=True):
        self._check(self.L.hk_set_counting(self.h, 1 if on else 0))

    def counters(self):
        c = np.zeros(3, np.uint64)
        self._check(self.L.hk_get_counters(self.h, ptr(c)))
        return c

    def synchronize(self):
        self._check(self.L.hk_synchronize(self.h))

    def set_stream(self, stream_ptr: int | None):
        self._check(self.L.hk_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def camera_rays(self, cam, w, h):
        out = np.zeros((w * h, 8), np.float32)
        self._check(self.L.hk_camera_rays(self.h, ptr(_f32(cam).ravel()), w, h, ptr(out)))
        return out

    def render(self, cam, lights, w, h, variant=_lib.SHORTSTACK, shade=_lib.SHADE_CPU):
        lights = _f32(lights).reshape(-1, 8)
        out = np.zeros(w * h, np.uint32)
        self._check(self.L.hk_render(self.h, ptr(_f32(cam).ravel()), ptr(lights), lights.shape[0], w, h,
                                     int(variant), int(shade), ptr(out)))
        return out

    def render_device(self, cam, lights, w, h, d_rgba: int, variant=_lib.SHORTSTACK, shade=_lib.SHADE_CPU):
        lights = _f32(lights).reshape(-1, 8)
        self._check(self.L.hk_render_device(self.h, ptr(_f32(cam).ravel()), ptr(lights), lights.shape[0], w, h,
                                            int(variant), int(shade), C.c_void_p(d_rgba)))

    def render_rows_device(self, cam, lights, w, h, y0, y1, d_rgba: int, variant=_lib.SHORTSTACK,
                           shade=_lib.SHADE_CPU):
        """Rows y0 .. y1 - 1 of the w x h frame into d_rgba (w x (y1 - y0))."""
        lights = _f32(lights).reshape(-1, 8)
        self._check(self.L.hk_render_rows_device(self.h, ptr(_f32(cam).ravel()), ptr(lights), lights.shape[0], w, h,
                                                 y0, y1, int(variant), int(shade), C.c_void_p(d_rgba)))

    def shade_picture(self, rays, hit4, lights):
        r = _f32(rays).reshape(-1, 8)
        lights = _f32(lights).reshape(-1, 8)
        out = np.zeros(r.shape[0], np.uint32)
        self._check(self.L.hk_shade_picture(self.h, ptr(r), ptr(_f32(hit4)), r.shape[0], ptr(lights),
                                            lights.shape[0], ptr(out)))
        return out

    def set_frame_shading(self, shade):
        self._check(self.L.hk_set_frame_shading(self.h, int(shade)))

    def frame(self, mats12, cam, lights, w, h, d_rgba: int, mode=_lib.BUILD_BINNED, variant=_lib.SHORTSTACK,
              use_graph=True, want_stats=False):
        lights = _f32(lights).reshape(-1, 8)
        m = None if mats12 is None else _f32(mats12)
        st = _lib.TreeStats() if want_stats else None
        self._check(self.L.hk_frame(self.h, ptr(m), ptr(_f32(cam).ravel()), ptr(lights), lights.shape[0], w, h,
                                    int(mode), int(variant), 1 if use_graph else 0, C.c_void_p(d_rgba),
                                    C.byref(st) if st is not None else None))
        return st.as_dict() if st is not None else None


    def set_debug_flags(self, flags):
        """Test aid (hk_set_debug_flags): bit 0 withholds one plan tile's done
        flag so that the build's bounded waits run out."""
        self._check(self.L.hk_set_debug_flags(self.h, int(flags)))

    # -- learned split proposer --
    def set_proposal_log(self, on=True):
        self._check(self.L.hk_set_proposal_log(self.h, 1 if on else 0))

    def proposal_log(self):
        """int32[nn, 8]: the bins proposed for each compact node of the last
        learned build (axis * 32 + bin, -1 for none)."""
        nn = C.c_uint32()
        self._check(self.L.hk_get_proposal_log(self.h, None, 0, C.byref(nn)))
        out = np.zeros((nn.value, 8), np.int32)
        self._check(self.L.hk_get_proposal_log(self.h, ptr(out), nn.value, C.byref(nn)))
        return out

    def mlp_init(self, seed=0):
        self._check(self.L.hk_mlp_init(self.h, seed))

    def mlp_save(self, path):
        self._check(self.L.hk_mlp_save(self.h, path.encode()))

    def mlp_load(self, path):
        self._check(self.L.hk_mlp_load(self.h, path.encode()))

    def mlp_params(self):
        p = np.zeros(_lib.MLP_PARAMS, np.float32)
        self._check(self.L.hk_mlp_get_params(self.h, ptr(p), p.size))
        return p

    def mlp_set_params(self, p):
        p = _f32(p)
        self._check(self.L.hk_mlp_set_params(self.h, ptr(p), p.size))

    def mlp_forward(self, X):
        X = _f32(X).reshape(-1, _lib.MLP_IN)
        out = np.zeros((X.shape[0], _lib.MLP_OUT), np.float32)
        self._check(self.L.hk_mlp_forward(self.h, ptr(X), X.shape[0], ptr(out)))
        return out

    def mlp_grad(self, X, y):
        X = _f32(X).reshape(-1, _lib.MLP_IN)
        y = np.ascontiguousarray(y, np.int32)
        g = np.zeros(_lib.MLP_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._check(self.L.hk_mlp_grad(self.h, ptr(X), ptr(y), X.shape[0], ptr(g), ptr(loss)))
        return g, float(loss[0])

    def mlp_record(self, capacity_rows):
        self._check(self.L.hk_mlp_record(self.h, int(capacity_rows)))

    def mlp_dataset(self, fetch=True):
        rows = C.c_uint32()
        self._check(self.L.hk_mlp_dataset(self.h, None, None, 0, C.byref(rows)))
        if not fetch:
            return rows.value
        X = np.zeros((rows.value, _lib.MLP_IN), np.float32)
        y = np.zeros(rows.value, np.int32)
        self._check(self.L.hk_mlp_dataset(self.h, ptr(X), ptr(y), rows.value, C.byref(rows)))
        return X, y

    def mlp_train(self, epochs=1, batch=1024, lr=1e-3, seed=0):
        losses = np.zeros(epochs, np.float32)
        self._check(self.L.hk_mlp_train(self.h, epochs, batch, lr, seed, ptr(losses)))
        return losses

    def autotune(self, d_rays: int, n: int, cache_path: str | None = None):
        r = _lib.TuneResult()
        self._check(self.L.hk_autotune(self.h, C.c_void_p(d_rays), n,
                                       cache_path.encode() if cache_path else None, C.byref(r)))
        return r.as_dict()

    def autotune_build(self, mode=_lib.BUILD_BINNED, reps: int = 5):
        """hk_autotune_build: the builder layout (subtree_max, subtree_depth)
        with the fastest builds on the current scene, set in the context."""
        r = _lib.BuildTuneResult()
        self._check(self.L.hk_autotune_build(self.h, int(mode), int(reps), C.byref(r)))
        return r.as_dict()

    def set_build_layout(self, subtree_max: int, subtree_depth: int, level_streams: int = 1):
        self._check(self.L.hk_set_build_layout(self.h, int(subtree_max), int(subtree_depth), int(level_streams)))

    def set_trace_config(self, block_size: int, short_stack: int):
        self._check(self.L.hk_set_trace_config(self.h, int(block_size), int(short_stack)))

    def ray_counts(self):
        p, sh = C.c_uint64(), C.c_uint64()
        self._check(self.L.hk_get_ray_counts(self.h, C.byref(p), C.byref(sh)))
        return p.value, sh.value

    def graph_info(self):
        k, a = C.c_uint32(), C.c_uint32()
        self._check(self.L.hk_frame_graph_info(self.h, C.byref(k), C.byref(a)))
        return k.value, a.value


class Batch:
    """Many scenes traced in one persistent launch (include/hulkcuda.h, hk_batch_*)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = C.c_void_p()
        ctx._check(ctx.L.hk_batch_create(ctx.h, C.byref(h)))
        self.h = h
        self.nscenes = 0

    def add_scene(self, verts, tris) -> int:
        v, t = _f32(verts), _u32(tris)
        sid = C.c_uint32()
        self.ctx._check(self.ctx.L.hk_batch_add_scene(self.h, ptr(v), v.shape[0], ptr(t), t.shape[0], C.byref(sid)))
        self.nscenes += 1
        return sid.value

    def trace_device(self, d_rays: int, offsets, d_hits: int, variant=_lib.ROPES, want_times=True):
        off = _u32(offsets)
        ms = np.zeros(self.nscenes, np.float32) if want_times else None
        self.ctx._check(self.ctx.L.hk_batch_trace_device(self.h, C.c_void_p(d_rays), ptr(off), self.nscenes,
                                                         int(variant), C.c_void_p(d_hits), ptr(ms)))
        return ms

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.hk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KDTreeCUDA:
    """``KDTreeCPU``'s interface on the GPU (HulkEngine/src/KDTreeCPU.hpp:53-72)."""

    def __init__(self, ctx: Context | None = None, mode=_lib.BUILD_BINNED):
        self.ctx = ctx or Context()
        self.mode = mode
        self.scene = None

    def buildKDTree(self, scene) -> int:
        """Upload the scene arrays, compute the triangle cache and build
        (KDTreeCPU::buildKDTree, KDTreeCPU.cpp:61-94). Returns e_ok."""
        self.scene = scene
        self.ctx.upload(scene.verts, scene.tris)
        self.ctx.precompute()
        self.last_stats = self.ctx.build(self.mode)
        return EHulkResult_ok

    def checkCollision(self, rays, variant=_lib.SHORTSTACK):
        """Batched KDTreeCPU::checkCollision (KDTreeCPU.cpp:230-253): per ray the
        closest hit time (inf on a miss) and triangle index (-1 on a miss)."""
        return self.ctx.trace(rays, variant)

    def getNodeArray(self):
        return self.ctx.export_tree()[0]

    def getPolygonArray(self):
        return self.ctx.export_tree()[1]


class TraceCUDA:
    """Headless GLVisitorGPUTrace: build the tree, trace primary + shadow rays
    and shade into a framebuffer (HulkEngine/src/GLVisitorGPUTrace.cpp:256-410)."""

    def __init__(self, ctx: Context | None = None, variant=_lib.SHORTSTACK, mode=_lib.BUILD_BINNED):
        self.ctx = ctx or Context()
        self.variant = variant
        self.mode = mode
        self.scene = None

    def initializeVisitor(self, scene):
        self.scene = scene
        self.ctx.upload(scene.verts, scene.tris)
        if scene.part_of_vertex is not None:
            self.ctx.set_parts(scene.part_of_vertex, scene.part_center.shape[0])

    def buildTree(self):
        self.ctx.precompute()
        return self.ctx.build(self.mode)

    def traceScene(self, shade=_lib.SHADE_CPU):
        sc = self.scene
        img = self.ctx.render(sc.camera, sc.lights, sc.width, sc.height, self.variant, shade)
        return img.reshape(sc.height, sc.width)
