"""ctypes bindings to the CPU oracle (``liboracle.so``) and to the compiled
reference (``_ref/libhulkref*.so``).

Test infrastructure only: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg, always as the checker, never as the product.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SHORTSTACK, FULLSTACK, RESTART, RESTART_EARLY, ROPES, BRUTE = range(6)
NORM_SSE, NORM_IEEE = 0, 1
ISECT_ACC, ISECT_POLY = 0, 1

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class _Tree(C.Structure):
    _fields_ = [("verts", C.c_void_p), ("tris", C.c_void_p), ("nt", C.c_uint32),
                ("cache", C.c_void_p), ("nodes", C.c_void_p), ("nn", C.c_uint32),
                ("refs", C.c_void_p), ("box", C.c_void_p), ("cnodes", C.c_void_p),
                ("cnn", C.c_uint32), ("cropes", C.c_void_p), ("cbox", C.c_void_p)]


class _SahParams(C.Structure):
    _fields_ = [("ct", C.c_float), ("ci", C.c_float), ("max_depth", C.c_uint32),
                ("leaf_below", C.c_uint32), ("reduction", C.c_uint32)]


class _BinnedParams(C.Structure):
    _fields_ = [("ct", C.c_float), ("ci", C.c_float), ("max_depth", C.c_uint32),
                ("leaf_size", C.c_uint32), ("bins", C.c_uint32), ("max_refs", C.c_uint32),
                ("max_nodes", C.c_uint32), ("exact_max", C.c_uint32), ("learned", C.c_uint32),
                ("topk", C.c_uint32), ("fallback_ratio", C.c_float), ("proposals", C.c_void_p),
                ("defer", C.c_uint32), ("defer_margin", C.c_uint32)]


# reference constants (KDTreeCPU.cpp:17-18, SharedStructs.hpp:16, KDTreeSAH.cpp:317,
# KDTreeCPU.hpp:23) and the benchmark-scene constants
REF_SAH = dict(ct=1.0, ci=5.0, max_depth=20, leaf_below=10, reduction=5)
CFG_SAH = dict(ct=1.0, ci=1.5, max_depth=24, leaf_below=5, reduction=1)


def build_oracle_lib() -> str:
    lib = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "hk_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return lib


class Tree:
    """Arrays of one KD tree + scene, kept alive for the C side."""

    def __init__(self, verts, tris, cache, nodes, refs, box, cnodes=None, ropes=None, cbox=None):
        self.verts = _c(verts, np.float32)
        self.tris = _c(tris, np.uint32)
        self.cache = _c(cache, np.float32)
        self.nodes = _c(nodes, np.uint32).reshape(-1, 4)
        self.refs = _c(refs, np.uint32) if len(refs) else np.zeros(1, np.uint32)
        self.box = _c(box, np.float32)
        self.cnodes = None if cnodes is None else _c(cnodes, np.uint32)
        self.ropes = None if ropes is None else _c(ropes, np.uint32)
        self.cbox = None if cbox is None else _c(cbox, np.float32)

    def cstruct(self) -> _Tree:
        p = lambda a: None if a is None else a.ctypes.data
        return _Tree(p(self.verts), p(self.tris), self.tris.shape[0], p(self.cache), p(self.nodes),
                     self.nodes.shape[0], p(self.refs), p(self.box), p(self.cnodes),
                     0 if self.cnodes is None else self.cnodes.size // 2, p(self.ropes), p(self.cbox))


class Oracle:
    def __init__(self):
        self.lib = C.CDLL(build_oracle_lib())
        L = self.lib
        L.hko_dot4.restype = C.c_float
        L.hko_dot4.argtypes = [_f32p, _f32p]
        L.hko_box_surface.restype = C.c_float
        L.hko_box_surface.argtypes = [_f32p]
        L.hko_box_volume.restype = C.c_float
        L.hko_box_volume.argtypes = [_f32p]
        L.hko_normalize.argtypes = [_f32p, C.c_int]
        L.hko_build_cache.argtypes = [_f32p, _u32p, C.c_uint32, C.c_int, _f32p]
        L.hko_transform.argtypes = [_f32p, _u32p, C.c_uint32, _f32p, _f32p]
        L.hko_scene_box.argtypes = [_f32p, C.c_uint32, _f32p]
        L.hko_camera_rays.argtypes = [_f32p, C.c_uint32, C.c_uint32, C.c_int, _f32p]
        pp = C.POINTER(C.POINTER(C.c_uint32))
        L.hko_build_sah_nlogn.argtypes = [_f32p, _u32p, C.c_uint32, _f32p, C.POINTER(_SahParams), pp,
                                          C.POINTER(C.c_uint32), pp, C.POINTER(C.c_uint32)]
        L.hko_build_sah_resort.argtypes = [_f32p, _u32p, C.c_uint32, _f32p, C.POINTER(_SahParams), pp,
                                          C.POINTER(C.c_uint32), pp, C.POINTER(C.c_uint32)]
        L.hko_build_binned.argtypes = [_f32p, _u32p, C.c_uint32, _f32p, C.POINTER(_BinnedParams), pp,
                                       C.POINTER(C.c_uint32), pp, C.POINTER(C.c_uint32)]
        L.hko_free.argtypes = [C.c_void_p]
        L.hko_set_isect_form.argtypes = [C.c_int]
        L.hko_tree_cost.restype = C.c_double
        L.hko_tree_cost.argtypes = [_u32p, C.c_uint32, _f32p, C.c_double, C.c_double]
        L.hko_node_boxes.argtypes = [_u32p, C.c_uint32, _f32p, _f32p]
        L.hko_ref_to_compact.restype = C.c_uint32
        L.hko_ref_to_compact.argtypes = [_u32p, C.c_uint32, _u32p]
        L.hko_compact_to_ref.argtypes = [_u32p, C.c_uint32, _u32p]
        L.hko_build_ropes.argtypes = [_u32p, C.c_uint32, _f32p, _u32p, _f32p]
        L.hko_trace.argtypes = [C.POINTER(_Tree), C.c_int, C.c_int, _f32p, C.c_uint32, _f32p, _i32p,
                                C.c_void_p, C.c_int]
        L.hko_render_cpu.argtypes = [C.POINTER(_Tree), C.c_int, C.c_int, _f32p, C.c_uint32, C.c_uint32,
                                     _f32p, C.c_uint32, C.c_int, _u32p, C.c_int]
        L.hko_shade_picture.argtypes = [_f32p, _f32p, C.c_uint32, _f32p, C.c_uint32, _u32p]
        L.hko_render_mirror.argtypes = [C.POINTER(_Tree), C.c_int, C.c_int, _f32p, C.c_uint32, C.c_uint32,
                                        _f32p, C.c_uint32, np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS"),
                                        C.c_int, _u32p, C.c_int]

    # -- helpers --
    def set_isect_form(self, form):
        """0: checkRayToPolyACC over the cache (default); 1: checkRayToPoly from
        the vertices (the reference's OpenCL form)."""
        self.lib.hko_set_isect_form(int(form))

    def dot4(self, a, b):
        return self.lib.hko_dot4(_c(a, np.float32), _c(b, np.float32))

    def normalize(self, v, mode=NORM_IEEE):
        v = _c(v, np.float32).copy()
        self.lib.hko_normalize(v, mode)
        return v

    def box_surface(self, box):
        return self.lib.hko_box_surface(_c(box, np.float32))

    def box_volume(self, box):
        return self.lib.hko_box_volume(_c(box, np.float32))

    def cache(self, verts, tris, mode=NORM_IEEE):
        tris = _c(tris, np.uint32)
        out = np.zeros((tris.shape[0], 16), np.float32)
        self.lib.hko_build_cache(_c(verts, np.float32), tris, tris.shape[0], mode, out)
        return out

    def transform(self, rest, part, mats):
        rest = _c(rest, np.float32)
        out = np.zeros_like(rest)
        self.lib.hko_transform(rest, _c(part, np.uint32), rest.shape[0], _c(mats, np.float32), out)
        return out

    def scene_box(self, verts):
        verts = _c(verts, np.float32)
        out = np.zeros(8, np.float32)
        self.lib.hko_scene_box(verts, verts.shape[0], out)
        return out

    def camera_rays(self, cam, w, h, mode=NORM_IEEE):
        out = np.zeros((h * w, 8), np.float32)
        self.lib.hko_camera_rays(_c(cam, np.float32).ravel(), w, h, mode, out)
        return out

    def _take(self, pn, nn, pr, nr, width):
        nodes = np.ctypeslib.as_array(pn, shape=(nn * width,)).copy().reshape(nn, width)
        refs = np.ctypeslib.as_array(pr, shape=(max(nr, 1),)).copy()[:nr]
        self.lib.hko_free(pn)
        self.lib.hko_free(pr)
        return nodes, refs

    def build_sah_nlogn(self, verts, tris, box, **kw):
        p = dict(REF_SAH)
        p.update(kw)
        prm = _SahParams(p["ct"], p["ci"], p["max_depth"], p["leaf_below"], p["reduction"])
        pn, pr = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
        nn, nr = C.c_uint32(), C.c_uint32()
        tris = _c(tris, np.uint32)
        self.lib.hko_build_sah_nlogn(_c(verts, np.float32), tris, tris.shape[0], _c(box, np.float32),
                                     C.byref(prm), C.byref(pn), C.byref(nn), C.byref(pr), C.byref(nr))
        return self._take(pn, nn.value, pr, nr.value, 4)

    def build_sah_resort(self, verts, tris, box, **kw):
        """buildKDTreeSAH / buildNodeSAH (the --treeType=SAH builder)."""
        p = dict(REF_SAH)
        p.update(kw)
        prm = _SahParams(p["ct"], p["ci"], p["max_depth"], p["leaf_below"], p["reduction"])
        pn, pr = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
        nn, nr = C.c_uint32(), C.c_uint32()
        tris = _c(tris, np.uint32)
        self.lib.hko_build_sah_resort(_c(verts, np.float32), tris, tris.shape[0], _c(box, np.float32),
                                      C.byref(prm), C.byref(pn), C.byref(nn), C.byref(pr), C.byref(nr))
        return self._take(pn, nn.value, pr, nr.value, 4)

    def build_binned(self, verts, tris, box, ct=1.0, ci=1.5, max_depth=24, leaf_size=4, bins=32,
                     max_refs=None, max_nodes=None, exact_max=0, proposals=None, topk=4, fallback_ratio=1.0,
                     defer=32, defer_margin=8):
        """The CUDA builder restated. With ``proposals`` (int32[nodes, 8], the
        GPU's proposal log of a learned build) it restates the learned build.
        ``defer`` (hk_config.subtree_max, the CUDA builder's layout) builds the
        subtrees of nodes of 2..defer references depth first after the levels;
        0 numbers every node level by level (the same tree, other node and
        reference order). ``defer_margin`` (hk_config.subtree_depth): only nodes
        at depth >= max_depth - defer_margin are deferred (0: any depth)."""
        nt = int(np.asarray(tris).shape[0])
        if max_refs is None:
            max_refs = max(16 * nt, 1024)
        if max_nodes is None:
            max_nodes = max(12 * nt, 1024)
        prop = None if proposals is None else _c(proposals, np.int32)
        prm = _BinnedParams(ct, ci, max_depth, leaf_size, bins, max_refs, max_nodes, exact_max,
                            0 if prop is None else 1, topk, fallback_ratio,
                            None if prop is None else prop.ctypes.data, min(int(defer), 32), int(defer_margin))
        pn, pr = C.POINTER(C.c_uint32)(), C.POINTER(C.c_uint32)()
        nn, nr = C.c_uint32(), C.c_uint32()
        tris = _c(tris, np.uint32)
        self.lib.hko_build_binned(_c(verts, np.float32), tris, tris.shape[0], _c(box, np.float32),
                                  C.byref(prm), C.byref(pn), C.byref(nn), C.byref(pr), C.byref(nr))
        return self._take(pn, nn.value, pr, nr.value, 2)

    def tree_cost(self, nodes, box, ct, ci):
        nodes = _c(nodes, np.uint32).reshape(-1, 4)
        return self.lib.hko_tree_cost(nodes.ravel(), nodes.shape[0], _c(box, np.float32), ct, ci)

    def ref_to_compact(self, nodes):
        nodes = _c(nodes, np.uint32).reshape(-1, 4)
        out = np.zeros((2 * nodes.shape[0] + 2, 2), np.uint32)
        n = self.lib.hko_ref_to_compact(nodes.ravel(), nodes.shape[0], out.ravel())
        return out[:n].copy()

    def compact_to_ref(self, cnodes):
        cnodes = _c(cnodes, np.uint32).reshape(-1, 2)
        out = np.zeros((cnodes.shape[0], 4), np.uint32)
        self.lib.hko_compact_to_ref(cnodes.ravel(), cnodes.shape[0], out.ravel())
        return out

    def ropes(self, cnodes, box):
        cnodes = _c(cnodes, np.uint32).reshape(-1, 2)
        r = np.zeros((cnodes.shape[0], 6), np.uint32)
        b = np.zeros((cnodes.shape[0], 8), np.float32)
        self.lib.hko_build_ropes(cnodes.ravel(), cnodes.shape[0], _c(box, np.float32), r.ravel(), b.ravel())
        return r, b

    def make_tree(self, verts, tris, cache, nodes, refs, box, with_ropes=False) -> Tree:
        cn = rp = cb = None
        if with_ropes:
            cn = self.ref_to_compact(nodes)
            rp, cb = self.ropes(cn, box)
        return Tree(verts, tris, cache, nodes, refs, box, cn, rp, cb)

    def trace(self, tree: Tree, rays, variant=SHORTSTACK, stack_depth=5, counters=False, nthreads=0):
        rays = _c(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        hits = np.zeros((n, 8), np.float32)
        ids = np.zeros(n, np.int32)
        cnt = np.zeros((n, 3), np.uint64) if counters else None
        ts = tree.cstruct()
        self.lib.hko_trace(C.byref(ts), variant, stack_depth, rays, n, hits, ids,
                           None if cnt is None else cnt.ctypes.data, nthreads)
        return (hits, ids, cnt) if counters else (hits, ids)

    def render_cpu(self, tree: Tree, rays, w, h, lights, variant=SHORTSTACK, stack_depth=5,
                   mode=NORM_IEEE, nthreads=0):
        out = np.zeros(w * h, np.uint32)
        lights = _c(lights, np.float32).reshape(-1, 8)
        ts = tree.cstruct()
        self.lib.hko_render_cpu(C.byref(ts), variant, stack_depth, _c(rays, np.float32).reshape(-1),
                                w, h, lights.ravel(), lights.shape[0], mode, out, nthreads)
        return out

    def render_mirror(self, tree: Tree, rays, w, h, lights, mirror, variant=SHORTSTACK, stack_depth=5,
                      mode=NORM_IEEE, nthreads=0):
        out = np.zeros(w * h, np.uint32)
        lights = _c(lights, np.float32).reshape(-1, 8)
        ts = tree.cstruct()
        self.lib.hko_render_mirror(C.byref(ts), variant, stack_depth, _c(rays, np.float32).reshape(-1), w, h,
                                   lights.ravel(), lights.shape[0], _c(mirror, np.uint8), mode, out, nthreads)
        return out

    def shade_picture(self, rays, hit4, lights):
        rays = _c(rays, np.float32).reshape(-1, 8)
        lights = _c(lights, np.float32).reshape(-1, 8)
        out = np.zeros(rays.shape[0], np.uint32)
        self.lib.hko_shade_picture(rays, _c(hit4, np.float32).reshape(-1), rays.shape[0], lights.ravel(),
                                   lights.shape[0], out)
        return out


class Reference:
    """The reference's own CPU path compiled from its sources (oracle/_ref)."""

    def __init__(self, cfg: bool = False):
        path = os.path.join(HERE, "_ref", "libhulkref%s.so" % ("_cfg" if cfg else ""))
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.hkref_create.restype = C.c_void_p
        L.hkref_create.argtypes = [_f32p, C.c_uint, _u32p, C.c_uint, _f32p]
        L.hkref_destroy.argtypes = [C.c_void_p]
        L.hkref_build.argtypes = [C.c_void_p]
        L.hkref_set_tree_type.argtypes = [C.c_int]
        L.hkref_set_vertices.argtypes = [C.c_void_p, _f32p, _f32p]
        L.hkref_node_count.restype = C.c_uint
        L.hkref_node_count.argtypes = [C.c_void_p]
        L.hkref_ref_count.restype = C.c_uint
        L.hkref_ref_count.argtypes = [C.c_void_p]
        L.hkref_get_nodes.argtypes = [C.c_void_p, _u32p]
        L.hkref_get_refs.argtypes = [C.c_void_p, _u32p]
        L.hkref_get_cache.argtypes = [C.c_void_p, _f32p]
        L.hkref_trace.argtypes = [C.c_void_p, _f32p, C.c_uint, _f32p, _i32p, C.c_void_p, C.c_int]
        L.hkref_render.argtypes = [C.c_void_p, _f32p, C.c_uint, C.c_uint, _f32p, C.c_uint, _u32p, C.c_int]
        L.hkref_normalize.argtypes = [_f32p, C.c_uint]
        L.hkref_box_surface.restype = C.c_float
        L.hkref_box_surface.argtypes = [_f32p]
        L.hkref_box_volume.restype = C.c_float
        L.hkref_box_volume.argtypes = [_f32p]
        self.h = None

    @staticmethod
    def available(cfg: bool = False) -> bool:
        return os.path.exists(os.path.join(HERE, "_ref", "libhulkref%s.so" % ("_cfg" if cfg else "")))

    def load(self, verts, tris, box):
        if self.h:
            self.lib.hkref_destroy(self.h)
        self._v = _c(verts, np.float32)
        self._t = _c(tris, np.uint32)
        self.nt = self._t.shape[0]
        self.h = self.lib.hkref_create(self._v, self._v.shape[0], self._t, self.nt, _c(box, np.float32))

    def set_vertices(self, verts, box):
        self._v = _c(verts, np.float32)
        self.lib.hkref_set_vertices(self.h, self._v, _c(box, np.float32))

    def build(self, tree_type: str = "SAHNlogN"):
        """KDTreeCPU::buildKDTree with --treeType (SAHNlogN, the default, or SAH)."""
        self.lib.hkref_set_tree_type(1 if tree_type == "SAH" else 0)
        self.lib.hkref_build(self.h)
        nn = self.lib.hkref_node_count(self.h)
        nr = self.lib.hkref_ref_count(self.h)
        nodes = np.zeros((nn, 4), np.uint32)
        refs = np.zeros(max(nr, 1), np.uint32)
        self.lib.hkref_get_nodes(self.h, nodes.ravel())
        self.lib.hkref_get_refs(self.h, refs)
        cache = np.zeros((self.nt, 16), np.float32)
        self.lib.hkref_get_cache(self.h, cache)
        return nodes, refs[:nr], cache

    def trace(self, rays, counters=False, nthreads=0):
        rays = _c(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        hits = np.zeros((n, 8), np.float32)
        ids = np.zeros(n, np.int32)
        cnt = np.zeros((n, 2), np.uint64) if counters else None
        self.lib.hkref_trace(self.h, rays, n, hits, ids, None if cnt is None else cnt.ctypes.data, nthreads)
        return (hits, ids, cnt) if counters else (hits, ids)

    def render(self, rays, w, h, lights, nthreads=0):
        lights = _c(lights, np.float32).reshape(-1, 8)
        out = np.zeros(w * h, np.uint32)
        self.lib.hkref_render(self.h, _c(rays, np.float32).reshape(-1), w, h, lights.ravel(),
                              lights.shape[0], out, nthreads)
        return out

    def normalize(self, v):
        v = _c(v, np.float32).reshape(-1, 4).copy()
        self.lib.hkref_normalize(v.ravel(), v.shape[0])
        return v

    def box_surface(self, box):
        return self.lib.hkref_box_surface(_c(box, np.float32))

    def box_volume(self, box):
        return self.lib.hkref_box_volume(_c(box, np.float32))

    def __del__(self):
        try:
            if self.h:
                self.lib.hkref_destroy(self.h)
        except Exception:
            pass


class ReferenceAff:
    """An AFF scene loaded by the reference's own AFFParser and animated by its
    AFFTransformVisitor (compiled from BartLoader/src into oracle/_ref)."""

    def __init__(self, path: str):
        lib_path = os.path.join(HERE, "_ref", "libhulkref.so")
        if not os.path.exists(lib_path):
            raise FileNotFoundError(lib_path)
        L = self.lib = C.CDLL(lib_path)
        L.hkref_aff_open.restype = C.c_void_p
        L.hkref_aff_open.argtypes = [C.c_char_p]
        L.hkref_aff_close.argtypes = [C.c_void_p]
        L.hkref_aff_counts.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.hkref_aff_view.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.hkref_aff_tris.argtypes = [C.c_void_p, _u32p]
        L.hkref_aff_lights.argtypes = [C.c_void_p, _f32p]
        L.hkref_aff_frame.argtypes = [C.c_void_p, C.c_float, _f32p, _f32p]
        L.hkref_aff_camera.argtypes = [C.c_void_p, C.c_float, _f32p]
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.h = L.hkref_aff_open(path.encode())
        if not self.h:
            raise FileNotFoundError(path)
        nv, nt, nl = C.c_uint(), C.c_uint(), C.c_uint()
        L.hkref_aff_counts(self.h, C.byref(nv), C.byref(nt), C.byref(nl))
        self.nv, self.nt, self.nl = nv.value, nt.value, nl.value
        fov, res, asp = C.c_float(), (C.c_int * 2)(), C.c_float()
        L.hkref_aff_view(self.h, C.byref(fov), res, C.byref(asp))
        self.fov, self.res, self.aspect = fov.value, (res[0], res[1]), asp.value

    def tris(self):
        t = np.zeros((self.nt, 4), np.uint32)
        self.lib.hkref_aff_tris(self.h, t)
        return t

    def lights(self):
        out = np.zeros((self.nl, 8), np.float32)
        if self.nl:
            self.lib.hkref_aff_lights(self.h, out)
        return out

    def frame(self, time: float):
        """Scene::m_vertices and the scene box after the frame at `time`."""
        v = np.zeros((self.nv, 4), np.float32)
        box = np.zeros(8, np.float32)
        self.lib.hkref_aff_frame(self.h, float(time), v, box)
        return v, box

    def camera(self, time: float):
        cam = np.zeros(16, np.float32)
        self.lib.hkref_aff_camera(self.h, float(time), cam)
        return cam

    def close(self):
        if self.h:
            self.lib.hkref_aff_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
