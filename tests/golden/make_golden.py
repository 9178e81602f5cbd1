"""Generate the golden fixtures of this directory from the reference itself.

The reference's CPU path (KDTreeCPU SAH-NlogN build, buildPolygonCache,
checkCollision, and the GLVisitorCPUTrace shading loop over its
checkCollision / FrameBuffer::replacePixel) is compiled from its own sources by
``oracle/build_ref.py`` into ``oracle/_ref``; this script runs it on seeded
scenes and stores inputs and outputs as compressed ``.npz`` files:

* ``soup3k.npz``   -- 3,000 random triangles, 4,096 random rays
* ``small24k.npz`` -- the 24,576-triangle ground + spheres scene, 128x128 rays

Quantities that depend on the CPU's ``rsqrtps`` approximation (the cached
normals, the rendered image) are stored with a probe (the reference's
normalisation of fixed vectors) so tests can tell whether the CPU they run on
reproduces them.

Usage: ``python tests/golden/make_golden.py`` (needs ``oracle/_ref``).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hulktracer_b200 import scenes  # noqa: E402
from oracle.oracle import Oracle, Reference, NORM_IEEE  # noqa: E402

PROBE = np.array([[1, 2, 3, 0], [0.3, -0.7, 0.1, 0], [1e-3, 5e2, -7.5, 0], [3, 4, 0, 0]], np.float32)


def random_rays(n, seed, box):
    rng = np.random.default_rng(seed)
    lo, hi = box[:3], box[4:7]
    ctr = (lo + hi) / 2
    ext = (hi - lo)
    o = ctr + (rng.uniform(-0.9, 0.9, size=(n, 3)) * ext)
    o[: n // 2] = ctr + rng.normal(size=(n // 2, 3)) * ext   # half from outside / far
    d = rng.normal(size=(n, 3))
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = o
    r[:, 4:7] = d
    O = Oracle()
    for i in range(n):
        r[i, 4:8] = O.normalize(r[i, 4:8], NORM_IEEE)
    return r


def make(name, sc, rays, render_wh=None):
    R = Reference()
    RC = Reference(cfg=True)
    box = sc.scene_box()
    R.load(sc.verts, sc.tris, box)
    nodes, refs, cache = R.build()
    hits, ids, cnt = R.trace(rays, counters=True)
    RC.load(sc.verts, sc.tris, box)
    cnodes, crefs, _ = RC.build()
    out = dict(verts=sc.verts, tris=sc.tris, box=box, lights=sc.lights, camera=sc.camera,
               ref_nodes=nodes, ref_refs=refs, ref_cache=cache, rays=rays, ref_hits=hits, ref_ids=ids,
               ref_counters=cnt, cfg_nodes=cnodes, cfg_refs=crefs, probe_in=PROBE,
               probe_out=R.normalize(PROBE))
    if render_wh is not None:
        w, h = render_wh
        O = Oracle()
        prim = O.camera_rays(sc.camera, w, h, NORM_IEEE)
        out["render_rays"] = prim
        out["render_wh"] = np.array([w, h], np.int32)
        out["ref_render"] = R.render(prim, w, h, sc.lights)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, {k: v.shape for k, v in out.items()})


def main():
    soup = scenes.random_soup(3000, seed=11, size=0.5)
    make("soup3k.npz", soup, random_rays(4096, 12, soup.scene_box()), render_wh=(64, 64))
    small = scenes.static_small()
    O = Oracle()
    rays = O.camera_rays(small.camera, 128, 128, NORM_IEEE)
    make("small24k.npz", small, rays, render_wh=(128, 128))


if __name__ == "__main__":
    main()
