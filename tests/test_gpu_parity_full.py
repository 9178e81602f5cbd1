"""Parity at the benchmark sizes, through the C ABI, on the GPU.

* The animated 64-part scene (199,692 triangles, 1280x720) at frames 0 and 17
  (the bench's workload): the GPU tree equals the oracle's restatement array
  for array for the binned build and the exact SAH on nodes of up to 1024
  references; on the reference's own tree with the reference's cache, every
  primary ray's hit id and t bits equal the compiled reference's
  checkCollision (ring 5) and, for every other traversal variant, the oracle;
  the frame image on the GPU's own tree equals the oracle's, and against the
  reference's own image the number and size of pixels beyond 1/255 are
  reported.
* The large static scene (1,049,152 triangles, one mirror bounce on 30% of
  the triangles) at 640x360 (230,400 primary rays): tree equality, hit ids on
  the reference tree, the mirror-shaded image against the oracle.
* A batch of 4 clustered-soup scenes with incoherent rays (primary, shadow
  and cosine-weighted bounce stand-ins) in one persistent launch against the
  oracle's traversal of each scene's GPU-built tree.

The compiled reference (oracle/_ref) runs live when it is present; without
it the reference comparisons skip and the oracle ones still run."""
import numpy as np
import pytest

from hulktracer_b200 import scenes
from oracle.oracle import (FULLSTACK as O_FULL, NORM_IEEE, RESTART as O_RESTART, RESTART_EARLY as O_RESTART_EARLY,
                           ROPES as O_ROPES, SHORTSTACK as O_SHORT, Reference)

pytestmark = pytest.mark.gpu

HAVE_REF = Reference.available()
CT, CI = 1.0, 1.5


@pytest.fixture(scope="module")
def animated():
    return scenes.animated_parts()


@pytest.fixture(scope="module")
def static_large():
    return scenes.static_large()


def frame_verts(hk, sc, frame):
    c = hk.Context()
    c.upload(sc.verts, sc.tris)
    c.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    c.transform(scenes.part_matrices(sc, frame))
    v, box = c.get_vertices(), c.get_box()
    c.close()
    return v, box


def check_tree(hk, oracle, verts, tris, box, exact_max, layout=(32, 8, 1)):
    """The GPU tree with builder layout (subtree_max, subtree_depth,
    level_streams) equals the oracle's with the same layout."""
    c = hk.Context(exact_max=exact_max, subtree_max=layout[0], subtree_depth=layout[1], level_streams=layout[2])
    c.upload(verts, tris)
    c.set_box(box)
    c.precompute()
    st = c.build()
    gn, gr = c.export_compact()
    on, orf = oracle.build_binned(verts, tris, box, ct=CT, ci=CI, max_depth=24, leaf_size=4, exact_max=exact_max,
                                  defer=layout[0], defer_margin=layout[1])
    assert st["capacity_hit"] == 0
    assert gn.shape == on.shape and gr.shape == orf.shape
    assert np.array_equal(gn, on) and np.array_equal(gr, orf)
    return c


def hits_equal(h, ids, t):
    assert np.array_equal(h["tri"], ids)
    m = ids >= 0
    assert np.array_equal(h["t"][m].view(np.uint32), np.asarray(t, np.float32)[m].view(np.uint32))


@pytest.mark.parametrize("frame", [0, 17])
@pytest.mark.parametrize("exact_max", [0, 1024])
def test_animated_full_size_tree_equals_oracle(hk, oracle, animated, frame, exact_max):
    v, box = frame_verts(hk, animated, frame)
    check_tree(hk, oracle, v, animated.tris, box, exact_max).close()


@pytest.mark.parametrize("layout", [(32, 0, 1), (0, 0, 2)])
def test_animated_full_size_tree_layouts(hk, oracle, animated, layout):
    """The layouts the builder autotuner picks for this scene (deferred
    subtrees at any depth) and for the BART scenes (level by level, large
    nodes on a second stream), at full size."""
    v, box = frame_verts(hk, animated, 17)
    check_tree(hk, oracle, v, animated.tris, box, 0, layout).close()


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not built")
@pytest.mark.parametrize("frame", [0, 17])
def test_animated_full_size_hits_on_reference_tree(hk, oracle, animated, frame):
    """All 921,600 primary rays on the reference's tree and cache: ring 5 ==
    the reference's checkCollision bit for bit; the other variants == the
    oracle bit for bit."""
    sc = animated
    v, box = frame_verts(hk, sc, frame)
    R = Reference()
    R.load(v, sc.tris, box)
    nodes, refs, cache = R.build()
    rays = oracle.camera_rays(sc.camera, sc.width, sc.height, NORM_IEEE)
    rh, rid = R.trace(rays)
    c5 = hk.Context(short_stack=5)
    c5.upload(v, sc.tris)
    c5.set_box(box)
    c5.import_cache(cache)
    c5.import_tree(nodes, refs)
    for var in (hk.SHORTSTACK, hk.SMEMSTACK):
        hits_equal(c5.trace(rays, var), rid, rh[:, 0])
    assert (rid >= 0).mean() > 0.5
    c5.close()
    c6 = hk.Context(short_stack=6)
    c6.upload(v, sc.tris)
    c6.set_box(box)
    c6.import_cache(cache)
    c6.import_tree(nodes, refs)
    for name, ov in (("fullstack", O_FULL), ("shortstack", O_SHORT), ("restart", O_RESTART),
                     ("restart_early", O_RESTART_EARLY), ("ropes", O_ROPES)):
        tree = oracle.make_tree(v, sc.tris, cache, nodes, refs, box, with_ropes=(ov == O_ROPES))
        oh, oid = oracle.trace(tree, rays, ov, 6)
        hits_equal(c6.trace(rays, hk.VARIANTS[name]), oid, oh[:, 0])
    c6.close()


@pytest.mark.parametrize("frame", [0, 17])
def test_animated_full_size_frame_image(hk, oracle, animated, frame):
    """One frame through hk_frame (transform, binned build, ropes trace,
    shadow rays, shading; the CUDA graph) equals the oracle's image on the
    same tree. Against the reference's own image (its tree, its rsqrt cache
    and shading) the pixels beyond 1/255 are counted and reported."""
    import torch
    sc = animated
    W, H = sc.width, sc.height
    c = hk.Context()
    c.upload(sc.verts, sc.tris)
    c.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    out = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    c.frame(scenes.part_matrices(sc, frame), sc.camera, sc.lights, W, H, out.data_ptr(), hk.BUILD_BINNED,
            hk.ROPES, True)
    c.synchronize()
    img = out.cpu().numpy().view(np.uint32)
    v, box = c.get_vertices(), c.get_box()
    cn, cr = c.export_compact()
    cache = c.export_cache()
    c.close()
    tree = oracle.make_tree(v, sc.tris, cache, oracle.compact_to_ref(cn), cr, box, with_ropes=True)
    rays = oracle.camera_rays(sc.camera, W, H, NORM_IEEE)
    oimg = oracle.render_cpu(tree, rays, W, H, sc.lights, O_ROPES, 6, NORM_IEEE)
    assert np.array_equal(img, oimg)
    if HAVE_REF:
        R = Reference()
        R.load(v, sc.tris, box)
        R.build()
        rimg = R.render(rays, W, H, sc.lights)
        a = img.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
        b = rimg.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
        d = np.abs(a - b).max(axis=1)
        print("frame %d vs the reference's image: %d of %d pixels beyond 1/255 (max %d/255), %d lit" %
              (frame, int((d > 1).sum()), d.size, int(d.max()), int((rimg != 0).sum())))
        assert (d <= 1).mean() >= 0.999


def test_static_large_tree_equals_oracle(hk, oracle, static_large):
    sc = static_large
    check_tree(hk, oracle, sc.verts, sc.tris, sc.scene_box(), 0).close()


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not built")
def test_static_large_hits_and_mirror_image(hk, oracle, static_large):
    """The 1.05M-triangle scene at 640x360: ring-5 hits on the reference tree
    == the reference's checkCollision; the mirror-shaded image on the
    reference tree == the oracle's restatement."""
    sc = static_large
    W, H = 640, 360
    box = sc.scene_box()
    R = Reference()
    R.load(sc.verts, sc.tris, box)
    nodes, refs, cache = R.build()
    rays = oracle.camera_rays(sc.camera, W, H, NORM_IEEE)
    rh, rid = R.trace(rays)
    c = hk.Context(short_stack=5)
    c.upload(sc.verts, sc.tris)
    c.set_box(box)
    c.import_cache(cache)
    c.import_tree(nodes, refs)
    hits_equal(c.trace(rays, hk.SHORTSTACK), rid, rh[:, 0])
    mirror = sc.extra["mirror"]
    c.set_mirrors(mirror)
    img = c.render(sc.camera, sc.lights, W, H, hk.SHORTSTACK, hk.SHADE_MIRROR)
    c.close()
    tree = oracle.make_tree(sc.verts, sc.tris, cache, nodes, refs, box)
    oimg = oracle.render_mirror(tree, rays, W, H, sc.lights, mirror, O_SHORT, 5, NORM_IEEE)
    assert np.array_equal(img, oimg)
    assert (img != 0).mean() > 0.3


def test_batch_incoherent_rays_equal_oracle(hk, oracle):
    """Four clustered-soup scenes with uneven, incoherent ray batches in one
    persistent launch (ropes and the full stack): every hit equals the
    oracle's traversal of that scene's GPU-built tree."""
    import torch
    sets = scenes.batch_scenes(n_scenes=4, tris=(20_000, 200_000), rays=(20_000, 120_000), seed=17)
    ctx = hk.Context()
    batch = hk.engine.Batch(ctx)
    rays, offsets, trees = [], [0], []
    for i, (sc, nr) in enumerate(sets):
        batch.add_scene(sc.verts, sc.tris)
        r = scenes.incoherent_rays(sc, nr, seed=500 + i)
        rays.append(r)
        offsets.append(offsets[-1] + nr)
        c = hk.Context()
        c.upload(sc.verts, sc.tris)
        c.precompute()
        c.build()
        cn, cr = c.export_compact()
        trees.append((sc, cn, cr, c.export_cache(), c.get_box()))
        c.close()
    allr = np.concatenate(rays)
    d_rays = torch.from_numpy(allr).cuda()
    d_hits = torch.zeros(2 * allr.shape[0], dtype=torch.int32, device="cuda")
    for var, ov in ((hk.ROPES, O_ROPES), (hk.FULLSTACK, O_FULL)):
        d_hits.fill_(0)
        batch.trace_device(d_rays.data_ptr(), offsets, d_hits.data_ptr(), var)
        torch.cuda.synchronize()
        h = d_hits.cpu().numpy().view(hk._lib.HIT_DTYPE)
        for i, (sc, cn, cr, cache, box) in enumerate(trees):
            tree = oracle.make_tree(sc.verts, sc.tris, cache, oracle.compact_to_ref(cn), cr, box,
                                    with_ropes=(ov == O_ROPES))
            oh, oid = oracle.trace(tree, rays[i], ov, 6)
            hits_equal(h[offsets[i]:offsets[i + 1]], oid, oh[:, 0])
    batch.close()
    ctx.close()


@pytest.mark.skipif(not HAVE_REF, reason="compiled reference not built")
def test_animated_full_size_rule4_own_cache(hk, oracle, animated):
    """Parity rule 4 on the GPU: with its own triangle cache (hk_precompute,
    IEEE 1 / sqrt) on the reference's tree, the GPU's ring-5 hit ids agree
    with the reference's checkCollision (and its rsqrt cache) on at least
    99.99% of the 921,600 primary rays of frame 17; every disagreement is an
    equal-t tie or a hit within 1e-5 of a triangle edge."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(__file__))
    from _agreement import explain
    sc = animated
    v, box = frame_verts(hk, sc, 17)
    R = Reference()
    R.load(v, sc.tris, box)
    nodes, refs, _ = R.build()
    rays = oracle.camera_rays(sc.camera, sc.width, sc.height, NORM_IEEE)
    rh, rid = R.trace(rays)
    c = hk.Context(short_stack=5)
    c.upload(v, sc.tris)
    c.set_box(box)
    c.precompute()
    c.import_tree(nodes, refs)
    h = c.trace(rays, hk.SHORTSTACK)
    c.close()
    n, ok = explain(v, sc.tris, rays, rid, rh[:, 0], h["tri"], h["t"])
    rate = 1.0 - n / rays.shape[0]
    print("GPU own cache vs reference: id agreement %.7f (%d of %d differ, %d explained)" %
          (rate, n, rays.shape[0], ok))
    assert rate >= 0.9999 and ok == n
