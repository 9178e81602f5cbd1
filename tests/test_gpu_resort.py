"""HK_BUILD_SAH_RESORT: the reference's --treeType=SAH builder on the GPU.

The GPU tree is compared node by node with the oracle's serial restatement of
buildNodeSAH (hko_build_sah_resort, itself equal to the compiled reference's
KDTreeCPU::buildKDTreeSAH, see test_resort_oracle.py) in the compact layout
hk_tree_import makes of a reference tree: same junctions (axis, child pair,
plane bits), same leaves with the same polygon lists. Hits through the tree
equal the compiled reference's checkCollision on its own SAH tree bit for bit,
and the ropes built with the tree trace like the stack traversals.
"""
import numpy as np
import pytest

from hulktracer_b200 import scenes
from oracle.oracle import NORM_IEEE, Reference

LEAF = 3
REF_CONSTANTS = dict(traverse_cost=1.0, intersect_cost=5.0, max_depth=20, leaf_size=9, sah_sample=5)
BENCH_CONSTANTS = dict(traverse_cost=1.0, intersect_cost=1.5, max_depth=24, leaf_size=4, sah_sample=1)
ORACLE_ARGS = {id(REF_CONSTANTS): dict(ct=1.0, ci=5.0, max_depth=20, leaf_below=10, reduction=5),
               id(BENCH_CONSTANTS): dict(ct=1.0, ci=1.5, max_depth=24, leaf_below=5, reduction=1)}


def compare_compact(cn, cr, ref_cn, ref_refs):
    """Same compact tree: junction words equal, leaves with equal lists."""
    assert cn.shape == ref_cn.shape, (cn.shape, ref_cn.shape)
    leaf = (cn[:, 0] & 3) == LEAF
    assert np.array_equal(leaf, (ref_cn[:, 0] & 3) == LEAF)
    assert np.array_equal(cn[~leaf], ref_cn[~leaf])
    assert np.array_equal(cn[leaf, 1], ref_cn[leaf, 1])
    for k in np.nonzero(leaf)[0]:
        c = cn[k, 1]
        if c:
            a, b = cn[k, 0] >> 2, ref_cn[k, 0] >> 2
            assert np.array_equal(cr[a:a + c], ref_refs[b:b + c]), "leaf %d" % k


def build_and_compare(hk, oracle, verts, tris, consts):
    c = hk.Context(**consts)
    c.upload(verts, tris)
    st = c.build(hk.BUILD_SAH_RESORT)
    box = c.get_box()
    cn, cr = c.export_compact()
    rn, rr = oracle.build_sah_resort(verts, tris, box, **ORACLE_ARGS[id(consts)])
    compare_compact(cn, cr, oracle.ref_to_compact(rn), rr)
    assert st["nodes"] == cn.shape[0] and st["refs"] == cr.shape[0]
    return c, box, rn, rr


@pytest.mark.gpu
@pytest.mark.parametrize("consts", [REF_CONSTANTS, BENCH_CONSTANTS], ids=["reference", "bench"])
@pytest.mark.parametrize("scene", ["soup3k", "small24k", "soup20k"])
def test_tree_equals_oracle(hk, oracle, scene, consts):
    sc = {"soup3k": lambda: scenes.random_soup(3000, seed=1),
          "small24k": lambda: scenes.static_small(width=64, height=64),
          "soup20k": lambda: scenes.random_soup(20000, seed=5)}[scene]()
    c, _, _, _ = build_and_compare(hk, oracle, sc.verts.astype(np.float32), sc.tris, consts)
    c.close()


@pytest.mark.gpu
def test_animated_frame_equals_oracle(hk, oracle):
    """The 199,692-triangle animated scene (frame 17), reference constants."""
    sc = scenes.animated_parts()
    c = hk.Context()
    c.upload(sc.verts, sc.tris)
    c.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    c.transform(scenes.part_matrices(sc, 17))
    v = c.get_vertices()
    c.close()
    c, _, _, _ = build_and_compare(hk, oracle, v, sc.tris, REF_CONSTANTS)
    c.close()


@pytest.mark.gpu
@pytest.mark.skipif(not Reference.available(), reason="compiled reference not built")
def test_hits_equal_reference_on_its_sah_tree(hk, oracle):
    sc = scenes.static_small(width=96, height=96)
    v = sc.verts.astype(np.float32)
    c = hk.Context(short_stack=5, **REF_CONSTANTS)
    c.upload(v, sc.tris)
    c.build(hk.BUILD_SAH_RESORT)
    box = c.get_box()
    R = Reference()
    R.load(v, sc.tris, box)
    nodes, refs, cache = R.build("SAH")
    rays = oracle.camera_rays(sc.camera, 96, 96, NORM_IEEE)
    rh, rid = R.trace(rays)
    c.import_cache(cache)
    h = c.trace(rays, hk.SHORTSTACK)
    assert np.array_equal(h["tri"], rid)
    m = rid >= 0
    assert m.mean() > 0.3
    assert np.array_equal(h["t"][m].view(np.uint32), rh[m, 0].view(np.uint32))
    # the ropes written by the builder trace like the stacks
    r = c.trace(rays, hk.ROPES)
    f = c.trace(rays, hk.FULLSTACK)
    assert np.array_equal(r["tri"], f["tri"]) and np.array_equal(r["t"].view(np.uint32), f["t"].view(np.uint32))
    c.close()


@pytest.mark.gpu
def test_empty_and_tiny_scenes(hk, oracle):
    # a scene below the leaf size is one leaf; degenerate (flat) triangles
    v = np.array([[0, 0, 0, 1], [1, 0, 0, 1], [0, 1, 0, 1], [1, 1, 0, 1]], np.float32)
    t = np.array([[0, 1, 2, 0], [1, 3, 2, 0]], np.uint32)
    c = hk.Context(**REF_CONSTANTS)
    c.upload(v, t)
    st = c.build(hk.BUILD_SAH_RESORT)
    cn, cr = c.export_compact()
    assert st["nodes"] == 2 and (cn[0, 0] & 3) == LEAF and cn[0, 1] == 2 and sorted(cr) == [0, 1]
    c.close()
    # many coincident flat triangles: every candidate is co-planar
    rng = np.random.default_rng(4)
    v = np.concatenate([rng.uniform(0, 1, size=(300, 3)), np.ones((300, 1))], 1).astype(np.float32)
    v[:, 2] = 0.5
    t = np.zeros((100, 4), np.uint32)
    t[:, :3] = np.arange(300).reshape(100, 3)
    c, _, _, _ = build_and_compare(hk, oracle, v, t, REF_CONSTANTS)
    c.close()
