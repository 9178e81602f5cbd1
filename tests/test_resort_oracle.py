"""The oracle's restatement of buildNodeSAH (--treeType=SAH, KDTreeSAH.cpp:
9-244) against the compiled reference: identical nodes (including the unlinked
node 1 the reference leaves behind) and leaf lists, with the reference's own
constants and with the benchmark constants."""
import numpy as np
import pytest

from hulktracer_b200 import scenes
from oracle.oracle import Reference

SCENES = {"soup3k": lambda: scenes.random_soup(3000, seed=1),
          "small24k": lambda: scenes.static_small(width=64, height=64),
          "soup20k": lambda: scenes.random_soup(20000, seed=5)}


@pytest.mark.skipif(not (Reference.available() and Reference.available(cfg=True)),
                    reason="compiled reference not built")
@pytest.mark.parametrize("cfg", [False, True], ids=["reference", "bench"])
@pytest.mark.parametrize("scene", sorted(SCENES))
def test_resort_oracle_equals_reference(oracle, scene, cfg):
    sc = SCENES[scene]()
    v = sc.verts.astype(np.float32)
    box = oracle.scene_box(v)
    R = Reference(cfg=cfg)
    R.load(v, sc.tris, box)
    rn, rr, _ = R.build("SAH")
    args = dict(ct=1.0, ci=1.5, max_depth=24, leaf_below=5, reduction=1) if cfg else {}
    on, orr = oracle.build_sah_resort(v, sc.tris, box, **args)
    assert np.array_equal(rn, on) and np.array_equal(rr, orr)
    assert np.array_equal(rn[1], [0, 0, 0, 0])   # the node buildKDTreeSAH pushes and never links
    # the default builder is a different tree
    n2, _, _ = R.build("SAHNlogN")
    assert n2.shape != rn.shape or not np.array_equal(n2, rn)


def test_resort_oracle_layout_rules(oracle):
    # leaves hold every listed polygon once per leaf, with sequential ids
    sc = scenes.random_soup(40, seed=9)
    v = sc.verts.astype(np.float32)
    n, r = oracle.build_sah_resort(v, sc.tris, oracle.scene_box(v))
    assert n.shape[0] >= 3 and n[0, 0] & 8
    leaves = n[(n[:, 0] & 4) != 0]
    assert leaves[:, 2].sum() == r.shape[0]
    assert np.array_equal(np.sort(leaves[:, 3]), np.arange(leaves.shape[0]))
