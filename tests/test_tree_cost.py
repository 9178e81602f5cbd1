"""SAH cost of the GPU builder's tree (its algorithm restated in the oracle;
GPU trees equal the restatement, tests/test_gpu_build.py) against the
reference's own SAH-NlogN tree built with the same constants (compiled
reference, Ct 1, Ci 1.5, depth 24, leaves below 5, no reduction). One cost
function (full surface areas) costs both. With the exact SAH on nodes of at
most 1024 references (hk_config.exact_max = 1024) the GPU tree must cost at
most 1.01x the reference's on the benchmark scenes (at the rest pose the reference loses polygons coplanar
with its candidate planes, KDTreeSAH.cpp:462-485, and the GPU tree is far
cheaper; at rotated frames the two are within a few tenths of a percent).
Soups of large random triangles are the builder's weakest case (the top
levels are binned); the second test bounds them."""
import numpy as np
import pytest

from hulktracer_b200 import scenes
from oracle.oracle import Reference

pytestmark = pytest.mark.skipif(not Reference.available(cfg=True), reason="compiled reference not built")

CT, CI = 1.0, 1.5


def ratio(oracle, verts, tris, box, exact_max=1024):
    R = Reference(cfg=True)
    R.load(verts, tris, box)
    rn, _, _ = R.build()
    cref = oracle.tree_cost(rn, box, CT, CI)
    cn, _ = oracle.build_binned(verts, tris, box, ct=CT, ci=CI, max_depth=24, leaf_size=4, exact_max=exact_max)
    return oracle.tree_cost(oracle.compact_to_ref(cn), box, CT, CI) / cref


@pytest.mark.parametrize("which", ["C1", "C2_100k", "C3_frame5", "C3_frame17", "C3_frame42"])
def test_exact_cost_within_1pct_on_benchmark_scenes(oracle, which):
    if which == "C1":
        sc = scenes.static_small()
        v = sc.verts
    elif which == "C2_100k":
        sc = scenes.static_large(n_cluster_tris=100_000)
        v = sc.verts
    else:
        sc = scenes.animated_parts()
        frame = int(which.split("frame")[1])
        v = oracle.transform(sc.rest_verts, sc.part_of_vertex, scenes.part_matrices(sc, frame))
    r = ratio(oracle, v, sc.tris, oracle.scene_box(v))
    assert r <= 1.01


@pytest.mark.parametrize("which", ["cluster4", "cluster5", "random20k"])
def test_exact_cost_on_soups(oracle, which):
    if which == "random20k":
        sc = scenes.random_soup(20000, seed=4)
        bound = 1.05
    else:
        sc = scenes.cluster_soup(30000, seed=int(which[-1]))
        bound = 1.01
    assert ratio(oracle, sc.verts, sc.tris, sc.scene_box()) <= bound


def test_binned_only_cost_recorded(oracle):
    """Binned everywhere (the default, 32 bins, the headline arm): a rotated
    frame costs 1.17x the reference's tree -- it does not meet the 1% bar,
    which is why the exact (exact_max = 1024) and learned arms exist."""
    sc = scenes.animated_parts()
    v = oracle.transform(sc.rest_verts, sc.part_of_vertex, scenes.part_matrices(sc, 5))
    r = ratio(oracle, v, sc.tris, oracle.scene_box(v), exact_max=0)
    assert 1.15 < r < 1.19, r
