"""AFF (BART) scenes on the device: hk_scene_load_aff / hk_scene_animate_aff.

The synthetic AFF scene of ``golden/aff`` is transformed on the GPU and
compared bit for bit with the vertices and scene box that the reference's own
AFFParser + AFFTransformVisitor produced (``golden/aff_golden.npz``). Then a
frame of it is traced: through the reference's tree (its checkCollision ==
the short-stack kernel bit for bit, as in the parity tests), through the GPU's
own tree (ropes == brute force), and through hk_frame with the AFF matrices,
camera and lights.
"""
import os

import numpy as np
import pytest

from hulktracer_b200.engine import Aff
from oracle.oracle import NORM_IEEE, Reference

HERE = os.path.dirname(os.path.abspath(__file__))
SCENE = os.path.join(HERE, "golden", "aff", "scene.aff")
GOLDEN = os.path.join(HERE, "golden", "aff_golden.npz")
W, H = 160, 100


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


@pytest.mark.gpu
def test_device_transform_matches_reference(hk, golden):
    aff = Aff(SCENE)
    c = hk.Context()
    c.load_aff(aff, float(golden["times"][0]))
    for k, t in enumerate(golden["times"]):
        if k:
            c.animate_aff(aff, float(t))
        assert np.array_equal(bits(c.get_vertices()), bits(golden["verts"][k])), "t=%g" % t
        assert np.array_equal(bits(c.get_box()), bits(golden["boxes"][k])), "box at t=%g" % t
    c.close()
    aff.close()


@pytest.mark.gpu
@pytest.mark.skipif(not Reference.available(), reason="compiled reference not built")
@pytest.mark.parametrize("k", [1, 3])
def test_frame_on_reference_tree(hk, oracle, golden, k):
    aff = Aff(SCENE)
    t = float(golden["times"][k])
    c = hk.Context(short_stack=5)
    c.load_aff(aff, t)
    v, box = c.get_vertices(), c.get_box()
    R = Reference()
    R.load(v, golden["tris"], box)
    nodes, refs, cache = R.build()
    rays = oracle.camera_rays(aff.camera(t), W, H, NORM_IEEE)
    rh, rid = R.trace(rays)
    c.import_cache(cache)
    c.import_tree(nodes, refs)
    h = c.trace(rays, hk.SHORTSTACK)
    assert np.array_equal(h["tri"], rid)
    m = rid >= 0
    assert m.sum() > 500   # the animated camera sees part of the scene
    assert np.array_equal(bits(h["t"][m]), bits(rh[m, 0]))
    c.close()
    aff.close()


@pytest.mark.gpu
def test_own_tree_and_frame_graph(hk, golden):
    import torch
    aff = Aff(SCENE)
    t = float(golden["times"][2])
    c = hk.Context()
    c.load_aff(aff, t)
    c.precompute()
    c.build()
    rays = c.camera_rays(aff.camera(t), W, H)
    b = c.trace(rays, hk.BRUTE)
    r = c.trace(rays, hk.ROPES)
    m = b["tri"] >= 0
    assert m.mean() > 0.1
    assert np.array_equal(r["tri"] >= 0, m) and np.array_equal(bits(r["t"][m]), bits(b["t"][m]))
    img = c.render(aff.camera(t), aff.lights(), W, H, hk.ROPES)
    # the per-frame graph (transform, build, trace, shadows, shading) from the
    # AFF matrices gives the same image as the separate calls
    out = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    c.frame(aff.part_matrices(t), aff.camera(t), aff.lights(), W, H, out.data_ptr(), hk.BUILD_BINNED, hk.ROPES,
            True)
    c.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint32), img)
    assert len(np.unique(img)) > 8
    c.close()
    aff.close()
