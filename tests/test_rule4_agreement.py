"""Parity rule 4 on the CPU: with the triangle cache computed the way the GPU
computes it (IEEE 1 / sqrt, hk_precompute) instead of the reference's rsqrt
approximation, and with the reference's OpenCL intersection form
(checkRayToPoly, SharedFunctions.hpp:47-103, restated in the oracle), the hit
ids on the reference's own tree agree with the reference's checkCollision
(KDTreeCPU.cpp:230-253) on at least 99.99% of the 512x512 primary rays of the
24,576-triangle scene, and every disagreement is an equal-t tie or a hit
within 1e-5 of a triangle edge. (The GPU's traversal equals the oracle's
IEEE-cache traversal bit for bit; tests/test_gpu_parity_full.py checks the
same agreement on the GPU at the animated scene's full size.)"""
import numpy as np
import pytest

from hulktracer_b200 import scenes
from oracle.oracle import ISECT_ACC, ISECT_POLY, NORM_IEEE, SHORTSTACK, Reference

from _agreement import explain  # noqa: E402

pytestmark = pytest.mark.skipif(not Reference.available(), reason="compiled reference not built")


@pytest.mark.parametrize("form", ["ieee_cache", "poly_form"])
def test_id_agreement_with_reference(oracle, form):
    sc = scenes.static_small()
    box = sc.scene_box()
    rays = oracle.camera_rays(sc.camera, 512, 512, NORM_IEEE)
    R = Reference()
    R.load(sc.verts, sc.tris, box)
    nodes, refs, _ = R.build()
    rh, rid = R.trace(rays)
    tree = oracle.make_tree(sc.verts, sc.tris, oracle.cache(sc.verts, sc.tris, NORM_IEEE), nodes, refs, box)
    oracle.set_isect_form(ISECT_POLY if form == "poly_form" else ISECT_ACC)
    try:
        oh, oid = oracle.trace(tree, rays, SHORTSTACK, 5)
    finally:
        oracle.set_isect_form(ISECT_ACC)
    n, ok = explain(sc.verts, sc.tris, rays, rid, rh[:, 0], oid, oh[:, 0])
    rate = 1.0 - n / rays.shape[0]
    print("%s: id agreement %.6f (%d of %d rays differ, %d explained)" % (form, rate, n, rays.shape[0], ok))
    assert rate >= 0.9999
    assert ok == n
    assert (rid >= 0).sum() > rays.shape[0] // 4
