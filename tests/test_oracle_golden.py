"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference compiled from its sources) and
the reference's unit tests (test/sharedFunctionTest.cpp)."""
import os

import numpy as np
import pytest

from oracle.oracle import (BRUTE, CFG_SAH, FULLSTACK, NORM_IEEE, NORM_SSE, RESTART, RESTART_EARLY, ROPES,
                           SHORTSTACK, Reference)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["soup3k.npz", "small24k.npz"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def same_rsqrt(oracle, g):
    """Does this CPU's rsqrtps reproduce the one the fixtures were made on?"""
    out = np.stack([oracle.normalize(v, NORM_SSE) for v in g["probe_in"]])
    return np.array_equal(out.view(np.uint32), g["probe_out"].view(np.uint32))


# ---- reference unit tests (test/sharedFunctionTest.cpp:7-55) ----
def test_box_volume(oracle):
    box = np.array([0, 0, 0, 1, 1.0, 2.0, 3.0, 1], np.float32)
    assert oracle.box_volume(box) == np.float32(1.0 * 2.0 * 3.0)


def test_box_surface(oracle):
    box = np.array([0, 0, 0, 1, 1.0, 2.0, 3.0, 1], np.float32)
    assert oracle.box_surface(box) == np.float32(2.0 * (1.0 * 2.0 + 2.0 * 3.0 + 1.0 * 3.0))


def test_dot_lane_order(oracle):
    # SPMatrix.hpp:284-289 reduces (p3 + p1) + (p2 + p0)
    a = np.array([1e8, 1.0, -1e8, 1.0], np.float32)
    b = np.array([1.0, 1.0, 1.0, 1.0], np.float32)
    p = a * b
    assert oracle.dot4(a, b) == np.float32(np.float32(p[3] + p[1]) + np.float32(p[2] + p[0]))


@pytest.mark.parametrize("name", CASES)
def test_sah_nlogn_tree_matches_reference(oracle, name):
    g = load(name)
    nodes, refs = oracle.build_sah_nlogn(g["verts"], g["tris"], g["box"])
    assert np.array_equal(nodes, g["ref_nodes"])
    assert np.array_equal(refs, g["ref_refs"])
    nodes, refs = oracle.build_sah_nlogn(g["verts"], g["tris"], g["box"], **CFG_SAH)
    assert np.array_equal(nodes, g["cfg_nodes"])
    assert np.array_equal(refs, g["cfg_refs"])


@pytest.mark.parametrize("name", CASES)
def test_cache_matches_reference(oracle, name):
    g = load(name)
    if not same_rsqrt(oracle, g):
        pytest.skip("this CPU's rsqrtps differs from the fixture CPU's")
    c = oracle.cache(g["verts"], g["tris"], NORM_SSE)
    ref = g["ref_cache"]
    eq = (c.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(c) & np.isnan(ref))
    assert eq.all()


@pytest.mark.parametrize("name", CASES)
def test_checkcollision_matches_reference(oracle, name):
    """The oracle's short stack (depth 5) == KDTreeCPU::checkCollision on the
    reference's own tree and cache: hit ids, t, normal and position bit-exact,
    node-visit and triangle-test counts equal."""
    g = load(name)
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"])
    hits, ids, cnt = oracle.trace(tree, g["rays"], SHORTSTACK, 5, counters=True)
    assert np.array_equal(ids, g["ref_ids"])
    hit = ids >= 0
    assert np.array_equal(hits[hit, :7].view(np.uint32), g["ref_hits"][hit, :7].view(np.uint32))
    assert np.array_equal(cnt[:, 0], g["ref_counters"][:, 0])
    assert np.array_equal(cnt[:, 2], g["ref_counters"][:, 1])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant", [FULLSTACK, RESTART, RESTART_EARLY, ROPES, BRUTE])
def test_other_variants_agree_with_reference(oracle, name, variant):
    """Full stack, kd-restart, ropes and brute force return the reference's
    closest hit (t bit-exact); ids may differ only between equal-t ties."""
    g = load(name)
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"],
                            with_ropes=(variant == ROPES))
    hits, ids = oracle.trace(tree, g["rays"], variant, 5)
    ref_t = g["ref_hits"][:, 0]
    assert np.array_equal(ids >= 0, g["ref_ids"] >= 0)
    hit = ids >= 0
    assert np.array_equal(hits[hit, 0], ref_t[hit])
    # t is bit-equal for every hit, so a different id is a triangle hit at the
    # same t: an equal-t tie (shared edges), resolved by test order
    diff = ids != g["ref_ids"]
    assert diff.mean() < 1e-2


@pytest.mark.parametrize("name", CASES)
def test_render_matches_reference(oracle, name):
    """Restated GLVisitorCPUTrace::traceScene: SSE mode equals the reference
    image exactly (same CPU), IEEE mode within 1/255 on >= 99.9% of pixels."""
    g = load(name)
    w, h = (int(x) for x in g["render_wh"])
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"])
    img_ieee = oracle.render_cpu(tree, g["render_rays"], w, h, g["lights"], mode=NORM_IEEE)
    a = img_ieee.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
    b = g["ref_render"].view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
    assert (np.abs(a - b).max(axis=1) <= 1).mean() >= 0.999
    if same_rsqrt(oracle, g):
        img_sse = oracle.render_cpu(tree, g["render_rays"], w, h, g["lights"], mode=NORM_SSE)
        assert np.array_equal(img_sse, g["ref_render"])


@pytest.mark.skipif(not Reference.available(), reason="compiled reference not built here")
def test_oracle_equals_compiled_reference_live(oracle):
    """Against the compiled reference itself (not only the stored vectors)."""
    from hulktracer_b200 import scenes
    sc = scenes.random_soup(1500, seed=5, size=0.8)
    box = sc.scene_box()
    R = Reference()
    R.load(sc.verts, sc.tris, box)
    nodes, refs, cache = R.build()
    on, orf = oracle.build_sah_nlogn(sc.verts, sc.tris, box)
    assert np.array_equal(nodes, on) and np.array_equal(refs, orf)
    rays = oracle.camera_rays(sc.camera, 48, 48)
    rh, rid = R.trace(rays)
    tree = oracle.make_tree(sc.verts, sc.tris, cache, nodes, refs, box)
    oh, oid = oracle.trace(tree, rays, SHORTSTACK, 5)
    assert np.array_equal(rid, oid)
