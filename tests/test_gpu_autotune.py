"""The autotuners: traversal configurations (the fastest applied and cached
per device; the tuned configuration returns the same hits) and the builder
layout (the fastest applied; the tree equals the oracle's with that layout)."""
import os

import numpy as np
import pytest

from hulktracer_b200 import scenes

pytestmark = pytest.mark.gpu


def test_autotune_and_cache(hk, tmp_path):
    import torch
    sc = scenes.animated_parts(n_parts=12, width=256, height=144)
    ctx = hk.Context()
    ctx.upload(sc.verts, sc.tris)
    ctx.precompute()
    ctx.build()
    rays = scenes.incoherent_rays(sc, 60_000, seed=3)
    ref = ctx.trace(rays, hk.ROPES)
    d = torch.from_numpy(rays).cuda()
    cache = str(tmp_path / "tune.txt")
    r = ctx.autotune(d.data_ptr(), rays.shape[0], cache)
    assert r["tried"] > 20 and r["best_ms"] > 0
    assert r["best_ms"] <= r["default_ms"] * 1.05
    assert os.path.exists(cache)
    hits = ctx.trace(rays, r["variant"])
    assert np.array_equal(hits["t"], ref["t"])
    r2 = ctx.autotune(d.data_ptr(), rays.shape[0], cache)
    assert r2["tried"] == 0 and r2["block_size"] == r["block_size"] and r2["short_stack"] == r["short_stack"]


def test_autotune_build_layout(hk, oracle):
    """hk_autotune_build times the builder layouts, keeps the fastest, and the
    next build with it equals the oracle's tree with the same layout; every
    candidate builds the same tree up to numbering (same cost)."""
    sc = scenes.animated_parts(n_parts=12, width=256, height=144)
    ctx = hk.Context()
    ctx.upload(sc.verts, sc.tris)
    ctx.set_box(sc.scene_box())
    ctx.precompute()
    ctx.build()
    cost0 = ctx.tree_cost(1.0, 1.5)
    r = ctx.autotune_build(hk.BUILD_BINNED, 3)
    assert r["tried"] == 10 and r["best_ms"] > 0 and r["best_ms"] <= r["default_ms"]
    assert r["level_streams"] in (1, 2)
    assert (r["subtree_max"], r["subtree_depth"]) in [(0, 0), (32, 0), (32, 10), (32, 8), (32, 6)]
    st = ctx.build()
    cn, cr = ctx.export_compact()
    on, orf = oracle.build_binned(sc.verts, sc.tris, sc.scene_box(), defer=r["subtree_max"],
                                  defer_margin=r["subtree_depth"])
    assert np.array_equal(cn, on) and np.array_equal(cr, orf)
    assert abs(ctx.tree_cost(1.0, 1.5) - cost0) <= 1e-6 * cost0
    assert st["nodes"] == on.shape[0]
    ctx.close()


def test_set_trace_and_build_config(hk):
    """hk_set_trace_config / hk_set_build_layout: invalid values are refused
    with HK_E_ILLEGAL_INPUT; valid ones change the launches, not the hits."""
    from hulktracer_b200._lib import HkError
    sc = scenes.animated_parts(n_parts=6, width=96, height=64)
    ctx = hk.Context()
    ctx.upload(sc.verts, sc.tris)
    ctx.precompute()
    ctx.build()
    rays = ctx.camera_rays(sc.camera, 96, 64)
    ref = ctx.trace(rays, hk.SHORTSTACK)
    for bad in ((48, 6), (512, 6), (128, 0), (128, 17)):
        with pytest.raises(HkError) as e:
            ctx.set_trace_config(*bad)
        assert e.value.status == 4
    with pytest.raises(HkError):
        ctx.set_build_layout(33, 0, 1)
    ctx.set_trace_config(64, 4)
    h = ctx.trace(rays, hk.SHORTSTACK)
    assert np.array_equal(h["tri"], ref["tri"]) and np.array_equal(h["t"], ref["t"])
    ctx.set_build_layout(0, 0, 2)
    ctx.build()
    h = ctx.trace(rays, hk.SHORTSTACK)
    assert np.array_equal(h["tri"], ref["tri"]) and np.array_equal(h["t"], ref["t"])
    ctx.close()
