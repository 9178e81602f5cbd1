"""The autotuner times traversal configurations, applies the fastest and
caches it per device; the tuned configuration returns the same hits."""
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
