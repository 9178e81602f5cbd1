"""Failure detection on the GPU, made to happen without a GPU fault: every
device-side wait of the builder is bounded and every traversal has a step
bound, and a test makes them run out.

* The builder's reference tiles wait (bounded) for the plan tile that wrote
  their nodes' reference destinations. A test aid (hk_set_debug_flags bit 0)
  makes the first plan tile of level 1 withhold its done flag; with a short
  spin limit the waits run out, the build stops (every later kernel returns
  at once) and hk_build returns HK_E_DEVICE_TIMEOUT. The failed output is not
  a tree (tracing it is refused), and the next build on the same context
  equals a normal build.
* A trace whose rays exceed the node-step bound (hk_config.max_steps) stops
  them and returns HK_E_BOUNDS; the context keeps working."""
import os

import numpy as np
import pytest

from hulktracer_b200 import scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
HK_E_DEVICE_TIMEOUT, HK_E_BOUNDS, HK_E_STATE = 17, 19, 20


def test_builder_wait_runs_out_and_context_recovers(hk):
    sc = scenes.animated_parts(n_parts=16, width=64, height=64)
    c = hk.Context(spin_limit=2000)
    c.upload(sc.verts, sc.tris)
    c.set_box(sc.scene_box())
    c.precompute()
    c.build()
    good_n, good_r = c.export_compact()
    rays = c.camera_rays(sc.camera, 64, 64)
    good_hits = c.trace(rays, hk.ROPES)
    c.set_debug_flags(1)
    for _ in range(2):
        with pytest.raises(hk.HkError) as e:
            c.build()
        assert e.value.status == HK_E_DEVICE_TIMEOUT
        with pytest.raises(hk.HkError) as e:
            c.trace(rays, hk.ROPES)
        assert e.value.status == HK_E_STATE
    c.set_debug_flags(0)
    c.build()
    n, r = c.export_compact()
    assert np.array_equal(n, good_n) and np.array_equal(r, good_r)
    h = c.trace(rays, hk.ROPES)
    assert np.array_equal(h["tri"], good_hits["tri"])
    c.close()


def test_trace_step_bound_returns_error(hk):
    g = dict(np.load(os.path.join(GOLDEN, "small24k.npz")))
    ok = hk.Context()
    bounded = hk.Context(max_steps=3)
    for c in (ok, bounded):
        c.upload(g["verts"], g["tris"])
        c.set_box(g["box"])
        c.import_cache(g["ref_cache"])
        c.import_tree(g["ref_nodes"], g["ref_refs"])
    for v in (hk.SHORTSTACK, hk.FULLSTACK, hk.RESTART):
        with pytest.raises(hk.HkError) as e:
            bounded.trace(g["rays"], v)
        assert e.value.status == HK_E_BOUNDS
    # the error word was cleared: the bounded context still traces short rays
    far = g["rays"].copy()
    far[:, 0:3] = 1e6       # every ray starts outside the scene box, heading away from it
    far[:, 4:7] = np.float32(1.0 / np.sqrt(3.0))
    h = bounded.trace(far, hk.SHORTSTACK)
    assert (h["tri"] == -1).all()
    h = ok.trace(g["rays"], hk.SHORTSTACK)
    assert (h["tri"] >= 0).any()
    ok.close()
    bounded.close()
