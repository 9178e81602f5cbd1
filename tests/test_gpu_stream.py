"""Out-of-core leaf geometry (hk_stream_setup / hk_trace_streamed): the
reference's residency protocol (GPUTrace_stackless.cl:6-120,
GLVisitorGPUTrace.cpp:412-502) with leaves paged into a device pool from pinned
host memory. Hits equal the fully resident kd-restart traversal bit for bit for
any pool that holds the largest leaf; a small pool pages and evicts."""
import numpy as np
import pytest

from hulktracer_b200 import scenes
from hulktracer_b200._lib import HkError
from oracle.oracle import NORM_IEEE, RESTART as O_RESTART

HK_E_CAPACITY, HK_E_STATE = 18, 20


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def setup_static(hk, w=96, h=96):
    sc = scenes.static_small(width=w, height=h)
    c = hk.Context()
    c.upload(sc.verts, sc.tris)
    c.precompute()
    c.build()
    rays = c.camera_rays(sc.camera, w, h)
    return sc, c, rays


@pytest.mark.gpu
@pytest.mark.parametrize("pool", [1024, 8192, 1 << 22])
def test_streamed_equals_restart(hk, pool):
    sc, c, rays = setup_static(hk)
    ref = c.trace(rays, hk.RESTART)
    largest = int(c.export_compact()[0][:, 1][(c.export_compact()[0][:, 0] & 3) == 3].max())
    c.stream_setup(max(pool, largest))
    hits, st = c.trace_streamed(rays)
    assert np.array_equal(hits["tri"], ref["tri"])
    m = ref["tri"] >= 0
    assert m.mean() > 0.3 and np.array_equal(bits(hits["t"][m]), bits(ref["t"][m]))
    assert st["launches"] >= 2 and st["leaves_loaded"] > 0
    if pool == 1024:
        assert st["leaves_evicted"] > 0      # the pool is smaller than the rays' working set
    elif pool > 8192:
        assert st["leaves_evicted"] == 0
        # a warm pool: the second call pages nothing and takes one launch
        hits2, st2 = c.trace_streamed(rays)
        assert st2["leaves_loaded"] == 0 and st2["launches"] == 1
        assert np.array_equal(hits2["tri"], hits["tri"])
    c.close()


@pytest.mark.gpu
def test_streamed_matches_oracle_restart(hk, oracle):
    sc, c, rays = setup_static(hk, 64, 64)
    cn, cr = c.export_compact()
    nodes, refs = c.export_tree()
    box = c.get_box()
    cache = c.export_cache()
    tree = oracle.make_tree(sc.verts, sc.tris, cache, nodes, refs, box)
    oh, oid = oracle.trace(tree, oracle.camera_rays(sc.camera, 64, 64, NORM_IEEE), O_RESTART, 6)
    c.stream_setup(2048)
    hits, _ = c.trace_streamed(oracle.camera_rays(sc.camera, 64, 64, NORM_IEEE))
    assert np.array_equal(hits["tri"], oid)
    m = oid >= 0
    assert np.array_equal(bits(hits["t"][m]), bits(oh[m, 0]))
    c.close()


@pytest.mark.gpu
def test_animated_frame_small_pool(hk):
    # a pool far smaller than the working set of the frame's primary rays
    sc = scenes.animated_parts()
    c = hk.Context()
    c.upload(sc.verts, sc.tris)
    c.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    c.transform(scenes.part_matrices(sc, 17))
    c.build()
    rays = c.camera_rays(sc.camera, 320, 180)
    ref = c.trace(rays, hk.RESTART)
    cn = c.export_compact()[0]
    leaves = cn[(cn[:, 0] & 3) == 3]
    pool = max(int(leaves[:, 1].max()), int(leaves[:, 1].sum()) // 200)   # 0.5% of the leaf records
    c.stream_setup(pool)
    hits, st = c.trace_streamed(rays)
    assert np.array_equal(hits["tri"], ref["tri"])
    m = ref["tri"] >= 0
    assert np.array_equal(bits(hits["t"][m]), bits(ref["t"][m]))
    assert st["leaves_evicted"] > 0 and st["bytes_paged"] > 0
    c.close()


@pytest.mark.gpu
def test_stream_errors(hk):
    sc, c, rays = setup_static(hk, 32, 32)
    with pytest.raises(HkError) as e:
        c.trace_streamed(rays)
    assert e.value.status == HK_E_STATE
    c.stream_setup(1)                            # smaller than any leaf of several triangles
    with pytest.raises(HkError) as e:
        c.trace_streamed(rays)
    assert e.value.status == HK_E_CAPACITY
    c.stream_setup(1 << 20)
    c.build()                                    # a new tree: the snapshot is stale
    with pytest.raises(HkError) as e:
        c.trace_streamed(rays)
    assert e.value.status == HK_E_STATE
    c.close()
