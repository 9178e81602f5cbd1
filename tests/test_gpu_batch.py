"""Many scenes with uneven ray batches in ONE persistent launch: every ray's
hit equals the single-scene trace of its own scene (ids and t bit-exact)."""
import numpy as np
import pytest

from hulktracer_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["ropes", "shortstack", "fullstack"])
def test_batch_equals_per_scene(hk, variant):
    import torch
    sets = scenes.batch_scenes(n_scenes=5, seed=9, tris=(2_000, 30_000), rays=(3_000, 40_000))
    ctx = hk.Context()
    batch = hk.engine.Batch(ctx)
    rays, offsets, expected = [], [0], []
    single = hk.Context()
    for i, (sc, nr) in enumerate(sets):
        assert batch.add_scene(sc.verts, sc.tris) == i
        r = scenes.incoherent_rays(sc, nr, seed=100 + i)
        rays.append(r)
        offsets.append(offsets[-1] + nr)
        single.upload(sc.verts, sc.tris)
        single.precompute()
        single.build()
        expected.append(single.trace(r, hk.VARIANTS[variant]))
    allr = np.concatenate(rays)
    d_rays = torch.from_numpy(allr).cuda()
    d_hits = torch.zeros(2 * allr.shape[0], dtype=torch.int32, device="cuda")
    ms = batch.trace_device(d_rays.data_ptr(), offsets, d_hits.data_ptr(), hk.VARIANTS[variant])
    torch.cuda.synchronize()
    hits = d_hits.cpu().numpy().view(hk._lib.HIT_DTYPE)
    for i in range(len(sets)):
        h = hits[offsets[i]:offsets[i + 1]]
        e = expected[i]
        assert np.array_equal(h["tri"], e["tri"])
        assert np.array_equal(h["t"], e["t"])
    assert ms.shape == (5,) and np.all(ms > 0)
    batch.close()


def test_batch_outliving_its_context(hk):
    """hk_destroy with a batch still alive frees the batch's device memory;
    later batch calls return HK_E_STATE, hk_batch_destroy frees the rest, and
    the process's CUDA state stays sound for the next context."""
    import ctypes as C
    from hulktracer_b200 import scenes
    sc = scenes.cluster_soup(5000, seed=3)
    ctx = hk.Context()
    batch = hk.engine.Batch(ctx)
    batch.add_scene(sc.verts, sc.tris)
    ctx.close()
    L = hk._lib.load()
    sid = C.c_uint32()
    assert L.hk_batch_add_scene(batch.h, hk._lib.ptr(np.ascontiguousarray(sc.verts, np.float32)), sc.verts.shape[0],
                                hk._lib.ptr(np.ascontiguousarray(sc.tris, np.uint32)), sc.tris.shape[0],
                                C.byref(sid)) == 20
    batch.close()
    c2 = hk.Context()
    c2.upload(sc.verts, sc.tris)
    c2.precompute()
    assert c2.build()["nodes"] > 0
    c2.close()
