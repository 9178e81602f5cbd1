"""hk_render_noalloc -- rendering for callers that cannot let the library
allocate device memory (a host with its own pooled allocator, code running
while a graph capture is open elsewhere, a fixed memory budget). The caller
owns the tree, triangle records and image buffers; the pipeline's scratch is
one static device array inside the library.

For every traversal variant the entry point accepts, the test renders twice
in a row through the C ABI from caller-held buffers and compares each image
with hk_render, the allocating entry point, on the same tree (pixels must be
equal; the tolerance used elsewhere is 1/255). Free device memory must be the
same before and after the second call: the first call on a device has already
looked up the scratch array and loaded every kernel the entry point launches,
so nothing is allocated afterwards. ROPES, which needs per-node cells and ropes
this call does not take, and a frame too large for the fixed scratch are
refused.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it passes alone and after the others."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

W, H = 256, 192
VARIANTS = ["shortstack", "fullstack", "smemstack", "restart", "restart_early", "brute"]


def _records(cache, verts, tris):
    rec = np.zeros((cache.shape[0], 16), np.float32)
    p1 = verts[tris[:, 0], :3]
    rec[:, 0:3], rec[:, 3] = cache[:, 0:3], cache[:, 12]
    rec[:, 4:7], rec[:, 7] = p1, cache[:, 13]
    rec[:, 8:11], rec[:, 11] = cache[:, 4:7], cache[:, 14]
    rec[:, 12:15], rec[:, 15] = cache[:, 8:11], cache[:, 15]
    return rec


@pytest.fixture(scope="module")
def setup(hk):
    import torch
    from hulktracer_b200 import scenes
    sc = scenes.static_small(width=W, height=H)
    ctx = hk.Context()
    ctx.upload(sc.verts, sc.tris)
    ctx.precompute()
    ctx.build()
    cn, cr = ctx.export_compact()
    rec = _records(ctx.export_cache(), sc.verts, sc.tris)
    # the caller's own device buffers
    bufs = dict(nodes=torch.from_numpy(cn.view(np.int32).copy()).cuda(),
                refs=torch.from_numpy(cr.view(np.int32).copy()).cuda(),
                rec=torch.from_numpy(rec).cuda(),
                rgba=torch.zeros(W * H, dtype=torch.int32, device="cuda"))
    yield sc, ctx, bufs
    ctx.close()


def _call(hk, sc, box, bufs, variant, w=W, h=H, rgba=None):
    import torch
    from hulktracer_b200._lib import ptr
    L = hk._lib.load()
    cam = np.ascontiguousarray(sc.camera, np.float32).ravel()
    lights = np.ascontiguousarray(sc.lights, np.float32)
    out = bufs["rgba"] if rgba is None else rgba
    return L.hk_render_noalloc(C.c_void_p(bufs["nodes"].data_ptr()), C.c_void_p(bufs["refs"].data_ptr()),
                               C.c_void_p(bufs["rec"].data_ptr()), sc.ntris, ptr(box), ptr(cam), ptr(lights),
                               lights.shape[0], w, h, variant, C.c_void_p(out.data_ptr()),
                               C.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("vname", VARIANTS)
def test_render_noalloc_matches_render(hk, setup, vname):
    import torch
    sc, ctx, bufs = setup
    variant = hk.VARIANTS[vname]
    expected = ctx.render(sc.camera, sc.lights, W, H, variant)
    box = ctx.get_box()
    torch.cuda.synchronize()
    for call in range(2):
        bufs["rgba"].fill_(-1)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        st = _call(hk, sc, box, bufs, variant)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert st == 0, "call %d returned %d" % (call, st)
        if call == 1:
            assert free1 == free0, "the second call changed free device memory by %d bytes" % (free0 - free1)
        img = bufs["rgba"].cpu().numpy().view(np.uint32)
        a = img.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
        b = expected.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
        assert np.abs(a - b).max() <= 1
        assert np.array_equal(img, expected)


def test_render_noalloc_refusals(hk, setup):
    import torch
    sc, ctx, bufs = setup
    box = ctx.get_box()
    # ROPES needs cells and ropes the call does not take
    assert _call(hk, sc, box, bufs, hk.ROPES) == 4   # HK_E_ILLEGAL_INPUT
    # a frame needing more scratch than the fixed array is refused up front
    big = torch.zeros(2048 * 2048, dtype=torch.int32, device="cuda")
    assert _call(hk, sc, box, bufs, hk.SHORTSTACK, 2048, 2048, big) == 18   # HK_E_CAPACITY
    assert int(big.abs().sum()) == 0
