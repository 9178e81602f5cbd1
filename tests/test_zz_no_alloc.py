"""hk_render_noalloc -- rendering for callers that cannot let the library
allocate device memory (a host with its own pooled allocator, code running
while a graph capture is open elsewhere, a fixed memory budget). The caller
owns the tree, triangle records and image buffers; the pipeline's scratch is
one static device array inside the library.

The test renders twice in a row through the C ABI from caller-held buffers and
compares each image with hk_render, the allocating entry point, on the same
tree (pixels must be equal; the tolerance used elsewhere is 1/255). It also
checks that a frame too large for the fixed scratch is refused.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it passes alone and after the others."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _records(cache, verts, tris):
    rec = np.zeros((cache.shape[0], 16), np.float32)
    p1 = verts[tris[:, 0], :3]
    rec[:, 0:3], rec[:, 3] = cache[:, 0:3], cache[:, 12]
    rec[:, 4:7], rec[:, 7] = p1, cache[:, 13]
    rec[:, 8:11], rec[:, 11] = cache[:, 4:7], cache[:, 14]
    rec[:, 12:15], rec[:, 15] = cache[:, 8:11], cache[:, 15]
    return rec


def test_render_noalloc_matches_render(hk):
    import torch
    from hulktracer_b200 import scenes
    from hulktracer_b200._lib import ptr

    W, H = 256, 192
    sc = scenes.static_small(width=W, height=H)
    ctx = hk.Context()
    ctx.upload(sc.verts, sc.tris)
    ctx.precompute()
    ctx.build()
    expected = ctx.render(sc.camera, sc.lights, W, H, hk.SHORTSTACK)
    cn, cr = ctx.export_compact()
    rec = _records(ctx.export_cache(), sc.verts, sc.tris)
    box = ctx.get_box()
    # the caller's own device buffers
    d_nodes = torch.from_numpy(cn.view(np.int32).copy()).cuda()
    d_refs = torch.from_numpy(cr.view(np.int32).copy()).cuda()
    d_rec = torch.from_numpy(rec).cuda()
    d_rgba = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    cam = np.ascontiguousarray(sc.camera, np.float32).ravel()
    lights = np.ascontiguousarray(sc.lights, np.float32)
    L = hk._lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    for call in range(2):
        d_rgba.fill_(-1)
        torch.cuda.synchronize()
        st = L.hk_render_noalloc(C.c_void_p(d_nodes.data_ptr()), C.c_void_p(d_refs.data_ptr()),
                                 C.c_void_p(d_rec.data_ptr()), sc.ntris, ptr(box), ptr(cam), ptr(lights),
                                 lights.shape[0], W, H, hk.SHORTSTACK, C.c_void_p(d_rgba.data_ptr()),
                                 C.c_void_p(stream))
        assert st == 0, "call %d returned %d" % (call, st)
        img = d_rgba.cpu().numpy().view(np.uint32)
        a = img.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
        b = expected.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
        assert np.abs(a - b).max() <= 1
        assert np.array_equal(img, expected)
    # a frame needing more scratch than the fixed array is refused up front
    big = torch.zeros(2048 * 2048, dtype=torch.int32, device="cuda")
    st = L.hk_render_noalloc(C.c_void_p(d_nodes.data_ptr()), C.c_void_p(d_refs.data_ptr()),
                             C.c_void_p(d_rec.data_ptr()), sc.ntris, ptr(box), ptr(cam), ptr(lights),
                             lights.shape[0], 2048, 2048, hk.SHORTSTACK, C.c_void_p(big.data_ptr()),
                             C.c_void_p(stream))
    assert st == 18  # HK_E_CAPACITY
    assert int(big.abs().sum()) == 0
    ctx.close()
