"""Ray-tile sharding of one frame on the GPU: bands of rows rendered with
hk_render_rows_device (as the ranks of a multi-GPU job render them) put
together equal hk_render's whole frame pixel for pixel, for every shading
mode and for bands that do and do not keep whole 8x4 ray tiles."""
import os

import numpy as np
import pytest

from hulktracer_b200.shard import rows_for_rank

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("world", [1, 2, 3, 5])
@pytest.mark.parametrize("variant,shade", [("ropes", 0), ("shortstack", 0), ("fullstack", 1), ("ropes", 2)])
def test_row_bands_equal_whole_frame(hk, world, variant, shade):
    import torch
    g = dict(np.load(os.path.join(GOLDEN, "small24k.npz")))
    W, H = 96, 70
    c = hk.Context()
    c.upload(g["verts"], g["tris"])
    c.set_box(g["box"])
    c.precompute()
    c.build()
    if shade == hk.SHADE_MIRROR:
        nt = g["tris"].shape[0]
        c.set_mirrors((np.arange(nt) % 3 == 0).astype(np.uint8))
    v = hk.VARIANTS[variant]
    full = c.render(g["camera"], g["lights"], W, H, v, shade)
    parts = []
    for r in range(world):
        y0, y1 = rows_for_rank(H, r, world)
        d = torch.zeros(W * (y1 - y0), dtype=torch.int32, device="cuda")
        c.render_rows_device(g["camera"], g["lights"], W, H, y0, y1, d.data_ptr(), v, shade)
        c.synchronize()
        parts.append(d.cpu().numpy().view(np.uint32))
    img = np.concatenate(parts)
    assert np.array_equal(img, full)
    assert (full != 0).sum() > 1000
    c.close()
