"""OBJ ingest (hk_obj_parse / hk_scene_load_obj): the reference OBJ loader's
token rules on a generated file, on the reference's own teapot when its
sources are at hand, and a GPU build + trace of a loaded mesh."""
import os

import numpy as np
import pytest

from hulktracer_b200 import scenes
from hulktracer_b200.engine import obj_parse
from hulktracer_b200._lib import HkError

from oracle.build_ref import reference_root

TEAPOT = os.path.join(reference_root(), "OBJLoader/Models/teapot/teapot.obj")


def write_obj(path, verts, tris, quads=()):
    with open(path, "w") as f:
        f.write("# generated mesh\n# with comments\no mesh\ng group1\nmtllib none.mtl\nusemtl red\n")
        for v in verts:
            f.write("v %.9g %.9g %.9g\n" % tuple(v[:3]))
            f.write("vn 0 1 0\nvt 0.5 0.5\n")
        for t in tris:
            f.write("f %d/%d/%d %d//%d %d\n" % (t[0] + 1, t[0] + 1, t[0] + 1, t[1] + 1, t[1] + 1, t[2] + 1))
        for q in quads:
            f.write("f %d %d %d %d\n" % tuple(x + 1 for x in q))


def test_parse_generated(tmp_path):
    sc = scenes.random_soup(500, seed=3)
    V = sc.verts.astype(np.float32)
    T = sc.tris
    p = str(tmp_path / "m.obj")
    # a quad face: the reference reads its first three tokens only
    write_obj(p, V, T[:, :3], quads=[(0, 1, 2, 3)])
    v, t = obj_parse(p)
    assert v.shape == (V.shape[0], 4) and np.all(v[:, 3] == 1.0)
    assert np.array_equal(v[:, :3], V[:, :3])
    assert t.shape[0] == T.shape[0] + 1
    assert np.array_equal(t[:-1, :3], T[:, :3]) and np.array_equal(t[-1, :3], [0, 1, 2])
    assert np.all(t[:, 3] == 0)


def test_parse_rejects_bad_index(tmp_path):
    p = str(tmp_path / "bad.obj")
    with open(p, "w") as f:
        f.write("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")
    with pytest.raises(HkError):
        obj_parse(p)


@pytest.mark.skipif(not os.path.exists(TEAPOT), reason="reference sources not present")
def test_parse_reference_teapot():
    v, t = obj_parse(TEAPOT)
    lines = open(TEAPOT).read().split("\n")
    vs = np.array([[float(x) for x in l.split()[1:4]] for l in lines if l.startswith("v ")], np.float32)
    fs = np.array([[int(tok.split("/")[0]) - 1 for tok in l.split()[1:4]] for l in lines if l.startswith("f ")],
                  np.uint32)
    assert v.shape[0] == vs.shape[0] == 1461 and t.shape[0] == fs.shape[0] == 2882
    assert np.array_equal(v[:, :3], vs) and np.array_equal(t[:, :3], fs)


@pytest.mark.gpu
def test_load_obj_build_trace(hk, tmp_path):
    sc = scenes.static_small(width=64, height=64)
    p = str(tmp_path / "s.obj")
    write_obj(p, sc.verts, sc.tris[:, :3])
    c = hk.Context()
    c.load_obj(p)
    assert c.ntris == sc.ntris
    c.precompute()
    c.build()
    rays = c.camera_rays(sc.camera, 64, 64)
    b = c.trace(rays, hk.BRUTE)
    h = c.trace(rays, hk.ROPES)
    m = b["tri"] >= 0
    assert m.any() and np.array_equal(h["tri"] >= 0, m) and np.array_equal(h["t"][m], b["t"][m])
