"""AFF (BART) ingest, host side: hk_aff_* against the reference's own loader.

The golden outputs in ``golden/aff_golden.npz`` were written by the reference's
AFFParser / AFFTransformVisitor / BoundingBoxVisitor compiled from its sources
(``golden/make_aff_golden.py``); the checks here are bit-exact. The product's
matrices are applied with the oracle's restatement of SPMatrix's VectorMult
(the same operation order the device transform uses). When the reference's
BART scenes are at hand, the robots, kitchen and museum scenes are compared
with the compiled reference frame by frame.
"""
import os

import numpy as np
import pytest

from hulktracer_b200.engine import Aff, fixed_tick_time
from hulktracer_b200._lib import HkError
from oracle.build_ref import reference_root
from oracle.oracle import Oracle, ReferenceAff

HERE = os.path.dirname(os.path.abspath(__file__))
SCENE = os.path.join(HERE, "golden", "aff", "scene.aff")
GOLDEN = os.path.join(HERE, "golden", "aff_golden.npz")
BART = os.path.join(reference_root(), "BartLoader")
HK_E_FILE_OPEN, HK_E_ILLEGAL_INPUT = 2, 4


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


@pytest.fixture(scope="module")
def aff():
    a = Aff(SCENE)
    yield a
    a.close()


def test_structure(aff, golden):
    i = aff.info
    assert (i["nv"], i["nt"]) == (golden["verts"].shape[1], golden["tris"].shape[0]) == (504, 812)
    # ground, the mesh under "xs", arm and elbow (included), bounce, still
    assert i["nmeshes"] == 6 and i["ndynamic"] == 4
    assert i["ntransforms"] == 6 and i["nanimations"] == 5 and i["nlights"] == 3
    assert i["has_view"] and i["fov_deg"] == golden["view"][0]
    assert (i["resx"], i["resy"]) == (int(golden["view"][1]), int(golden["view"][2])) == (320, 200)
    assert i["has_anim_params"] and (i["anim_start"], i["anim_end"], i["anim_frames"]) == (0.0, 10.0, 100)
    assert i["has_camera_anim"]
    assert np.allclose(i["from"], [3.5, 2.0, 9.0]) and np.allclose(i["up"], [0, 1, 0])


def test_triangles_lights(aff, golden):
    v, t, part = aff.geometry()
    assert np.array_equal(t, golden["tris"])
    assert np.all(v[:, 3] == 1.0)
    # parts are the meshes in file order, each a contiguous vertex range
    assert np.all(np.diff(part.astype(np.int64)) >= 0) and part[-1] == aff.info["nmeshes"] - 1
    assert np.array_equal(bits(aff.lights()), bits(golden["lights"]))


def test_frames_bit_exact(aff, golden, oracle):
    rest, _, part = aff.geometry()
    for k, t in enumerate(golden["times"]):
        v = oracle.transform(rest, part, aff.part_matrices(float(t)))
        assert np.array_equal(bits(v), bits(golden["verts"][k])), "vertices differ at t=%g" % t
        assert np.array_equal(bits(oracle.scene_box(v)), bits(golden["boxes"][k]))
        assert np.array_equal(bits(aff.camera(float(t))), bits(golden["cameras"][k])), "camera at t=%g" % t


def test_static_parts_do_not_move(aff):
    # the ground is under no transform: identity at every time
    m0 = aff.part_matrices(0.0)
    for t in (0.3, 7.0):
        m = aff.part_matrices(t)
        assert np.array_equal(m[0], m0[0])
        assert np.array_equal(m[0], [1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0])
    assert not np.array_equal(aff.part_matrices(0.3)[4], aff.part_matrices(2.0)[4])


def test_fixed_tick_time():
    # GLWindow::display's --fixedTic clock: tick / 10, skipping ticks 59 and 421
    t = [fixed_tick_time(f) for f in range(62)]
    assert t[:3] == [0.0, np.float32(0.1), np.float32(0.2)]
    assert t[58] == np.float32(5.8) and t[59] == np.float32(6.0) and t[60] == np.float32(6.1)
    assert fixed_tick_time(419) == np.float32(42.0) and fixed_tick_time(420) == np.float32(42.2)


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


MESH = "m\n vertices 3\n 0 0 0\n 1 0 0\n 0 1 0\n triangles 1\n 0 1 2\n"


@pytest.mark.parametrize("text,needle", [
    ("q 1 2 3\n", "unknown command"),
    ("}\n", "without an open transform"),
    ("x a\n{\n" + MESH, "not closed"),
    ("k a\n{\n transl 3\n 0 0 0 0 0 0 0\n 1 0 0 0 0 0 0\n 2 0 0 0 0 0 0\n}\n", "at least 4"),
    ("k a\n{\n wobble 4\n}\n", "keyframe type"),
    ("m\n vertices 3\n 0 0 0\n 1 0 0\n 0 1 0\n triangles 1\n 0 1 3\n", "outside the mesh"),
    ("m\n vertices 3\n 0 0 0\n 1 0 0\n", "mesh vertex"),
    ("m\n vertices 3\n 0 0 0\n 1 0 0\n 0 1 0\n faces 1\n 0 1 2\n", "'triangles' expected"),
    ("v\nfrom 0 0 0\nat 0 0 1\nangle 40\n", "viewpoint up"),
    ("xs 1 1 1 0 1 0\n{\n}\n", "static transform"),
    ("l 1 2 3 0.5\n", "light color"),
    ("tz\n", "valid t codes"),
])
def test_syntax_errors(tmp_path, text, needle):
    p = _write(tmp_path, "bad.aff", text)
    with pytest.raises(HkError) as e:
        Aff(p)
    assert e.value.status == HK_E_ILLEGAL_INPUT and needle in str(e.value)


def test_missing_files(tmp_path):
    with pytest.raises(HkError) as e:
        Aff(str(tmp_path / "nope.aff"))
    assert e.value.status == HK_E_FILE_OPEN
    p = _write(tmp_path, "main.aff", MESH + "i 0 missing_part.aff\n")
    with pytest.raises(HkError) as e:
        Aff(p)
    assert e.value.status == HK_E_FILE_OPEN and "missing_part.aff" in str(e.value)
    # above the detail level an include is skipped without being opened
    p = _write(tmp_path, "main2.aff", "d 1\n" + MESH + "i 2 missing_part.aff\n")
    a = Aff(p)
    assert a.info["nt"] == 1


def test_index_kept_in_16_bits(tmp_path):
    p = _write(tmp_path, "w.aff", "m\n vertices 3\n 0 0 0\n 1 0 0\n 0 1 0\n triangles 1\n 0 65537 2\n")
    _, t, _ = Aff(p).geometry()
    assert np.array_equal(t[0], [0, 1, 2, 0])


def test_defaults_without_view(tmp_path):
    a = Aff(_write(tmp_path, "plain.aff", MESH))
    i = a.info
    # the reference Scene's defaults (HulkEngine/src/Scene.cpp:21-27)
    assert not i["has_view"] and i["fov_deg"] == 45.0 and (i["resx"], i["resy"]) == (800, 600)
    assert not i["has_camera_anim"] and i["nlights"] == 0
    cam = a.camera(3.0)
    assert np.array_equal(cam[:4], [0, 0, 0, 0])          # eye at the origin
    assert cam[12 + 2] == -1.0                             # looking down -z


BART_SCENES = ["robots/Robot.aff", "kitchen/kitchen.aff", "museum/museum3.aff", "museum/museum6.aff"]


@pytest.mark.skipif(not (os.path.isdir(BART) and os.path.exists(
    os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libhulkref.so"))),
    reason="reference BART scenes or the compiled reference not present")
@pytest.mark.parametrize("scene", BART_SCENES)
def test_bart_scene_against_reference(scene, oracle):
    path = os.path.join(BART, scene)
    a = Aff(path)
    r = ReferenceAff(path)
    assert (a.info["nv"], a.info["nt"]) == (r.nv, r.nt)
    rest, tris, part = a.geometry()
    assert np.array_equal(tris, r.tris())
    assert np.array_equal(bits(a.lights()), bits(r.lights()))
    assert a.info["fov_deg"] == r.fov and (a.info["resx"], a.info["resy"]) == r.res
    for frame in (0, 1, 30, 59, 137, 400):
        t = fixed_tick_time(frame)
        ref_v, ref_box = r.frame(t)
        v = oracle.transform(rest, part, a.part_matrices(t))
        assert np.array_equal(bits(v), bits(ref_v)), "%s frame %d" % (scene, frame)
        assert np.array_equal(bits(oracle.scene_box(v)), bits(ref_box))
        assert np.array_equal(bits(a.camera(t)), bits(r.camera(t)))
    r.close()
    a.close()


@pytest.mark.skipif(not os.path.isdir(BART), reason="reference BART scenes not present")
def test_bart_museum_missing_blob():
    # animart7.aff is not in the reference checkout; the reference exits, here
    # the open fails with a status
    with pytest.raises(HkError) as e:
        Aff(os.path.join(BART, "museum", "museum7.aff"))
    assert e.value.status == HK_E_FILE_OPEN and "animart7.aff" in str(e.value)


def test_scene_from_aff(aff, oracle):
    """The bench's AFF workload: one part per mesh, the file's lights and
    resolution, matrices and camera on the fixed-tick clock."""
    from hulktracer_b200 import scenes
    sc = scenes.from_aff(SCENE)
    assert sc.ntris == 812 and (sc.width, sc.height) == (320, 200)
    assert sc.part_center.shape[0] == aff.info["nmeshes"] and sc.lights.shape == (3, 8)
    t = fixed_tick_time(7)
    assert np.array_equal(scenes.part_matrices(sc, 7), aff.part_matrices(t))
    assert np.array_equal(scenes.frame_camera(sc, 7).ravel(), aff.camera(t))
    assert not np.array_equal(scenes.frame_camera(sc, 0), scenes.frame_camera(sc, 30))
