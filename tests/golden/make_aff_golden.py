"""Write the synthetic AFF scene of ``aff/`` and its golden outputs.

The scene is generated here from a seed (it is not one of the BART scenes): a
hierarchy of static ("xs") and keyframed ("x" + "k") transforms over triangle
meshes, with includes, a detail level, every command the reference parses and
drops, a "camera" animation, rotation keys whose quaternions flip sign between
neighbours (the reference rewrites such keys), Kochanek-Bartels tension /
continuity / bias values away from zero, a duplicated animation name (the first
one wins), an animated transform without keyframes, and one triangle index above
65535 (the reference keeps indices in 16 bits).

The golden outputs come from the reference itself: its AFFParser,
AFFTransformVisitor, BoundingBoxVisitor and updateCamera compiled from its own
sources by ``oracle/build_ref.py`` into ``oracle/_ref`` (``oracle.oracle.
ReferenceAff``). ``aff_golden.npz`` holds the triangles, lights, view
parameters, and the transformed vertices, scene box and CameraPos at the times
in ``times``.

Usage: ``python tests/golden/make_aff_golden.py`` (needs ``oracle/_ref``).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

AFF_DIR = os.path.join(HERE, "aff")
MAIN = os.path.join(AFF_DIR, "scene.aff")
GOLDEN = os.path.join(HERE, "aff_golden.npz")
# frames 0, 1, 7, 59 (tick 60) of the reference's fixed-tick clock, times
# inside and past the key ranges, and one before them (clamped)
TIMES = np.array([0.0, 0.1, 0.7, 6.0, 2.45, 4.9, 9.5, -1.0], np.float32)


def _mesh(rng, nv, nt, center, size, normals=False, tex=False, wrap=False):
    v = center + rng.normal(size=(nv, 3)) * size
    out = ["m", " vertices %d" % nv]
    out += ["  %.6g %.6g %.6g" % tuple(p) for p in v]
    if normals:
        n = rng.normal(size=(nv, 3))
        out.append(" normals %d" % nv)
        out += ["  %.6g %.6g %.6g" % tuple(p) for p in n]
    if tex:
        out.append(" texturecoords %d tex.ppm" % nv)
        out += ["  %.4g %.4g" % tuple(p) for p in rng.uniform(size=(nv, 2))]
    out.append(" triangles %d" % nt)
    for k in range(nt):
        t = rng.choice(nv, 3, replace=False)
        if wrap and k == 0:
            t[1] += 65536   # stored in 16 bits by the reference: the same vertex
        row = "  %d %d %d" % tuple(t)
        if normals:
            row += "  %d %d %d" % tuple(t % 65536)
        if tex:
            row += "  %d %d %d" % tuple(t % 65536)
        out.append(row)
    return "\n".join(out) + "\n"


def _pos_keys(rng, kind, n, t0, t1, base, amp):
    ts = np.linspace(t0, t1, n)
    rows = ["  %s %d" % (kind, n)]
    for t in ts:
        p = base + rng.normal(size=3) * amp
        tcb = rng.uniform(-0.6, 0.6, size=3)
        rows.append("   %.4g  %.6g %.6g %.6g  %.3g %.3g %.3g" % ((t,) + tuple(p) + tuple(tcb)))
    return "\n".join(rows)


def _rot_keys(rng, n, t0, t1, flips=True):
    ts = np.linspace(t0, t1, n)
    rows = ["  rot %d" % n]
    # angles that wander past 180 degrees so neighbouring quaternions flip
    angles = np.cumsum(rng.uniform(60, 200, size=n)) if flips else rng.uniform(-90, 90, size=n)
    for t, a in zip(ts, angles):
        ax = rng.normal(size=3)
        if rng.uniform() < 0.7:
            ax /= np.linalg.norm(ax)        # mostly unit axes; the rest are used as given
        tcb = rng.uniform(-0.5, 0.5, size=3)
        rows.append("   %.4g  %.6g %.6g %.6g  %.5g  %.3g %.3g %.3g" % ((t,) + tuple(ax) + (a,) + tuple(tcb)))
    return "\n".join(rows)


def write_scene(seed=2024):
    rng = np.random.default_rng(seed)
    os.makedirs(AFF_DIR, exist_ok=True)
    main = []
    main.append("# synthetic scene for the AFF ingest tests (generated by make_aff_golden.py)")
    main.append("% second comment form")
    main.append("v\nfrom 3.5 2.0 9.0\nat 0 0.5 0\nup 0 1 0\nangle 40\nhither 0.01\nresolution 320 200")
    main.append("b 0.1 0.2 0.3\nam 0.5 0.5 0.5")
    main.append("l 10 20 30\nl -5 8 2 0.4 0.5 0.6\nla sun 0 50 0 1 1 0.9\n")
    main.append("a 0 10 100")
    main.append("f 0.8 0.2 0.1 0.7 0.3 20 0 1")
    main.append("fm 0.1 0.1 0.1  0.5 0.5 0.5  0.9 0.9 0.9  30 0 1.5")
    main.append("s 1 2 3 0.5\nc 0 0 0 1 0 1 0 0.5")
    main.append("p 3\n0 0 0\n1 0 0\n0 1 0\npp 3\n0 0 0 0 0 1\n1 0 0 0 0 1\n0 1 0 0 0 1")
    main.append("tt tex.ppm\n0 0 0 0 0\n1 0 0 1 0\n0 1 0 0 1")
    main.append("ttp tex.ppm\n0 0 0 0 0 1 0 0\n1 0 0 0 0 1 1 0\n0 1 0 0 0 1 0 1")
    main.append("tpa 2\n0.0\n0 0 0 0 0 1\n1 0 0 0 0 1\n0 1 0 0 0 1\n1.0\n0 0 1 0 0 1\n1 0 1 0 0 1\n0 1 1 0 0 1")
    main.append("d 1")
    main.append("i 0 ground.aff")
    main.append("i 2 not_included.aff")
    main.append("xs 2 1 0.5  0.3 0.9 0.1 35  1 -2 0.5\n{")
    main.append(_mesh(rng, 120, 200, np.array([0, 1, 0]), 0.7, normals=True))
    main.append("x spin\n{\n xs 1 1 1  0 1 0 90  0 1 0\n {\n  i 1 arm.aff\n }\n}")
    main.append("}")
    main.append("x bounce\n{")
    main.append(_mesh(rng, 150, 260, np.array([-2, 0, 1]), 0.5, normals=True, tex=True, wrap=True))
    main.append("}")
    main.append("x still\n{")
    main.append(_mesh(rng, 80, 120, np.array([2, 0, -1]), 0.4))
    main.append("}")
    main.append("k spin\n{")
    main.append(_rot_keys(rng, 7, -0.5, 5.5))
    main.append(_pos_keys(rng, "transl", 5, -0.5, 4.5, np.zeros(3), 0.8))
    main.append("}")
    main.append("k bounce\n{")
    main.append(_pos_keys(rng, "transl", 6, -1.0, 6.0, np.array([0, 1, 0]), 1.0))
    main.append(_pos_keys(rng, "scale", 5, -0.5, 7.5, np.ones(3), 0.3))
    main.append(_rot_keys(rng, 4, 0.0, 3.0, flips=False))
    main.append("  visibility 2\n   0.5 0\n   2.0 1")
    main.append("}")
    main.append("k bounce\n{")      # a second animation of that name: never used
    main.append(_pos_keys(rng, "transl", 4, 0.0, 3.0, np.array([9, 9, 9]), 1.0))
    main.append("}")
    main.append("k camera\n{")
    main.append(_pos_keys(rng, "transl", 5, -1.0, 10.0, np.array([0, 1, 8]), 1.5))
    main.append(_rot_keys(rng, 5, -1.0, 10.0, flips=False))
    main.append("}")
    with open(MAIN, "w") as f:
        f.write("\n".join(main) + "\n")
    with open(os.path.join(AFF_DIR, "ground.aff"), "w") as f:
        f.write("# ground plane, under no transform\n")
        f.write("m\n vertices 4\n  -10 -1 -10\n  10 -1 -10\n  10 -1 10\n  -10 -1 10\n")
        f.write(" triangles 2\n  0 1 2\n  0 2 3\n")
    with open(os.path.join(AFF_DIR, "arm.aff"), "w") as f:
        f.write("% arm: a keyframed transform inside an included file\n")
        f.write(_mesh(rng, 90, 140, np.array([0, 2, 0]), 0.3, tex=True))
        f.write("x elbow\n{\n")
        f.write(_mesh(rng, 60, 90, np.array([0, 3, 0]), 0.25))
        f.write("}\n")
        f.write("k elbow\n{\n")
        f.write(_rot_keys(rng, 6, -0.2, 4.8) + "\n")
        f.write(_pos_keys(rng, "scale", 4, 0.0, 4.0, np.ones(3), 0.2) + "\n")
        f.write("}\n")


def main():
    from oracle.oracle import ReferenceAff
    write_scene()
    ref = ReferenceAff(MAIN)
    out = {"times": TIMES, "tris": ref.tris(), "lights": ref.lights(),
           "view": np.array([ref.fov, ref.res[0], ref.res[1], ref.aspect], np.float32)}
    verts, boxes, cams = [], [], []
    for t in TIMES:
        v, b = ref.frame(float(t))
        verts.append(v)
        boxes.append(b)
        cams.append(ref.camera(float(t)))
    out["verts"] = np.stack(verts)
    out["boxes"] = np.stack(boxes)
    out["cameras"] = np.stack(cams)
    np.savez_compressed(GOLDEN, **out)
    print("%s: %d vertices, %d triangles, %d times" % (GOLDEN, ref.nv, ref.nt, len(TIMES)))


if __name__ == "__main__":
    main()
