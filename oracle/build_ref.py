#!/usr/bin/env python3
"""Compile the reference HulkEngine CPU KD-tree path and BART loader into ``oracle/_ref``.

Test infrastructure only: the product never links or loads what this builds.

The reference is MSVC code. Its KD build + CPU traversal sources compile with
g++ once a small Win32 shim (``oracle/refshim/windows.h``) is force-included
and a few MSVC-only constructs are patched in *generated copies* that live in
``oracle/_ref/gen*`` (git-ignored; nothing from the reference is committed):

* ``HulkEngine/public/Stack.hpp``: ``toher`` typo in the iterator copy
  constructor (line 46), non-const copy constructor, unqualified ``min`` (163).
* ``HulkEngine/public/SseUtils.hpp``: ``__m128`` operator overloads that GCC
  vector types already define (70-96, 142-148, 158-160) and the function named
  ``not`` (150).
* ``HulkEngine/public/FrameBuffer.hpp``: MSVC ``m128i_i32[k]`` (212-214).
* ``HulkEngine/public/Visitor.hpp:68``, ``HulkEngine/src/DeleteVisitor.cpp:29``:
  a temporary bound to a non-const reference.
* ``HulkEngine/src/KDTreeCPU.cpp``: instrumented copy that records the winning
  polygon index in ``testNodePolygons`` (the reference has no hit ID) and counts
  node visits / triangle tests in ``searchKDTreeStackless``.

The BART loader (``BartLoader/src``: AFFParser, AFFTransformVisitor and the
keyframe code) is compiled into both libraries unchanged except for two
process-wide statics that the driver re-arms per scene: the detail level
(``AFFParser.cpp:23``) and the first-traversal flag of the transform visitor
(``AFFTransformVisitor.cpp:134-140``).

Two libraries are produced:

* ``libhulkref.so``      -- reference constants (Ct 1, Ci 5, depth 20, leaf < 10,
  every 5th triangle sampled).
* ``libhulkref_cfg.so``  -- the same code with the constants of the benchmark
  scenes (Ct 1, Ci 1.5, depth 24, leaf <= 4, no subsampling), for SAH-cost
  comparisons against the GPU builder.

Usage: ``python oracle/build_ref.py [--reference DIR]``. Where the reference
sources are is decided here and nowhere else (``reference_root()``): ``--reference``,
else ``$HK_REFERENCE_ROOT``, else the directory the reference checkout is
mounted at on the build machine (``DEFAULT_REFERENCE``). When none holds the
sources, nothing is built and the checkers that need the compiled reference
skip.
"""
import argparse
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
DEFAULT_REFERENCE = "/root/reference"


def reference_root() -> str:
    """The reference checkout this recipe compiles from (it may not exist)."""
    return os.environ.get("HK_REFERENCE_ROOT", DEFAULT_REFERENCE)

SOURCES = [
    "src/KDTreeSAH.cpp", "src/SPMatrix.cpp", "src/SseUtils.cpp", "src/Settings.cpp",
    "src/Statistics.cpp", "src/Scene.cpp", "src/Node.cpp", "src/Intersectable.cpp",
    "src/BoundingBoxVisitor.cpp", "src/StaticMeshNode.cpp", "src/RigidTransform.cpp",
]

CXXFLAGS = ["-std=c++14", "-O2", "-DPRODUCTION", "-ffp-contract=off", "-fpermissive",
            "-msse4.1", "-fno-operator-names", "-fPIC", "-fopenmp", "-w"]


def _read(path):
    with open(path, "r", encoding="latin-1") as f:
        return f.read().replace("\r\n", "\n")


def _write(path, text):
    with open(path, "w", encoding="latin-1") as f:
        f.write(text)


def _replace(text, old, new, count=1, what=""):
    n = text.count(old)
    if n < count:
        raise RuntimeError("patch anchor not found (%s): %r" % (what, old))
    return text.replace(old, new)


def _patch_stack(src):
    t = _read(src)
    t = _replace(t, "iterator(iterator & other): m_vec(toher.m_vec)",
                 "iterator(const iterator & other): m_vec(other.m_vec)", what="Stack iterator")
    t = _replace(t, "i < min(m_size,newSize)", "i < std::min(m_size,newSize)", what="Stack min")
    t = t.replace('#include "util.hpp"', '#include <algorithm>\n#include <cstring>\n#include "util.hpp"', 1)
    return t


def _patch_sseutils(src):
    t = _read(src)
    # drop every free operator overload taking __m128 / __m128i (GCC provides them)
    t, n = re.subn(r"inline [^\n{]*operator[^\n{]*__m128[^\n{]*\{[^{}]*\};?", "", t)
    if n == 0:
        raise RuntimeError("patch anchor not found (SseUtils operators)")
    t = _replace(t, "inline __m128 not(__m128 a)", "inline __m128 not_(__m128 a)", what="SseUtils not")
    return t


def _patch_framebuffer(src):
    t = _read(src)
    for k in range(3):
        t = _replace(t, "intVaule.m128i_i32[%d]" % k, "_mm_extract_epi32(intVaule,%d)" % k,
                     what="FrameBuffer m128i")
    return t


def _patch_end_loop(src):
    t = _read(src)
    t = _replace(t, "while (it != node->end())",
                 "Node::SonIterator hk_end_it = node->end();\n\twhile (it != hk_end_it)",
                 what="SonIterator end")
    return t


def _patch_kdtree_cpp(src, cfg):
    t = _read(src)
    head = ("#include <cstdint>\n"
            "extern thread_local unsigned hkref_last_poly;\n"
            "extern thread_local unsigned long long hkref_nodes;\n"
            "extern thread_local unsigned long long hkref_tests;\n")
    t = head + t
    # winning polygon index (KDTreeCPU.cpp:273-279)
    t = _replace(t, "\t\t\t\thit.normal = hitPos.normal;\n",
                 "\t\t\t\thit.normal = hitPos.normal;\n\t\t\t\thkref_last_poly = polyIndex;\n",
                 what="testNodePolygons winner")
    # triangle tests (KDTreeCPU.cpp:261-271 loop body)
    t = _replace(t, "\t\tunsigned int polyIndex  = m_leafPolygons[i];\n",
                 "\t\tunsigned int polyIndex  = m_leafPolygons[i];\n\t\thkref_tests++;\n",
                 what="testNodePolygons count")
    # node visits in the short-stack search (KDTreeCPU.cpp:396-437)
    t = _replace(t, "\t    while (pNode->m_flags & EPlaneAxis::e_junction) //if this is a leaf node\n\t    {\n",
                 "\t    while (pNode->m_flags & EPlaneAxis::e_junction) //if this is a leaf node\n\t    {\n\t\t\thkref_nodes++;\n",
                 what="stackless junction count")
    t = _replace(t, "\t\tif  (pNode->m_flags & EPlaneAxis::e_leaf)\n\t\t{\n",
                 "\t\tif  (pNode->m_flags & EPlaneAxis::e_leaf)\n\t\t{\n\t\t\thkref_nodes++;\n",
                 what="stackless leaf count")
    if cfg:
        t = _replace(t, "KDTreeCPU::c_intersectionCost = 5.0f;", "KDTreeCPU::c_intersectionCost = 1.5f;",
                     what="Ci")
    return t


def _patch_cfg_structs(src):
    return _replace(_read(src), "#define c_maxKDTreeDepth 20", "#define c_maxKDTreeDepth 24", what="depth")


def _patch_cfg_kdtree_hpp(src):
    return _replace(_read(src), "static const uint c_reductionFactor = 5;",
                    "static const uint c_reductionFactor = 1;", what="reduction")


def _patch_cfg_sah(src):
    t = _read(src)
    # leaf test of the NlogN builder (KDTreeSAH.cpp:316-317) and the per-node
    # re-sort builder (KDTreeSAH.cpp:38-39)
    t = _replace(t, "( itrData.polygonList.size() < 10 ))", "( itrData.polygonList.size() < 5 ))",
                 count=2, what="leaf size")
    return t


BART_SOURCES = ["animation.cpp", "kbsplpos.cpp", "kbsplrot.cpp", "quat.cpp"]


def _patch_aff_parser(src):
    # gDetailLevel is a file static that outlives one load; the driver loads
    # many scenes in one process, so every top-level parse starts at level 0
    # as a fresh process does (AFFParser.cpp:23,1462-1467)
    t = _read(src)
    return _replace(t, "\tm_relPath = relPath;\n", "\tgDetailLevel = 0;\n\tm_relPath = relPath;\n",
                    what="AFFParser detail level")


def _patch_aff_visitor(src):
    # traverseBegin transforms static meshes on the first traversal of the
    # process only (a function static, AFFTransformVisitor.cpp:134-140); the
    # driver re-arms it for every new visitor it creates
    t = _read(src)
    t = "extern int hkref_aff_rearm;\n" + t
    return _replace(t, "\tstatic int count = 0;\n",
                    "\tstatic int count = 0;\n\tif (hkref_aff_rearm) { count = 0; hkref_aff_rearm = 0; }\n",
                    what="AFFTransformVisitor static count")


def _make_gen(ref, gen, cfg):
    if os.path.isdir(gen):
        shutil.rmtree(gen)
    os.makedirs(gen)
    he = os.path.join(ref, "HulkEngine")
    shim = os.path.join(HERE, "refshim", "windows.h")
    shutil.copy(shim, os.path.join(gen, "windows.h"))
    shutil.copy(shim, os.path.join(gen, "Windows.h"))
    patched = {
        "Stack.hpp": _patch_stack(os.path.join(he, "public", "Stack.hpp")),
        "SseUtils.hpp": _patch_sseutils(os.path.join(he, "public", "SseUtils.hpp")),
        "FrameBuffer.hpp": _patch_framebuffer(os.path.join(he, "public", "FrameBuffer.hpp")),
        "Visitor.hpp": _patch_end_loop(os.path.join(he, "public", "Visitor.hpp")),
    }
    if cfg:
        patched["SharedStructs.hpp"] = _patch_cfg_structs(os.path.join(he, "public", "SharedStructs.hpp"))
        patched["KDTreeCPU.hpp"] = _patch_cfg_kdtree_hpp(os.path.join(he, "src", "KDTreeCPU.hpp"))
    for name, text in patched.items():
        _write(os.path.join(gen, name), text)
    # case-insensitive include aliases (MSVC resolves "scene.hpp" to Scene.hpp)
    for sub in ("public", "src"):
        d = os.path.join(he, sub)
        for name in os.listdir(d):
            if not name.endswith((".hpp", ".h")):
                continue
            target = os.path.join(gen, name) if name in patched else os.path.join(d, name)
            for alias in {name, name.lower(), name[0].lower() + name[1:]}:
                p = os.path.join(gen, alias)
                if not os.path.exists(p):
                    os.symlink(target, p)
    srcs = {
        "KDTreeCPU.cpp": _patch_kdtree_cpp(os.path.join(he, "src", "KDTreeCPU.cpp"), cfg),
        "DeleteVisitor.cpp": _patch_end_loop(os.path.join(he, "src", "DeleteVisitor.cpp")),
    }
    if cfg:
        srcs["KDTreeSAH.cpp"] = _patch_cfg_sah(os.path.join(he, "src", "KDTreeSAH.cpp"))
    bart = os.path.join(ref, "BartLoader", "src")
    srcs["AFFParser.cpp"] = _patch_aff_parser(os.path.join(bart, "AFFParser.cpp"))
    srcs["AFFTransformVisitor.cpp"] = _patch_aff_visitor(os.path.join(bart, "AFFTransformVisitor.cpp"))
    for name, text in srcs.items():
        _write(os.path.join(gen, name), text)
    return srcs


def build(ref, cfg):
    tag = "_cfg" if cfg else ""
    gen = os.path.join(OUT, "gen" + tag)
    objdir = os.path.join(OUT, "obj" + tag)
    os.makedirs(objdir, exist_ok=True)
    gen_srcs = _make_gen(ref, gen, cfg)
    he = os.path.join(ref, "HulkEngine")
    bl = os.path.join(ref, "BartLoader")
    incs = ["-I" + gen, "-I" + os.path.join(he, "public"), "-I" + os.path.join(he, "src"),
            "-I" + os.path.join(bl, "public"), "-I" + os.path.join(bl, "src")]
    pre = ["-include", os.path.join(gen, "windows.h")]
    units = [os.path.join(gen, n) for n in gen_srcs]
    units += [os.path.join(he, s) for s in SOURCES if os.path.basename(s) not in gen_srcs]
    units += [os.path.join(bl, "src", s) for s in BART_SOURCES]
    units.append(os.path.join(HERE, "ref_driver.cpp"))
    objs = []
    for u in units:
        o = os.path.join(objdir, os.path.basename(u) + ".o")
        cmd = ["g++"] + CXXFLAGS + pre + incs + ["-c", u, "-o", o]
        subprocess.check_call(cmd)
        objs.append(o)
    lib = os.path.join(OUT, "libhulkref%s.so" % tag)
    subprocess.check_call(["g++", "-shared", "-fopenmp", "-o", lib] + objs)
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_root())
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.reference, "HulkEngine")):
        print("reference sources not found at %s; nothing built" % a.reference)
        return 1
    os.makedirs(OUT, exist_ok=True)
    for cfg in (False, True):
        print(build(a.reference, cfg))
    return 0


if __name__ == "__main__":
    sys.exit(main())
