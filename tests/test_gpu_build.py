"""GPU binned-SAH builder, per-frame transform and the frame graph against the
oracle's serial restatement of the same algorithm, through the C ABI."""
import os

import numpy as np
import pytest

from hulktracer_b200 import scenes
from oracle.oracle import NORM_IEEE, ROPES as O_ROPES, SHORTSTACK as O_SHORT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.fixture(scope="module")
def ctx(hk):
    return hk.Context()


def small_animated():
    return scenes.animated_parts(n_parts=6, width=96, height=64)


@pytest.mark.parametrize("exact_max", [0, 256, 1024])
@pytest.mark.parametrize("which", ["soup3k", "small24k", "animated6"])
def test_build_identical_to_oracle(hk, oracle, which, exact_max):
    """Binned everywhere (exact_max 0), and with the exact SAH on nodes of
    at most 256 / 1024 references (warp in registers up to 32, one CTA per
    medium node above): the GPU tree equals the oracle's, array for array."""
    ctx = hk.Context(exact_max=exact_max)
    if which == "animated6":
        sc = small_animated()
        verts, tris, box = sc.verts, sc.tris, sc.scene_box()
    else:
        g = load(which + ".npz")
        verts, tris, box = g["verts"], g["tris"], g["box"]
    ctx.upload(verts, tris)
    ctx.set_box(box)
    ctx.precompute()
    st = ctx.build()
    cn, cr = ctx.export_compact()
    on, orf = oracle.build_binned(verts, tris, box, ct=1.0, ci=1.5, max_depth=24, leaf_size=4, exact_max=exact_max)
    assert cn.shape == on.shape
    assert np.array_equal(cn, on)
    assert np.array_equal(cr, orf)
    assert st["nodes"] == on.shape[0] and st["refs"] == orf.shape[0]


@pytest.mark.parametrize("subtree_max,subtree_depth,streams", [(0, 8, 1), (16, 8, 1), (32, 0, 1), (32, 4, 1),
                                                                (0, 0, 2), (32, 8, 2)])
def test_subtree_threshold_identical_to_oracle(hk, oracle, subtree_max, subtree_depth, streams):
    """hk_config.subtree_max / subtree_depth / level_streams: no deferred
    subtrees (every node level by level), subtrees of nodes of at most 16
    references, deferral at any depth, and only in the last 4 levels; the
    large nodes decided in the small nodes' launch or on a second stream; the
    GPU tree equals the oracle's with the same rule."""
    sc = small_animated()
    verts, tris, box = sc.verts, sc.tris, sc.scene_box()
    ctx = hk.Context(subtree_max=subtree_max, subtree_depth=subtree_depth, level_streams=streams)
    ctx.upload(verts, tris)
    ctx.set_box(box)
    ctx.precompute()
    st = ctx.build()
    cn, cr = ctx.export_compact()
    on, orf = oracle.build_binned(verts, tris, box, ct=1.0, ci=1.5, max_depth=24, leaf_size=4, defer=subtree_max,
                                  defer_margin=subtree_depth)
    assert np.array_equal(cn, on) and np.array_equal(cr, orf)
    sub = ctx.subtree_counts()
    assert (sub["roots"] == 0) == (subtree_max == 0)
    assert st["nodes"] == on.shape[0]
    ctx.close()


def test_trace_on_built_tree(ctx, hk, oracle):
    g = load("small24k.npz")
    ctx.upload(g["verts"], g["tris"])
    ctx.set_box(g["box"])
    ctx.precompute()
    ctx.build()
    nodes, refs = ctx.export_tree()
    cache = ctx.export_cache()
    hits = ctx.trace(g["rays"], hk.SHORTSTACK)
    tree = oracle.make_tree(g["verts"], g["tris"], cache, nodes, refs, g["box"])
    oh, oid = oracle.trace(tree, g["rays"], O_SHORT, 6)
    assert np.array_equal(hits["tri"], oid)
    m = oid >= 0
    assert np.array_equal(hits["t"][m], oh[m, 0])
    # the same closest hits as brute force over all triangles (t exact)
    bh = ctx.trace(g["rays"], hk.BRUTE)
    assert np.array_equal(bh["tri"] >= 0, m)
    assert np.array_equal(bh["t"][m], hits["t"][m])


def test_ropes_on_built_tree(ctx, hk, oracle):
    """Ropes written by the GPU builder: the ropes traversal equals the
    oracle's ropes traversal on the same (identical) tree, and finds the same
    closest hits as the stack traversal."""
    g = load("small24k.npz")
    ctx.upload(g["verts"], g["tris"])
    ctx.set_box(g["box"])
    ctx.precompute()
    ctx.build()
    cn, cr = ctx.export_compact()
    cache = ctx.export_cache()
    hits = ctx.trace(g["rays"], hk.ROPES)
    nodes = oracle.compact_to_ref(cn)
    tree = oracle.make_tree(g["verts"], g["tris"], cache, nodes, cr, g["box"])
    tree.cnodes = np.ascontiguousarray(cn, np.uint32)
    r, b = oracle.ropes(cn, g["box"])
    tree.ropes, tree.cbox = r, b
    oh, oid = oracle.trace(tree, g["rays"], O_ROPES, 6)
    assert np.array_equal(hits["tri"], oid)
    m = oid >= 0
    assert np.array_equal(hits["t"][m], oh[m, 0])
    sh = ctx.trace(g["rays"], hk.SHORTSTACK)
    assert np.array_equal(sh["t"], hits["t"])


def test_transform_and_box(ctx, oracle):
    sc = small_animated()
    ctx.upload(sc.verts, sc.tris)
    ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    mats = scenes.part_matrices(sc, 7)
    ctx.transform(mats)
    v = ctx.get_vertices()
    o = oracle.transform(sc.rest_verts, sc.part_of_vertex, mats)
    assert np.array_equal(v.view(np.uint32), o.view(np.uint32))
    box = ctx.get_box()
    ob = oracle.scene_box(o)
    assert np.array_equal(box[:3], ob[:3]) and np.array_equal(box[4:7], ob[4:7])


def test_frame_graph_matches_oracle_pipeline(ctx, hk, oracle):
    import torch
    sc = small_animated()
    w, h = sc.width, sc.height
    ctx.upload(sc.verts, sc.tris)
    ctx.set_parts(sc.part_of_vertex, sc.part_center.shape[0])
    out = torch.zeros(w * h, dtype=torch.int32, device="cuda")
    for frame in (0, 3, 11):
        mats = scenes.part_matrices(sc, frame)
        ctx.frame(mats, sc.camera, sc.lights, w, h, out.data_ptr(), use_graph=True)
        ctx.synchronize()
        img_g = out.cpu().numpy().view(np.uint32).copy()
        ctx.frame(mats, sc.camera, sc.lights, w, h, out.data_ptr(), use_graph=False)
        ctx.synchronize()
        img_n = out.cpu().numpy().view(np.uint32).copy()
        assert np.array_equal(img_g, img_n)
        verts = oracle.transform(sc.rest_verts, sc.part_of_vertex, mats)
        box = oracle.scene_box(verts)
        cache = oracle.cache(verts, sc.tris, NORM_IEEE)
        cn, cr = oracle.build_binned(verts, sc.tris, box)
        nodes = oracle.compact_to_ref(cn)
        tree = oracle.make_tree(verts, sc.tris, cache, nodes, cr, box)
        rays = oracle.camera_rays(sc.camera, w, h, NORM_IEEE)
        oimg = oracle.render_cpu(tree, rays, w, h, sc.lights, O_SHORT, 6, NORM_IEEE)
        assert np.array_equal(img_g, oimg)


def test_tree_file_layout_and_reload(ctx, hk, tmp_path):
    """hk_tree_save_file writes the reference's dataset layout (compared with
    the oracle's restatement of saveDataSetToFile); the file reloads onto its
    scene as the same tree, and on its own (per-leaf triangles as the scene)
    traces to the same hit distances."""
    from oracle import treefile
    g = load("small24k.npz")
    ctx.upload(g["verts"], g["tris"])
    ctx.set_box(g["box"])
    ctx.import_cache(g["ref_cache"])
    ctx.import_tree(g["ref_nodes"], g["ref_refs"])
    nodes, refs = ctx.export_tree()
    f = str(tmp_path / "tree.bin")
    ctx.save_tree_file(f)
    data = open(f, "rb").read()
    want = treefile.dataset_bytes(nodes, refs, g["verts"], g["tris"])
    assert data[:len(want)] == want
    assert data[len(want):len(want) + 8] == b"HKLEAFPL"
    hits = ctx.trace(g["rays"], hk.SHORTSTACK)
    # reload onto the same scene: the same tree
    c2 = hk.Context(short_stack=6)
    c2.upload(g["verts"], g["tris"])
    c2.import_cache(g["ref_cache"])
    c2.load_tree_file(f)
    n2, r2 = c2.export_tree()
    assert np.array_equal(n2, nodes) and np.array_equal(r2, refs)
    assert np.array_equal(c2.trace(g["rays"], hk.SHORTSTACK)["tri"], hits["tri"])
    # on its own: triangle k of the new scene is leaf polygon k of the file
    c3 = hk.Context()
    c3.load_tree_file(f, load_scene=True)
    assert c3.ntris == refs.shape[0]
    h3 = c3.trace(g["rays"], hk.BRUTE)
    ctx.precompute()   # the same (IEEE) triangle records as c3's
    b = ctx.trace(g["rays"], hk.BRUTE)
    m = b["tri"] >= 0
    assert np.array_equal(h3["tri"] >= 0, m)
    assert np.array_equal(h3["t"][m], b["t"][m])
    h4 = c3.trace(g["rays"], hk.SHORTSTACK)
    assert np.array_equal(h4["t"][m], b["t"][m])


def test_frame_mirror_shading_equals_render(ctx, hk):
    """hk_frame with HK_SHADE_MIRROR (graph) equals hk_render with the same
    shading on the tree the frame built."""
    import torch
    sc = scenes.static_small(width=64, height=64)
    nt = sc.ntris
    h32 = (np.arange(nt, dtype=np.uint64) * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    mirror = (h32.astype(np.float64) / 4294967296.0 < 0.3).astype(np.uint8)
    ctx.upload(sc.verts, sc.tris)
    ctx.set_mirrors(mirror)
    ctx.set_frame_shading(hk.SHADE_MIRROR)
    try:
        out = torch.zeros(64 * 64, dtype=torch.int32, device="cuda")
        ctx.frame(None, sc.camera, sc.lights, 64, 64, out.data_ptr(), use_graph=True)
        ctx.synchronize()
        img_f = out.cpu().numpy().view(np.uint32).copy()
        img_r = ctx.render(sc.camera, sc.lights, 64, 64, hk.SHORTSTACK, hk.SHADE_MIRROR)
        assert np.array_equal(img_f, img_r)
        assert (img_r != ctx.render(sc.camera, sc.lights, 64, 64, hk.SHORTSTACK)).any()
    finally:
        ctx.set_frame_shading(hk.SHADE_CPU)


def test_capacity_guard_stops_splitting(hk):
    """A reference arena of twice the triangles: the level whose children would
    not fit stops splitting (its nodes become leaves, capacity_hit = 1) and the
    build succeeds; the tree stays within the arena and traces like brute force
    (full stack, ropes)."""
    g = load("small24k.npz")
    nt = g["tris"].shape[0]
    c = hk.Context(max_refs=2 * nt)
    c.upload(g["verts"], g["tris"])
    c.set_box(g["box"])
    c.precompute()
    st = c.build()
    assert st["capacity_hit"] == 1
    assert st["refs"] <= 2 * nt
    b = c.trace(g["rays"], hk.BRUTE)
    m = b["tri"] >= 0
    for v in (hk.FULLSTACK, hk.ROPES):
        h = c.trace(g["rays"], v)
        assert np.array_equal(h["tri"] >= 0, m)
        assert np.array_equal(h["t"][m], b["t"][m])
    c.close()
