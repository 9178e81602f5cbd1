"""CUDA traversal, intersection and shading against the oracle and the
reference's golden outputs, through the C ABI (libhulkcuda.so).

Parity bar: hit triangle ids and t bit-exact (the stated tolerance for t is
1e-5 relative; the kernels reproduce the reference's arithmetic exactly, so
the tests demand equality); pixels within 1/255."""
import os

import numpy as np
import pytest

from oracle.oracle import (BRUTE as O_BRUTE, FULLSTACK as O_FULL, NORM_IEEE, RESTART as O_RESTART,
                           RESTART_EARLY as O_RESTART_EARLY, ROPES as O_ROPES, SHORTSTACK as O_SHORT)

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["soup3k.npz", "small24k.npz"]
T_RTOL = 1e-5


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.fixture(scope="module")
def ctx6(hk):
    return hk.Context(short_stack=6)


@pytest.fixture(scope="module")
def ctx5(hk):
    return hk.Context(short_stack=5)


def setup_ref_tree(ctx, g):
    ctx.upload(g["verts"], g["tris"])
    ctx.set_box(g["box"])
    ctx.import_cache(g["ref_cache"])
    ctx.import_tree(g["ref_nodes"], g["ref_refs"])


def check_hits(hits, ids, t):
    assert np.array_equal(hits["tri"], ids)
    m = ids >= 0
    assert np.array_equal(hits["t"][m], t[m])
    assert np.all(np.abs(hits["t"][m] - t[m]) <= T_RTOL * np.abs(t[m]))
    assert np.all(np.isinf(hits["t"][~m]))


@pytest.mark.parametrize("name", CASES)
def test_shortstack5_equals_reference_checkcollision(ctx5, hk, name):
    """Ring depth 5 reproduces KDTreeCPU::checkCollision on the reference tree
    and cache: hit ids and t bit-exact against the reference's own output."""
    g = load(name)
    setup_ref_tree(ctx5, g)
    for v in (hk.SHORTSTACK, hk.SMEMSTACK):
        hits = ctx5.trace(g["rays"], v)
        check_hits(hits, g["ref_ids"], g["ref_hits"][:, 0])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant,ovariant", [("fullstack", O_FULL), ("shortstack", O_SHORT),
                                              ("smemstack", O_SHORT), ("restart", O_RESTART),
                                              ("restart_early", O_RESTART_EARLY), ("brute", O_BRUTE),
                                              ("ropes", O_ROPES)])
def test_variant_bit_exact_vs_oracle(ctx6, hk, oracle, name, variant, ovariant):
    g = load(name)
    setup_ref_tree(ctx6, g)
    hits = ctx6.trace(g["rays"], hk.VARIANTS[variant])
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"],
                            with_ropes=(ovariant == O_ROPES))
    oh, oid = oracle.trace(tree, g["rays"], ovariant, 6)
    check_hits(hits, oid, oh[:, 0])


@pytest.mark.parametrize("name", CASES)
def test_counters_match_oracle(ctx5, hk, oracle, name):
    g = load(name)
    setup_ref_tree(ctx5, g)
    ctx5.set_counting(True)
    try:
        ctx5.trace(g["rays"], hk.SHORTSTACK)
        c = ctx5.counters()
    finally:
        ctx5.set_counting(False)
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"])
    _, _, oc = oracle.trace(tree, g["rays"], O_SHORT, 5, counters=True)
    assert int(c[0]) == int(oc[:, 0].sum())
    assert int(c[2]) == int(oc[:, 2].sum())
    assert int(c[2]) == int(g["ref_counters"][:, 1].sum())


@pytest.mark.parametrize("name", CASES)
def test_precompute_bit_exact(ctx6, oracle, name):
    g = load(name)
    ctx6.upload(g["verts"], g["tris"])
    ctx6.precompute()
    c = ctx6.export_cache()
    o = oracle.cache(g["verts"], g["tris"], NORM_IEEE)
    eq = (c.view(np.uint32) == o.view(np.uint32)) | (np.isnan(c) & np.isnan(o))
    assert eq.all()


def test_camera_rays_bit_exact(ctx6, oracle):
    g = load("small24k.npz")
    r = ctx6.camera_rays(g["camera"], 96, 64)
    o = oracle.camera_rays(g["camera"], 96, 64, NORM_IEEE)
    assert np.array_equal(r.view(np.uint32), o.view(np.uint32))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant", ["shortstack", "fullstack", "restart_early", "ropes"])
def test_render_cpu_semantics(ctx6, hk, oracle, name, variant):
    """GLVisitorCPUTrace::traceScene semantics (shadow rays, replacePixel):
    equal to the oracle with IEEE normalisation, and within 1/255 of the
    reference's own image on >= 99.9% of pixels."""
    g = load(name)
    setup_ref_tree(ctx6, g)
    w, h = (int(x) for x in g["render_wh"])
    img = ctx6.render(g["camera"], g["lights"], w, h, hk.VARIANTS[variant])
    ovar = {"shortstack": O_SHORT, "fullstack": O_FULL, "restart_early": O_RESTART_EARLY, "ropes": O_ROPES}[variant]
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"],
                            with_ropes=(ovar == O_ROPES))
    oimg = oracle.render_cpu(tree, g["render_rays"], w, h, g["lights"], ovar, 6, NORM_IEEE)
    assert np.array_equal(img, oimg)
    a = img.view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
    b = g["ref_render"].view(np.uint8).reshape(-1, 4)[:, :3].astype(int)
    assert (np.abs(a - b).max(axis=1) <= 1).mean() >= 0.999


def test_shade_picture(ctx6, hk, oracle):
    g = load("small24k.npz")
    setup_ref_tree(ctx6, g)
    w, h = (int(x) for x in g["render_wh"])
    img = ctx6.render(g["camera"], g["lights"], w, h, hk.SHORTSTACK, hk.SHADE_PICTURE)
    rays = g["render_rays"]
    hits = ctx6.trace(rays, hk.SHORTSTACK)
    cache = g["ref_cache"]
    hit4 = np.zeros((rays.shape[0], 4), np.float32)
    hit4[:, 3] = np.finfo(np.float32).max
    m = hits["tri"] >= 0
    hit4[m, :3] = cache[hits["tri"][m], :3]
    hit4[m, 3] = hits["t"][m]
    o = oracle.shade_picture(rays, hit4, g["lights"])
    assert np.array_equal(img, o)
    assert np.array_equal(ctx6.shade_picture(rays, hit4, g["lights"]), o)


def test_rejects_bad_inputs(ctx6, hk):
    g = load("soup3k.npz")
    v = g["verts"].copy()
    v[0, 3] = 0.5
    with pytest.raises(hk.HkError) as e:
        ctx6.upload(v, g["tris"])
    assert e.value.status == 4
    t = g["tris"].copy()
    t[5, 1] = 10 ** 7
    with pytest.raises(hk.HkError):
        ctx6.upload(g["verts"], t)
    ctx6.upload(g["verts"], g["tris"])
    bad = g["ref_nodes"].copy()
    junc = np.nonzero(bad[:, 0] & 8)[0]
    bad[junc[3], 1] = junc[1]          # a child shared by two parents
    with pytest.raises(hk.HkError):
        ctx6.import_tree(bad, g["ref_refs"])
    rays = g["rays"][:8].copy()
    rays[0, 7] = 1.0
    ctx6.import_cache(g["ref_cache"])
    ctx6.import_tree(g["ref_nodes"], g["ref_refs"])
    with pytest.raises(hk.HkError):
        ctx6.trace(rays)


@pytest.mark.parametrize("variant", ["ropes", "shortstack"])
def test_render_mirror_bounce(ctx6, hk, oracle, variant):
    """HK_SHADE_MIRROR (no reference counterpart) equals the oracle's
    restatement: reflected rays on 30% of triangles, then the usual shading."""
    g = load("small24k.npz")
    setup_ref_tree(ctx6, g)
    nt = g["tris"].shape[0]
    h32 = (np.arange(nt, dtype=np.uint64) * np.uint64(2654435761)) & np.uint64(0xFFFFFFFF)
    mirror = (h32.astype(np.float64) / 4294967296.0 < 0.3).astype(np.uint8)
    ctx6.set_mirrors(mirror)
    w, h = (int(x) for x in g["render_wh"])
    img = ctx6.render(g["camera"], g["lights"], w, h, hk.VARIANTS[variant], hk.SHADE_MIRROR)
    ovar = O_ROPES if variant == "ropes" else O_SHORT
    tree = oracle.make_tree(g["verts"], g["tris"], g["ref_cache"], g["ref_nodes"], g["ref_refs"], g["box"],
                            with_ropes=(ovar == O_ROPES))
    oimg = oracle.render_mirror(tree, g["render_rays"], w, h, g["lights"], mirror, ovar, 6, NORM_IEEE)
    assert np.array_equal(img, oimg)
    assert (img != ctx6.render(g["camera"], g["lights"], w, h, hk.VARIANTS[variant])).any()


def test_ropes_ties_and_signed_zero(hk):
    """Closest-hit ropes shares a warp's leaf tests out over its lanes and
    keeps each ray's hit by (t, position in the leaf): on a floor whose
    triangles are each listed three times (every hit is a three-way tie), and
    for rays that start on the floor heading up, away from its -y normal
    (t = -0.0 on a hit), the ids and the bits of t equal brute force and the
    in-order full stack."""
    rng = np.random.default_rng(21)
    n = 16
    xs = np.linspace(-4.0, 4.0, n + 1, dtype=np.float32)
    floor = np.array([[x, 0.0, z, 1.0] for z in xs for x in xs], np.float32)
    roof = floor.copy()
    roof[:, 1] = 2.0
    verts = np.concatenate([floor, roof])
    quads = []
    for j in range(n):
        for i in range(n):
            a = j * (n + 1) + i
            quads += [[a, a + 1, a + n + 2, 0], [a, a + n + 2, a + n + 1, 0]]
    quads = np.array(quads, np.uint32)
    roof_tris = quads.copy()
    roof_tris[:, :3] += floor.shape[0]
    tris = np.concatenate([quads, quads, quads, roof_tris]).astype(np.uint32)   # the floor three times
    ctx = hk.Context()
    ctx.upload(verts, tris)
    ctx.set_box(np.float32([-4, 0, -4, 1, 4, 2, 4, 1]))
    ctx.precompute()
    ctx.build()
    m = 20000
    rays = np.zeros((2 * m, 8), np.float32)
    # from between floor and roof, downwards with a tilt (every one lands on the floor)
    rays[:m, 0] = rng.uniform(-3.0, 3.0, m)
    rays[:m, 1] = rng.uniform(0.2, 1.8, m)
    rays[:m, 2] = rng.uniform(-3.0, 3.0, m)
    d = np.stack([rng.uniform(-0.5, 0.5, m), -np.ones(m), rng.uniform(-0.5, 0.5, m)], 1)
    rays[:m, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    # starting on the floor, heading up: the floor's hit has t = -0.0
    rays[m:, 0] = rng.uniform(-3.9, 3.9, m)
    rays[m:, 2] = rng.uniform(-3.9, 3.9, m)
    rays[m:, 4:7] = rays[:m, 4:7] * np.float32([1, -1, 1])
    b = ctx.trace(rays, hk.BRUTE)
    assert (b["tri"][:m] >= 0).all() and (b["tri"][:m] < quads.shape[0]).all()   # the first copy wins
    assert (np.signbit(b["t"][m:]) & (b["tri"][m:] >= 0)).sum() > m // 2
    for v in (hk.ROPES, hk.FULLSTACK):
        h = ctx.trace(rays, v)
        assert np.array_equal(h["tri"], b["tri"])
        assert np.array_equal(h["t"].view(np.uint32), b["t"].view(np.uint32))
    ctx.close()


@pytest.mark.parametrize("stack,block,ok", [(16, 256, False), (8, 512, None), (15, 256, True), (8, 128, True)])
def test_shared_memory_bound_of_the_shared_ring(hk, stack, block, ok):
    """SMEMSTACK keeps its ring in shared memory (stack x block x 12 bytes) next
    to the warp-shared leaf test's slots (block x 8 bytes). A configuration past
    48 KB is refused with HK_E_ILLEGAL_INPUT before anything is launched; one
    within it traces like the register ring. A block above the kernel's bound
    of 256 threads is refused when the context is created (ok None)."""
    g = load("soup3k.npz")
    if ok is None:
        with pytest.raises(hk.HkError) as e:
            hk.Context(short_stack=stack, block_size=block)
        assert e.value.status == 4
        return
    ctx = hk.Context(short_stack=stack, block_size=block)
    setup_ref_tree(ctx, g)
    rays = g["rays"]
    if not ok:
        with pytest.raises(hk.HkError) as e:
            ctx.trace(rays, hk.SMEMSTACK)
        assert e.value.status == 4 and "48 KB" in str(e.value)
    else:
        a = ctx.trace(rays, hk.SMEMSTACK)
        b = ctx.trace(rays, hk.SHORTSTACK)
        assert np.array_equal(a["tri"], b["tri"]) and np.array_equal(a["t"].view(np.uint32), b["t"].view(np.uint32))
    ctx.close()
