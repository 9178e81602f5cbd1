"""The CUDA builder's node layout, restated by the oracle: subtrees of nodes of
2..T references (hk_config.subtree_max, default 32) are built depth first
after the levels and numbered after every level's nodes. That changes the
numbering only: walked from the root, the tree is node for node the tree that
numbers every node level by level (same splits, same leaf references in the
same order), in binned, exact and degenerate cases. The capacity rule is
checked too: when the subtrees do not fit the node arena, every deferred root
stays a leaf with its references."""
import numpy as np
import pytest

from hulktracer_b200 import scenes

CLEAF = 3


def walk(cn, refs):
    """Pre-order list of (axis, plane bits) / ('leaf', refs) from the root."""
    out, stack = [], [0]
    while stack:
        n = stack.pop()
        x, y = int(cn[n, 0]), int(cn[n, 1])
        if x & 3 == CLEAF:
            out.append(("leaf", tuple(refs[(x >> 2):(x >> 2) + y].tolist())))
        else:
            out.append((x & 3, y))
            stack.append((x >> 2) + 1)
            stack.append(x >> 2)
    return out


def scene_cases():
    sc = scenes.animated_parts(n_parts=6, width=96, height=64)
    yield "animated6", sc.verts, sc.tris, sc.scene_box()
    rng = np.random.default_rng(3)
    n = 3000
    c = rng.random((n, 3)).astype(np.float32) * 10
    v = np.concatenate([c + rng.normal(0, 0.3, (n, 3)).astype(np.float32) for _ in range(3)])
    verts = np.concatenate([v, np.ones((3 * n, 1), np.float32)], 1)
    tris = np.stack([np.arange(n), np.arange(n) + n, np.arange(n) + 2 * n, np.zeros(n, np.int64)], 1)
    box = np.array([*verts[:, :3].min(0), 0, *verts[:, :3].max(0), 0], np.float32)
    yield "soup3k", verts, tris.astype(np.uint32), box
    # many coplanar, overlapping and flat triangles (flat-on-plane references)
    k = 400
    g = rng.integers(0, 4, (k, 3)).astype(np.float32)
    pv = np.concatenate([g, g + [1, 0, 0], g + [0, 1, 0]])
    verts = np.concatenate([pv, np.ones((3 * k, 1), np.float32)], 1)
    tris = np.stack([np.arange(k), np.arange(k) + k, np.arange(k) + 2 * k, np.zeros(k, np.int64)], 1)
    box = np.array([-0.5, -0.5, -0.5, 0, 5.5, 5.5, 5.5, 0], np.float32)
    yield "flat_grid", verts, tris.astype(np.uint32), box


@pytest.mark.parametrize("defer,margin", [(32, 0), (12, 0), (32, 8), (32, 3)])
@pytest.mark.parametrize("exact_max", [0, 1024])
@pytest.mark.parametrize("case", list(range(3)))
def test_deferred_layout_is_the_same_tree(oracle, case, exact_max, defer, margin):
    name, verts, tris, box = list(scene_cases())[case]
    a, ar = oracle.build_binned(verts, tris, box, exact_max=exact_max, defer=0)
    b, br = oracle.build_binned(verts, tris, box, exact_max=exact_max, defer=defer, defer_margin=margin)
    assert a.shape == b.shape and ar.shape == br.shape
    assert walk(a, ar) == walk(b, br), name
    if a.shape[0] > 64 and margin == 0:
        assert not np.array_equal(a, b)    # the numbering does differ


def test_deferred_subtrees_numbered_after_the_levels(oracle):
    """Every node reached through a deferred root (a node of 2..32 references)
    has a larger index than every node the levels numbered, and sibling pairs
    stay adjacent (pair = 2k)."""
    sc = scenes.animated_parts(n_parts=6, width=96, height=64)
    cn, refs = oracle.build_binned(sc.verts, sc.tris, sc.scene_box(), defer_margin=0)
    leaf = (cn[:, 0] & 3) == CLEAF
    pairs = cn[~leaf, 0] >> 2
    assert np.all(pairs % 2 == 0)
    # the distinct references below every node, bottom up
    order, stack = [], [0]
    while stack:
        k = stack.pop()
        order.append(k)
        if not leaf[k]:
            p = int(cn[k, 0] >> 2)
            stack += [p, p + 1]
    uniq = {}
    for k in reversed(order):
        if leaf[k]:
            s = int(cn[k, 0] >> 2)
            uniq[k] = set(refs[s:s + int(cn[k, 1])].tolist())
        else:
            p = int(cn[k, 0] >> 2)
            uniq[k] = uniq[p] | uniq[p + 1]
    roots = [k for k in order if not leaf[k] and 2 <= len(uniq[k]) <= 32]
    inner = [k for k in order if not leaf[k] and len(uniq[k]) > 32]
    if roots and inner:
        first_sub = min(int(cn[k, 0] >> 2) for k in roots)
        last_level = max(int(cn[k, 0] >> 2) + 1 for k in inner)
        assert first_sub > last_level


def test_subtrees_that_do_not_fit_stay_leaves(oracle):
    """A node arena that holds the levels but not the subtrees: every deferred
    root becomes a leaf over its 2..32 references; the rest of the tree is
    unchanged."""
    sc = scenes.animated_parts(n_parts=6, width=96, height=64)
    box = sc.scene_box()
    full, fr = oracle.build_binned(sc.verts, sc.tris, box)
    small, sr = oracle.build_binned(sc.verts, sc.tris, box, max_nodes=full.shape[0] - 1)
    assert small.shape[0] < full.shape[0]
    assert set(sr.tolist()) == set(fr.tolist())
    # walk both trees together: they agree down to the deferred roots, which
    # are leaves in the small tree and split in the full one
    stack, cut = [(0, 0)], 0
    while stack:
        a, b = stack.pop()
        xa, ya, xb, yb = (int(v) for v in (small[a, 0], small[a, 1], full[b, 0], full[b, 1]))
        if xa & 3 == CLEAF and xb & 3 != CLEAF:
            assert 2 <= ya <= 32
            cut += 1
            continue
        assert (xa & 3, ya if xa & 3 != CLEAF else 0) == (xb & 3, yb if xb & 3 != CLEAF else 0)
        if xa & 3 == CLEAF:
            assert np.array_equal(sr[xa >> 2:(xa >> 2) + ya], fr[xb >> 2:(xb >> 2) + yb])
        else:
            stack += [((xa >> 2) + 1, (xb >> 2) + 1), (xa >> 2, xb >> 2)]
    assert cut > 0
