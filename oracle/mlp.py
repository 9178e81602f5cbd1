"""CPU oracle of the learned split proposer's network (test infrastructure
only: tests use it as the checker of the CUDA kernels; no product path calls
it).

The network has no reference counterpart: hulkTracer's builders
(HulkEngine/src/KDTreeSAH.cpp, HulkEngine/src/KDTreeCPU.cpp) cost every
candidate plane. This file restates, in numpy, what the CUDA side computes:

* ``forward_fp32`` / ``grad_fp32``: the FP32 training path -- 200 -> 256 ->
  256 -> 256 -> 96 with ReLU, mean softmax cross-entropy, and the gradient of
  every parameter in the flat layout of ``hk_mlp_get_params``;
* ``forward_bf16``: the inference path -- inputs, weights and hidden
  activations rounded to BF16 (round to nearest even), products accumulated in
  FP32 (here in float64, then rounded), biases in FP32;
* ``hist_features`` / ``exact_label``: the 200 node features the builder
  computes from a node's binned histogram, and the training label of an
  exactly searched node.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 200, 256, 96
SHAPES = [("W1", (IN, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, HID)), ("b3", (HID,)), ("W4", (HID, OUT)), ("b4", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unflatten(p):
    """Views of the flat parameter vector: W (in x out, row-major) and b."""
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = p[o:o + n].reshape(shp)
        o += n
    return out


def flatten(d):
    return np.concatenate([np.asarray(d[name], np.float32).ravel() for name, _ in SHAPES])


def bf16(x):
    """Round FP32 to BF16 (nearest, ties to even), returned as FP32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def forward_fp32(p, X):
    P = unflatten(np.asarray(p, np.float32))
    X = np.asarray(X, np.float32)
    H1 = np.maximum(X @ P["W1"] + P["b1"], 0)
    H2 = np.maximum(H1 @ P["W2"] + P["b2"], 0)
    H3 = np.maximum(H2 @ P["W3"] + P["b3"], 0)
    Z = H3 @ P["W4"] + P["b4"]
    return Z, (X, H1, H2, H3)


def loss_and_dz(Z, y):
    Z = Z.astype(np.float64)
    Z = Z - Z.max(axis=1, keepdims=True)
    E = np.exp(Z)
    Pr = E / E.sum(axis=1, keepdims=True)
    n = Z.shape[0]
    loss = -np.log(np.maximum(Pr[np.arange(n), y], 1e-30)).mean()
    dZ = Pr.copy()
    dZ[np.arange(n), y] -= 1.0
    return float(loss), (dZ / n).astype(np.float32)


def grad_fp32(p, X, y):
    """Mean softmax cross-entropy and its gradient (flat layout)."""
    P = unflatten(np.asarray(p, np.float32))
    Z, (X, H1, H2, H3) = forward_fp32(p, X)
    loss, d4 = loss_and_dz(Z, np.asarray(y))
    g = {}
    g["W4"], g["b4"] = H3.T @ d4, d4.sum(0)
    d3 = (d4 @ P["W4"].T) * (H3 > 0)
    g["W3"], g["b3"] = H2.T @ d3, d3.sum(0)
    d2 = (d3 @ P["W3"].T) * (H2 > 0)
    g["W2"], g["b2"] = H1.T @ d2, d2.sum(0)
    d1 = (d2 @ P["W2"].T) * (H1 > 0)
    g["W1"], g["b1"] = X.T @ d1, d1.sum(0)
    return flatten(g), loss


def forward_bf16(p, X):
    P = unflatten(np.asarray(p, np.float32))
    a = bf16(X).astype(np.float64)
    for i in (1, 2, 3):
        z = (a @ bf16(P["W%d" % i]).astype(np.float64)).astype(np.float32) + P["b%d" % i]
        a = bf16(np.maximum(z, 0)).astype(np.float64)
    return (a @ bf16(P["W4"]).astype(np.float64)).astype(np.float32) + P["b4"]


def hist_features(node_lo, node_hi, tri_lo, tri_hi, depth, max_depth):
    """The 200 features of one node as the builder computes them from its
    binned-SAH histogram (every reference of the node): per axis the counts
    of the clipped lower bounds per bin b (p_b <= lo < p_{b+1}) and of the
    clipped upper bounds per bin c (p_c < hi <= p_{c+1}), p_k = min + ext *
    (k / 32), as fractions of the node's references; the node extents over the
    largest extent; depth / max_depth; references / 1024; three zeros."""
    f = np.zeros(200, np.float32)
    cnt = tri_lo.shape[0]
    lo_n = np.asarray(node_lo, np.float32)
    hi_n = np.asarray(node_hi, np.float32)
    for a in range(3):
        l, h = lo_n[a], hi_n[a]
        ext = np.float32(h - l)
        if not ext > 0:
            continue
        k = np.arange(1, 32, dtype=np.float32) * np.float32(0.03125)
        planes = (l + ext * k).astype(np.float32)          # p_1 .. p_31, non-decreasing
        lo = np.maximum(tri_lo[:, a].astype(np.float32), l)
        hi = np.minimum(tri_hi[:, a].astype(np.float32), h)
        b = np.searchsorted(planes, lo, side="right")       # planes <= lo
        c = np.searchsorted(planes, hi, side="left")        # planes < hi
        f[a * 64: a * 64 + 32] = np.bincount(b, minlength=32).astype(np.float32)
        f[a * 64 + 32: a * 64 + 64] = np.bincount(c, minlength=32).astype(np.float32)
    if cnt:
        f[:192] *= np.float32(1.0) / np.float32(cnt)
    e = (hi_n[:3] - lo_n[:3]).astype(np.float32)
    m = e.max()
    f[192:195] = e * (np.float32(1.0) / m if m > 0 else np.float32(0.0))
    f[195] = np.float32(depth) / np.float32(max_depth)
    f[196] = np.float32(cnt) * np.float32(1.0 / 1024.0)
    return f


def exact_label(node_lo, node_hi, axis, plane):
    """axis * 32 + the bin b holding the plane: p_b <= plane < p_{b+1}."""
    l = np.float32(node_lo[axis])
    ext = np.float32(np.float32(node_hi[axis]) - l)
    k = np.arange(1, 32, dtype=np.float32) * np.float32(0.03125)
    planes = (l + ext * k).astype(np.float32)
    return int(axis) * 32 + int(np.searchsorted(planes, np.float32(plane), side="right"))
