"""The proposer network's CPU oracle (oracle/mlp.py) checked against torch
autograd in float64, and its BF16 rounding against torch's conversion."""
import numpy as np
import torch

from oracle import mlp


def rand_params(seed=0):
    rng = np.random.default_rng(seed)
    p = np.zeros(mlp.NPARAMS, np.float32)
    P = mlp.unflatten(p)
    for name, shp in mlp.SHAPES:
        fan_in = shp[0] if len(shp) == 2 else 64
        P[name][...] = rng.normal(0, np.sqrt(2.0 / fan_in), size=shp)
    return p


def test_grad_fp32_matches_autograd():
    p = rand_params(1)
    rng = np.random.default_rng(2)
    X = rng.random((48, mlp.IN), dtype=np.float32)
    y = rng.integers(0, mlp.OUT, size=48).astype(np.int32)
    g, loss = mlp.grad_fp32(p, X, y)
    P = {k: torch.tensor(v.astype(np.float64), requires_grad=True) for k, v in mlp.unflatten(p).items()}
    x = torch.tensor(X.astype(np.float64))
    h = torch.relu(x @ P["W1"] + P["b1"])
    h = torch.relu(h @ P["W2"] + P["b2"])
    h = torch.relu(h @ P["W3"] + P["b3"])
    z = h @ P["W4"] + P["b4"]
    lt = torch.nn.functional.cross_entropy(z, torch.tensor(y.astype(np.int64)))
    lt.backward()
    ref = np.concatenate([P[name].grad.numpy().ravel() for name, _ in mlp.SHAPES])
    assert abs(loss - lt.item()) < 1e-5 * max(1.0, abs(lt.item()))
    o = 0
    for name, shp in mlp.SHAPES:
        n = int(np.prod(shp))
        a, b = g[o:o + n].astype(np.float64), ref[o:o + n]
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b) + 1e-9, name
        o += n


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(100000) * 10.0 ** rng.integers(-6, 6, 100000)).astype(np.float32)
    t = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(mlp.bf16(x).view(np.uint32), t.view(np.uint32))


def test_hist_features_shape_sums_and_bins():
    """Per axis the lower-bound and upper-bound bin counts each sum to the
    node's references; a bound exactly on a bin plane goes to the bin above
    it (lower bounds) or below it (upper bounds), as the builder's
    corrections place them."""
    rng = np.random.default_rng(4)
    lo = rng.uniform(-1, 0.5, size=(100, 3)).astype(np.float32)
    hi = lo + rng.uniform(0, 0.5, size=(100, 3)).astype(np.float32)
    nlo, nhi = np.float32([-1, -1, -1, 0]), np.float32([1, 2, 1, 0])
    f = mlp.hist_features(nlo, nhi, lo, hi, 3, 24)
    assert f.shape == (200,)
    for a in range(3):
        assert abs(f[a * 64:a * 64 + 32].sum() - 1) < 1e-5
        assert abs(f[a * 64 + 32:(a + 1) * 64].sum() - 1) < 1e-5
    third = np.float32(1) / np.float32(3)
    assert np.array_equal(f[192:195], np.float32([2 * third, 3 * third, 2 * third]))
    assert f[195] == np.float32(3) / np.float32(24)
    assert f[196] == np.float32(100) / np.float32(1024)
    # x in [-1, 1]: p_16 = 0 exactly; a bound on it
    lo2 = np.zeros((1, 3), np.float32)
    f2 = mlp.hist_features(nlo, nhi, lo2, lo2, 0, 24)
    assert f2[16] == 1.0 and f2[32 + 15] == 1.0
    assert mlp.exact_label(nlo, nhi, 0, np.float32(0.0)) == 16
    assert mlp.exact_label(nlo, nhi, 1, np.float32(-0.99)) == 32
