"""Learned surrogate (no counterpart in the reference; parity unpinned).

The MLP kernels (tcgen05 GEMMs with fused epilogues) are checked against the
CPU restatement of the network in oracle/dmph_mlp_oracle.c, which rounds the
same operands to BF16; sums differ by accumulation order only, so the bars
are a few BF16 ulps.  The driver (collect, train, judged surrogate calls,
fallback) is checked for its bookkeeping and for leaving a finite state."""
import numpy as np
import pytest

from oracle import oracle as orc
from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import MLP_FEATURES, MLP_IN, MLP_OUT, PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu


def make(bodies=False, **kw):
    s = scenes.small()
    p = s.params.copy()
    p.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(p, s.type, s.x, s.v)
    if bodies:
        g.set_bodies(s.body, s.body_density)
    args = dict(batch=8192, pool_rows=1 << 17, check_interval=5)
    args.update(kw)
    g.enable_surrogate(**args)
    return g


def random_rows(n, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, MLP_IN), np.float32)
    X[:, :MLP_FEATURES] = rng.normal(size=(n, MLP_FEATURES))
    return X


def test_mlp_forward_matches_oracle():
    g = make()
    w = g.surrogate_weights()
    rng = np.random.default_rng(3)
    w = (w + 0.05 * rng.normal(size=w.shape)).astype(np.float32)  # non-zero biases and outputs
    g.set_surrogate_weights(w)
    X = random_rows(3000, 1)
    Y = g.mlp_forward(X)
    Yo = orc.mlp_forward(w, X)
    scale = np.abs(Yo[:, :6]).max()
    assert scale > 0.1
    err = np.abs(Y[:, :6] - Yo[:, :6]).max() / scale
    assert err <= 2e-2, err
    assert np.sqrt(np.mean((Y[:, :6] - Yo[:, :6]) ** 2)) / np.sqrt(np.mean(Yo[:, :6] ** 2)) <= 5e-3
    g.close()


def test_mlp_gradient_matches_oracle():
    g = make()
    w = g.surrogate_weights()
    rng = np.random.default_rng(5)
    w = (w + 0.05 * rng.normal(size=w.shape)).astype(np.float32)
    g.set_surrogate_weights(w)
    X = random_rows(8192, 2)
    T = np.zeros((8192, MLP_OUT), np.float32)
    T[:, :6] = rng.normal(size=(8192, 6))
    G, loss = g.mlp_gradient(X, T)
    Go, loss_o = orc.mlp_grad(w, X, T)
    assert abs(loss - loss_o) <= 1e-3 * loss_o
    # per layer: relative L2 error of the gradient
    offs, o = [], 0
    for i, h in ((64, 128), (128, 128), (128, 128), (128, 16)):
        offs.append((o, o + i * h, o + i * h + h))
        o += i * h + h
    assert o == len(G)
    for a, b, c in offs:
        for lo, hi in ((a, b), (b, c)):
            rel = np.linalg.norm(G[lo:hi] - Go[lo:hi]) / (np.linalg.norm(Go[lo:hi]) + 1e-30)
            assert rel <= 2e-2, (lo, hi, rel)
    g.close()


@pytest.mark.parametrize("bodies", [False, True])
def test_surrogate_collect_train_advance(bodies):
    g = make(bodies=bodies)
    g.step(20)
    g.surrogate_collect(12)
    st = g.surrogate_stats()
    assert st["plain_blocks"] == 12 and st["pool_rows"] > 8192
    l0 = g.surrogate_train(1)
    l1 = g.surrogate_train(200)
    assert np.isfinite(l1) and l1 < l0, (l0, l1)
    t0 = g.info().time
    g.surrogate_advance(12)
    st = g.surrogate_stats()
    K = g.surrogate_params.substeps
    assert abs(g.info().time - (t0 + 12 * K * g.params.dt)) < 1e-9
    assert st["calls"] + st["plain_blocks"] == 12 + 12
    assert st["judged"] >= 1
    _, x, v, _ = g.state()
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
    g.close()


def test_fallback_on_large_error_and_none_on_loose_tolerance():
    g = make(tolerance=1e-12, fallback_blocks=3, check_interval=2)
    g.step(20)
    g.surrogate_collect(4)
    g.surrogate_advance(3)  # 2 surrogate calls, then a judged block
    st = g.surrogate_stats()
    assert st["judged"] == 1 and st["fallbacks"] == 1 and st["in_fallback"] == 1
    g.surrogate_advance(3)
    st = g.surrogate_stats()
    assert st["in_fallback"] == 0 and st["plain_blocks"] == 4 + 1 + 3
    g.close()
    h = make(tolerance=1e9, check_interval=2)
    h.step(20)
    h.surrogate_collect(4)
    h.surrogate_advance(6)
    st = h.surrogate_stats()
    assert st["judged"] == 2 and st["fallbacks"] == 0 and st["calls"] == 4
    h.close()
