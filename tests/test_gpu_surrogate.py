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


@pytest.mark.parametrize("n", [1, 127, 3000, 30000])
def test_fused_forward_equals_the_layer_gemms(n):
    """the fused forward kernel (TMA-fed tiles, weights in shared memory,
    activations through TMEM and shared memory) gives the bits of the four
    per-layer GEMMs: the same MMAs in the same K order, the same epilogues"""
    if n > 7000:  # more tiles than SMs: each CTA loops over several, double-buffered
        sc = scenes.small(dx=0.01)
        p = sc.params.copy()
        p.precision = PRECISION_FP32_SPLIT
        g = solver.Solver(p, sc.type, sc.x, sc.v)
        g.enable_surrogate(batch=8192, pool_rows=1 << 17, check_interval=5)
        assert g.n >= n
    else:
        g = make()
    w = g.surrogate_weights()
    rng = np.random.default_rng(5)
    g.set_surrogate_weights((w + 0.05 * rng.normal(size=w.shape)).astype(np.float32))
    X = random_rows(n, 2)
    a = g.mlp_forward(X)
    b = g.mlp_forward(X, layers=True)
    assert np.array_equal(a, b), np.abs(a - b).max()
    assert np.abs(a[:, :6]).max() > 0.05
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


def test_front_judge():
    """the surge-front judge alone (velocity-increment judge off): a tolerance
    no prediction meets falls back at the judged block, a loose one never;
    the estimate and the last block's deviation are reported"""
    g = make(tolerance=0.0, front_tolerance=1e-6, fallback_blocks=3, check_interval=2)
    # a network that predicts a strong push along x (output bias of dv_x),
    # so that its front runs ahead of the solver's by several histogram bins
    w = g.surrogate_weights()
    w[-16] = 2000.0
    g.set_surrogate_weights(w)
    g.step(20)
    g.surrogate_collect(4)
    g.surrogate_advance(3)  # 2 surrogate calls, then a judged block
    st = g.surrogate_stats()
    assert st["judged"] == 1 and st["fallbacks"] == 1 and st["in_fallback"] == 1
    assert st["front_estimate"] > 1e-6 and st["last_front_dev"] > 0
    g.close()
    h = make(tolerance=0.0, front_tolerance=1e9, check_interval=2)
    h.step(20)
    h.surrogate_collect(4)
    h.surrogate_advance(6)
    st = h.surrogate_stats()
    assert st["judged"] == 2 and st["fallbacks"] == 0 and st["calls"] == 4
    assert 0 <= st["front_estimate"] < 1e9
    h.close()


def test_list_features_match_stencil_features():
    """the features computed over the Verlet lists (the default) and over the
    27-cell stencil are the same sums up to FP32 summation order"""
    g = make()
    g.step(60)
    fl = g.surrogate_features()
    g.set_pair_mode("stencil")
    fs = g.surrogate_features()
    assert fl.shape == fs.shape and len(fl) > 0
    scale = np.maximum(np.abs(fs).max(axis=0), 1e-3)
    err = np.abs(fl - fs).max(axis=0) / scale
    assert err.max() <= 2e-3, (err.max(), int(err.argmax()))
    g.close()


def test_trained_network_gains_over_no_network():
    """What the network adds.  The network is trained on the latest plain
    blocks and judged on the next one, as the surrogate's own training during
    a run does: from the same state, the K-step velocity increments of the
    fluid predicted with the trained network (residual form:
    dv = K dt (a0 + |g| y / 16)) and without it (dv = K dt a0: constant
    acceleration over the block) are compared with the increments the plain
    solver then makes, over six rounds of (judge the next block, then collect
    two more blocks and train on).  Config 1 with rigid debris, K = 4.
    The relation between the features and the increments drifts in this
    early flow within about a hundred steps, so a network trained once and
    judged far from its data does not gain; trained on the latest blocks it
    does, by the margin asserted here."""
    K = 4
    s = scenes.config1()  # the surrogate bench's scene: 72k fluid particles
    p = s.params.copy()
    p.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(p, s.type, s.x, s.v)
    g.set_bodies(s.body, s.body_density)
    g.enable_surrogate(substeps=K, pool_rows=1 << 20)
    g.step(300)
    g.surrogate_collect(16)
    g.surrogate_train(800)
    V = p.particle_spacing ** 3
    dens = np.array(list(p.density))
    gmag = float(np.linalg.norm(list(p.gravity)))
    kdt = K * p.dt
    et, e0 = [], []
    for _ in range(6):
        F = g.surrogate_features()  # fluid and debris slots, slot order
        t, _, v0, ids = g.state()
        a0 = g.field("Force") / (dens[t] * V)[:, None]
        X = np.zeros((len(F), MLP_IN), np.float32)
        X[:, :MLP_FEATURES] = F
        Y = g.mlp_forward(X)
        rows = np.flatnonzero(t[:len(F)] < 2)  # fluid
        dv_net = (Y[rows, :3] * (gmag / 16.0) + a0[rows]) * kdt  # outputs in units of |g| / 16
        dv_none = a0[rows] * kdt
        g.step(K)
        t1, _, v1, ids1 = g.state()
        slot = np.empty(len(ids1), np.int64)
        slot[ids1] = np.arange(len(ids1))
        dv = v1[slot[ids[rows]]] - v0[rows]
        et.append(np.linalg.norm(dv_net - dv) / np.linalg.norm(dv))
        e0.append(np.linalg.norm(dv_none - dv) / np.linalg.norm(dv))
        g.surrogate_collect(2)
        g.surrogate_train(100)
    mt, m0 = float(np.mean(et)), float(np.mean(e0))
    print("K-step velocity-increment error: trained network %.4f, without it %.4f" % (mt, m0))
    assert mt < 0.97 * m0, (mt, m0)
    g.close()
