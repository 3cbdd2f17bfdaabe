"""The surrogate's training corpus (dem_mph_b200.corpus, config 4 in small):
rows recorded on several seeded scenes, moved between contexts through the
pool's host interface (dmph_surrogate_get_samples / _add_samples, features
rounded to BF16 as recorded), and one network trained on them on the GPU,
which fits the corpus better than the network it started from."""
import numpy as np
import pytest

from dem_mph_b200 import corpus, scenes

pytestmark = pytest.mark.gpu


def bf16(x):
    """round-to-nearest-even to BF16, as the pool stores features"""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def test_corpus_roundtrip_and_training():
    sc = [scenes.small(seed=11 + k, n_debris=2, yaw=True) for k in range(2)]
    X, T = corpus.build(sc, steps=96, substeps=4, rows_per_scene=6000)
    assert X.shape[1] == 64 and T.shape[1] == 16 and len(X) == len(T) > 4000
    assert np.all(np.isfinite(X)) and np.all(np.isfinite(T)) and np.all(T[:, 6:] == 0)
    g = corpus._solver(sc[0], 4, 1 << 14)
    g.surrogate_add_samples(X[:10000], T[:10000])
    Xb, Tb = g.surrogate_samples(1 << 14)
    n = min(len(X), 10000)
    assert len(Xb) == n
    assert np.array_equal(Xb, bf16(X[:n])) and np.array_equal(Tb, T[:n])
    w0 = g.surrogate_weights()
    g.close()
    w, losses = corpus.train(sc[0], X, T, iters=300, substeps=4, batch=8192, report_every=100)
    assert len(losses) == 3 and np.all(np.isfinite(losses))
    g = corpus._solver(sc[1], 4, 1 << 14)
    m = min(len(X), g.n)  # rows of one forward call: at most the particle count

    def mse(weights):
        g.set_surrogate_weights(weights)
        Y = g.mlp_forward(X[:m])
        return float(np.mean((Y[:, :6] - T[:m, :6]) ** 2))
    before, after = mse(w0), mse(w)
    print("corpus MSE before %.4f after %.4f, losses %s" % (before, after, losses))
    assert after < 0.8 * before
    g.close()


def test_committed_corpus_network_gains_on_an_unseen_scene():
    """the network trained on the config-4 corpus (dem_mph_b200/weights,
    made by bench.py --corpus --save-weights) on config 1, a scene outside
    its corpus: its K = 8 velocity increments are closer to the solver's than
    constant acceleration over the block"""
    import os
    w = np.load(os.path.join(os.path.dirname(corpus.__file__), "weights", "surrogate_config4_k8.npy"))
    e_net, e_none = corpus.evaluate(scenes.config1(), w, substeps=8)
    print("held-out config 1, K = 8: with the network %.4f, without %.4f" % (e_net, e_none))
    assert e_net < 0.75 * e_none
