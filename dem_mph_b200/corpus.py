"""Training corpus of the surrogate network (config 4): plain K-step blocks
recorded on many seeded scenes, pooled on the host, and one network trained
on the pool by the library's own tensor-core forward and backward kernels.

The surrogate's features and targets are dimensionless (velocities in units
of c0 / 10, accelerations and the velocity-increment targets in units of
|g|, lengths in dx), so blocks of scenes with other spacings, column heights
and time steps share one pool.  A context records into its own pool ring
(dmph_surrogate_collect keeps about pool/16 rows of every block); `record`
reads the ring out every 16 blocks and keeps a uniform subset, so the rows
it returns cover the whole trajectory.
"""
import numpy as np

from . import solver
from .abi import PRECISION_FP32_SPLIT


def _solver(scene, substeps, pool_rows, batch=8192):
    p = scene.params.copy()
    p.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(p, scene.type, scene.x, scene.v)
    if len(scene.body_density):
        g.set_bodies(scene.body, scene.body_density)
    g.enable_surrogate(substeps=substeps, pool_rows=pool_rows, batch=batch)
    return g


def record(scene, steps=4000, substeps=8, rows=131072, seed=0):
    """(X [n, 64], T [n, 16]) recorded on `scene` over `steps` solver steps
    (plain blocks of `substeps` steps), n <= rows drawn uniformly over the
    blocks"""
    rng = np.random.default_rng(seed)
    pool = 1 << 17
    chunk = 16  # blocks that fill the ring once
    blocks = max(1, steps // substeps)
    nchunks = max(1, -(-blocks // chunk))
    per = max(1, rows // nchunks)
    g = _solver(scene, substeps, pool)
    xs, ts = [], []
    done = 0
    while done < blocks:
        nb = min(chunk, blocks - done)
        g.surrogate_collect(nb)
        done += nb
        X, T = g.surrogate_samples(pool)
        # the rows of these nb blocks are the newest of the ring
        fresh = min(len(X), nb * (pool // chunk))
        X, T = X[len(X) - fresh:], T[len(T) - fresh:]
        pick = rng.choice(len(X), size=min(per, len(X)), replace=False)
        xs.append(X[pick])
        ts.append(T[pick])
    g.close()
    return np.concatenate(xs)[:rows], np.concatenate(ts)[:rows]


def build(scenes, steps=4000, substeps=8, rows_per_scene=131072, seed=0):
    """(X, T) of all scenes, in scene order"""
    xs, ts = [], []
    for k, s in enumerate(scenes):
        X, T = record(s, steps, substeps, rows_per_scene, seed + k)
        xs.append(X)
        ts.append(T)
    return np.concatenate(xs), np.concatenate(ts)


def train(scene, X, T, iters=20000, substeps=8, batch=262144, report_every=1000):
    """weights of a network trained on the rows (Adam on the GPU, batches
    drawn from the pool), and the losses every `report_every` iterations;
    `scene` only hosts the training context"""
    pool = 1 << max(20, int(np.ceil(np.log2(max(len(X), batch)))))
    g = _solver(scene, substeps, pool, batch=batch)
    g.surrogate_add_samples(X, T)
    losses = []
    left = iters
    while left > 0:
        n = min(report_every, left)
        losses.append(g.surrogate_train(n))
        left -= n
    w = g.surrogate_weights()
    g.close()
    return w, losses


def evaluate(scene, weights, substeps=8, settle=300, blocks=6):
    """mean relative error of the fluid's K-step velocity increments on a
    scene the network has not seen, from the network's prediction (its
    residual over constant acceleration, in units of |g| / 16) and without
    it (constant acceleration over the block): (with, without)"""
    from .abi import MLP_FEATURES, MLP_IN
    g = _solver(scene, substeps, 1 << 17)
    g.set_surrogate_weights(weights)
    p = scene.params
    V = p.particle_spacing ** 3
    dens = np.array(list(p.density))
    gmag = float(np.linalg.norm(list(p.gravity)))
    kdt = substeps * p.dt
    g.step(settle)
    et, e0 = [], []
    for _ in range(blocks):
        F = g.surrogate_features()
        t, _, v0, ids = g.state()
        a0 = g.field("Force") / (dens[t] * V)[:, None]
        X = np.zeros((len(F), MLP_IN), np.float32)
        X[:, :MLP_FEATURES] = F
        Y = g.mlp_forward(X)
        rows = np.flatnonzero(t[:len(F)] < 2)
        dv_net = (Y[rows, :3] * (gmag / 16.0) + a0[rows]) * kdt
        dv_none = a0[rows] * kdt
        g.step(substeps)
        _, _, v1, ids1 = g.state()
        slot = np.empty(len(ids1), np.int64)
        slot[ids1] = np.arange(len(ids1))
        dv = v1[slot[ids[rows]]] - v0[rows]
        et.append(np.linalg.norm(dv_net - dv) / np.linalg.norm(dv))
        e0.append(np.linalg.norm(dv_none - dv) / np.linalg.norm(dv))
        g.step(20 * substeps)
    g.close()
    return float(np.mean(et)), float(np.mean(e0))
