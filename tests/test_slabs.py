"""x-slab domain decomposition (dem_mph_b200.slabs) on the host: two gloo
ranks, each with one slab of a small dam break, exchange ghost states every
step and decide the rebuilds together.  The per-slab engine here is the
oracle (no GPU in this test; on GPUs the same driver steps libdmph contexts,
tests/test_gpu_slabs.py): the test checks the decomposition itself, that
the slabs' owned particles have the single-domain neighbour sets exactly and
follow the single-domain run to rounding, through rebuilds and the
re-partition each rebuild makes.

Free debris are compared only over a few steps: the reference's DEM takes
its contact constants from the last neighbour within dx in list order
(source/DEM-MPH.cpp:2305-2341), and each rank orders the particles of a cell
by its own sort, so debris contacts differ from the single-domain run and
the reference's non-dissipative contact model amplifies that."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))


class OracleEngine:
    """the oracle behind the slab driver's engine interface (test only)"""

    def __init__(self, p, typ, x, v):
        from oracle.oracle import Oracle
        self.o = Oracle(p, typ, x, v)

    def step_begin(self):
        return self.o.step_begin()

    def step_finish(self, rebuild):
        self.o.step_finish(rebuild)

    def get_rows(self, rows):
        return self.o.get_rows(rows)

    def set_rows(self, rows, x, v):
        self.o.set_rows(rows, x, v)

    def close(self):
        self.o.close()


def neighbour_sets(o, gid):
    """per particle (global id) the sorted global ids of its neighbour list"""
    ptr, ind, pidx = o.get("NeighborPtr"), o.get("NeighborInd"), o.get("ParticleIndex")
    out = {}
    for i in range(len(pidx)):
        out[int(gid[pidx[i]])] = np.sort(gid[pidx[ind[ptr[i]:ptr[i + 1]]]])
    return out


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, steps, out):
    import datetime
    import sys
    sys.path[:0] = [ROOT, HERE]
    import torch.distributed as dist
    from helpers import load_scene
    from oracle.oracle import Oracle
    from dem_mph_b200 import slabs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        p, typ, x, v = load_scene(name)
        typ = np.asarray(typ)
        n = len(typ)
        whole = Oracle(p, typ, x, v)
        slab = slabs.Slab(p, rank, world, OracleEngine)
        slab.partition(np.arange(n), typ, x, v)
        # neighbour sets of the owned particles at creation
        mine = neighbour_sets(slab.engine.o, slab.gid)
        ref = neighbour_sets(whole, np.arange(n))
        owned = slab.gid[:slab.n_owned]
        nb_ok = all(np.array_equal(mine[int(g)], ref[int(g)]) for g in owned)
        comm = slabs.TorchComm("cpu")
        for _ in range(steps):
            slabs.step_distributed(slab, comm, typ)
            whole.step(1)
        g, t, xs, vs = slab.owned_state(typ)
        pid = whole.get("ParticleIndex")
        slot = np.empty(n, np.int64)
        slot[pid] = np.arange(n)
        xo, vo = whole.get("Position")[slot[g]], whole.get("Velocity")[slot[g]]
        fluid = t < 2
        L = float(np.ptp(whole.get("Position"), axis=0).max())
        vmax = float(np.abs(whole.get("Velocity")).max())
        out[rank] = dict(nb_ok=nb_ok, owned=len(g), local=len(slab.gid), rebuilds=slab.rebuilds,
                         ref_rebuilds=int(whole.scalar("Rebuilds")), fluid=int(fluid.sum()),
                         dx=float(np.abs(xs - xo)[fluid].max(initial=0.0) / L),
                         dv=float(np.abs(vs - vo)[fluid].max(initial=0.0) / vmax))
        dist.barrier()
        slab.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,steps", [("small3d_fluid", 65), ("small3d", 10)])
def test_two_slabs_match_one_domain(name, steps):
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), name, steps, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0]["nb_ok"] and res[1]["nb_ok"], "owned particles' neighbour sets differ"
    from helpers import load_scene
    n = len(load_scene(name)[1])
    assert res[0]["owned"] + res[1]["owned"] == n  # every particle owned once
    assert res[0]["local"] > res[0]["owned"] and res[1]["local"] > res[1]["owned"]  # ghosts present
    assert res[0]["fluid"] > 0 and res[1]["fluid"] > 0  # the cut goes through the fluid
    for r in (0, 1):
        assert res[r]["rebuilds"] == res[r]["ref_rebuilds"]
        assert res[r]["dx"] <= 1e-13 and res[r]["dv"] <= 1e-11, res[r]
    if name == "small3d_fluid":
        assert res[0]["rebuilds"] >= 1  # the re-partition at a rebuild is covered


def test_slab_split_and_ghosts():
    """slabs of equal mobile-particle count; every particle owned once;
    ghosts within 2 rc + 0.1 dx, across the periodic end too"""
    import sys
    sys.path.insert(0, ROOT)
    from dem_mph_b200 import scenes, slabs
    s = scenes.small(n_debris=0)
    lo, hi = slabs.split_slabs(s.params, s.x, 3, s.type)
    G = slabs.ghost_width(s.params)
    seen = np.zeros(s.n, int)
    W = s.params.domain_max[0] - s.params.domain_min[0]
    for r in range(3):
        own, gh = slabs.slab_members(s.params, s.x, lo, hi, r, G)
        seen += own
        d = np.minimum(np.mod(lo[r] - s.x[:, 0], W), np.mod(s.x[:, 0] - hi[r], W))
        assert np.all(d[gh] < G) and not np.any(gh & own)
    assert np.all(seen == 1)
    mobile = [int(((s.type < 4) & slabs.slab_members(s.params, s.x, lo, hi, r, G)[0]).sum()) for r in range(3)]
    # a lattice plane of equal x goes to one side of a boundary
    plane = np.unique(s.x[s.type < 4, 0], return_counts=True)[1].max()
    assert max(mobile) - min(mobile) <= 2 * plane
