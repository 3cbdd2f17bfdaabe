"""Domain decomposition of one scene into x-slabs, one slab per rank.

The reference steps one scene in one process (its MPI include is commented
out, source/DEM-MPH.cpp:27); a scene too large for one GPU is split here along
x, gravity being along -y so that the slabs cut through the flow rather than
along its depth.

Each rank holds a solver context over the particles it owns (x in its slab)
and GHOSTS: the particles of the other slabs within G = 2 rc + 0.1 dx of its
slab (rc = MaxRadius + MARGIN, the list radius; periodic in x).  Two levels of
neighbours are inside G, so every pass-A result that an owned particle's
pass B reads (the pressure and, with surface tension, the attractive pressure
of a neighbour) comes out right on the rank itself, and one exchange per
step suffices:

1. the owners send the start-of-step positions and velocities of the
   particles that are ghosts elsewhere; every rank writes them into its
   ghost rows (dmph_set_rows);
2. every rank runs the drift of the step (dmph_step_begin) and the ranks
   combine their largest displacement since the last rebuild with one
   all-reduce (MAX): the reference's rebuild trigger (:1264-1286) is a
   maximum over all particles, so all ranks rebuild together, on the same
   steps as one context holding the whole scene;
3. on a rebuild step the ranks gather their owned particles, split the scene
   afresh into slabs of equal mobile (fluid and debris) particle count, and
   each creates its context over its new owned and ghost particles from the
   drifted state (the creation sorts them and builds the lists: that step's
   rebuild); then dmph_step_finish completes the step.  Between rebuilds
   every particle moves less than MARGIN / 2, so the ghosts chosen at a
   rebuild stay enough until the next.

Owned particles then follow the same arithmetic as in one context over the
whole scene, up to the order of the neighbour sums (each rank's contexts sort
only their own particles), and the neighbour sets of owned particles are the
same.  Ghost results are discarded.  Rigid debris bodies and moving walls are
not supported here (a body would span slabs; the wall centres live in the
context's clock).  Free debris follow the reference's DEM, whose contact
constants come from the last neighbour within dx in list order (:2305-2341):
with another order inside a cell those constants, and so the debris, differ
from the single-context run.

Communication: `TorchComm` (torch.distributed, gloo on the host or NCCL on the
GPUs: the exchanged arrays travel as tensors of the group's device) for one
rank per process, or `run_local`, which steps all slabs of one process in
turn and combines their results directly.
"""
import numpy as np

FLUID_END, SOLID_END = 2, 4


def ghost_width(params):
    """G = 2 rc + 0.1 dx: two levels of neighbours plus the drift a particle
    may make before the next rebuild"""
    dx = params.particle_spacing
    rc = max(params.radius_ratio_a, params.radius_ratio_p, params.radius_ratio_v) * dx + 0.1 * dx
    return 2.0 * rc + 0.1 * dx


def rebuild_threshold(params):
    """the reference's trigger: max |x - x_ref|^2 > (MARGIN / 2)^2, MARGIN = 0.1 dx"""
    margin = 0.1 * params.particle_spacing
    return 0.5 * margin * 0.5 * margin


def split_slabs(params, x, world, typ=None):
    """x-boundaries of `world` slabs holding equal numbers of mobile (fluid
    and debris) particles, whose pass B and integration make most of the
    work (all particles when typ is None or none is mobile): slab r holds
    lo[r] <= x < hi[r] (the last slab up to the domain end)"""
    xx = np.asarray(x)[:, 0]
    if typ is not None and np.any(np.asarray(typ) < SOLID_END):
        xx = xx[np.asarray(typ) < SOLID_END]
    xs = np.sort(xx)
    lo = np.empty(world)
    hi = np.empty(world)
    lo[0] = params.domain_min[0]
    hi[-1] = params.domain_max[0]
    for r in range(1, world):
        b = xs[min(len(xs) - 1, (r * len(xs)) // world)]
        lo[r] = b
        hi[r - 1] = b
    return lo, hi


def slab_members(params, x, lo, hi, r, G):
    """(owned, ghost) masks of slab r: owned lo <= x < hi; ghosts the others
    within G of the slab, measured around the periodic x extent"""
    W = params.domain_max[0] - params.domain_min[0]
    xx = np.asarray(x)[:, 0]
    last = r == len(lo) - 1
    owned = (xx >= lo[r]) & ((xx < hi[r]) | (last & (xx <= hi[r])))
    left = np.mod(lo[r] - xx, W)    # distance from x up to the slab's start
    right = np.mod(xx - hi[r], W)   # distance from the slab's end up to x
    ghost = ~owned & ((left < G) | (right < G))
    return owned, ghost


class Slab:
    """One rank's part of the scene: its owned and ghost rows (global input
    rows, gid) and the engine (a solver context, or the oracle in the CPU
    tests) over them, owned rows first."""

    def __init__(self, params, rank, world, engine_factory):
        self.params = params
        self.rank = rank
        self.world = world
        self.factory = engine_factory
        self.G = ghost_width(params)
        self.engine = None
        self.steps = 0
        self.rebuilds = 0

    def partition(self, gid, typ, x, v):
        """split the scene (all ranks' particles, in gid order) and create
        this rank's engine; records which of its owned rows are ghosts on
        other ranks (its exports)"""
        lo, hi = split_slabs(self.params, x, self.world, typ)
        owned, ghost = slab_members(self.params, x, lo, hi, self.rank, self.G)
        elsewhere = np.zeros(len(gid), bool)
        for s in range(self.world):
            if s != self.rank:
                elsewhere |= slab_members(self.params, x, lo, hi, s, self.G)[1]
        rows = np.concatenate([np.flatnonzero(owned), np.flatnonzero(ghost)])
        self.gid = np.asarray(gid)[rows]
        self.n_owned = int(owned.sum())
        self.local_of = {int(g): k for k, g in enumerate(self.gid)}
        self.export_local = np.flatnonzero(elsewhere[rows[:self.n_owned]]).astype(np.int32)
        self.ghost_local = np.arange(self.n_owned, len(rows), dtype=np.int32)
        self.bounds = (lo, hi)
        if self.engine is not None:
            self.engine.close()
        p = self.params.copy()
        p.time = self.time
        self.engine = self.factory(p, np.asarray(typ)[rows], np.asarray(x)[rows], np.asarray(v)[rows])

    @property
    def time(self):
        """Time at the start of the step in progress"""
        return self.params.time + self.steps * self.params.dt

    def exports(self):
        """(gid, x, v) of the owned particles that are ghosts elsewhere"""
        x, v = self.engine.get_rows(self.export_local)
        return self.gid[self.export_local], x, v

    def import_ghosts(self, gid, x, v):
        """write the states of this rank's ghosts from the owners' exports"""
        want = {int(g): k for k, g in enumerate(gid)}
        pick = np.array([want[int(g)] for g in self.gid[self.ghost_local]], dtype=np.int64)
        if len(pick):
            self.engine.set_rows(self.ghost_local, np.asarray(x)[pick], np.asarray(v)[pick])

    def owned_state(self, typ_of_gid):
        """(gid, type, x, v) of the owned particles (current state)"""
        rows = np.arange(self.n_owned, dtype=np.int32)
        x, v = self.engine.get_rows(rows)
        g = self.gid[:self.n_owned]
        return g, typ_of_gid[g], x, v

    def close(self):
        if self.engine is not None:
            self.engine.close()
            self.engine = None


def _concat(parts):
    """concatenate per-rank (gid, ...) tuples and order them by gid"""
    cols = [np.concatenate([np.asarray(p[k]) for p in parts]) for k in range(len(parts[0]))]
    order = np.argsort(cols[0], kind="stable")
    return [c[order] for c in cols]


class TorchComm:
    """the two collectives the slab step needs, over torch.distributed"""

    def __init__(self, device="cpu"):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.device = torch, dist, device

    def allreduce_max(self, value):
        t = self.torch.tensor([float(value)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def allgather(self, arrays):
        """list over ranks of tuples like `arrays` (arrays of one common
        length per rank)"""
        torch, dist = self.torch, self.dist
        world = dist.get_world_size()
        n = torch.tensor([len(arrays[0])], dtype=torch.int64, device=self.device)
        ns = [torch.zeros_like(n) for _ in range(world)]
        dist.all_gather(ns, n)
        ns = [int(t.item()) for t in ns]
        m = max(ns)
        out = [[None] * len(arrays) for _ in range(world)]
        for k, a in enumerate(arrays):
            a = np.asarray(a)
            pad = np.zeros((m,) + a.shape[1:], a.dtype)
            pad[:len(a)] = a
            t = torch.from_numpy(pad).to(self.device)
            bufs = [torch.empty_like(t) for _ in range(world)]
            dist.all_gather(bufs, t)
            for r in range(world):
                out[r][k] = bufs[r].cpu().numpy()[:ns[r]]
        return [tuple(o) for o in out]


def step_distributed(slab, comm, typ_of_gid):
    """one step of this rank's slab (every rank calls it, in lock step)"""
    parts = comm.allgather(slab.exports())
    slab.import_ghosts(*_concat(parts))
    m2 = slab.engine.step_begin()
    if comm.allreduce_max(m2) > rebuild_threshold(slab.params):
        # the drifted owned particles of all ranks make the new slabs; each
        # new context's creation is this step's rebuild
        g, t, x, v = _concat(comm.allgather(slab.owned_state(typ_of_gid)))
        slab.partition(g, t, x, v)
        slab.rebuilds += 1
    slab.engine.step_finish(False)
    slab.steps += 1


def run_local(slabs, typ_of_gid, nsteps):
    """nsteps steps of all slabs of this process, the collectives done
    directly (one process standing in for the ranks; no kernel of one slab
    waits on another's)"""
    for _ in range(nsteps):
        g, x, v = _concat([s.exports() for s in slabs])
        for s in slabs:
            s.import_ghosts(g, x, v)
        m2 = max(s.engine.step_begin() for s in slabs)
        if m2 > rebuild_threshold(slabs[0].params):
            g, t, x, v = _concat([s.owned_state(typ_of_gid) for s in slabs])
            for s in slabs:
                s.partition(g, t, x, v)
                s.rebuilds += 1
        for s in slabs:
            s.engine.step_finish(False)
            s.steps += 1
