"""Benchmark of the DEM-MPH explicit timestep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config2|config1|config3|config5] [--precision fp64|fp32]

One "step" is one explicit timestep of the whole scene (the reference main
loop body, source/DEM-MPH.cpp:450-579): drift, walls, periodic wrap, the
rebuild trigger (and a neighbour rebuild when it fires), the density and
pressure pass, the force pass with drag/buoyancy/gravity and the fluid
update, and the DEM substeps.  The workload is the 3D dam break with debris
of dem_mph_b200.scenes (config2: 3.2 x 1.0 x 1.0 m tank at 5 mm, ~1.2 M
fluid + ~1.4 M wall particles + 200 debris bodies; seeded synthetic
particles, since the reference ships no such scene).

Metric: particle-steps/s = N_total x steps / device seconds (whole job, all
ranks; inputs resident in HBM).  Multi-GPU: every rank advances its own
independent seeded replica (weak scaling, no data-path collective); time is
the max over ranks.  Rank 0 prints one JSON line.

`--impl reference` times the reference's own CPU implementation (built from
its source into oracle/_ref/ by oracle/Makefile) on this machine's host cores
with all OpenMP threads, on a bounded number of steps of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}

# Untimed steps before the warm-up, per workload.  Config 2's configured run
# (10,000 steps, CUDA events per 250-step block) rebuilds every ~16 steps at
# first, every 2nd step from step ~2,450 (2.2 ms/step) and every step from
# step ~6,450 on (3.3 ms/step), 6,219 rebuilds and 2.49 ms/step on average.
# A short timed window therefore settles into the late flow, the costliest
# regime of the run, so that it does not overstate the run.
SETTLE_DEFAULT = {"config2": 7000, "config1": 200, "config3": 200, "config5": 2000}
WINDOW = {"config2": "late flow after 7,000 settle steps: a neighbour rebuild every step, the costliest regime of "
                     "the 10,000-step configured run (which rebuilds in 62% of its steps)"}
# Rebuild fraction of the timed window that SETTLE_DEFAULT leads to, as the
# GPU arm measures it (run.rebuild_fraction_timed); the reference arm, which
# cannot settle thousands of steps on the host, adds its own timed neighbour
# rebuild at this cadence.  None: no rebuild added.
WINDOW_REBUILD_FRACTION = {"config2": 1.0, "config1": None}
# networks trained on the config-4 corpus (bench.py --corpus --save-weights),
# by surrogate K
CORPUS_WEIGHTS = {8: "dem_mph_b200/weights/surrogate_config4_k8.npy"}
# the reference arm times at most this many steps (each config-2 step takes
# seconds on the host); fewer than requested are reported as such
REFERENCE_MAX_STEPS, REFERENCE_MAX_WARMUP = 30, 5


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


def max_over_ranks(x, world, device):
    """the largest value over the ranks (timings are taken as the slowest
    rank's); a plain float with one rank"""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_scene(workload, rank):
    from dem_mph_b200 import scenes
    seed = 1234 + rank
    if workload == "config1":
        return scenes.config1(seed=seed)
    if workload == "config2":
        return scenes.config2(seed=seed)
    if workload == "config5":
        return scenes.config5(seed=seed)
    raise ValueError(workload)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region"""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        try:
            for line in open(self.path):
                f = [s.strip() for s in line.split(",")]
                if len(f) < 9:
                    continue
                sm.append(float(f[1]))
                mx.append(float(f[2]))
                for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                      "sw_power_cap"), f[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_time(scene, steps, warmup, threads=None):
    """Time the reference's own step (oracle/_ref/ref_dump3d --bench: the
    reference's functions called in its main-loop order) on the host cores."""
    from dem_mph_b200 import files
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_dump3d")
    if not os.path.exists(exe):
        return None, "oracle/_ref/ref_dump3d not built"
    with tempfile.TemporaryDirectory() as tmp:
        data, grid = os.path.join(tmp, "dem.data"), os.path.join(tmp, "scene.grid")
        files.write_data_file(data, scene.params)
        files.write_grid(grid, scene.params, scene.type, scene.x, scene.v)
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        r = subprocess.run([exe, "--bench", data, grid, str(steps), str(warmup)], capture_output=True, text=True,
                           env=env)
        if r.returncode != 0:
            return None, "reference run failed: " + r.stderr[-200:]
        line = [l for l in r.stdout.splitlines() if l.startswith("{")][-1]
        return json.loads(line), None


def workload_config(scene, args, world):
    """The `config` object of both arms' JSON lines: what the workload is,
    with nothing that depends on the run (those facts go under `run`), so
    the reference arm states the very same dict."""
    c = scene.counts()
    p = scene.params
    bodies = not args.no_bodies and len(scene.body_density) > 0
    ours = ("FP32 split pair forces on cell-relative positions, FP64 rigid-body debris (DEM contacts and "
            "body update)" if args.precision == "fp32" else "FP64 throughout (the parity build)")
    ours += "; debris as rigid bodies" if bodies else "; debris as individual DEM particles"
    if list_reuse_on(args, scene):
        ours += ("; the reference's rebuild trigger refreshes the trigger positions and neighbour counts every "
                 "time, the cell sort and Verlet lists (skin up to 0.4 dx) are remade only when they could "
                 "miss a pair (list reuse)")
    return {"workload": scene.name, "n_particles": c["total"], "n_fluid": c["fluid"], "n_solid": c["solid"],
            "n_wall": c["wall"], "n_debris_bodies": len(scene.body_density), "dt": p.dt,
            "dem_substeps": int(p.dt / p.dem_dt), "settle_steps": args.settle,
            "window": WINDOW.get(args.workload, "after %d settle steps" % args.settle),
            "arms": {"ours": ours + "; neighbour rebuild triggers by the reference's test",
                     "reference": "the reference's own CPU step (FP64, debris as individual DEM particles: it "
                                  "has no rigid bodies) on all host cores, its neighbour rebuild timed and "
                                  "added at the GPU window's cadence"},
            "parallelism": "replicas x%d" % world,
            "l2": "inputs larger than L2 (particle state alone %.0f MB)" % (c["total"] * 60 / 1e6)}


def list_reuse_on(args, scene):
    """list reuse (DMPH_FLAG_LIST_REUSE) in the GPU arm: FP32 split build,
    debris as rigid bodies or none, unless --no-list-reuse"""
    bodies = not args.no_bodies and len(scene.body_density) > 0
    return (args.precision == "fp32" and not getattr(args, "no_list_reuse", False)
            and (bodies or len(scene.body_density) == 0))


def reference_rate(res, n, steps, rebuild_fraction):
    """Reference particle-steps/s over `steps` steps with a neighbour rebuild
    in `rebuild_fraction` of them: the timed steps without their own
    rebuilds, plus that many rebuilds at the measured rebuild time (the mean
    of the timed steps' rebuilds, else the initial one).  Returns (value,
    seconds, rebuilds added)."""
    t_steps = res["seconds"] - res.get("rebuild_seconds", 0.0)
    t_reb = (res["rebuild_seconds"] / res["rebuilds"] if res.get("rebuilds") else res.get("init_rebuild_seconds",
                                                                                         0.0))
    per_step = t_steps / res["steps"]
    R = 0 if rebuild_fraction is None else int(round(rebuild_fraction * steps))
    secs = per_step * steps + R * t_reb
    return n * steps / secs, secs, R


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# list-mode kernels on config 2, FP32 split, late in the flow (after 6,000
# steps), from ncu captures of the bench's own command
TRAFFIC_CONFIG2_FP32 = {"pass_a": 765.5e6, "pass_b": 690.9e6, "list_build": 824.2e6}
# DRAM bytes per launch of the ensemble's shared pass launches on config 3
# (one launch each, after the bench's settle steps); empty until captured
TRAFFIC_CONFIG3 = {"pass_a": 3629.5e6, "pass_b": 3237.3e6}
TRAFFIC_SOURCE_CONFIG3 = "ncu capture of one launch of each ensemble pass kernel on config 3"
# the same with list reuse (lists with a skin of up to 0.4 dx, cells 3.5 dx)
TRAFFIC_CONFIG2_FP32_REUSE = {"pass_a": 959.6e6, "pass_b": 868.4e6, "list_build": 1064.7e6}
TRAFFIC_SOURCE = "ncu capture of one launch of the same kernel and workload in the late flow"


def algorithmic_bytes(prec):
    """Compulsory HBM bytes per particle of the dominant kernel (pass B) with
    neighbour re-reads served on chip: read position, velocity, pressure and
    type, write force and (fluid) velocity."""
    if prec == "fp64":
        return 24 + 24 + 8 + 4 + 24 + 24
    return 16 + 16 + 4 + 16 + 16


def kernel_table(ph, precision, n, n_fs, entries, steps, rebuilds):
    """Per-kernel figures for the roofline block and the kernel with the most
    device time over the timed run.

    ph: {phase: (total_ms, launches)} of the profiled steps; n particles, n_fs
    fluid and debris; entries: list entries of all particles; steps and
    rebuilds of the timed run.  Each kernel gets its mean launch time, its
    time over the timed run (launch time x launches in the run), and its
    compulsory HBM bytes per launch: pass B reads p4, v4 and pressure and
    writes force and velocity of the fluid and debris; pass A reads p4 and v4
    and writes pressure and the divergence terms of every particle; the list
    build writes every list entry (4 B) and count (4 B) and reads each
    particle's position once (16 B).  Returns (table, name of the top kernel),
    the name None when no phase was timed.
    """
    bpp = algorithmic_bytes(precision)
    kern = {}
    for ph_name, kname, nbytes, n_launch in (
            ("pass_a", "k_pass_a32_list", n * (bpp - 24), steps),
            ("pass_b", "k_pass_b32_list", n_fs * bpp, steps),
            ("list_build", "k_build_list32", 4 * entries + 20 * n, rebuilds)):
        tot, cnt = ph.get(ph_name, (0.0, 0))
        if cnt == 0 or (ph_name == "list_build" and precision != "fp32"):
            continue
        if precision != "fp32":
            kname = "k_" + ph_name
        kern[ph_name] = {"kernel": kname, "launch_ms": tot / cnt, "bytes": nbytes,
                         "run_ms": tot / cnt * n_launch}
    if not kern:
        return kern, None
    return kern, max(kern, key=lambda k: kern[k]["run_ms"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: the configured run, 10000 for config 2, 2000 for config 1, "
                         "300 for config 3, 1000 for config 5)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config2", choices=["config2", "config1", "config3", "config5"])
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--settle", type=int, default=None,
                    help="untimed steps run before warm-up (default per workload: 7000 for config2, the late flow; "
                         "2000 for config5; 200 otherwise)")
    ap.add_argument("--no-graph", action="store_true", help="launch kernels one by one instead of graph replay")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch variants of the pair passes")
    ap.add_argument("--profiler-range", action="store_true",
                    help="open the CUDA profiler range around the timed steps only (ncu --profile-from-start off)")
    ap.add_argument("--variants", type=int, nargs=2, default=None, metavar=("A", "B"),
                    help="set the pair-pass launch variants (pass A, pass B) instead of autotuning")
    ap.add_argument("--surrogate", action="store_true",
                    help="plain vs surrogate sim-s/hour and surge-front / debris-centroid error (config1 by default)")
    ap.add_argument("--substeps", type=int, default=8, help="surrogate K")
    ap.add_argument("--corpus", action="store_true",
                    help="build the config-4 training corpus, train the surrogate on it, judge it held out")
    ap.add_argument("--save-weights", default=None, help="--corpus: write the trained weights (.npy) here")
    ap.add_argument("--weights", default=None,
                    help="--surrogate: start from these weights (.npy; default for K = 8: the config-4 corpus network)")
    ap.add_argument("--online-only", action="store_true",
                    help="--surrogate: no corpus network, train on the run's own first blocks only")
    ap.add_argument("--pretrain-iters", type=int, default=None,
                    help="--surrogate: Adam iterations on the run's own first blocks (default 2000, 0 with --weights)")
    ap.add_argument("--corpus-scenes", type=int, default=32)
    ap.add_argument("--corpus-steps", type=int, default=4000)
    ap.add_argument("--train-iters", type=int, default=20000)
    ap.add_argument("--sg-tolerance", type=float, default=0.5,
                    help="surrogate judge tolerance on the velocity-increment error of a judged block (a guard "
                         "against a network that has lost the flow)")
    ap.add_argument("--front-tolerance", type=float, default=0.02,
                    help="surrogate judge on the surge front: fall back when its estimated deviation exceeds "
                         "this fraction of its travel (0: off)")
    ap.add_argument("--no-bodies", action="store_true",
                    help="move debris particles individually (reference DEM) instead of as rigid bodies")
    ap.add_argument("--no-list-reuse", action="store_true",
                    help="remake the cell sort and Verlet lists at every rebuild trigger (FP32 build)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.settle is None:
        args.settle = SETTLE_DEFAULT.get(args.workload, 200)
    if args.steps is None:
        args.steps = 2000 if args.surrogate else {"config2": 10000, "config1": 2000, "config3": 300,
                                                  "config5": 1000}[args.workload]

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from dem_mph_b200 import solver
    from dem_mph_b200.abi import FLAG_LIST_REUSE, PRECISION_FP64, PRECISION_FP32_SPLIT

    if args.workload == "config3":
        return run_ensemble(args, rank, world)
    if args.surrogate:
        return run_surrogate(args, rank, world)
    if args.corpus:
        return run_corpus(args, rank, world)
    scene = make_scene(args.workload, rank)
    p = scene.params.copy()
    p.precision = PRECISION_FP64 if args.precision == "fp64" else PRECISION_FP32_SPLIT
    if list_reuse_on(args, scene):
        p.flags |= FLAG_LIST_REUSE
    g = solver.Solver(p, scene.type, scene.x, scene.v)
    bodies = not args.no_bodies and len(scene.body_density) > 0
    if bodies:
        g.set_bodies(scene.body, scene.body_density)
    n = scene.n
    # the list-build autotuner times real rebuilds while stepping: its steps
    # are the last of the settle steps
    tune_build = args.precision == "fp32" and not args.no_autotune and args.settle >= 60
    g.step(args.settle - (30 if tune_build else 0))
    build_variant = None
    if tune_build:
        build_variant, build_ms = g.autotune_list_build(10)
        build_variant = {"variant": build_variant, "list_build_ms": [round(float(x), 4) for x in build_ms]}
    variants = None
    if args.variants is not None:
        g.set_variants(*args.variants)
        variants = list(args.variants)
    elif args.precision == "fp32" and not args.no_autotune:
        va, vb, _, _ = g.autotune()
        variants = [va, vb]
    if not args.no_graph:
        g.set_graph(True)
    g.step(args.warmup)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- timed region: K steps, device time on the solver's stream
    barrier()
    torch.cuda.synchronize()
    l0 = g.info().kernel_launches
    rebuilds_before = int(g.info().rebuilds)
    builds_before = g.rebuild_stats()[1]
    if args.profiler_range:
        torch.cuda.profiler.start()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = g.step_timed(args.steps)
        torch.cuda.synchronize()
    if args.profiler_range:
        torch.cuda.profiler.stop()
    barrier()
    inf_t = g.info()
    launches = int(inf_t.kernel_launches - l0)
    rebuilds_timed = int(inf_t.rebuilds) - rebuilds_before
    builds_timed = g.rebuild_stats()[1] - builds_before
    ms_max = max_over_ranks(ms, world, "cuda")
    value = n * world * args.steps / (ms_max / 1e3)

    # ---- per-phase device times (separate pass, events around each phase,
    # over the next 300 steps at most, in the same flow regime)
    prof_steps = min(args.steps, 300)
    g.set_profiling(True)
    g.step(prof_steps)
    ph = g.phase_times()
    g.set_profiling(False)
    inf = g.info()
    n_fs = inf.n_fluid + inf.n_solid
    ea, eb = g.list_stats()
    # the list build runs at the full rebuilds only (all of them without list reuse)
    roofline = roofline_block(ph, args, n, n_fs, ea, eb, builds_timed, prof_steps, list_reuse_on(args, scene))

    # ---- end to end through the C ABI with host buffers: every step uploads
    # the particle state from pinned host memory, steps, reads it back
    host = (torch.empty(n, dtype=torch.int32, pin_memory=True).numpy(),
            torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy(),
            torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy(),
            torch.empty(n, dtype=torch.int32, pin_memory=True).numpy())
    _, x_h, v_h, _ = g.state(out=host)
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        g.set_state(x_h, v_h)
        g.step(1)
        g.state(out=host)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e = {"value": n * world * e2e_steps / max_over_ranks(e2e_s, world, "cuda"), "unit": "particle-steps/s",
           "h2d_bytes_per_step": int(n * 48), "d2h_bytes_per_step": int(n * 48 + n * 8),
           "steps": e2e_steps}
    g.close()

    frac_timed = rebuilds_timed / args.steps
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res, why = reference_time(scene, 1, 0)
        if res:
            v, _, R = reference_rate(res, res["particles"], 1, frac_timed)
            cpu = {"value": v, "unit": "particle-steps/s", "cores": res["threads"], "kind": "reference",
                   "sample": "1 reference step of the same scene after its initialisation, plus its neighbour "
                             "rebuild (calculateCellParticle + calculateNeighbor, %.2f s, timed in the "
                             "initialisation) at the timed window's cadence of %.2f rebuilds per step"
                             % (res.get("init_rebuild_seconds", 0.0), frac_timed)}
        else:
            cpu = {"value": None, "unit": "particle-steps/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": why}

    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded dam break with debris, dem_mph_b200.scenes)",
        "config": workload_config(scene, args, world),
        "run": {"rebuilds_in_timed_steps": rebuilds_timed, "rebuild_fraction_timed": frac_timed,
                "list_reuse": list_reuse_on(args, scene), "list_builds_in_timed_steps": builds_timed,
                "timed_from_step": args.settle + args.warmup, "graph_replay": not args.no_graph,
                "pass_variants": variants, "list_build_variant": build_variant, "precision": args.precision,
                "debris": "rigid bodies (FP64)" if bodies else "individual DEM particles"},
        "sim_s_per_hour": p.dt * args.steps / (ms_max / 1e3) * 3600.0,
        "clocks": clk.summary(),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def roofline_block(ph, args, n, n_fs, ea, eb, builds_timed, prof_steps, reuse=False):
    """The roofline object for the kernel with the most device time over the
    timed run, with the other timed kernels beside it; None when no phase was
    timed.  builds_timed: list builds in the timed steps; reuse: list reuse
    on (longer lists: the traffic table's captures were made without it)."""
    peaks, peak_src = load_peaks()
    kern, top = kernel_table(ph, args.precision, n, n_fs, ea, args.steps, builds_timed)
    if top is None:
        return None
    dur = kern[top]["launch_ms"]
    achieved = kern[top]["bytes"] / (dur / 1e3) / 1e9
    # DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
    # an ncu capture of the same kernels on config 2 in the late flow
    traffic_tab = {}
    if args.workload == "config2" and args.precision == "fp32":
        traffic_tab = TRAFFIC_CONFIG2_FP32_REUSE if reuse else TRAFFIC_CONFIG2_FP32
    # pair work: Verlet-list entries each pass walks per launch (each entry is
    # one candidate pair: two 16-byte neighbour gathers and the pair arithmetic)
    pa_dur = kern["pass_a"]["launch_ms"] if "pass_a" in kern else float("nan")
    pb_dur = kern["pass_b"]["launch_ms"] if "pass_b" in kern else float("nan")
    pairs = {"pass_a": {"entries_per_launch": ea, "launch_ms": pa_dur, "entries_per_s": ea / (pa_dur / 1e3)},
             "pass_b": {"entries_per_launch": eb, "launch_ms": pb_dur, "entries_per_s": eb / (pb_dur / 1e3)}}
    return {"bound": "hbm", "kernel": kern[top]["kernel"],
            "achieved": achieved, "peak": peaks["hbm_gbs"],
            "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic_tab.get(top),
            "traffic_source": TRAFFIC_SOURCE if traffic_tab.get(top) else None,
            "peak_source": peak_src, "launch_ms": dur,
            "algorithmic_bytes_per_launch": kern[top]["bytes"],
            "kernels": {k: {"kernel": v["kernel"], "launch_ms": v["launch_ms"],
                            "ms_over_timed_run": v["run_ms"],
                            "achieved_gbs": v["bytes"] / (v["launch_ms"] / 1e3) / 1e9,
                            "traffic": traffic_tab.get(k)}
                        for k, v in kern.items()},
            "phase_ms_per_step": {k: v[0] / max(prof_steps, 1) for k, v in ph.items()},
            "phase_steps": prof_steps,
            "pairs": pairs}


def run_surrogate(args, rank, world):
    """Plain solver against the learned K-step surrogate on the same scene and
    the same span of simulated time: both start from the initial state; the
    surrogate run first advances `settle` plain steps, collects 480 steps of
    training blocks and trains (reported separately as a one-off cost), then
    advances by judged surrogate calls (with any fallback blocks and their
    training inside the timed span).  Errors: 99th-percentile fluid x (the
    surge front) relative to the plain run's front travel, and debris body
    centroids relative to the tank length.  Wall-clock timing around
    synchronised calls: the surrogate driver reads its decisions on the host."""
    import numpy as np
    import torch
    from dem_mph_b200 import solver
    from dem_mph_b200.abi import PRECISION_FP32_SPLIT

    wl = "config1" if args.workload == "config2" and "--workload" not in sys.argv else args.workload
    scene = make_scene(wl, rank)
    K = args.substeps
    settle = args.settle if "--settle" in sys.argv else SETTLE_DEFAULT.get(wl, 200)
    weights = args.weights
    if weights is None and not args.online_only and K in CORPUS_WEIGHTS:
        weights = os.path.join(ROOT, CORPUS_WEIGHTS[K])
    # the surrogate's blocks follow the settle and collection steps
    total = max(args.steps, 2000, settle + 480 + 100 * K)

    def make():
        p = scene.params.copy()
        p.precision = PRECISION_FP32_SPLIT
        g = solver.Solver(p, scene.type, scene.x, scene.v)
        if len(scene.body_density):
            g.set_bodies(scene.body, scene.body_density)
        return g

    def front(g):
        t, x, _, _ = g.state()
        return float(np.quantile(x[t < 2, 0], 0.99))

    a = make()
    a.set_graph(True)
    f0 = front(a)
    c0 = a.bodies()["X"].copy() if len(scene.body_density) else None
    a.step(args.warmup)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.step(total - args.warmup)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    fa = front(a)
    ca = a.bodies()["X"].copy() if c0 is not None else None
    dt = scene.params.dt

    b = make()
    vtol = args.sg_tolerance
    b.enable_surrogate(substeps=K, check_interval=50, tolerance=vtol, front_tolerance=args.front_tolerance,
                       fallback_blocks=20, train_iters_per_block=20)
    if weights:
        # a network trained beforehand on the config-4 corpus
        b.set_surrogate_weights(np.load(weights))
    b.step(settle)
    nb_collect = 480 // K
    b.surrogate_collect(nb_collect)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    pre = args.pretrain_iters if args.pretrain_iters is not None else (0 if weights else 2000)
    losses = [b.surrogate_train(200) for _ in range(pre // 200)]
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    done = settle + nb_collect * K
    nblocks = (total - done) // K
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    b.surrogate_advance(nblocks)
    torch.cuda.synchronize()
    t_sg = time.perf_counter() - t2
    b.step(total - done - nblocks * K)
    st = b.surrogate_stats()
    fb = front(b)
    cb = b.bodies()["X"].copy() if c0 is not None else None
    plain_rate = (total - args.warmup) * dt / t_plain * 3600.0
    sg_rate = nblocks * K * dt / t_sg * 3600.0
    front_err = abs(fb - fa) / max(fa - f0, 1e-9)
    L = float(np.ptp(scene.x[:, 0]))
    cent_err = float(np.linalg.norm(cb - ca, axis=1).max()) if c0 is not None else 0.0
    out = {
        "metric": "sim-s/hour (surrogate-accelerated)", "value": sg_rate, "unit": "sim-s/hour", "n_gpus": world,
        "steps": total, "warmup": args.warmup, "ms_per_step": 1e3 * t_sg / max(nblocks * K, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 MLP + f32/f64 solver",
        "data": "synthetic (seeded dam break with debris, dem_mph_b200.scenes)",
        "config": {"workload": scene.name, "n_particles": scene.n, "substeps_K": K, "check_interval": 50,
                   "tolerance": vtol, "front_tolerance": args.front_tolerance,
                   "settle_steps": settle, "collect_steps": nb_collect * K,
                   "surrogate_blocks": nblocks, "dt": dt,
                   "weights": os.path.relpath(weights, ROOT) if weights else "trained on this run's first blocks",
                   "pretrain_iters": pre},
        "plain_sim_s_per_hour": plain_rate, "speedup_vs_plain": sg_rate / plain_rate,
        "front_error_rel_travel": front_err, "front_plain_m": fa, "front_surrogate_m": fb, "front_start_m": f0,
        "debris_centroid_error_max_m": cent_err, "debris_centroid_error_rel_tank": cent_err / L,
        "train_seconds_before_advance": t_train,
        "train_loss_first_last": [losses[0], losses[-1]] if losses else None,
        "surrogate_stats": st, "cpu_baseline": None, "roofline": None, "e2e": None,
        "timing": "wall clock around synchronised calls",
    }
    # the surrogate network's forward pass alone (device time): on the rows of
    # this run's calls, and on config 2's 1.23 M fluid and debris rows
    peaks, peak_src = load_peaks()
    flop_row = 2 * (64 * 128 + 128 * 128 + 128 * 128 + 128 * 16)
    inf_b = b.info()

    def mlp_line(g, rows):
        fused = g.mlp_forward_ms(rows, reps=20)
        layers = g.mlp_forward_ms(rows, reps=20, layers=True)
        tf = rows * flop_row / (fused / 1e3) / 1e12
        return {"rows": rows, "fused_ms": fused, "per_layer_gemms_ms": layers,
                "fused_tflops": tf, "frac_of_bf16_peak": tf / (peaks["bf16_tflops"]),
                "flop_per_row": flop_row}
    mlp = {"workload_rows": mlp_line(b, inf_b.n_fluid + inf_b.n_solid)}
    a.close()
    b.close()
    big = make_scene("config2", rank)
    p2 = big.params.copy()
    p2.precision = PRECISION_FP32_SPLIT
    g2 = solver.Solver(p2, big.type, big.x, big.v)
    g2.set_bodies(big.body, big.body_density)
    g2.enable_surrogate(substeps=K)
    inf2 = g2.info()
    mlp["config2_rows"] = mlp_line(g2, inf2.n_fluid + inf2.n_solid)
    g2.close()
    mlp["peak_source"] = peak_src
    out["mlp_forward"] = mlp
    if rank == 0:
        print(json.dumps(out))


def run_corpus(args, rank, world):
    """Config 4: the surrogate's training corpus (seeded config-1-type scenes
    at 8.8 mm, ~250k particles, `--corpus-steps` solver steps each recorded
    in K-step blocks), one network trained on it on the GPU (Adam, batch
    262,144), judged on held-out scenes: the K-step velocity-increment error
    with the network and without it (constant acceleration over the block).
    Wall clock around synchronised calls."""
    import torch
    from dem_mph_b200 import corpus, scenes

    K = args.substeps
    sc = scenes.config4(seed=1234 + rank, n_scenes=args.corpus_scenes)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    X, T = corpus.build(sc, steps=args.corpus_steps, substeps=K, rows_per_scene=131072)
    t1 = time.perf_counter()
    w, losses = corpus.train(sc[0], X, T, iters=args.train_iters, substeps=K, batch=262144)
    t2 = time.perf_counter()
    if args.save_weights and rank == 0:
        np.save(args.save_weights, w)
    held = {"config1": scenes.config1(), "config4_unseen": scenes.config4(seed=999, n_scenes=1)[0]}
    ev = {}
    for name, s in held.items():
        e_net, e_none = corpus.evaluate(s, w, substeps=K)
        ev[name] = {"error_with_network": e_net, "error_without": e_none, "gain": e_none / max(e_net, 1e-30)}
    out = {"metric": "K-step velocity-increment error, held-out config 1 (surrogate trained on the config-4 corpus)",
           "value": ev["config1"]["error_with_network"], "unit": "relative L2", "n_gpus": world,
           "higher_is_better": False, "vs_baseline": None, "dtype": "bf16 MLP (FP32 Adam)",
           "data": "synthetic (seeded dam breaks, dem_mph_b200.scenes.config4)",
           "config": {"workload": "config4_corpus_%d_scenes" % len(sc), "scene_particles":
                      [int(min(s.n for s in sc)), int(max(s.n for s in sc))], "steps_per_scene": args.corpus_steps,
                      "substeps_K": K, "rows": int(len(X)), "train_iters": args.train_iters, "batch": 262144},
           "corpus_seconds": t1 - t0, "train_seconds": t2 - t1, "loss_every_1000": losses, "held_out": ev,
           "timing": "wall clock around synchronised calls"}
    if rank == 0:
        print(json.dumps(out))


def run_ensemble(args, rank, world):
    """Config 3: 64 independent scenes of uneven size advanced as one ensemble
    (FP32 split, rigid bodies): pass A and pass B of all scenes are one
    persistent launch each and a whole ensemble step is one CUDA graph."""
    import torch
    import torch.distributed as dist
    from dem_mph_b200 import scenes, solver
    from dem_mph_b200.abi import PRECISION_FP32_SPLIT

    sc = scenes.config3(seed=1234 + rank)
    sv = []
    for s in sc:
        p = s.params.copy()
        p.precision = PRECISION_FP32_SPLIT
        g = solver.Solver(p, s.type, s.x, s.v)
        if len(s.body_density):
            g.set_bodies(s.body, s.body_density)
        sv.append(g)
    ens = solver.Ensemble(sv)
    n = sum(s.n for s in sc)
    ens.step(args.settle)
    variants = None
    if not args.no_autotune:
        va, vb, _, _ = ens.autotune()
        variants = [va, vb]
    ens.set_graph(not args.no_graph)
    ens.step(args.warmup)

    def barrier():
        if world > 1:
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    l0 = ens.info()["kernel_launches"] + sum(g.info().kernel_launches for g in sv)
    if args.profiler_range:
        torch.cuda.profiler.start()
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = ens.step_timed(args.steps)
        torch.cuda.synchronize()
    if args.profiler_range:
        torch.cuda.profiler.stop()
    barrier()
    launches = ens.info()["kernel_launches"] + sum(g.info().kernel_launches for g in sv) - l0
    ms_max = max_over_ranks(ms, world, "cuda")
    value = n * world * args.steps / (ms_max / 1e3)
    peaks, peak_src = load_peaks()
    bpp = algorithmic_bytes("fp32")
    achieved = n * bpp / (ms_max / args.steps / 1e3) / 1e9
    # per-kernel device times of the two shared pass launches (events around
    # each, no graph replay) over the next steps
    prof_steps = min(args.steps, 50)
    ens.set_profiling(True)
    ens.step(prof_steps)
    ph = ens.phase_times()
    ens.set_profiling(False)
    n_fs = int(sum(s.counts()["fluid"] + s.counts()["solid"] for s in sc))
    kern, top = kernel_table(ph, "fp32", n, n_fs, 0, prof_steps, 0)
    ens_names = {"pass_a": "k_ens_pass_list<0>", "pass_b": "k_ens_pass_list<1>"}
    if top is not None:
        k = kern[top]
        ach_k = k["bytes"] / (k["launch_ms"] / 1e3) / 1e9
        roof = {"bound": "hbm", "kernel": ens_names[top], "achieved": ach_k, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": ach_k / peaks["hbm_gbs"], "traffic": TRAFFIC_CONFIG3.get(top),
                "traffic_source": TRAFFIC_SOURCE_CONFIG3 if TRAFFIC_CONFIG3.get(top) else None,
                "peak_source": peak_src, "launch_ms": k["launch_ms"], "algorithmic_bytes_per_launch": k["bytes"],
                "kernels": {name: {"kernel": ens_names[name], "launch_ms": v["launch_ms"],
                                   "achieved_gbs": v["bytes"] / (v["launch_ms"] / 1e3) / 1e9,
                                   "traffic": TRAFFIC_CONFIG3.get(name)} for name, v in kern.items()},
                "whole_step": {"achieved_gbs": achieved, "frac": achieved / peaks["hbm_gbs"],
                               "algorithmic_bytes_per_step": n * bpp}}
    else:
        roof = {"bound": "hbm", "kernel": "whole ensemble step", "achieved": achieved, "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": None, "peak_source": peak_src}
    # end to end: per step, upload every scene's state from pinned host memory,
    # one ensemble step, read every scene's state back
    host = []
    for g in sv:
        host.append((torch.empty(g.n, dtype=torch.int32, pin_memory=True).numpy(),
                     torch.empty((g.n, 3), dtype=torch.float64, pin_memory=True).numpy(),
                     torch.empty((g.n, 3), dtype=torch.float64, pin_memory=True).numpy(),
                     torch.empty(g.n, dtype=torch.int32, pin_memory=True).numpy()))
        g.state(out=host[-1])
    e2e_steps = 3
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for g, h in zip(sv, host):
            g.set_state(h[1], h[2])
        ens.step(1)
        for g, h in zip(sv, host):
            g.state(out=h)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_max = max_over_ranks(e2e_s, world, "cuda")
    dts = [s.params.dt for s in sc]
    out = {
        "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded ensemble of dam breaks, dem_mph_b200.scenes.config3)",
        "config": {"workload": "config3_ensemble_64_scenes", "n_scenes": len(sc), "n_particles": n,
                   "scene_particles_min": min(s.n for s in sc), "scene_particles_max": max(s.n for s in sc),
                   "n_debris_bodies": int(sum(len(s.body_density) for s in sc)), "precision": "fp32",
                   "dt_range": [min(dts), max(dts)], "settle_steps": args.settle,
                   "graph_replay": not args.no_graph, "pass_variants": variants,
                   "parallelism": "replicas x%d" % world,
                   "l2": "inputs larger than L2 (particle state alone %.0f MB)" % (n * 60 / 1e6)},
        "clocks": clk.summary(),
        "roofline": roof,
        "cpu_baseline": None,
        "e2e": {"value": n * world * e2e_steps / e2e_max, "unit": "particle-steps/s",
                "h2d_bytes_per_step": int(n * 48), "d2h_bytes_per_step": int(n * 56), "steps": e2e_steps},
        "gpu_launches": int(launches),
    }
    ens.close()
    for g in sv:
        g.close()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU step on this box's cores,
    on the same workload and config as the GPU arm.  It times the requested
    steps after the requested warm-up (at most REFERENCE_MAX_STEPS and
    REFERENCE_MAX_WARMUP, each config-2 step taking seconds), starting from
    the scene's initial state: it cannot settle thousands of steps on the
    host.  To stand for the GPU arm's window it replaces the rebuilds of its
    own timed steps by its neighbour rebuild, timed, at the cadence of that
    window (WINDOW_REBUILD_FRACTION)."""
    if rank != 0:
        return
    scene = make_scene(args.workload, 0)
    steps = max(1, min(args.steps, REFERENCE_MAX_STEPS))
    warm = min(args.warmup, REFERENCE_MAX_WARMUP)
    res, why = reference_time(scene, steps, warm)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    frac = WINDOW_REBUILD_FRACTION.get(args.workload)
    v, secs, R = reference_rate(res, res["particles"], steps, frac)
    t_reb = res["rebuild_seconds"] / res["rebuilds"] if res.get("rebuilds") else res.get("init_rebuild_seconds")
    sample = ("%d reference steps after %d warm-up from the initial state, without the %d rebuilds they met, plus "
              "%d neighbour rebuilds (calculateCellParticle + calculateNeighbor) of %.2f s each: the GPU window's "
              "cadence" % (res["steps"], warm, res["rebuilds"], R, t_reb or 0.0))
    out = {"impl": "reference", "metric": "particle-steps/s", "value": v, "unit": "particle-steps/s",
           "n_gpus": world, "steps": res["steps"], "warmup": warm, "ms_per_step": secs * 1e3 / res["steps"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded dam break with debris, dem_mph_b200.scenes)",
           "config": workload_config(scene, args, world),
           "run": {"rebuilds_added": R, "rebuild_seconds_each": t_reb, "rebuilds_met_in_timed_steps": res["rebuilds"],
                   "step_seconds_without_rebuild": (res["seconds"] - res.get("rebuild_seconds", 0.0)) / res["steps"],
                   "threads": res["threads"]},
           "cpu_baseline": {"value": v, "unit": "particle-steps/s", "cores": res["threads"], "kind": "reference",
                            "sample": sample},
           "e2e": {"value": v, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
