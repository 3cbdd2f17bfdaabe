"""The bench's choice of the kernel its roofline block describes: the one with
the most device time over the timed run, from per-launch phase times and the
launch counts of the run (host logic, no GPU)."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)

N, NFS, ENTRIES = 1000, 400, 120000


def test_rare_rebuilds_leave_a_pass_on_top():
    # 300 profiled steps, 2 rebuilds; the timed run has 10,000 steps and 100 rebuilds
    ph = {"pass_a": (210.0, 300), "pass_b": (180.0, 300), "list_build": (3.0, 2), "rebuild": (4.0, 2)}
    kern, top = bench.kernel_table(ph, "fp32", N, NFS, ENTRIES, 10000, 100)
    assert top == "pass_a"
    assert abs(kern["pass_a"]["launch_ms"] - 0.7) < 1e-12
    assert abs(kern["list_build"]["run_ms"] - 150.0) < 1e-9
    assert kern["pass_a"]["bytes"] == N * (bench.algorithmic_bytes("fp32") - 24)
    assert kern["pass_b"]["bytes"] == NFS * bench.algorithmic_bytes("fp32")
    assert kern["list_build"]["bytes"] == 4 * ENTRIES + 20 * N


def test_frequent_rebuilds_put_the_list_build_on_top():
    ph = {"pass_a": (210.0, 300), "pass_b": (180.0, 300), "list_build": (450.0, 300)}
    kern, top = bench.kernel_table(ph, "fp32", N, NFS, ENTRIES, 10000, 6000)
    assert top == "list_build" and kern[top]["kernel"] == "k_build_list32"
    assert abs(kern[top]["run_ms"] - 9000.0) < 1e-9


def test_fp64_has_no_fp32_list_build_row():
    ph = {"pass_a": (500.0, 300), "pass_b": (600.0, 300), "list_build": (900.0, 300)}
    kern, top = bench.kernel_table(ph, "fp64", N, NFS, ENTRIES, 300, 300)
    assert set(kern) == {"pass_a", "pass_b"} and top == "pass_b"
    assert kern["pass_b"]["kernel"] == "k_pass_b"


def test_no_timed_phase_gives_no_top_kernel():
    kern, top = bench.kernel_table({}, "fp32", N, NFS, ENTRIES, 20, 0)
    assert kern == {} and top is None
    kern, top = bench.kernel_table({"pass_a": (0.0, 0)}, "fp64", N, NFS, ENTRIES, 20, 0)
    assert kern == {} and top is None


def test_reference_rate_adds_rebuilds_at_the_window_cadence():
    # 4 timed steps of 10 s of which one rebuild of 30 s: 7.5 s per step
    # without rebuilds; half the steps of the GPU window rebuild
    res = {"seconds": 40.0, "steps": 4, "rebuilds": 1, "rebuild_seconds": 10.0, "init_rebuild_seconds": 99.0}
    v, secs, R = bench.reference_rate(res, 1000, 4, 0.5)
    assert R == 2 and abs(secs - (4 * 7.5 + 2 * 10.0)) < 1e-12 and abs(v - 4000 / secs) < 1e-9
    # no rebuild in the timed steps: the initialisation's rebuild time is used
    res = {"seconds": 20.0, "steps": 2, "rebuilds": 0, "rebuild_seconds": 0.0, "init_rebuild_seconds": 30.0}
    v, secs, R = bench.reference_rate(res, 1000, 2, 1.0)
    assert R == 2 and abs(secs - 80.0) < 1e-12
    # no cadence known: the timed steps alone, their own rebuilds removed
    v, secs, R = bench.reference_rate(res, 1000, 2, None)
    assert R == 0 and abs(secs - 20.0) < 1e-12
