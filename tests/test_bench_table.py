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
