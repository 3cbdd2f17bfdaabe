"""Build libdmph.so (CUDA for sm_100a + host C++) and the `dem_mph` executable.

Usage:  python -m dem_mph_b200.build [--force]

Everything is compiled in-tree: objects go to dem_mph_b200/_build/, the
library to dem_mph_b200/libdmph.so and the executable to dem_mph_b200/dem_mph.
FP64 kernels are compiled with -fmad=false so that no multiply-add is fused
(the reference's x86-64 FP64 code has none), host code with
-ffp-contract=off for the same reason.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdmph.so")
EXE = os.path.join(HERE, "dem_mph")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cuda_home():
    for c in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if c and os.path.exists(os.path.join(c, "bin", "nvcc")):
            return c
    nvcc = shutil.which("nvcc")
    if nvcc:
        return os.path.dirname(os.path.dirname(nvcc))
    raise RuntimeError("nvcc not found")


# (source, extra flags); FP32 kernels keep FMA contraction
CU_SOURCES = [
    ("dmph_f64.cu", ["-fmad=false"]),
    ("dmph_rebuild.cu", ["-fmad=false"]),
    ("dmph_api.cu", ["-fmad=false"]),
    ("dmph_f32.cu", []),
    ("dmph_noalloc.cu", ["-fmad=false"]),
    ("dmph_checkpoint.cu", ["-fmad=false"]),
    ("dmph_bodies.cu", []),
    ("dmph_mlp.cu", []),
    ("dmph_surrogate.cu", []),
]
CPP_SOURCES = ["dmph_params.cpp", "dmph_io.cpp", "dmph_bodies_io.cpp"]
HEADERS = ["dmph_device.cuh", "dmph_state.cuh", "dmph_traverse.cuh", "dmph_internal.h", "dmph_ctx.h", "dmph_mlp.h"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(force=False, verbose=False):
    cuda = _cuda_home()
    nvcc = os.path.join(cuda, "bin", "nvcc")
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "dmph.h")]
    jobs = []
    objs = []
    for src, extra in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([nvcc] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                         "-Xcompiler", "-ffp-contract=off", "-Xptxas", "-v"] + extra +
                        ["-I", CSRC, "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall",
                         "-I", os.path.join(cuda, "include"), "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                         "-c", s, "-o", o])
    logs = []
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            logs = list(ex.map(_run, jobs))
    if force or jobs or _newer(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    host_src = os.path.join(HOST, "dem_mph.cpp")
    if os.path.exists(host_src) and (force or _newer(EXE, [host_src, LIB, os.path.join(ROOT, "include", "dmph.h")])):
        _run(["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
              "-I", os.path.join(cuda, "include"), host_src, "-o", EXE, "-L", HERE, "-ldmph",
              "-L", os.path.join(cuda, "lib64"), "-lcudart", "-Wl,-rpath,$ORIGIN",
              "-Wl,-rpath," + os.path.join(cuda, "lib64")])
    if verbose:
        for l in logs:
            sys.stdout.write(l)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
