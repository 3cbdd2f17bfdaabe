import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests of libdmph.so")


def _ensure_built():
    """Build the oracle (gcc) and libdmph.so (nvcc) in-tree when missing or
    stale; on a machine without the toolchains the prebuilt files are used."""
    ora = os.path.join(ROOT, "oracle", "liboracle.so")
    src = os.path.join(ROOT, "oracle", "dmph_oracle.c")
    if not os.path.exists(ora) or os.path.getmtime(ora) < os.path.getmtime(src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)
    from dem_mph_b200 import build
    try:
        build.build()
    except RuntimeError as e:
        if not os.path.exists(build.LIB):
            raise
        sys.stderr.write("using prebuilt libdmph.so (%s)\n" % str(e).splitlines()[0])


_ensure_built()
