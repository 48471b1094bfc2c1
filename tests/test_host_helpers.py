"""Host-side helpers of the engine (csrc/kw_host.h) without a GPU: the parallel loop of the
simulation setup, the ascending mask scan that orders sensor points and source rows, and the
sensor-series transpose of the output copy (device rows [t][sensor] to the [sensor][t] output).
A small C++ program checks each against a plain loop."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "k-wave-swift_b200", "csrc")
SRC = os.path.join(ROOT, "tests", "host", "check_kw_host.cpp")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_parallel_for_mask_scan_and_series_transpose(tmp_path):
    exe = str(tmp_path / "check_kw_host")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC, SRC, "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
