"""Writes the long-horizon parity fixtures tests/golden/long_<case>.npz from the FP64 oracle.

    python tests/golden/make_long.py [--threads N] [case ...]

The cases (tests/long_cases.py) are the benchmark workloads at their own grid sizes and time
horizons; the oracle needs minutes to tens of minutes per case on a few cores, too long to run
inside the GPU test suite, so its outputs are kept here, subsampled (kept sensor rows, every
t_stride-th sample, a sub-lattice of pFinal) and rounded to float32. Test infrastructure only.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "k-wave-swift_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle  # noqa: E402
from long_cases import CASES, subsample  # noqa: E402


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("cases", nargs="*")
    a = ap.parse_args()
    for name in a.cases or list(CASES):
        case = CASES[name]
        b = case["build"]()
        t0 = time.time()
        out, loop_s = oracle.run(b, nthreads=a.threads)
        keep = subsample(case, out)
        path = os.path.join(HERE, f"long_{name}.npz")
        np.savez_compressed(path, nt=np.int64(b.grid.nt), shape=np.array(b.shape), **keep)
        print(f"{name}: nt {b.grid.nt}, oracle {time.time() - t0:.0f} s -> {os.path.basename(path)} "
              f"({os.path.getsize(path) // 1024} KB)", flush=True)


if __name__ == "__main__":
    main()
