"""Build libkwave_cuda.so in-tree (k-wave-swift_b200/_build/) for sm_100a with nvcc.

    python k-wave-swift_b200/build.py [--verbose-ptxas]

The library is self-contained (static CUDA runtime) and exports only the C ABI of
include/kwave_cuda.h. Sources are compiled in parallel; a source is rebuilt when it or any
header in csrc/ or include/ is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libkwave_cuda.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_compiler() -> list[str]:
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _newest_header() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def build(verbose_ptxas: bool = False, force: bool = False, out_dir: str = OUT, defines: tuple = ()) -> str:
    """Compile every source and link the library into out_dir (defines: extra -D flags)."""
    os.makedirs(out_dir, exist_ok=True)
    lib = os.path.join(out_dir, "libkwave_cuda.so")
    nvcc = _nvcc()
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr = _newest_header()
    jobs = []
    objs = []
    for s in srcs:
        obj = os.path.join(out_dir, os.path.basename(s) + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(s), hdr):
            cmd = [nvcc, *_host_compiler(), *ARCH, *COMMON, *[f"-D{d}" for d in defines], "-c", s, "-o", obj]
            if s.endswith(".cpp"):
                cmd[cmd.index("-c"):cmd.index("-c")] = ["-x", "cu"]
            if verbose_ptxas and s.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed: " + " ".join(cmd[-3:]))
            if verbose_ptxas:
                sys.stderr.write(r.stderr)
    if jobs or not os.path.exists(lib):
        link = [nvcc, *_host_compiler(), *ARCH, "-shared", "-cudart", "static", "-o", lib, *objs]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--out", default=OUT)
    ap.add_argument("-D", dest="defines", action="append", default=[])
    a = ap.parse_args()
    print(build(a.verbose_ptxas, a.force, a.out, tuple(a.defines)))
