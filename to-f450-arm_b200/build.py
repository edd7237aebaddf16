"""Build libtof.so (sm_100a) in-tree with nvcc.

    python to-f450-arm_b200/build.py [-v]

Compiles every .cu under csrc/ for compute_100a/sm_100a and links them into
tof_b200/libtof.so next to the Python package that loads it.  Object files
go to _build/ (git-ignored).  Rebuilds only when a source is newer than the
library.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "tof_b200", "libtof.so")
BUILD = os.path.join(ROOT, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_v: bool = False) -> str:
    srcs = sources()
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    if not force and not _stale(OUT, srcs + headers + [__file__]):
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, "-c", s, "-o", o]
        if ptxas_v:
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(o)
    failed = False
    for s, p in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode or ptxas_v):
            print(out)
        if p.returncode:
            failed = True
            print(f"nvcc failed on {os.path.basename(s)}", file=sys.stderr)
    if failed:
        raise RuntimeError("libtof build failed")
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_v="--ptxas" in sys.argv))
