"""Build libsputnik_b200.so in-tree: CUDA sources for sm_100a with nvcc, C
sources with gcc (no floating-point contraction, so the host-side tables and
container operations round exactly as the reference's build does), linked
against the static CUDA runtime.

    python -m madmax_b200.build [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libsputnik_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -static-global-template-stub=false: the batched kernel's instantiations live
# in their own translation units and are launched from rve_batch.cu
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-static-global-template-stub=false", "-Xptxas", "-v"] + ARCH
CC_FLAGS = ["-O2", "-ffp-contract=off", "-fPIC", "-std=gnu11", "-Wall", "-Wno-unused-function"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu"))), sorted(glob.glob(os.path.join(CSRC, "*.c")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(cmd, log):
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return log


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cu, c = _sources()
    hdrs = _headers()
    nvcc = _nvcc()
    inc = ["-I", INCLUDE, "-I", CSRC]
    tasks = []
    objs = []
    for src in cu + c:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + hdrs):
            if src.endswith(".cu"):
                cmd = [nvcc] + NVCC_FLAGS + inc + ["-c", src, "-o", obj]
            else:
                cmd = ["gcc"] + CC_FLAGS + inc + ["-c", src, "-o", obj]
            tasks.append((cmd, obj + ".log"))
    if tasks:
        n = jobs or min(len(tasks), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=n) as ex:
            for log in ex.map(lambda t: _compile(*t), tasks):
                if verbose:
                    print(open(log).read())
    if force or tasks or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static", "-lm", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def ptxas_report() -> str:
    """Register / shared-memory / spill lines from the last build."""
    out = []
    for log in sorted(glob.glob(os.path.join(BUILD, "*.cu.o.log"))):
        for line in open(log):
            if ("ptxas info" in line and ("registers" in line or "Compiling" in line)) or \
                    "bytes spill" in line:
                out.append(line.rstrip())
    return "\n".join(out)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--ptxas", action="store_true", help="print register/spill report")
    a = ap.parse_args(argv)
    lib = build(force=a.force, jobs=a.j)
    print(lib)
    if a.ptxas:
        print(ptxas_report())


if __name__ == "__main__":
    sys.exit(main())
