"""Builds libtomostar_cuda.so in-tree for sm_100a with nvcc (no torch in the library).

Every source under csrc/ is compiled to an object under _build/ (in parallel, skipped when up to
date) and linked into tomostar_b200/libtomostar_cuda.so. Host code is compiled with
-ffp-contract=off so the host geometry rounds as the reference's does.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtomostar_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NO_FMA = {"rays.cu", "locate.cu", "domain.cu"}
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math",
          "-I", os.path.join(HERE, "..", "include")]


def _deps() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    # The ray tracer rounds every operation on its own, as the reference's .NET arithmetic does:
    # a contracted multiply-add at one call site and not another breaks identities such as
    # "the same point twice gives a zero-length segment".
    flags = ["-fmad=false"] if os.path.basename(src) in NO_FMA else []
    cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", src, "-o", obj]
    stamp = obj + ".cmd"
    newest = max(os.path.getmtime(p) for p in [src, *_deps(), os.path.abspath(__file__)])
    if (os.path.exists(obj) and os.path.getmtime(obj) >= newest and os.path.exists(stamp)
            and open(stamp).read() == " ".join(cmd)):
        return obj
    if verbose and src.endswith(".cu"):
        cmd = cmd[:-4] + ["-Xptxas", "-v"] + cmd[-4:]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    with open(stamp, "w") as f:
        f.write(" ".join(c for c in cmd if c not in ("-Xptxas", "-v")))
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
