"""Build the native library in-tree: ``python -m yafray_b200.build``.

Every .cu and .cpp under csrc/ is compiled with nvcc for sm_100a only
(`-gencode arch=compute_100a,code=sm_100a`) and linked into
yafray_b200/libyafray_b200.so.  `--fmad=false` keeps single-precision
arithmetic unfused, as on the x86-64 SSE reference, so that hit distances,
entry/exit points and shading terms round the same way.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("YR_BUILD_DIR", os.path.join(HERE, "_build"))
OUT = os.environ.get("YR_OUT", os.path.join(HERE, "libyafray_b200.so"))
EXTRA = os.environ.get("YR_DEFINES", "").split()  # variant builds for A/B measurements
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-O2,-ffp-contract=off",
          "-I" + os.path.join(HERE, "..", "include")]


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(
            [os.path.getmtime(src)] + [os.path.getmtime(h) for h in glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))]
            + [os.path.getmtime(os.path.join(HERE, "..", "include", "yr.h"))]):
        return obj
    cmd = [NVCC] + ARCH + COMMON + EXTRA + ["-c", src, "-o", obj]
    if src.endswith(".cu") and os.environ.get("YR_PTXAS_V"):
        cmd[1:1] = ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if os.environ.get("YR_PTXAS_V"):
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(_compile, srcs))
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(OUT)
    return OUT


if __name__ == "__main__":
    build(verbose=True)
