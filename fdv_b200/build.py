"""Build libfdvb200.so in-tree with nvcc for sm_100a.

The library is a plain C-ABI shared object (include/fdv_b200.h): the CUDA
kernels and the engine that drives them (csrc/device), the host entropy tail,
container writers and public API (csrc/host).  ``-fmad=false`` keeps every
floating-point multiply and add of the rate-distortion decisions separately
rounded, as the reference's C11 build does.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfdvb200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O2",
          "-I", os.path.join(ROOT, "include")]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "device", "*.cu")) +
                  glob.glob(os.path.join(CSRC, "host", "*.cpp")))


def headers() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*", "*.cuh")) + glob.glob(os.path.join(CSRC, "*", "*.h")) +
                  [os.path.join(ROOT, "include", "fdv_b200.h")])


def _obj(src: str) -> str:
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(OBJ, rel + ".o")


def _compile(src: str, extra: list[str]) -> str:
    out = _obj(src)
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", src, "-o", out]
    if src.endswith(".cpp"):
        cmd = [NVCC, *COMMON, *extra, "-x", "c++", "-c", src, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return out


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdr_t = max(os.path.getmtime(h) for h in headers())
    todo = []
    for s in sources():
        o = _obj(s)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t,
                                                                        os.path.getmtime(__file__)):
            todo.append(s)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            futs = {ex.submit(_compile, s, extra): s for s in todo}
            for f in cf.as_completed(futs):
                f.result()
                if verbose:
                    print("compiled", os.path.relpath(futs[f], ROOT))
    objs = [_obj(s) for s in sources()]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        # -z defs: an unresolved symbol fails the link instead of the first call
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lpthread", "-ldl", "-lrt",
               "-Xlinker", "-z", "-Xlinker", "defs"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
