"""Build recipe for the oracle (test infrastructure, never shipped or timed as the product).

Two things are built here:

* ``oracle/_ref/libfdvref_r{16,32,64}.so`` -- the reference codec itself, compiled
  from ``include/fdv.h`` of the reference tree (yhbsh/fdv) with gcc, exactly as its
  own Makefile would (C11, ``-D_DEFAULT_SOURCE``, ``-O2``, pthreads, libm).  The
  reference hard-codes ``FDV_BORDER 32`` (fdv.h:220) and ties ``FDV_ME_RANGE``
  (fdv.h:5163-5170) to ``FDV_SPLIT_NUM/DEN``, so the +-32 and +-64 search-range
  variants are compiled from a patched copy of the header that lives only in a
  temporary directory for the length of the compile.  Only the ``.so`` files land
  in ``oracle/_ref/`` (git-ignored; they travel to the GPU box with the tree).
  This step needs the reference tree and is skipped when it is absent.
* ``oracle/_build/liboracle.so`` -- the CPU restatement in ``oracle/fdv_oracle.c``.

Every oracle library is a checker: only tests, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` load them.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.environ.get("FDV_REFERENCE_DIR", "/root/reference")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_OUT = os.path.join(HERE, "_build")

# search range -> (border, extra defines).  The border must be a multiple of 32
# (FDV_ALIGN) and cover range + 4 (static assert at fdv.h:5178).
VARIANTS = {
    16: (32, []),
    32: (64, ["-DFDV_ME_RANGE=32", "-DFDV_SPLIT_NUM=9", "-DFDV_SPLIT_DEN=10"]),
    64: (96, ["-DFDV_ME_RANGE=64", "-DFDV_SPLIT_NUM=9", "-DFDV_SPLIT_DEN=10"]),
}

CFLAGS = ["-std=c11", "-D_DEFAULT_SOURCE", "-O2", "-pthread", "-fPIC", "-shared"]


def ref_lib_path(search_range: int) -> str:
    return os.path.join(REF_OUT, f"libfdvref_r{search_range}.so")


def oracle_lib_path() -> str:
    return os.path.join(ORACLE_OUT, "liboracle.so")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources if os.path.exists(s))


def build_ref(force: bool = False) -> bool:
    """Compile the reference into oracle/_ref.  Returns False when the reference
    tree is not present (the GPU box only uses prebuilt libraries)."""
    header = os.path.join(REF_DIR, "include", "fdv.h")
    if not os.path.exists(header):
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim.c")
    for rng, (border, defs) in VARIANTS.items():
        out = ref_lib_path(rng)
        if not force and not _stale(out, [header, shim, __file__]):
            continue
        with tempfile.TemporaryDirectory(prefix="fdvref_") as tmp:
            inc = os.path.join(REF_DIR, "include")
            if border != 32:
                with open(header, "r", encoding="utf-8") as f:
                    text = f.read()
                old = "#define FDV_BORDER 32\n"
                if text.count(old) != 1:
                    raise RuntimeError("reference FDV_BORDER define not found exactly once")
                with open(os.path.join(tmp, "fdv.h"), "w", encoding="utf-8") as f:
                    f.write(text.replace(old, f"#define FDV_BORDER {border}\n"))
                inc = tmp
            cmd = ["gcc", *CFLAGS, *defs, "-I", inc, shim, "-o", out, "-lm"]
            subprocess.run(cmd, check=True)
    return True


def build_oracle(force: bool = False) -> str:
    """Compile the CPU restatement (oracle/fdv_oracle.c) into oracle/_build."""
    os.makedirs(ORACLE_OUT, exist_ok=True)
    src = os.path.join(HERE, "fdv_oracle.c")
    out = oracle_lib_path()
    if force or _stale(out, [src, __file__]):
        cmd = ["gcc", "-std=c11", "-D_DEFAULT_SOURCE", "-O2", "-fPIC", "-shared",
               src, "-o", out, "-lm"]
        subprocess.run(cmd, check=True)
    return out


def build_all(force: bool = False) -> None:
    build_ref(force)
    if os.path.exists(os.path.join(HERE, "fdv_oracle.c")):
        build_oracle(force)


if __name__ == "__main__":
    build_all(force=True)
    print("oracle built:", os.listdir(REF_OUT) if os.path.isdir(REF_OUT) else [], oracle_lib_path())
