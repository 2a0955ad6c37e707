"""Algorithmic integer-op count of the hd720 workload -- test infrastructure.

Runs the CPU restatement (oracle/fdv_oracle.c) built with -DORACLE_OPCOUNT --
every primitive adds its op cost, see the table at the top of that file -- over
the first frames of the hd720 workload (1280x720 as 8 bands of 6 macroblock
rows, QP 24, search range 32, the generator's seed 1): one key frame, then
P-frames.  Writes the count per P-frame (all bands), by category, to
profiles/pframe_ops_hd720.json, which bench.py reads for the integer-pipe
roofline of the P-frame kernel (the count is of the reference algorithm's
work, as the reference computes it; the GPU computes the same decisions).

    python -m oracle.opcount [--pframes N]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_LIB = os.path.join(HERE, "_build", "liboracle_ops.so")
CATS = ["sad", "mc", "satd", "transform4", "quant4", "rdoq", "transform8", "quant8", "pixel", "intra_pred",
        "deblock"]


def build_counting() -> str:
    os.makedirs(os.path.dirname(OUT_LIB), exist_ok=True)
    src = os.path.join(HERE, "fdv_oracle.c")
    if not os.path.exists(OUT_LIB) or os.path.getmtime(OUT_LIB) < os.path.getmtime(src):
        subprocess.run(["gcc", "-std=c11", "-D_DEFAULT_SOURCE", "-O2", "-fPIC", "-shared", "-DORACLE_OPCOUNT", src,
                        "-o", OUT_LIB, "-lm"], check=True)
    return OUT_LIB


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--pframes", type=int, default=3)
    args = ap.parse_args(argv)
    sys.path.insert(0, ROOT)
    import numpy as np
    import oracle as O
    import fdv_b200 as F
    W, H, QP, RANGE, BAND_MBROWS = 1280, 720, 24, 32, 6
    build_counting()
    # the counting build behind the oracle's own unit wrapper
    O._orc = None
    path0 = O._build.oracle_lib_path
    O._build.oracle_lib_path = lambda: OUT_LIB
    try:
        O.restatement()
    finally:
        O._build.oracle_lib_path = path0
    L = O._orc
    L.oracle_opcount.argtypes = [C.POINTER(C.c_ulonglong), C.c_int]
    n = len(CATS)
    buf = (C.c_ulonglong * n)()

    def take():
        L.oracle_opcount(buf, 1)
        return [int(v) for v in buf]

    nf = 1 + args.pframes
    sc = F.Scene(W, H, 120, nrects=40, rect_min=8, rect_max=64, vmax_qpel=24, pan_qx=9, pan_qy=0, static_pct=40,
                 seed=1)
    frames = [sc.frame(f) for f in range(nf)]
    bands, y = [], 0
    while y < H:
        bh = min(BAND_MBROWS * 16, H - y)
        bands.append((y, bh))
        y += bh
    units = [O.OracleUnit(W, bh, RANGE) for _, bh in bands]
    cw = W // 2
    per = []
    t0 = time.time()
    take()
    for f in range(nf):
        fr = frames[f]
        Y = fr[:W * H].reshape(H, W)
        U = fr[W * H:W * H + cw * (H // 2)].reshape(H // 2, cw)
        V = fr[W * H + cw * (H // 2):].reshape(H // 2, cw)
        for (y0, bh), u in zip(bands, units):
            band = np.concatenate([Y[y0:y0 + bh].ravel(), U[y0 // 2:(y0 + bh) // 2].ravel(),
                                   V[y0 // 2:(y0 + bh) // 2].ravel()])
            u.frame(band, int(f == 0), QP)
        per.append(take())
    key = dict(zip(CATS, per[0]))
    pf = [dict(zip(CATS, p)) for p in per[1:]]
    avg = {k: sum(p[k] for p in pf) // len(pf) for k in CATS}
    out = {
        "workload": "hd720: 1280x720, 8 bands x 6 macroblock rows, QP 24, range 32, generator seed 1",
        "frames": f"1 key + {args.pframes} P",
        "ops_per_pframe": sum(avg.values()),
        "ops_per_pframe_by_category": avg,
        "ops_keyframe": sum(key.values()),
        "ops_keyframe_by_category": key,
        "cost_table": "oracle/fdv_oracle.c (ORACLE_OPCOUNT)",
        "command": "python -m oracle.opcount --pframes %d" % args.pframes,
        "cpu_seconds": round(time.time() - t0, 1),
    }
    dst = os.path.join(ROOT, "profiles", "pframe_ops_hd720.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
