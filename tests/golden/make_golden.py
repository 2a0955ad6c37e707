"""Generate tests/golden/golden.json from the reference encoder.

Run in a container that holds the reference sources: the reference is compiled
from them into oracle/_ref (oracle/build.py) and encodes the seeded workloads;
this records SHA-256 digests and lengths of its streams and of the rendered
source frames, plus a few known-answer vectors of its exported kernels.  The
GPU tests compare the library's output with these digests, so they do not need
the reference tree at run time.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import fdv_b200 as F  # noqa: E402
import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


# (name, scene kwargs, encode kwargs)
CASES = [
    ("cif30", dict(w=352, h=288, nframes=30, nrects=6, seed=1),
     dict(qp=28, keyint=0, band_mbrows=None, search_range=16)),
    ("hd720_g12", dict(w=1280, h=720, nframes=12, nrects=40, pan_qx=9, static_pct=40, seed=1),
     dict(qp=24, keyint=60, band_mbrows=6, search_range=32)),
    ("pan256_k5", dict(w=256, h=144, nframes=10, nrects=10, pan_qx=9, static_pct=40, seed=5),
     dict(qp=24, keyint=5, band_mbrows=None, search_range=32)),
    ("tiny_q0", dict(w=64, h=48, nframes=4, nrects=3, rect_max=24, pan_qx=5, seed=7),
     dict(qp=0, keyint=0, band_mbrows=None, search_range=16)),
    ("tiny_q51_r64", dict(w=64, h=48, nframes=4, nrects=3, rect_max=24, pan_qx=5, seed=7),
     dict(qp=51, keyint=2, band_mbrows=None, search_range=64)),
    ("bands_q12", dict(w=192, h=160, nframes=6, nrects=8, pan_qx=-6, pan_qy=3, static_pct=20, seed=9),
     dict(qp=12, keyint=4, band_mbrows=3, search_range=16)),
    # the 1080p stress shape: 1920x1088 (the format has no crop), 17 bands of 4
    # macroblock rows, range +-64, QP 20, fast objects (up to 24 px/frame)
    ("c3_1088_r64", dict(w=1920, h=1088, nframes=4, nrects=200, rect_min=8, rect_max=96, vmax_qpel=96, pan_qx=6,
                         pan_qy=-3, static_pct=0, seed=3),
     dict(qp=20, keyint=60, band_mbrows=4, search_range=64)),
]

# Independent streams of mixed sizes and QPs coded together (one engine, one
# launch per frame step): each must equal the reference's fdv_video_encode.
BATCH = [
    dict(w=320, h=240, nframes=5, nrects=6, seed=21, qp=18),
    dict(w=640, h=368, nframes=5, nrects=12, pan_qx=5, seed=22, qp=27),
    dict(w=1280, h=720, nframes=5, nrects=40, pan_qx=9, static_pct=40, seed=23, qp=36),
    dict(w=1920, h=1088, nframes=5, nrects=60, pan_qx=-4, pan_qy=2, seed=24, qp=22),
    dict(w=320, h=240, nframes=5, nrects=10, pan_qy=7, seed=25, qp=31),
]
BATCH_KEYINT = 3


# Streaming encodes (fdv_enc_*) under average-bitrate control: (name, scene
# kwargs, encoder kwargs).  The low bitrates make frames overshoot their
# allocation, so the reference codes them again, coarser (fdv.h:8281-8335).
STREAMS = [
    ("rc_single_low", dict(w=256, h=144, nframes=14, nrects=10, pan_qx=9, static_pct=40, seed=5),
     dict(qp=24, keyint=6, search_range=16, bitrate=8000, fps=30, bufsecs=1.0, band_mbrows=None, nthreads=1,
          repeat_after=[4])),
    ("rc_single_cif", dict(w=352, h=288, nframes=12, nrects=6, seed=1),
     dict(qp=28, keyint=0, search_range=16, bitrate=300000, fps=30, bufsecs=0.5, band_mbrows=None, nthreads=1,
          repeat_after=[])),
    ("rc_single_r32", dict(w=256, h=144, nframes=10, nrects=12, pan_qx=-7, pan_qy=2, static_pct=10, seed=11),
     dict(qp=30, keyint=5, search_range=32, bitrate=60000, fps=25, bufsecs=2.0, band_mbrows=None, nthreads=1,
          repeat_after=[6])),
    ("rc_tiled", dict(w=192, h=160, nframes=10, nrects=8, pan_qx=-6, pan_qy=3, static_pct=20, seed=9),
     dict(qp=20, keyint=4, search_range=16, bitrate=30000, fps=30, bufsecs=1.0, band_mbrows=3, nthreads=2,
          repeat_after=[2])),
]


def scene(kw) -> list[np.ndarray]:
    kw = dict(kw)
    n = kw.pop("nframes")
    w, h = kw.pop("w"), kw.pop("h")
    return F.Scene(w, h, n, **kw).frames(n)


def main() -> None:
    out = {"cases": {}, "kernels": {}}
    for name, skw, ekw in CASES:
        fr = scene(skw)
        w, h = skw["w"], skw["h"]
        if ekw["band_mbrows"] is None:
            s = O.ref_video_encode(fr, w, h, ekw["qp"], ekw["keyint"], ekw["search_range"])
            dec = O.ref_video_decode(s, ekw["search_range"])
        else:
            s = O.ref_vtile_encode(fr, w, h, ekw["qp"], ekw["keyint"], ekw["band_mbrows"], 1, ekw["search_range"])
            dec = O.ref_vtile_decode(s, ekw["search_range"])
        out["cases"][name] = {
            "scene": skw, "encode": ekw, "stream_sha256": sha(s), "stream_len": len(s),
            "frames_sha256": sha(b"".join(f.tobytes() for f in fr)),
            "decoded_sha256": sha(dec.tobytes()),
        }
        print(name, len(s), flush=True)
    out["batch"] = {"keyint": BATCH_KEYINT, "search_range": 16, "streams": []}
    for bk in BATCH:
        skw = {k: v for k, v in bk.items() if k != "qp"}
        fr = scene(skw)
        s = O.ref_video_encode(fr, bk["w"], bk["h"], bk["qp"], BATCH_KEYINT, 16)
        out["batch"]["streams"].append({"scene": skw, "qp": bk["qp"], "stream_sha256": sha(s), "stream_len": len(s)})
        print("batch", bk["w"], bk["h"], len(s), flush=True)
    out["streams"] = {}
    for name, skw, ekw in STREAMS:
        fr = scene(skw)
        s = O.ref_enc_stream(fr, skw["w"], skw["h"], ekw["qp"], ekw["keyint"], ekw["search_range"], ekw["bitrate"],
                             ekw["fps"], ekw["bufsecs"], ekw["band_mbrows"], ekw["nthreads"], tuple(ekw["repeat_after"]))
        out["streams"][name] = {"scene": skw, "encode": ekw, "file_sha256": sha(s), "file_len": len(s)}
        print(name, len(s), flush=True)
    # known answers of the reference's kernels (its own tests pin the first two:
    # test_enc.c:466-476 flat block -> DC only; :817-826 motion search recovers
    # a pure translation with SAD 0)
    L = O.ref(16)
    res = (C.c_int16 * 16)(*([10] * 16))
    co = (C.c_int32 * 16)()
    L.fdv_fdct4x4(res, co)
    out["kernels"]["fdct4x4_flat10"] = list(co)
    rng = np.random.default_rng(42)
    blk = rng.integers(-255, 256, 16).astype(np.int16)
    co2 = (C.c_int32 * 16)()
    L.fdv_fdct4x4(blk.ctypes.data_as(C.POINTER(C.c_int16)), co2)
    lev = (C.c_int16 * 16)()
    L.fdv_quant4x4(co2, lev, 24)
    out["kernels"]["fdct4x4_seed42"] = {"in": blk.tolist(), "coeff": list(co2), "level_qp24": list(lev)}
    c8 = (C.c_int32 * 64)()
    q8 = (C.c_int32 * 52)()
    L.fdvref_c8_tables(c8, q8)
    out["kernels"]["c8"] = list(c8)
    out["kernels"]["qstep8"] = list(q8)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
