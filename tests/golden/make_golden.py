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
    # the whole 720p workload the benchmark times: 120 frames, two key frames
    # (0 and 60), P-frames in launches of up to thirty, the reference ring
    # wrapping several times
    ("hd720_full", dict(w=1280, h=720, nframes=120, nrects=40, pan_qx=9, static_pct=40, seed=1),
     dict(qp=24, keyint=60, band_mbrows=6, search_range=32)),
]

# The camera-like stress content at the 1080p stress shape: a 1/f^2 fractal
# canvas under a 0.5 %/frame zoom and a pan, 200 objects at up to 24 px/frame,
# sensor noise sd 2 / 1, a hard cut every 100 frames; 17 bands of 4 macroblock
# rows, range +-64, QP 20, key interval 60.
C3_SCENE = dict(kind="camera", w=1920, h=1088, nframes=300, nobjects=200, obj_min=8, obj_max=96, vmax_qpel=96,
                zoom_ppm=5000, pan_qx=9, pan_qy=-4, noise_y_x16=32, noise_c_x16=16, cut_every=100, seed=3)
C3_ENCODE = dict(qp=20, keyint=60, band_mbrows=4, search_range=64)
# The reference's whole-array tiled encoder gives each band twice its raw
# frame size plus 64 KiB for the whole stream (fdv.h:7111-7113), which this
# noisy content outgrows within the first GOP: it returns 0 there, and so must
# the library.  The streaming tiled encoder grows its buffer (fdv.h:8341-8347)
# and codes all 300 frames; the full-length parity case goes through it.
C3_VTILE_FRAMES = 60

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
    if kw.pop("kind", "rects") == "camera":
        return F.CamScene(w, h, n, **kw).frames(n)
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
            s = O.ref_vtile_encode(fr, w, h, ekw["qp"], ekw["keyint"], ekw["band_mbrows"], os.cpu_count() or 1,
                                   ekw["search_range"])
            dec = O.ref_vtile_decode(s, ekw["search_range"])
        out["cases"][name] = {
            "scene": skw, "encode": ekw, "stream_sha256": sha(s), "stream_len": len(s),
            "frames_sha256": sha(b"".join(f.tobytes() for f in fr)),
            "decoded_sha256": sha(dec.tobytes()), "last_decoded_sha256": sha(dec[-1].tobytes()),
        }
        print(name, len(s), flush=True)
    # the camera-like stress case: the whole-array tiled encoder's capacity
    # failure, and the full 300 frames through the streaming tiled encoder
    fr = scene(C3_SCENE)
    e = C3_ENCODE
    w, h = C3_SCENE["w"], C3_SCENE["h"]
    try:
        O.ref_vtile_encode(fr[:C3_VTILE_FRAMES], w, h, e["qp"], e["keyint"], e["band_mbrows"], os.cpu_count() or 1,
                           e["search_range"])
        vtile_fails = False
    except RuntimeError:
        vtile_fails = True
    s = O.ref_enc_stream(fr, w, h, e["qp"], e["keyint"], e["search_range"], 0, 30, 1.0, e["band_mbrows"],
                         os.cpu_count() or 1)
    dec = O.ref_vtile_decode(s[12:], e["search_range"], os.cpu_count() or 1)
    out["c3"] = {"scene": C3_SCENE, "encode": e, "vtile_frames": C3_VTILE_FRAMES, "vtile_fails": vtile_fails,
                 "file_sha256": sha(s), "file_len": len(s), "fps": 30,
                 "frames_sha256": sha(b"".join(f.tobytes() for f in fr)),
                 "decoded_sha256": sha(dec.tobytes()), "last_decoded_sha256": sha(dec[-1].tobytes())}
    print("c3", vtile_fails, len(s), flush=True)
    del fr, dec
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
