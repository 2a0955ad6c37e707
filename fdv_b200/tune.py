"""Autotuner of the encoder engine's launch shape.

The P-frame analysis runs as one persistent wavefront kernel per batch of
consecutive P-frames.  Two choices set how well that kernel fills the SMs,
and both depend on the unit geometry and the search range:

* P-frames per launch (1..60).  The frames of a batch overlap: frame k + 1's
  macroblock rows start as soon as frame k has written the reference tiles
  they read.  More frames keep more rows in flight and spread the launch's
  ramp-up and drain over more frames; fewer frames start the host's entropy
  coding of a batch sooner.
* Blocks of the wavefront kernel (the number of macroblock rows in flight at
  once; one block per SM by default).  A row's block holds its SM while the
  row waits for the row above or for the previous frame's tiles, so fewer
  blocks can leave SMs to other work at a small cost.

The threads per macroblock (512) and the shared-memory window of the
reference planes are fixed when the kernel is compiled; they are not swept.

``autotune`` codes a short seeded sequence of the geometry on the device for
each candidate shape (device-resident sources, CUDA-event kernel time per
P-frame), keeps the fastest, stores it per GPU model and geometry in a JSON
cache (``$FDVB_TUNE_CACHE``, default ``~/.cache/fdv_b200/tuning.json``), and
records it for the fdv_* encoders of that geometry (``fdvb_set_tuning``).
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import Engine, Scene, lib, set_search_range, get_search_range, set_tuning, u8p

BATCHES = (6, 12, 20, 30, 60)
GRID_CUTS = (0, 8, 20, 40)          # SMs left free by the wavefront kernel


def cache_path() -> str:
    return os.environ.get("FDVB_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "fdv_b200", "tuning.json"))


def _key(gpu: str, sizes, search_range: int) -> str:
    return f"{gpu}|r{search_range}|" + ",".join(f"{w}x{h}" for w, h in sizes)


def _gpu_name(device: int) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def load(sizes, search_range: int, device: int = 0) -> dict | None:
    """The cached choice for this GPU model and geometry, or None."""
    try:
        with open(cache_path()) as f:
            return json.load(f).get(_key(_gpu_name(device), sizes, search_range))
    except (OSError, ValueError):
        return None


def _store(key: str, entry: dict) -> None:
    path = cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        try:
            with open(path) as f:
                db = json.load(f)
        except (OSError, ValueError):
            db = {}
        db[key] = entry
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(db, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home: the choice still applies to this process


def _sequence(sizes, nframes: int, seed: int):
    """Seeded moving-rectangle content for every unit, as the benchmarks use."""
    out = []
    for u, (w, h) in enumerate(sizes):
        sc = Scene(w, h, nframes, nrects=max(2, w * h // 20000), rect_min=8, rect_max=64, vmax_qpel=24, pan_qx=9,
                   pan_qy=-2, static_pct=30, seed=seed + u)
        out.append(np.stack(sc.frames(nframes)))
    return out


def measure(eng: Engine, planes, intra, qps, nframes: int, reps: int = 2) -> float:
    """Kernel time per P-frame (ms) of `nframes` frame steps from device sources."""
    L = lib()
    if L.fdvg_frames_device(eng._g, nframes, planes, intra, qps) != 0:   # warm-up
        raise RuntimeError("tuning run failed")
    best = None
    for _ in range(reps):
        eng.stats_reset()
        if L.fdvg_frames_device(eng._g, nframes, planes, intra, qps) != 0:
            raise RuntimeError("tuning run failed")
        st = eng.stats()
        v = st["p_ms"] / max(1, st["p_launches"])
        best = v if best is None else min(best, v)
    return best


def autotune(sizes, search_range: int, device: int = 0, nframes: int = 61, qp: int = 24, use_cache: bool = True,
             record: bool = True, seed: int = 7) -> dict:
    """Choose the launch shape for units of `sizes` at `search_range`
    (the default shape: the largest batch size at one block per SM).

    Sweeps the P-frames per launch at one block per SM, then the block count
    at the best batch size; returns {"max_batch", "p_grid", "p_ms_per_frame",
    "default_p_ms_per_frame", "candidates", "cached"}."""
    import torch
    sizes = [tuple(s) for s in sizes]
    key = _key(_gpu_name(device), sizes, search_range)
    if use_cache:
        hit = load(sizes, search_range, device)
        if hit is not None:
            if record:
                set_tuning(sizes, search_range, hit["max_batch"], hit["p_grid"])
            return dict(hit, cached=True)
    old_range = get_search_range()
    set_search_range(search_range)
    try:
        seq = _sequence(sizes, nframes, seed)
        dev = [torch.from_numpy(s).to(f"cuda:{device}") for s in seq]
        torch.cuda.synchronize(device)
        nu = len(sizes)
        planes = (u8p * (3 * nu * nframes))()
        for f in range(nframes):
            for u, (w, h) in enumerate(sizes):
                b = dev[u].data_ptr() + f * w * h * 3 // 2
                j = 3 * (f * nu + u)
                planes[j], planes[j + 1], planes[j + 2] = (C.cast(b, u8p), C.cast(b + w * h, u8p),
                                                           C.cast(b + w * h * 5 // 4, u8p))
        intra = (C.c_int * (nu * nframes))(*([1] * nu + [0] * (nu * (nframes - 1))))
        qps = (C.c_int * (nu * nframes))(*([qp] * (nu * nframes)))
        eng = Engine(sizes, search_range, device)
        nsm = eng.tuning()["nsm"]
        cands = []
        try:
            for k in BATCHES:
                eng.set_tuning(k, 0)
                cands.append({"max_batch": k, "p_grid": nsm, "p_ms_per_frame": measure(eng, planes, intra, qps, nframes)})
            kbest = min(cands, key=lambda c: c["p_ms_per_frame"])["max_batch"]
            for cut in GRID_CUTS[1:]:
                eng.set_tuning(kbest, nsm - cut)
                cands.append({"max_batch": kbest, "p_grid": nsm - cut,
                              "p_ms_per_frame": measure(eng, planes, intra, qps, nframes)})
        finally:
            eng.close()
    finally:
        set_search_range(old_range)
    best = min(cands, key=lambda c: c["p_ms_per_frame"])
    default = next(c for c in cands if c["max_batch"] == BATCHES[-1] and c["p_grid"] == nsm)
    entry = {"max_batch": best["max_batch"], "p_grid": best["p_grid"], "p_ms_per_frame": round(best["p_ms_per_frame"], 4),
             "default_p_ms_per_frame": round(default["p_ms_per_frame"], 4),
             "candidates": [dict(c, p_ms_per_frame=round(c["p_ms_per_frame"], 4)) for c in cands],
             "sequence": f"{nframes} frames (1 key), QP {qp}, seeded moving rectangles", "nsm": nsm}
    _store(key, entry)
    if record:
        set_tuning(sizes, search_range, entry["max_batch"], entry["p_grid"])
    return dict(entry, cached=False)
