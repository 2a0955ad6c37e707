"""The launch-shape autotuner (fdv_b200.tune) and the shapes it chooses from.

* Any launch shape -- P-frames per launch, blocks of the wavefront kernel --
  gives byte-identical streams: the shape changes when rows run, never what
  they compute.  Checked through fdv_vtile_encode with shapes recorded by
  fdvb_set_tuning, against the reference's golden digest.
* The tuner measures every candidate, keeps the fastest, persists it per GPU
  model and geometry, and answers later calls from its cache.
* Out-of-range shapes are rejected.
"""
import hashlib
import json

import pytest

from conftest import scene_frames

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def test_launch_shape_never_changes_the_stream(built, golden):
    import fdv_b200 as F
    case = golden["cases"]["bands_q12"]
    sc, e = case["scene"], case["encode"]
    fr = scene_frames(sc)
    w, h, bm = sc["w"], sc["h"], e["band_mbrows"]
    bh = 16 * bm
    sizes = [(w, min(bh, h - y0)) for y0 in range(0, h, bh)]
    F.set_search_range(e["search_range"])
    try:
        for k, grid in ((1, 0), (2, 3), (5, 0), (60, 1), (60, 0)):
            F.set_tuning(sizes, e["search_range"], k, grid)
            s = F.vtile_encode(fr, w, h, e["qp"], e["keyint"], bm, 4)
            assert sha(s) == case["stream_sha256"], (k, grid)
    finally:
        F.set_tuning(sizes, e["search_range"], 0, 0)
        F.set_search_range(16)


def test_engine_tuning_bounds(built):
    import fdv_b200 as F
    eng = F.Engine([(64, 48)], 16)
    t = eng.tuning()
    assert t["max_batch"] == 60 and t["p_grid"] == t["nsm"] > 0
    eng.set_tuning(7, 5)
    assert eng.max_batch() == 7 and eng.tuning()["p_grid"] == 5
    eng.set_tuning(30, 100000)
    assert eng.tuning()["p_grid"] == t["nsm"]
    for bad in ((0, 0), (61, 0), (5, -1)):
        with pytest.raises(F.FdvError):
            eng.set_tuning(*bad)
    eng.close()


def test_autotune_measures_candidates_and_caches(built, tmp_path, monkeypatch):
    import fdv_b200.tune as T
    monkeypatch.setenv("FDVB_TUNE_CACHE", str(tmp_path / "tuning.json"))
    sizes, rng = [(160, 96), (160, 64)], 32
    r = T.autotune(sizes, rng, nframes=25, record=False)
    assert not r["cached"]
    ks = {c["max_batch"] for c in r["candidates"]}
    assert set(T.BATCHES) <= ks
    best = min(r["candidates"], key=lambda c: c["p_ms_per_frame"])
    assert (r["max_batch"], r["p_grid"]) == (best["max_batch"], best["p_grid"])
    assert r["p_ms_per_frame"] <= r["default_p_ms_per_frame"]
    db = json.load(open(tmp_path / "tuning.json"))
    assert len(db) == 1
    again = T.autotune(sizes, rng, nframes=25, record=False)
    assert again["cached"] and again["max_batch"] == r["max_batch"] and again["p_grid"] == r["p_grid"]
