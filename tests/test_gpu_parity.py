"""GPU parity: the CUDA analysis loop against the CPU oracle and the reference.

* Engine level, P-frames: references seeded identically on both sides, then
  the 16 symbol streams and the reconstruction must be identical to the
  oracle's, over sizes, QPs (0..51), search ranges (16/32/64) and one or two
  references.
* Engine level, key frames: the 3 x 12 intra streams and reconstruction.
* Whole streams through the C ABI: byte-identical to the reference encoder's
  (golden SHA-256 digests recorded from it), and the reference decoder's
  output equals the GPU reconstruction.
* The streaming encoder with held frames and a due key frame.
* Bounded waits: an injected stall makes the wavefront waits expire; the step
  returns an error and the engine stays usable.
"""
import hashlib

import numpy as np
import pytest

from conftest import scene_frames

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def _p_case(w, h, rng, qp, nref, seed):
    import fdv_b200 as F
    import oracle as O
    sc = F.Scene(w, h, 3, nrects=max(2, w * h // 4000), pan_qx=9, pan_qy=-3, static_pct=30, seed=seed)
    f0, f1, f2 = sc.frames(3)
    eng = F.Engine([(w, h)], rng)
    u = O.OracleUnit(w, h, rng)
    if nref == 2:
        eng.set_refs(0, f1, f0)
        u.set_refs(f1, f0)
    else:
        eng.set_refs(0, f1)
        u.set_refs(f1)
    eng.step([f2], [0], [qp])
    g = eng.pframe_streams(0)
    o, _ = u.frame(f2, 0, qp)
    for k in range(16):
        assert g[k] == o[k], f"stream {k}"
    assert np.array_equal(eng.recon(0), u.recon())
    eng.close()


@pytest.mark.parametrize("w,h,rng,qp,nref,seed", [
    (64, 64, 16, 28, 1, 1), (64, 64, 16, 28, 2, 2), (256, 144, 32, 24, 2, 3), (352, 288, 16, 12, 2, 4),
    (352, 288, 16, 40, 1, 5), (128, 64, 64, 0, 2, 6), (160, 96, 32, 51, 2, 7), (96, 96, 16, 5, 1, 8),
    (320, 176, 32, 33, 2, 9), (64, 128, 64, 20, 2, 10),
])
def test_pframe_matches_oracle(built, w, h, rng, qp, nref, seed):
    _p_case(w, h, rng, qp, nref, seed)


@pytest.mark.parametrize("w,h,qp,seed", [
    (64, 64, 28, 1), (128, 96, 24, 2), (352, 288, 12, 3), (256, 144, 40, 4), (96, 48, 0, 5),
    (160, 80, 7, 6), (192, 112, 51, 7),
])
def test_keyframe_matches_oracle(built, w, h, qp, seed):
    import fdv_b200 as F
    import oracle as O
    f0 = F.Scene(w, h, 1, nrects=3, seed=seed).frame(0)
    eng = F.Engine([(w, h)], 16)
    u = O.OracleUnit(w, h, 16)
    eng.step([f0], [1], [qp])
    o, _ = u.frame(f0, 1, qp)
    for p in range(3):
        g = eng.iframe_streams(0, p)
        for k in range(12):
            assert g[k] == o[p][k], f"plane {p} stream {k}"
    assert np.array_equal(eng.recon(0), u.recon())
    eng.close()


@pytest.mark.parametrize("name", ["cif30", "pan256_k5", "tiny_q0", "tiny_q51_r64", "bands_q12", "hd720_g12",
                                  "c3_1088_r64", "hd720_full"])
def test_stream_matches_reference(built, golden, name):
    import fdv_b200 as F
    case = golden["cases"][name]
    sc, e = case["scene"], case["encode"]
    fr = scene_frames(sc)
    F.set_search_range(e["search_range"])
    try:
        if e["band_mbrows"] is None:
            s = F.video_encode(fr, sc["w"], sc["h"], e["qp"], e["keyint"])
        else:
            s = F.vtile_encode(fr, sc["w"], sc["h"], e["qp"], e["keyint"], e["band_mbrows"], 4)
    finally:
        F.set_search_range(16)
    assert len(s) == case["stream_len"]
    assert sha(s) == case["stream_sha256"]


def test_reconstruction_matches_reference_decoder(built, golden):
    """Decoder parity: the reference decoder's frames equal the GPU's
    reconstruction of every frame."""
    import fdv_b200 as F
    case = golden["cases"]["pan256_k5"]
    sc, e = case["scene"], case["encode"]
    fr = scene_frames(sc)
    eng = F.Engine([(sc["w"], sc["h"])], e["search_range"])
    recs = []
    for f, x in enumerate(fr):
        eng.step([x], [int(f % e["keyint"] == 0)], [e["qp"]])
        recs.append(eng.recon(0))
    assert sha(np.concatenate(recs).tobytes()) == case["decoded_sha256"]


def test_streaming_encoder_matches_whole_array(built, golden):
    import fdv_b200 as F
    import oracle as O
    case = golden["cases"]["tiny_q51_r64"]
    sc = dict(case["scene"])
    fr = scene_frames(sc)
    w, h = sc["w"], sc["h"]
    F.set_search_range(64)
    try:
        enc = F.Encoder(w, h, 51, 2)
        for x in fr:
            enc.frame(x)
        assert enc.count() == len(fr)
        data = enc.finish(25)
        assert data[:4] == b"FDV1" and data[5] == 0
        assert sha(data[12:]) == case["stream_sha256"]
        # held frames: all-SKIP re-emissions, a key frame that falls on a held
        # slot is carried to the next real frame
        enc = F.Encoder(w, h, 30, 3)
        enc.frame(fr[0]); enc.frame(fr[1]); enc.frame(fr[2])
        enc.repeat()
        enc.frame(fr[3])
        a = enc.finish(30)
        if O.have_ref(64):
            import ctypes as C
            R = O.ref(64)
            R.fdv_enc_open.restype = C.c_void_p
            R.fdv_enc_frame.argtypes = [C.c_void_p, C.POINTER(C.c_uint8)]
            R.fdv_enc_repeat.argtypes = [C.c_void_p]
            R.fdv_enc_finish.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
            R.fdv_enc_finish.restype = C.c_void_p
            e = R.fdv_enc_open(w, h, 30, 3)
            u8p = C.POINTER(C.c_uint8)
            for i in [0, 1, 2]:
                R.fdv_enc_frame(e, fr[i].ctypes.data_as(u8p))
            R.fdv_enc_repeat(e)
            R.fdv_enc_frame(e, fr[3].ctypes.data_as(u8p))
            n = C.c_size_t()
            p = R.fdv_enc_finish(e, 30, C.byref(n))
            assert a == C.string_at(p, n.value)
        # tiled streaming == fdv_vtile_encode
        enc = F.Encoder(w, h, 51, 2, band_mbrows=1, nthreads=2)
        for x in fr:
            enc.frame(x)
        t = enc.finish(25)
        assert t[5] == 1 and t[12:] == F.vtile_encode(fr, w, h, 51, 2, 1, 2)
    finally:
        F.set_search_range(16)


def test_bounded_wait_reports_timeout_and_recovers(built):
    import ctypes as C
    import fdv_b200 as F
    import oracle as O
    L = F.lib()
    L.fdvg_set_wait_timeout_ns.argtypes = [C.c_void_p, C.c_ulonglong]
    L.fdvg_set_wait_timeout_ns.restype = None
    L.fdvg_inject_stall.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.fdvg_inject_stall.restype = None
    w, h = 96, 96
    sc = F.Scene(w, h, 3, nrects=3, seed=4)
    f0, f1, f2 = sc.frames(3)
    eng = F.Engine([(w, h)], 16)
    eng.set_refs(0, f1, f0)
    L.fdvg_set_wait_timeout_ns(eng._g, 50_000_000)
    L.fdvg_inject_stall(eng._g, 0, 2)          # row 2 never runs: rows 3.. wait on a flag nothing sets
    with pytest.raises(F.FdvError, match="timed out"):
        eng.step([f2], [0], [26])
    # the context is intact: a clean step afterwards matches the oracle
    eng.set_refs(0, f1, f0)
    eng.step([f2], [0], [26])
    u = O.OracleUnit(w, h, 16)
    u.set_refs(f1, f0)
    o, _ = u.frame(f2, 0, 26)
    assert eng.pframe_streams(0) == o
    eng.close()


@pytest.mark.parametrize("name", ["rc_single_low", "rc_single_cif", "rc_single_r32", "rc_tiled"])
def test_bitrate_controlled_stream_matches_reference(built, golden, name):
    """fdv_enc_set_bitrate: the controller's quantisers, the lambda fractions of
    P-frames and the re-coding of frames that overshoot reproduce the
    reference's .fdv file byte for byte (held frames included)."""
    import fdv_b200 as F
    case = golden["streams"][name]
    sc, e = case["scene"], case["encode"]
    fr = scene_frames(sc)
    F.set_search_range(e["search_range"])
    try:
        enc = F.Encoder(sc["w"], sc["h"], e["qp"], e["keyint"], e["band_mbrows"], e["nthreads"])
        enc.set_bitrate(e["bitrate"], e["fps"], e["bufsecs"])
        with pytest.raises(F.FdvError):
            enc2 = F.Encoder(sc["w"], sc["h"], e["qp"], e["keyint"])
            enc2.frame(fr[0])
            enc2.set_bitrate(e["bitrate"], e["fps"], e["bufsecs"])   # only before the first frame
        enc2.close()
        for i, x in enumerate(fr):
            enc.frame(x)
            if i in e["repeat_after"]:
                enc.repeat()
        data = enc.finish(e["fps"])
    finally:
        F.set_search_range(16)
    assert len(data) == case["file_len"]
    assert sha(data) == case["file_sha256"]


def test_gpu_stream_counts_equal_host_counts(built):
    """The symbol counts the compaction kernel makes equal a host count of the
    streams it delivers, for P-frames and every key-frame plane (the counts
    the entropy tail builds its tables from; the stream digests above show the
    tail's output is unchanged when it uses them)."""
    import fdv_b200 as F
    w, h = 320, 176
    fr = F.Scene(w, h, 3, nrects=8, pan_qx=9, static_pct=30, seed=12).frames(3)
    eng = F.Engine([(w, 96), (w, 80)], 32)
    def bands(f):
        Y = f[:w * h].reshape(h, w); U = f[w * h:w * h * 5 // 4].reshape(h // 2, w // 2); V = f[w * h * 5 // 4:].reshape(h // 2, w // 2)
        return [np.concatenate([Y[y0:y0 + bh].ravel(), U[y0 // 2:(y0 + bh) // 2].ravel(), V[y0 // 2:(y0 + bh) // 2].ravel()])
                for y0, bh in ((0, 96), (96, 80))]
    for f in range(3):
        eng.step(bands(fr[f]), [int(f == 0)] * 2, [22, 30])
        for u in range(2):
            if f == 0:
                for p in range(3):
                    st, hg = eng.iframe_streams(u, p), eng.iframe_hist(u, p)
                    for k in range(12):
                        assert np.array_equal(hg[k], np.bincount(np.frombuffer(st[k], np.uint8), minlength=256)), (u, p, k)
            else:
                st, hg = eng.pframe_streams(u), eng.pframe_hist(u)
                for k in range(16):
                    assert np.array_equal(hg[k], np.bincount(np.frombuffer(st[k], np.uint8), minlength=256)), (u, k)
    eng.close()


def test_batched_streams_match_reference(built, golden):
    """Independent streams of mixed sizes (320x240 .. 1920x1088) and QPs coded
    by one engine -- every frame step one P-frame launch (or one key-frame
    launch) for all of them -- each equal to the reference's fdv_video_encode."""
    import fdv_b200 as F
    import oracle as O
    B = golden["batch"]
    K, specs = B["keyint"], B["streams"]
    frames = [scene_frames(sp["scene"]) for sp in specs]
    sizes = [(sp["scene"]["w"], sp["scene"]["h"]) for sp in specs]
    nf = specs[0]["scene"]["nframes"]
    eng = F.Engine(sizes, B["search_range"])
    tcs = [F.TabCache() for _ in specs]
    blobs = [[] for _ in specs]
    for f in range(nf):
        intra = int(f % K == 0)
        eng.step([fr[f] for fr in frames], [intra] * len(specs), [sp["qp"] for sp in specs])
        for u, sp in enumerate(specs):
            (w, h), qp = sizes[u], sp["qp"]
            if intra:
                tcs[u].reset()
                pw, ph = [w, w // 2, w // 2], [h, h // 2, h // 2]
                blobs[u].append(O.iframe_blob([F.entropy_image(eng.iframe_streams(u, p), pw[p], ph[p], qp)
                                               for p in range(3)]))
            else:
                blobs[u].append(F.entropy_pframe(eng.pframe_streams(u), qp, tcs[u]))
    eng.close()
    for u, sp in enumerate(specs):
        st = O.compose_video(sizes[u][0], sizes[u][1], nf, sp["qp"], K, blobs[u])
        assert len(st) == sp["stream_len"], u
        assert sha(st) == sp["stream_sha256"], u


def test_submit_collect_pipeline_equals_step(built):
    """fdvg_submit / fdvg_collect with two frames in flight give every frame
    the same streams and reconstruction as fdvg_frame one at a time."""
    import fdv_b200 as F
    w, h = 160, 96
    fr = F.Scene(w, h, 5, nrects=5, pan_qx=7, seed=31).frames(5)
    ref = F.Engine([(w, h)], 16)
    want = []
    for f in range(5):
        ref.step([fr[f]], [int(f == 0)], [26])
        want.append([ref.iframe_streams(0, p) for p in range(3)] if f == 0 else ref.pframe_streams(0))
    ref.close()
    eng = F.Engine([(w, h)], 16)
    got = []
    for f in range(6):
        if f < 5:
            eng.submit([fr[f]], [int(f == 0)], [26])
        if f > 0:
            eng.collect()
            got.append([eng.iframe_streams(0, p) for p in range(3)] if f == 1 else eng.pframe_streams(0))
    eng.close()
    assert got == want


def test_camera_stress_tiled_capacity_matches_reference(built, golden):
    """The camera-like stress content (noise at QP 20) outgrows the capacity the
    reference's whole-array tiled encoder gives each band (twice its raw frame
    plus 64 KiB, fdv.h:7111-7113) within the first GOP: the reference returns
    0 there, and so does fdv_vtile_encode."""
    import fdv_b200 as F
    c3 = golden["c3"]
    sc, e = dict(c3["scene"]), c3["encode"]
    sc["nframes"] = c3["vtile_frames"]
    fr = scene_frames(sc)
    F.set_search_range(e["search_range"])
    try:
        if c3["vtile_fails"]:
            with pytest.raises(F.FdvError, match="capacity"):
                F.vtile_encode(fr, sc["w"], sc["h"], e["qp"], e["keyint"], e["band_mbrows"], 8)
        else:
            F.vtile_encode(fr, sc["w"], sc["h"], e["qp"], e["keyint"], e["band_mbrows"], 8)
    finally:
        F.set_search_range(16)


def test_camera_stress_stream_matches_reference(built, golden):
    """The camera-like stress configuration at full length: 1920x1088, 300
    frames (a 1/f^2 canvas under a 0.5 %/frame zoom and a pan, 200 objects at
    up to 24 px/frame, sensor noise, hard cuts at frames 100 and 200), 17
    bands of 4 macroblock rows, range +-64, QP 20, key interval 60, through
    the streaming tiled encoder (fdv_enc_open_tiled): the .fdv file equals the
    reference's byte for byte, and the GPU decoder's frames equal the
    reference decoder's."""
    import fdv_b200 as F
    c3 = golden["c3"]
    sc, e = c3["scene"], c3["encode"]
    fr = scene_frames(sc)
    assert sha(b"".join(f.tobytes() for f in fr)) == c3["frames_sha256"]
    F.set_search_range(e["search_range"])
    try:
        enc = F.Encoder(sc["w"], sc["h"], e["qp"], e["keyint"], e["band_mbrows"], 8)
        for x in fr:
            enc.frame(x)
        data = enc.finish(c3["fps"])
        del fr
        assert len(data) == c3["file_len"]
        assert sha(data) == c3["file_sha256"]
        dec = F.vtile_decode(data[12:])
    finally:
        F.set_search_range(16)
    assert sha(dec.tobytes()) == c3["decoded_sha256"]
