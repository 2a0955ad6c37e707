"""GPU decoder parity: fdv_video_decode / fdv_vtile_decode against the
reference decoder (fdv.h:6856-6930, :7303-7372).

* The golden streams (encoded here, byte-identical to the reference's) decode
  to the frames whose SHA-256 digest was recorded from the reference decoder.
* Streams over sizes, QPs 0..51, key intervals and search ranges 16/32/64
  decode exactly as the reference decoder decodes them; tiled streams with
  1-, 2- and 5-row bands likewise.
* Learned-form streams (every macroblock class) decode to the encoder's own
  reconstruction.
* Malformed streams (truncated, corrupt header, corrupt blob, out-of-range
  vector) are rejected with -1, as the reference rejects them, and the decoder
  keeps working afterwards.
"""
import hashlib
import struct

import numpy as np
import pytest

from conftest import scene_frames

pytestmark = pytest.mark.gpu


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def _encode(F, fr, w, h, e):
    if e["band_mbrows"] is None:
        return F.video_encode(fr, w, h, e["qp"], e["keyint"])
    return F.vtile_encode(fr, w, h, e["qp"], e["keyint"], e["band_mbrows"], 4)


@pytest.mark.parametrize("name", ["cif30", "pan256_k5", "tiny_q0", "tiny_q51_r64", "bands_q12", "hd720_g12",
                                  "c3_1088_r64", "hd720_full"])
def test_golden_streams_decode_like_reference(built, golden, name):
    import fdv_b200 as F
    case = golden["cases"][name]
    sc, e = case["scene"], case["encode"]
    fr = scene_frames(sc)
    F.set_search_range(e["search_range"])
    try:
        s = _encode(F, fr, sc["w"], sc["h"], e)
        assert sha(s) == case["stream_sha256"]
        dec = F.video_decode(s) if e["band_mbrows"] is None else F.vtile_decode(s)
    finally:
        F.set_search_range(16)
    assert dec.shape == (sc["nframes"], sc["w"] * sc["h"] * 3 // 2)
    assert sha(dec.tobytes()) == case["decoded_sha256"]


@pytest.mark.parametrize("w,h,qp,keyint,rng,seed", [
    (64, 64, 28, 0, 16, 1), (128, 96, 0, 3, 16, 2), (256, 144, 51, 4, 32, 3), (352, 288, 12, 0, 64, 4),
    (96, 208, 36, 2, 32, 5), (320, 176, 20, 5, 64, 6),
])
def test_streams_decode_like_reference(built, w, h, qp, keyint, rng, seed):
    import fdv_b200 as F
    import oracle as O
    fr = F.Scene(w, h, 7, nrects=max(3, w * h // 3000), pan_qx=7, pan_qy=-2, static_pct=30, vmax_qpel=4 * rng,
                 seed=seed).frames(7)
    F.set_search_range(rng)
    try:
        s = F.video_encode(fr, w, h, qp, keyint)
        dec = F.video_decode(s)
    finally:
        F.set_search_range(16)
    ref = O.ref_video_decode(s, rng)
    assert np.array_equal(dec, ref)


@pytest.mark.parametrize("band_mbrows", [1, 2, 5])
def test_tiled_streams_decode_like_reference(built, band_mbrows):
    import fdv_b200 as F
    import oracle as O
    w, h = 192, 176
    fr = F.Scene(w, h, 6, nrects=9, pan_qx=-5, pan_qy=4, static_pct=20, seed=band_mbrows).frames(6)
    s = F.vtile_encode(fr, w, h, 22, 4, band_mbrows, 4)
    dec = F.vtile_decode(s, 4)
    assert np.array_equal(dec, O.ref_vtile_decode(s, 16))
    assert np.array_equal(F.vtile_decode(s, 1), dec)


def test_learned_stream_decodes_to_encoder_reconstruction(built):
    import fdv_b200 as F
    import fdv_b200.learned as L
    w, h, qp = 320, 192, 23
    frames = F.Scene(w, h, 6, seed=78, **L.CONTENT).frames(6)
    p = L.load_params(L.DEFAULT_WEIGHTS)
    stream, recs, _ = L.encode_engine(frames, w, h, qp, 0, params=p, conf=0.8)
    dec = F.video_decode(stream)
    for f in range(len(frames)):
        assert np.array_equal(dec[f], recs[f]), f


def test_malformed_streams_are_rejected(built):
    import fdv_b200 as F
    import oracle as O
    w, h = 64, 48
    fr = F.Scene(w, h, 4, nrects=3, pan_qx=5, rect_max=24, seed=7).frames(4)
    s = F.video_encode(fr, w, h, 24, 0)
    good = F.video_decode(s)
    bad = [
        s[:len(s) - 3],                                   # truncated last blob
        s[:8],                                            # header only
        struct.pack("<HHH", 4, 40, 48) + s[6:],           # width not a multiple of 16
        s[:6] + bytes([52]) + s[7:],                      # qp out of range
        s[:16] + bytes([9]) + s[17:],                     # key-frame plane header: wrong width
    ]
    # the second frame's blob: an entropy mode that does not exist
    n0 = struct.unpack_from("<I", s, 8)[0]
    p1 = 12 + n0 + 4
    bad.append(s[:p1 + 1] + bytes([7]) + s[p1 + 2:])
    for b in bad:
        with pytest.raises(F.FdvError):
            F.video_decode(b)
        with pytest.raises(RuntimeError):
            O.ref_video_decode(b, 16)
    # a vector past the reference border: the range-16 decoder (32-sample
    # border) rejects a range-64 stream that reaches further, like the reference
    fr2 = F.Scene(128, 64, 3, nrects=4, rect_max=32, pan_qx=220, seed=9).frames(3)
    F.set_search_range(64)
    try:
        far = F.video_encode(fr2, 128, 64, 20, 0)
    finally:
        F.set_search_range(16)
    try:
        ref = O.ref_video_decode(far, 16)
    except RuntimeError:
        ref = None
    if ref is None:
        with pytest.raises(F.FdvError):
            F.video_decode(far)
    else:
        assert np.array_equal(F.video_decode(far), ref)
    assert np.array_equal(F.video_decode(s), good)


def test_corrupted_blobs_match_reference_verdict(built):
    """Single-byte corruptions inside frame blobs: the GPU decoder accepts
    exactly the streams the reference accepts, with the same frames."""
    import fdv_b200 as F
    import oracle as O
    w, h = 64, 64
    fr = F.Scene(w, h, 3, nrects=4, pan_qx=6, seed=12).frames(3)
    s = F.video_encode(fr, w, h, 26, 0)
    rng = np.random.default_rng(5)
    for _ in range(24):
        pos = int(rng.integers(12, len(s)))
        b = bytearray(s)
        b[pos] ^= int(rng.integers(1, 256))
        b = bytes(b)
        try:
            ref = O.ref_video_decode(b, 16)
        except RuntimeError:
            ref = None
        if ref is None:
            with pytest.raises(F.FdvError):
                F.video_decode(b)
        else:
            assert np.array_equal(F.video_decode(b), ref), pos


def test_decoder_timing_counts_launches(built):
    """fdvd_timing brackets every launch: one inter launch per P-frame step,
    one key-frame launch per key step, one frame step per frame."""
    import fdv_b200 as F
    w, h = 128, 96
    fr = F.Scene(w, h, 7, nrects=4, pan_qx=5, seed=3).frames(7)
    s = F.vtile_encode(fr, w, h, 24, 3, 2, 4)
    L = F.lib()
    F.decode_stats(reset=True)
    L.fdvd_timing(1)
    try:
        F.vtile_decode(s)
    finally:
        L.fdvd_timing(0)
    st = F.decode_stats(reset=True)
    assert st["frame"][1] == 7 and st["key"][1] == 3 and st["inter"][1] == 4 and st["frame_ops"][1] == 7
    assert all(v[0] > 0 for k, v in st.items() if v[1] and not k.startswith("host_"))
    assert st["host_symbols"][1] == 7 and st["host_symbols"][0] > 0 and st["host_records"][0] > 0
    F.vtile_decode(s)
    assert F.decode_stats()["frame"][1] == 0
