"""The CPU restatement oracle, pinned to the reference encoder.

* Whole streams: the oracle's analysis composed with the library's host
  entropy tail must equal the reference encoder's bytes (golden SHA-256 digests
  from tests/golden/golden.json, and the reference itself when its library
  oracle/_ref is present).
* Kernels: the restated transforms, quantisers, RDOQ, 8x8 tables, SATD,
  intra predictors, motion compensation, motion search and deblocking against
  the reference's exported functions on seeded inputs, plus the reference
  tests' own known answers (flat block -> DC only; a pure translation is
  recovered with SAD 0).
"""
import ctypes as C
import hashlib

import numpy as np
import pytest

from conftest import scene_frames

i16p = C.POINTER(C.c_int16)
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)


def sha(b):
    return hashlib.sha256(bytes(b)).hexdigest()


def orc():
    import oracle as O
    L = O.restatement()
    return L


def need_ref(rng=16):
    import oracle as O
    if not O.have_ref(rng):
        pytest.skip("reference library not built (no reference sources here)")
    return O.ref(rng)


@pytest.mark.parametrize("name", ["cif30", "pan256_k5", "tiny_q0", "tiny_q51_r64"])
def test_oracle_stream_equals_reference(built, golden, name):
    import oracle as O
    case = golden["cases"][name]
    e = case["encode"]
    fr = scene_frames(case["scene"])
    assert sha(b"".join(f.tobytes() for f in fr)) == case["frames_sha256"], "scene generator changed"
    s = O.oracle_video_stream(fr, case["scene"]["w"], case["scene"]["h"], e["qp"], e["keyint"], e["search_range"])
    assert len(s) == case["stream_len"]
    assert sha(s) == case["stream_sha256"]


def test_oracle_recon_equals_reference_decoder(built, golden):
    import oracle as O
    case = golden["cases"]["pan256_k5"]
    e, sc = case["encode"], case["scene"]
    fr = scene_frames(sc)
    u = O.OracleUnit(sc["w"], sc["h"], e["search_range"])
    recs = []
    for f, x in enumerate(fr):
        u.frame(x, int(f % e["keyint"] == 0), e["qp"])
        recs.append(u.recon())
    assert sha(np.concatenate(recs).tobytes()) == case["decoded_sha256"]


def test_known_answers(built, golden):
    L = orc()
    k = golden["kernels"]
    res = (C.c_int16 * 16)(*([10] * 16))
    co = (C.c_int32 * 16)()
    L.oracle_fdct4x4(res, co)
    assert list(co) == k["fdct4x4_flat10"] == [160] + [0] * 15
    v = k["fdct4x4_seed42"]
    blk = (C.c_int16 * 16)(*v["in"])
    L.oracle_fdct4x4(blk, co)
    assert list(co) == v["coeff"]
    lev = (C.c_int16 * 16)()
    L.oracle_quant4x4(co, lev, 24)
    assert list(lev) == v["level_qp24"]
    c8 = (C.c_int32 * 64)()
    q8 = (C.c_int32 * 52)()
    L.oracle_c8_tables(c8, q8)
    assert list(c8) == k["c8"] and list(q8) == k["qstep8"]


def test_motion_search_recovers_translation(built):
    # the reference's own check (test_enc.c:817-826): content shifted by
    # (12, -8) pels is found exactly, with zero SAD
    L = orc()
    L.oracle_me_search.argtypes = [u8p, C.c_int, u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                   C.POINTER(C.c_int)]
    rng = np.random.default_rng(3)
    W = H = 96
    ref = rng.integers(0, 256, (H, W)).astype(np.uint8)
    # smooth so the diamond can descend
    ref = (np.cumsum(np.cumsum(ref.astype(np.int64), 0), 1) // 64 % 256).astype(np.uint8)
    cur = np.zeros_like(ref)
    for y in range(H):
        for x in range(W):
            cur[y, x] = ref[min(max(y - 8, 0), H - 1), min(max(x + 12, 0), W - 1)]
    mx, my = C.c_int(), C.c_int()
    sad = L.oracle_me_search(cur.ctypes.data_as(u8p), W, ref.ctypes.data_as(u8p), W, H, W, 40, 40, 16, 16, 16,
                             48, -32, C.byref(mx), C.byref(my))
    assert (mx.value, my.value, sad) == (48, -32, 0)


def test_kernels_vs_reference(built):
    R = need_ref(16)
    L = orc()
    rng = np.random.default_rng(11)
    for trial in range(400):
        qp = int(rng.integers(0, 52))
        lam = 0.425 * 2.0 ** ((qp - 12) / 3.0)
        res = rng.integers(-60, 61, 16).astype(np.int16) if trial % 2 else rng.integers(-255, 256, 16).astype(np.int16)
        a, b = (C.c_int32 * 16)(), (C.c_int32 * 16)()
        R.fdv_fdct4x4(res.ctypes.data_as(i16p), a)
        L.oracle_fdct4x4(res.ctypes.data_as(i16p), b)
        assert list(a) == list(b)
        la, lb = (C.c_int16 * 16)(), (C.c_int16 * 16)()
        R.fdv_quant4x4(a, la, qp)
        L.oracle_quant4x4(b, lb, qp)
        assert list(la) == list(lb)
        R.fdv_rdoq4x4.argtypes = [i16p, i16p, C.c_int, C.c_double]
        L.oracle_rdoq4x4.argtypes = [i16p, i16p, C.c_int, C.c_double]
        R.fdv_rdoq4x4(la, res.ctypes.data_as(i16p), qp, lam)
        L.oracle_rdoq4x4(lb, res.ctypes.data_as(i16p), qp, lam)
        assert list(la) == list(lb)
        da, db = (C.c_int32 * 16)(), (C.c_int32 * 16)()
        R.fdv_dequant4x4(la, da, qp)
        L.oracle_dequant4x4(lb, db, qp)
        assert list(da) == list(db)
        ra, rb = (C.c_int16 * 16)(), (C.c_int16 * 16)()
        R.fdv_idct4x4(da, ra)
        L.oracle_idct4x4(db, rb)
        assert list(ra) == list(rb)
        # 8x8
        x8 = rng.integers(-255, 256, 64).astype(np.int16)
        y8a, y8b = (C.c_int32 * 64)(), (C.c_int32 * 64)()
        R.fdv_fdct8x8(x8.ctypes.data_as(i16p), y8a)
        L.oracle_fdct8x8(x8.ctypes.data_as(i16p), y8b)
        assert list(y8a) == list(y8b)
        l8a, l8b = (C.c_int16 * 64)(), (C.c_int16 * 64)()
        R.fdv_quant8x8(y8a, l8a, qp)
        L.oracle_quant8x8(y8b, l8b, qp)
        assert list(l8a) == list(l8b)
        R.fdv_dequant8x8(l8a, y8a, qp)
        L.oracle_dequant8x8(l8b, y8b, qp)
        r8a, r8b = (C.c_int16 * 64)(), (C.c_int16 * 64)()
        R.fdv_idct8x8(y8a, r8a)
        L.oracle_idct8x8(y8b, r8b)
        assert list(r8a) == list(r8b)
        # SATD and the 4x4 / n x n intra predictors
        src = rng.integers(0, 256, 16).astype(np.uint8)
        pred = rng.integers(0, 256, 16).astype(np.uint8)
        assert R.fdv_satd4x4(src.ctypes.data_as(u8p), 4, pred.ctypes.data_as(u8p)) == \
            L.oracle_satd4x4(src.ctypes.data_as(u8p), 4, pred.ctypes.data_as(u8p))
        top = rng.integers(0, 256, 64).astype(np.uint8)
        left = rng.integers(0, 256, 64).astype(np.uint8)
        tl = int(rng.integers(0, 256))
        ht, hl = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        m = int(rng.integers(0, 9))
        pa, pb = (C.c_uint8 * 16)(), (C.c_uint8 * 16)()
        R.fdv_intra_predict_4x4(m, top.ctypes.data_as(u8p), left.ctypes.data_as(u8p), C.c_uint8(tl), 1, 1, pa)
        L.oracle_intra4x4(m, top.ctypes.data_as(u8p), left.ctypes.data_as(u8p), C.c_uint8(tl), 1, 1, pb)
        assert list(pa) == list(pb)
        n = int(rng.choice([8, 16, 32, 64]))
        pa, pb = (C.c_uint8 * (n * n))(), (C.c_uint8 * (n * n))()
        mm = int(rng.integers(0, 4))
        R.fdv_intra_nxn(mm, top.ctypes.data_as(u8p), left.ctypes.data_as(u8p), C.c_uint8(tl), n, ht, hl, pa)
        L.oracle_intra_nxn(mm, top.ctypes.data_as(u8p), left.ctypes.data_as(u8p), C.c_uint8(tl), n, ht, hl, pb)
        assert list(pa) == list(pb)


class FdvPlane(C.Structure):
    _fields_ = [("base", C.c_void_p), ("data", C.c_void_p), ("width", C.c_int), ("height", C.c_int),
                ("stride", C.c_int), ("border", C.c_int)]


class FdvFrame(C.Structure):
    _fields_ = [("planes", FdvPlane * 3), ("width", C.c_int), ("height", C.c_int),
                ("subsample_x", C.c_int), ("subsample_y", C.c_int)]


def test_mc_deblock_vs_reference(built):
    """Every quarter-pel phase of luma MC and bilinear chroma MC, block sizes 16
    and 8 / 8 and 4, including vectors reaching into the border, and the
    deblocking filter at several QPs -- restated (edge clamping) vs reference
    (replicated border planes)."""
    R = need_ref(16)
    L = orc()
    rng = np.random.default_rng(5)
    W, H = 96, 64
    img = rng.integers(0, 256, (H, W)).astype(np.uint8)
    f = FdvFrame()
    assert R.fdv_frame_alloc(C.byref(f), W, H) == 0
    pl = f.planes[0]
    for y in range(H):
        C.memmove(pl.data + y * pl.stride, img[y].ctypes.data, W)
    R.fdv_frame_extend_borders(C.byref(f))
    R.fdv_mc_luma.argtypes = [C.POINTER(FdvPlane), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, u8p, C.c_int]
    R.fdv_mc_chroma.argtypes = R.fdv_mc_luma.argtypes
    for trial in range(300):
        bw = int(rng.choice([8, 16]))
        bx = int(rng.integers(0, W - bw + 1)) // 4 * 4
        by = int(rng.integers(0, H - bw + 1)) // 4 * 4
        mvx, mvy = int(rng.integers(-4 * 19, 4 * 19)), int(rng.integers(-4 * 19, 4 * 19))
        a = np.zeros(bw * bw, np.uint8)
        b = np.zeros(bw * bw, np.uint8)
        R.fdv_mc_luma(C.byref(pl), bx, by, bw, bw, mvx, mvy, a.ctypes.data_as(u8p), bw)
        L.oracle_mc_luma(img.ctypes.data_as(u8p), W, H, W, bx, by, bw, bw, mvx, mvy, b.ctypes.data_as(u8p), bw)
        assert np.array_equal(a, b), (bx, by, bw, mvx, mvy)
        cbw = bw // 2
        R.fdv_mc_chroma(C.byref(pl), bx, by, cbw, cbw, mvx // 2, mvy // 2, a.ctypes.data_as(u8p), cbw)
        L.oracle_mc_chroma(img.ctypes.data_as(u8p), W, H, W, bx, by, cbw, cbw, mvx // 2, mvy // 2,
                           b.ctypes.data_as(u8p), cbw)
        assert np.array_equal(a[:cbw * cbw], b[:cbw * cbw])
    R.fdv_frame_free(C.byref(f))
    for qp in [0, 10, 24, 37, 51]:
        x = rng.integers(0, 256, (40, 56)).astype(np.uint8)
        x = (x // 16 * 16 + rng.integers(0, 6, x.shape)).astype(np.uint8)
        a, b = x.copy(), x.copy()
        R.fdv_deblock_plane(a.ctypes.data_as(u8p), 56, 40, 56, qp)
        L.oracle_deblock(b.ctypes.data_as(u8p), 56, 40, 56, qp)
        assert np.array_equal(a, b)


def test_oracle_stream_equals_reference_live(built, golden):
    """Direct comparison with the reference encoder (when its library is here)."""
    import oracle as O
    need_ref(32)
    case = golden["cases"]["bands_q12"]
    sc, e = case["scene"], case["encode"]
    fr = scene_frames(sc)
    # each band of the tiled stream is an independent video; compare band 0
    w, bh = sc["w"], e["band_mbrows"] * 16
    band = [np.concatenate([f[:w * sc["h"]].reshape(sc["h"], w)[:bh].ravel(),
                            f[w * sc["h"]:w * sc["h"] * 5 // 4].reshape(sc["h"] // 2, w // 2)[:bh // 2].ravel(),
                            f[w * sc["h"] * 5 // 4:].reshape(sc["h"] // 2, w // 2)[:bh // 2].ravel()]) for f in fr]
    ours = O.oracle_video_stream(band, w, bh, e["qp"], e["keyint"], e["search_range"])
    assert ours == O.ref_video_encode(band, w, bh, e["qp"], e["keyint"], e["search_range"])


def test_opcount_build_counts_every_category():
    """The op-counting build of the restatement (oracle.opcount) counts a P-frame's
    searches, compensation, transforms and pixels; the normal build has no counter."""
    import ctypes as C
    import fdv_b200 as F
    import oracle as O
    import oracle.opcount as OC
    path = OC.build_counting()
    L = C.CDLL(path)
    L.oracle_opcount.argtypes = [C.POINTER(C.c_ulonglong), C.c_int]
    assert not hasattr(O.restatement(), "oracle_opcount")
    saved, O._orc = O._orc, None
    p0 = O._build.oracle_lib_path
    O._build.oracle_lib_path = lambda: path
    try:
        u = O.OracleUnit(64, 48, 16)
        fr = F.Scene(64, 48, 2, nrects=3, pan_qx=5, rect_max=24, seed=7).frames(2)
        buf = (C.c_ulonglong * len(OC.CATS))()
        u.frame(fr[0], 1, 24)
        O._orc.oracle_opcount(buf, 1)
        u.frame(fr[1], 0, 24)
        O._orc.oracle_opcount(buf, 1)
        got = dict(zip(OC.CATS, list(buf)))
    finally:
        O._build.oracle_lib_path = p0
        O._orc = saved
    for k in ("sad", "mc", "transform4", "quant4", "pixel", "deblock"):
        assert got[k] > 0, k
