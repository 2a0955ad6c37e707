"""The allocation-free P-frame entry point (fdvg_pframe_static).

Callers that cannot allocate device memory mid-encode (a host that owns the
GPU's memory pool, a real-time capture path that cannot take cudaMalloc's
implicit synchronisation) use fdvg_pframe_static, whose scratch is a fixed
array inside the library.  Its symbol streams and reconstruction must equal
the CPU oracle's (and so the engine's, fdvg_frame) for the same frames and
references, on calls in a row -- a later call must not see an earlier one's
leftovers -- at search ranges 16, 32 and 64, up to the 1280x720 unit the
scratch is sized for.  Bad arguments (misaligned buffers, units beyond the
scratch) are rejected before anything is queued, and an output buffer too
small for the streams is reported as such.
This file is collected last so a failure here leaves every other test run.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lib():
    import fdv_b200 as F
    L = F.lib()
    L.fdvg_pframe_static.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                     C.c_double, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]
    L.fdvg_pframe_static.restype = C.c_int
    L.fdvg_pframe_static_error.restype = C.c_char_p
    L.fdvg_pframe_static_capacity.restype = C.c_size_t
    return L


def _oracle_result(w, h, rng, qp, cur, near, far):
    import oracle as O
    u = O.OracleUnit(w, h, rng)
    u.set_refs(near, far)
    streams, _ = u.frame(cur, 0, qp)
    return streams, u.recon()


def _engine_result(w, h, rng, qp, cur, near, far):
    import fdv_b200 as F
    eng = F.Engine([(w, h)], rng)
    eng.set_refs(0, near, far)
    eng.step([cur], [0], [qp])
    out = eng.pframe_streams(0), eng.recon(0)
    eng.close()
    return out


def _static_call(L, w, h, rng, qp, cur, near, far, cap=None):
    import torch
    dev = "cuda:0"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    cur_d, near_d = t(cur), t(near)
    far_d = t(far) if far is not None else None
    rec_d = torch.zeros(w * h * 3 // 2, dtype=torch.uint8, device=dev)
    if cap is None:
        cap = 64 + (w // 16) * (h // 16) * 2400
    out_d = torch.zeros(cap, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    rc = L.fdvg_pframe_static(cur_d.data_ptr(), near_d.data_ptr(), far_d.data_ptr() if far_d is not None else None,
                              rec_d.data_ptr(), w, h, qp, 1.0, rng, out_d.data_ptr(), cap, None)
    return rc, out_d, rec_d


def _static_result(L, w, h, rng, qp, cur, near, far):
    rc, out_d, rec_d = _static_call(L, w, h, rng, qp, cur, near, far)
    assert rc == 0, L.fdvg_pframe_static_error()
    out = out_d.cpu().numpy()
    lens = out[:64].view(np.uint32)
    streams, p = [], 64
    for k in range(16):
        streams.append(out[p:p + lens[k]].tobytes())
        p += int(lens[k])
    return streams, rec_d.cpu().numpy()


# (w, h, range, qp, seed, two references): consecutive calls of different
# sizes, ranges and reference counts share the one scratch array
CASES = [(352, 288, 16, 28, 11, True), (256, 144, 32, 20, 12, False), (160, 96, 64, 24, 13, True),
         (1280, 720, 64, 24, 14, True), (352, 288, 16, 28, 11, True)]


def test_static_entry_matches_oracle_on_calls_in_a_row():
    import fdv_b200 as F
    L = _lib()
    for i, (w, h, rng, qp, seed, two) in enumerate(CASES):
        n = max(8, w * h // 6000)
        f0, f1, f2 = F.Scene(w, h, 3, nrects=n, pan_qx=9, pan_qy=-2, static_pct=30, seed=seed).frames(3)
        far = f0 if two else None
        want_streams, want_rec = _oracle_result(w, h, rng, qp, f2, f1, far)
        st, rec = _static_result(L, w, h, rng, qp, f2, f1, far)
        for k in range(16):
            assert st[k] == want_streams[k], f"call {i} ({w}x{h} range {rng}): stream {k}"
        assert np.array_equal(rec, want_rec), f"call {i} ({w}x{h} range {rng}): reconstruction"


def test_static_entry_matches_engine():
    import fdv_b200 as F
    L = _lib()
    w, h, rng, qp = 256, 144, 32, 30
    f0, f1, f2 = F.Scene(w, h, 3, nrects=8, pan_qx=-5, static_pct=20, seed=15).frames(3)
    for _ in range(2):
        want_streams, want_rec = _engine_result(w, h, rng, qp, f2, f1, f0)
        st, rec = _static_result(L, w, h, rng, qp, f2, f1, f0)
        assert st == list(want_streams)
        assert np.array_equal(rec, want_rec)


def test_static_entry_rejects_units_beyond_its_scratch():
    L = _lib()
    assert L.fdvg_pframe_static_capacity() == 24 << 20
    import torch
    b = torch.zeros(16, dtype=torch.uint8, device="cuda:0")
    p = b.data_ptr()
    rc = L.fdvg_pframe_static(p, p, None, p, 1920, 1088, 24, 1.0, 64, p, 16 << 20, None)
    assert rc < 0
    msg = L.fdvg_pframe_static_error().decode()
    assert "scratch" in msg and "1920x1088" in msg


def test_static_entry_rejects_misaligned_buffers():
    """Rejected on the host before any launch: nothing is read or written."""
    L = _lib()
    import torch
    b = torch.zeros(64 * 48 * 3 // 2 + 64, dtype=torch.uint8, device="cuda:0")
    p = b.data_ptr()
    assert p % 16 == 0
    for bad in range(5):
        ptrs = [p, p, p, p, p]
        ptrs[bad] = p + 1
        rc = L.fdvg_pframe_static(ptrs[0], ptrs[1], ptrs[2], ptrs[3], 64, 48, 24, 1.0, 16, ptrs[4], 4096, None)
        assert rc < 0
        assert "16-byte aligned" in L.fdvg_pframe_static_error().decode()


def test_static_entry_reports_a_small_output_buffer():
    import fdv_b200 as F
    L = _lib()
    w, h = 128, 96
    f0, f1 = F.Scene(w, h, 2, nrects=6, pan_qx=9, seed=16).frames(2)
    rc, _, _ = _static_call(L, w, h, 16, 10, f1, f0, None, cap=80)
    assert rc < 0
    assert "output buffer too small" in L.fdvg_pframe_static_error().decode()
    # the next call with room succeeds
    st, rec = _static_result(L, w, h, 16, 10, f1, f0, None)
    want_streams, want_rec = _oracle_result(w, h, 16, 10, f1, f0, None)
    assert st == list(want_streams) and np.array_equal(rec, want_rec)
