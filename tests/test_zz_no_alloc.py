"""The allocation-free P-frame entry point (fdvg_pframe_static).

Callers that cannot allocate device memory mid-encode (a host that owns the
GPU's memory pool, a real-time capture path that cannot take cudaMalloc's
implicit synchronisation) use fdvg_pframe_static, whose scratch is a fixed
array inside the library.  Its symbol streams and reconstruction must be
identical to the engine's (fdvg_frame) for the same frames and references, on
two calls in a row -- the second call must not see the first one's leftovers.
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


def _engine_result(w, h, rng, qp, cur, near, far):
    import fdv_b200 as F
    eng = F.Engine([(w, h)], rng)
    eng.set_refs(0, near, far)
    eng.step([cur], [0], [qp])
    out = eng.pframe_streams(0), eng.recon(0)
    eng.close()
    return out


def _static_result(L, w, h, rng, qp, cur, near, far):
    import torch
    dev = "cuda:0"
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    cur_d, near_d = t(cur), t(near)
    far_d = t(far) if far is not None else None
    rec_d = torch.zeros(w * h * 3 // 2, dtype=torch.uint8, device=dev)
    cap = 64 + (w // 16) * (h // 16) * 2400
    out_d = torch.zeros(cap, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize()
    rc = L.fdvg_pframe_static(cur_d.data_ptr(), near_d.data_ptr(), far_d.data_ptr() if far_d is not None else None,
                              rec_d.data_ptr(), w, h, qp, 1.0, rng, out_d.data_ptr(), cap, None)
    assert rc == 0, L.fdvg_pframe_static_error()
    out = out_d.cpu().numpy()
    lens = out[:64].view(np.uint32)
    streams, p = [], 64
    for k in range(16):
        streams.append(out[p:p + lens[k]].tobytes())
        p += int(lens[k])
    return streams, rec_d.cpu().numpy()


def test_static_entry_matches_engine_on_two_calls():
    import fdv_b200 as F
    L = _lib()
    cases = [(352, 288, 16, 28, 11), (256, 144, 32, 20, 12)]
    for i, (w, h, rng, qp, seed) in enumerate(cases):
        f0, f1, f2 = F.Scene(w, h, 3, nrects=8, pan_qx=9, static_pct=30, seed=seed).frames(3)
        far = f0 if i == 0 else None
        ref_streams, ref_rec = _engine_result(w, h, rng, qp, f2, f1, far)
        st, rec = _static_result(L, w, h, rng, qp, f2, f1, far)
        for k in range(16):
            assert st[k] == ref_streams[k], f"call {i}: stream {k}"
        assert np.array_equal(rec, ref_rec), f"call {i}: reconstruction"


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
