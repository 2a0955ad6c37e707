"""Host timing of a whole-array encode (fdvb_encode_stats).

After an fdv_vtile_encode call the encoder reports, in milliseconds since
the call entered it, the first submission, the last frame collected and the
end, in that order, and the collect waits and coding time it summed, each
within the call's own wall time."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_encode_stats_are_ordered_and_within_the_call(built):
    import fdv_b200 as F
    L = F.lib()
    L.fdvb_encode_stats.argtypes = [C.POINTER(C.c_double)]
    w, h, nf = 320, 192, 12
    frames = [np.ascontiguousarray(f) for f in F.Scene(w, h, nf, nrects=8, pan_qx=9, seed=21).frames(nf)]
    arr = (F.u8p * nf)(*[f.ctypes.data_as(F.u8p) for f in frames])
    out = np.empty(w * h * 3 // 2 * nf, np.uint8)
    t0 = time.perf_counter()
    n = L.fdv_vtile_encode(arr, nf, w, h, 24, 6, 4, 4, out.ctypes.data_as(F.u8p), out.size)
    wall = (time.perf_counter() - t0) * 1e3
    assert n > 0, F.last_error()
    ms = (C.c_double * 6)()
    L.fdvb_encode_stats(ms)
    first, last, coded, total, waits, coding = list(ms)
    assert 0.0 < first <= last <= total <= wall
    assert coded <= total
    assert 0.0 <= waits <= total and 0.0 < coding <= total
