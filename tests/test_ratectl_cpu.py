"""The average-bitrate controller (fdv_rc_*, fdv.h:7886-8029) against the
reference's compiled one: the same call sequences must leave the two fdv_rc
states equal field for field (doubles compared exactly), and the chosen
quantisers and lambda fractions must agree."""
import ctypes as C
import random

import pytest


class RC(C.Structure):
    _fields_ = [("bitrate", C.c_int), ("fps", C.c_int), ("bufbits", C.c_double), ("qpmin", C.c_int),
                ("qpmax", C.c_int), ("keyint", C.c_int), ("qp_p", C.c_double), ("ip_off", C.c_double),
                ("last_target", C.c_double), ("fill", C.c_double), ("used_qp", C.c_int), ("lscale", C.c_double)]


def _bind(L):
    p = C.POINTER(RC)
    L.fdv_rc_init.argtypes = [p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int]
    L.fdv_rc_pick.argtypes = [p, C.c_int]
    L.fdv_rc_update.argtypes = [p, C.c_int, C.c_size_t]
    L.fdv_rc_skip.argtypes = [p, C.c_size_t]
    L.fdv_rc_adopt.argtypes = [p, C.c_int, C.c_double]
    L.fdv_rc_split.argtypes = [p, C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    return L


def _state(r):
    return tuple(getattr(r, f) for f, _ in RC._fields_)


@pytest.mark.parametrize("seed", range(6))
def test_rate_controller_matches_reference(built, seed):
    import fdv_b200 as F
    import oracle as O
    if not O.have_ref(16):
        pytest.skip("reference library not built")
    ours, ref = _bind(F.lib()), _bind(O.ref(16))
    rnd = random.Random(seed)
    args = (rnd.choice([8000, 250000, 1000000, 6000000]), rnd.choice([0, 25, 30, 60]), rnd.choice([176, 640, 1280]),
            rnd.choice([144, 360, 720]), rnd.choice([0, 1, 30, 60]), rnd.choice([0.0, 0.5, 2.0]),
            rnd.choice([0, 10]), rnd.choice([0, 40]))
    a, b = RC(), RC()
    ours.fdv_rc_init(C.byref(a), *args)
    ref.fdv_rc_init(C.byref(b), *args)
    assert _state(a) == _state(b)
    for step in range(400):
        op = rnd.random()
        intra = int(rnd.random() < 0.1)
        if op < 0.55:
            assert ours.fdv_rc_pick(C.byref(a), intra) == ref.fdv_rc_pick(C.byref(b), intra)
            nbytes = int(rnd.lognormvariate(8, 2))
            ours.fdv_rc_update(C.byref(a), intra, nbytes)
            ref.fdv_rc_update(C.byref(b), intra, nbytes)
        elif op < 0.7:
            nbytes = rnd.randrange(0, 5000)
            ours.fdv_rc_skip(C.byref(a), nbytes)
            ref.fdv_rc_skip(C.byref(b), nbytes)
        elif op < 0.85:
            q = rnd.uniform(-5, 60)
            ours.fdv_rc_adopt(C.byref(a), intra, q)
            ref.fdv_rc_adopt(C.byref(b), intra, q)
        else:
            q = rnd.uniform(-5, 60)
            qa, qb, la, lb = C.c_int(), C.c_int(), C.c_double(), C.c_double()
            ours.fdv_rc_split(C.byref(a), q, C.byref(qa), C.byref(la))
            ref.fdv_rc_split(C.byref(b), q, C.byref(qb), C.byref(lb))
            assert (qa.value, la.value) == (qb.value, lb.value)
        assert _state(a) == _state(b), f"step {step}"
