"""Oracle loaders -- test infrastructure only.

* ``ref(range)``: the reference codec compiled from its own sources
  (oracle/_ref/libfdvref_r{16,32,64}.so, see oracle/build.py).
* ``restatement()``: the CPU restatement of the analysis loop
  (oracle/fdv_oracle.c -> oracle/_build/liboracle.so).
* ``oracle_video_stream``: a whole .fdv video stream composed from the
  restatement's symbol streams and the library's host entropy tail -- the
  check that both match the reference byte for byte.

Only tests, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import os
import struct

import numpy as np

from . import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))
u8p = C.POINTER(C.c_uint8)
_refs: dict[int, C.CDLL] = {}
_orc = None


def have_ref(search_range: int = 16) -> bool:
    return os.path.exists(_build.ref_lib_path(search_range))


def ref(search_range: int = 16) -> C.CDLL:
    if search_range not in _refs:
        path = _build.ref_lib_path(search_range)
        if not os.path.exists(path):
            _build.build_ref()
        L = C.CDLL(path)
        sz, i = C.c_size_t, C.c_int
        L.fdv_video_encode.argtypes = [C.POINTER(u8p), i, i, i, i, i, u8p, sz]
        L.fdv_video_encode.restype = sz
        L.fdv_vtile_encode.argtypes = [C.POINTER(u8p), i, i, i, i, i, i, i, u8p, sz]
        L.fdv_vtile_encode.restype = sz
        L.fdv_video_decode.argtypes = [u8p, sz, u8p, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.fdv_vtile_decode.argtypes = [u8p, sz, u8p, C.POINTER(i), C.POINTER(i), C.POINTER(i), i]
        L.fdv_image_encode.argtypes = [u8p, i, i, i, i, u8p, sz, u8p]
        L.fdv_image_encode.restype = sz
        _refs[search_range] = L
    return _refs[search_range]


def restatement() -> C.CDLL:
    global _orc
    if _orc is None:
        path = _build.oracle_lib_path()
        if not os.path.exists(path):
            _build.build_oracle()
        L = C.CDLL(path)
        L.oracle_open.argtypes = [C.c_int, C.c_int, C.c_int]
        L.oracle_open.restype = C.c_void_p
        L.oracle_close.argtypes = [C.c_void_p]
        L.oracle_frame.argtypes = [C.c_void_p, u8p, C.c_int, C.c_int, C.c_double, C.c_int,
                                   C.c_void_p, C.POINTER(C.c_int)]
        L.oracle_recon.argtypes = [C.c_void_p, u8p]
        L.oracle_free.argtypes = [C.c_void_p]
        L.oracle_mb_info.argtypes = [C.c_void_p, u8p, C.POINTER(C.c_int16)]
        L.oracle_set_refs.argtypes = [C.c_void_p, u8p, u8p]
        _orc = L
    return _orc


class OStreams(C.Structure):
    _fields_ = [("s", C.c_void_p * 16), ("n", C.c_size_t * 16)]


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(u8p)


class OracleUnit:
    """One encoder unit of the CPU restatement."""

    def __init__(self, w: int, h: int, search_range: int = 16):
        self.w, self.h = w, h
        self._u = restatement().oracle_open(w, h, search_range)
        if not self._u:
            raise ValueError("bad oracle unit")

    def frame(self, i420, is_intra: int, qp: int, lscale: float = 1.0, force_skip: int = 0):
        """Returns (streams, tally): 16 P-frame streams, or 3 x 12 key-frame plane streams."""
        a = np.ascontiguousarray(i420, dtype=np.uint8).reshape(-1) if i420 is not None else None
        outs = (OStreams * 3)()
        tally = (C.c_int * 4)()
        restatement().oracle_frame(self._u, _ptr(a) if a is not None else None, is_intra, qp, lscale,
                                   force_skip, C.cast(outs, C.c_void_p), tally)

        def take(o: OStreams, n: int) -> list[bytes]:
            res = []
            for k in range(n):
                p, ln = o.s[k], o.n[k]
                res.append(C.string_at(p, ln) if (p and ln) else b"")
                if p:
                    restatement().oracle_free(p)
            return res
        if is_intra:
            return [take(outs[p], 12) for p in range(3)], None
        return take(outs[0], 16), list(tally)

    def recon(self) -> np.ndarray:
        out = np.empty(self.w * self.h * 3 // 2, np.uint8)
        restatement().oracle_recon(self._u, _ptr(out))
        return out

    def mb_info(self):
        nmb = (self.w // 16) * (self.h // 16)
        modes = np.empty(nmb, np.uint8)
        mvs = np.empty(nmb * 2, np.int16)
        restatement().oracle_mb_info(self._u, _ptr(modes), mvs.ctypes.data_as(C.POINTER(C.c_int16)))
        return modes, mvs.reshape(-1, 2)

    def set_refs(self, near, far=None) -> None:
        a = np.ascontiguousarray(near, dtype=np.uint8).reshape(-1)
        b = np.ascontiguousarray(far, dtype=np.uint8).reshape(-1) if far is not None else None
        restatement().oracle_set_refs(self._u, _ptr(a), _ptr(b) if b is not None else None)

    def __del__(self):
        try:
            restatement().oracle_close(self._u)
        except Exception:
            pass


def compose_video(w: int, h: int, nframes: int, qp: int, keyint: int, frame_blobs: list[bytes]) -> bytes:
    """The video stream container around per-frame blobs (fdv.h:6764-6805)."""
    out = bytearray(struct.pack("<HHHBB", nframes, w, h, qp, keyint))
    for b in frame_blobs:
        out += struct.pack("<I", len(b)) + b
    return bytes(out)


def iframe_blob(planes_blobs: list[bytes]) -> bytes:
    out = bytearray()
    for b in planes_blobs:
        out += struct.pack("<I", len(b)) + b
    return bytes(out)


def oracle_video_stream(frames, w: int, h: int, qp: int, keyint: int, search_range: int = 16) -> bytes:
    """A video stream from the CPU restatement's analysis + the library's entropy tail."""
    import fdv_b200 as F
    u = OracleUnit(w, h, search_range)
    tc = F.TabCache()
    blobs = []
    for f, fr in enumerate(frames):
        is_intra = f == 0 or (keyint > 0 and f % keyint == 0)
        st, _ = u.frame(fr, int(is_intra), qp)
        if is_intra:
            tc.reset()
            pw = [w, w // 2, w // 2]
            ph = [h, h // 2, h // 2]
            blobs.append(iframe_blob([F.entropy_image(st[p], pw[p], ph[p], qp) for p in range(3)]))
        else:
            blobs.append(F.entropy_pframe(st, qp, tc))
    return compose_video(w, h, len(frames), qp, keyint, blobs)


def ref_video_encode(frames, w: int, h: int, qp: int, keyint: int, search_range: int = 16) -> bytes:
    L = ref(search_range)
    fr = [np.ascontiguousarray(f, dtype=np.uint8).reshape(-1) for f in frames]
    arr = (u8p * len(fr))(*[_ptr(a) for a in fr])
    cap = w * h * 3 * len(fr) + 65536
    out = np.empty(cap, np.uint8)
    n = L.fdv_video_encode(arr, len(fr), w, h, qp, keyint, _ptr(out), cap)
    if n == 0:
        raise RuntimeError("reference fdv_video_encode failed")
    return out[:n].tobytes()


def ref_vtile_encode(frames, w: int, h: int, qp: int, keyint: int, band_mbrows: int, nthreads: int = 1,
                     search_range: int = 16) -> bytes:
    L = ref(search_range)
    fr = [np.ascontiguousarray(f, dtype=np.uint8).reshape(-1) for f in frames]
    arr = (u8p * len(fr))(*[_ptr(a) for a in fr])
    cap = w * h * 3 * len(fr) + 65536
    out = np.empty(cap, np.uint8)
    n = L.fdv_vtile_encode(arr, len(fr), w, h, qp, keyint, band_mbrows, nthreads, _ptr(out), cap)
    if n == 0:
        raise RuntimeError("reference fdv_vtile_encode failed")
    return out[:n].tobytes()


def ref_video_decode(stream: bytes, search_range: int = 16) -> np.ndarray:
    """Decoded frames (nframes x I420) of a video stream, by the reference decoder."""
    L = ref(search_range)
    nf, w, h = struct.unpack_from("<HHH", stream, 0)
    buf = np.frombuffer(stream, np.uint8).copy()
    out = np.empty(nf * w * h * 3 // 2, np.uint8)
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    if L.fdv_video_decode(_ptr(buf), len(stream), _ptr(out), C.byref(a), C.byref(b), C.byref(c)) != 0:
        raise RuntimeError("reference decode failed")
    return out.reshape(nf, -1)


def ref_vtile_decode(stream: bytes, search_range: int = 16, nthreads: int = 1) -> np.ndarray:
    """Decoded frames of a tiled stream, by the reference's fdv_vtile_decode on nthreads threads."""
    L = ref(search_range)
    w, h, nf = struct.unpack_from("<HHH", stream, 0)
    buf = np.frombuffer(stream, np.uint8).copy()
    out = np.empty(nf * w * h * 3 // 2, np.uint8)
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    if L.fdv_vtile_decode(_ptr(buf), len(stream), _ptr(out), C.byref(a), C.byref(b), C.byref(c), nthreads) != 0:
        raise RuntimeError("reference tiled decode failed")
    return out.reshape(nf, -1)


def ref_enc_stream(frames, w: int, h: int, qp: int, keyint: int, search_range: int = 16, bitrate: int = 0,
                   fps: int = 30, bufsecs: float = 1.0, band_mbrows: int | None = None, nthreads: int = 1,
                   repeat_after: tuple = ()) -> bytes:
    """The reference's streaming encoder (fdv_enc_*, fdv.h:1157-1198) over
    `frames`, optionally under its average-bitrate control
    (fdv_enc_set_bitrate, :8385); after each frame index in repeat_after a
    held frame (fdv_enc_repeat) is pushed.  Returns the finished .fdv file."""
    L = ref(search_range)
    vp = C.c_void_p
    L.fdv_enc_open.restype = vp
    L.fdv_enc_open.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int]
    L.fdv_enc_open_tiled.restype = vp
    L.fdv_enc_open_tiled.argtypes = [C.c_int] * 6
    L.fdv_enc_set_bitrate.argtypes = [vp, C.c_int, C.c_int, C.c_double]
    L.fdv_enc_frame.argtypes = [vp, u8p]
    L.fdv_enc_repeat.argtypes = [vp]
    L.fdv_enc_finish.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t)]
    L.fdv_enc_finish.restype = vp
    e = L.fdv_enc_open(w, h, qp, keyint) if band_mbrows is None else L.fdv_enc_open_tiled(w, h, qp, keyint,
                                                                                         band_mbrows, nthreads)
    if not e:
        raise RuntimeError("reference fdv_enc_open failed")
    if bitrate and L.fdv_enc_set_bitrate(e, bitrate, fps, bufsecs) != 0:
        raise RuntimeError("reference fdv_enc_set_bitrate failed")
    for i, f in enumerate(frames):
        a = np.ascontiguousarray(f, dtype=np.uint8).reshape(-1)
        if L.fdv_enc_frame(e, _ptr(a)) != 0:
            raise RuntimeError("reference fdv_enc_frame failed")
        if i in repeat_after and L.fdv_enc_repeat(e) != 0:
            raise RuntimeError("reference fdv_enc_repeat failed")
    n = C.c_size_t()
    p = L.fdv_enc_finish(e, fps, C.byref(n))
    if not p:
        raise RuntimeError("reference fdv_enc_finish failed")
    return C.string_at(p, n.value)
