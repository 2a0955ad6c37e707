"""fdv_b200: the fdv encoder analysis loop on B200, behind the fdv.h encode API.

Python mirror of the library's C ABI (include/fdv_b200.h).  The functions keep
the reference's names, argument meaning and error behaviour (``fdv.h``): the
encoders return the coded bytes, or raise ``FdvError`` where the C call
returns 0 / NULL.  The native library ``libfdvb200.so`` is required; there is
no CPU fallback for the analysis loop.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfdvb200.so")

u8p = C.POINTER(C.c_uint8)


class FdvError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    """The loaded native library (built on first use when nvcc is present)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _b
            _b.build()
        L = C.CDLL(LIB_PATH)
        sz, i, p = C.c_size_t, C.c_int, C.c_void_p
        L.fdv_video_encode.argtypes = [C.POINTER(u8p), i, i, i, i, i, u8p, sz]
        L.fdv_video_encode.restype = sz
        L.fdv_vtile_encode.argtypes = [C.POINTER(u8p), i, i, i, i, i, i, i, u8p, sz]
        L.fdv_vtile_encode.restype = sz
        L.fdv_enc_open.argtypes = [i, i, i, i]
        L.fdv_enc_open.restype = p
        L.fdv_enc_open_tiled.argtypes = [i, i, i, i, i, i]
        L.fdv_enc_open_tiled.restype = p
        L.fdv_enc_frame.argtypes = [p, u8p]
        L.fdv_enc_repeat.argtypes = [p]
        L.fdv_enc_set_bitrate.argtypes = [p, i, i, C.c_double]
        L.fdv_enc_count.argtypes = [p]
        L.fdv_enc_bytes.argtypes = [p]
        L.fdv_enc_bytes.restype = sz
        L.fdv_enc_finish.argtypes = [p, i, C.POINTER(sz)]
        L.fdv_enc_finish.restype = p
        L.fdv_enc_close.argtypes = [p]
        L.fdv_enc_close.restype = None
        L.fdv_wrap.argtypes = [u8p, sz, i, i, u8p, sz]
        L.fdv_wrap.restype = sz
        L.fdvb_set_search_range.argtypes = [i]
        L.fdvb_get_search_range.argtypes = []
        L.fdvb_set_device.argtypes = [i]
        L.fdvb_last_error.restype = C.c_char_p
        L.fdvg_create.argtypes = [i, C.POINTER(i), C.POINTER(i), i, i]
        L.fdvg_create.restype = p
        L.fdvg_destroy.argtypes = [p]
        L.fdvg_destroy.restype = None
        L.fdvg_frame.argtypes = [p, C.POINTER(u8p), C.POINTER(i), C.POINTER(i), C.POINTER(C.c_double), C.POINTER(i)]
        L.fdvg_pframe_streams.argtypes = [p, i, C.POINTER(u8p), C.POINTER(sz)]
        L.fdvg_iframe_streams.argtypes = [p, i, i, C.POINTER(u8p), C.POINTER(sz)]
        L.fdvg_pframe_hist.argtypes = [p, i, C.POINTER(C.c_uint32)]
        L.fdvg_submit.argtypes = [p, C.POINTER(u8p), C.POINTER(i), C.POINTER(i), C.c_void_p, C.c_void_p]
        L.fdvg_collect.argtypes = [p]
        L.fdvg_submit_batch.argtypes = [p, i, C.POINTER(u8p), C.POINTER(i), C.POINTER(i), C.c_void_p, C.c_void_p]
        L.fdvg_max_batch.argtypes = [p]
        L.fdvg_set_tuning.argtypes = [p, i, i]
        L.fdvg_get_tuning.argtypes = [p, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.fdvg_get_tuning.restype = None
        L.fdvb_set_tuning.argtypes = [i, C.POINTER(i), C.POINTER(i), i, i, i]
        L.fdvg_frames_device.argtypes = [p, i, C.POINTER(u8p), C.POINTER(i), C.POINTER(i)]
        L.fdvg_iframe_hist.argtypes = [p, i, i, C.POINTER(C.c_uint32)]
        L.fdvg_recon.argtypes = [p, i, u8p]
        L.fdvg_set_learned.argtypes = [p, C.POINTER(C.c_float), C.c_float]
        L.fdvg_set_records.argtypes = [p, i]
        L.fdvg_set_learned_conf.argtypes = [p, C.POINTER(C.c_float)]
        L.fdvg_mb_records.argtypes = [p, i, u8p, C.POINTER(C.c_int16), u8p, C.POINTER(C.c_float)]
        L.fdvb_set_learned.argtypes = [C.POINTER(C.c_float), C.c_float]
        dd, ll = C.c_double, C.c_longlong
        L.fdvg_stats.argtypes = [p] + [C.POINTER(t) for t in (dd, dd, ll, dd, ll, ll, ll, ll)]
        L.fdvg_stats.restype = None
        L.fdvg_stats_reset.argtypes = [p]
        L.fdvg_stats_reset.restype = None
        L.fdvg_set_refs.argtypes = [p, i, u8p, u8p]
        L.fdvb_tabcache_new.restype = p
        L.fdvb_tabcache_reset.argtypes = [p]
        L.fdvb_tabcache_reset.restype = None
        L.fdvb_tabcache_free.argtypes = [p]
        L.fdvb_tabcache_free.restype = None
        L.fdvb_entropy_pframe.argtypes = [C.POINTER(u8p), C.POINTER(sz), i, p, u8p, sz]
        L.fdvb_entropy_pframe.restype = sz
        L.fdvb_entropy_image.argtypes = [C.POINTER(u8p), C.POINTER(sz), i, i, i, u8p, sz]
        L.fdvb_entropy_image.restype = sz
        L.fdvb_scene_open.argtypes = [p]
        L.fdvb_scene_open.restype = p
        L.fdvb_scene_frame.argtypes = [p, i, u8p]
        L.fdvb_scene_close.argtypes = [p]
        L.fdvb_scene_close.restype = None
        L.fdvb_measure_int_rate.argtypes = [i, i]
        L.fdvb_measure_int_rate.restype = C.c_double
        L.fdvb_camscene_open.argtypes = [p]
        L.fdvb_camscene_open.restype = p
        L.fdvb_camscene_frame.argtypes = [p, i, u8p]
        L.fdvb_camscene_close.argtypes = [p]
        L.fdvb_camscene_close.restype = None
        ip = C.POINTER(i)
        L.fdv_video_decode.argtypes = [u8p, sz, u8p, ip, ip, ip]
        L.fdv_vtile_decode.argtypes = [u8p, sz, u8p, ip, ip, ip, i]
        L.fdvd_last_error.restype = C.c_char_p
        L.fdvd_timing.argtypes = [i]
        L.fdvd_timing.restype = None
        L.fdvd_stats.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_longlong), i]
        L.fdvd_stats.restype = None
        _lib = L
    return _lib


def last_error() -> str:
    return (lib().fdvb_last_error() or b"").decode()


def _ptr(a: np.ndarray) -> "C._Pointer":
    return a.ctypes.data_as(u8p)


def _frames_arg(frames: Sequence[np.ndarray]):
    arr = (u8p * len(frames))(*[_ptr(f) for f in frames])
    return arr


def _as_frames(frames, w: int, h: int) -> list[np.ndarray]:
    fs = w * h * 3 // 2
    out = []
    for f in frames:
        a = np.ascontiguousarray(np.frombuffer(f, dtype=np.uint8) if isinstance(f, (bytes, bytearray)) else f,
                                 dtype=np.uint8).reshape(-1)
        if a.size != fs:
            raise ValueError(f"frame has {a.size} bytes, expected {fs}")
        out.append(a)
    return out


def set_tuning(sizes, search_range: int, max_batch: int, p_grid: int = 0) -> None:
    """Record a launch shape for the fdv_* encoders' engines of this geometry
    (fdvb_set_tuning); max_batch 0 removes it."""
    n = len(sizes)
    w = (C.c_int * n)(*[s[0] for s in sizes])
    h = (C.c_int * n)(*[s[1] for s in sizes])
    if lib().fdvb_set_tuning(n, w, h, search_range, max_batch, p_grid) != 0:
        raise FdvError(last_error())


def measure_int_rate(device: int = 0, reps: int = 5) -> float:
    """32-bit integer lane-operations per second the device retires
    (fdvb_measure_int_rate); 0.0 on error."""
    return float(lib().fdvb_measure_int_rate(device, reps))


def set_search_range(r: int) -> int:
    """Run-time FDV_ME_RANGE: 16, 32 or 64 pels."""
    prev = lib().fdvb_set_search_range(r)
    if prev < 0:
        raise FdvError(last_error())
    return prev


def get_search_range() -> int:
    return lib().fdvb_get_search_range()


def set_learned(params, conf: float = 0.8) -> None:
    """Learned proposals for the fdv_* encoders from the next call on (fdvb_set_learned); None: off."""
    a = None if params is None else np.ascontiguousarray(params, np.float32)
    if lib().fdvb_set_learned(a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None, conf) != 0:
        raise FdvError(last_error())


def video_encode(frames, w: int, h: int, qp: int, keyint: int) -> bytes:
    """fdv_video_encode (fdv.h:903)."""
    fr = _as_frames(frames, w, h)
    cap = w * h * 3 * max(1, len(fr)) + 65536
    out = np.empty(cap, np.uint8)
    n = lib().fdv_video_encode(_frames_arg(fr), len(fr), w, h, qp, keyint, _ptr(out), cap)
    if n == 0:
        raise FdvError(last_error() or "fdv_video_encode failed")
    return out[:n].tobytes()


def vtile_encode(frames, w: int, h: int, qp: int, keyint: int, band_mbrows: int, nthreads: int = 8) -> bytes:
    """fdv_vtile_encode (fdv.h:973)."""
    fr = _as_frames(frames, w, h)
    cap = w * h * 3 * max(1, len(fr)) + 65536
    out = np.empty(cap, np.uint8)
    n = lib().fdv_vtile_encode(_frames_arg(fr), len(fr), w, h, qp, keyint, band_mbrows, nthreads, _ptr(out), cap)
    if n == 0:
        raise FdvError(last_error() or "fdv_vtile_encode failed")
    return out[:n].tobytes()


def _decode(fn, stream: bytes, nf: int, w: int, h: int, *extra) -> np.ndarray:
    if nf <= 0 or w <= 0 or h <= 0 or w % 16 or h % 16:
        raise FdvError("bad stream header")
    src = np.frombuffer(stream, np.uint8)
    out = np.empty(nf * w * h * 3 // 2, np.uint8)
    n, ww, hh = C.c_int(), C.c_int(), C.c_int()
    if fn(_ptr(src), src.size, _ptr(out), C.byref(n), C.byref(ww), C.byref(hh), *extra) != 0:
        raise FdvError((lib().fdvd_last_error() or b"").decode() or "decode failed")
    return out.reshape(n.value, -1)


def video_decode(stream: bytes) -> np.ndarray:
    """fdv_video_decode (fdv.h:907): [nframes][w*h*3/2] I420 frames."""
    if len(stream) < 8:
        raise FdvError("bad stream header")
    nf, w, h = np.frombuffer(stream[:6], "<u2")
    return _decode(lib().fdv_video_decode, stream, int(nf), int(w), int(h))


def vtile_decode(stream: bytes, nthreads: int = 8) -> np.ndarray:
    """fdv_vtile_decode (fdv.h:980): [nframes][w*h*3/2] I420 frames."""
    if len(stream) < 12:
        raise FdvError("bad stream header")
    w, h, nf = np.frombuffer(stream[:6], "<u2")
    return _decode(lib().fdv_vtile_decode, stream, int(nf), int(w), int(h), nthreads)


def decode_stats(reset: bool = True) -> dict:
    """Decoder kernel timing accumulated while fdvd_timing was on (fdvd_stats)."""
    ms = (C.c_double * 9)()
    n = (C.c_longlong * 9)()
    lib().fdvd_stats(ms, n, int(reset))
    keys = ("inter", "intra16", "key", "frame_ops", "frame", "host_symbols", "host_scatter", "host_submit_wait",
            "host_records")
    return {k: (ms[j], n[j]) for j, k in enumerate(keys)}


class Encoder:
    """The streaming encoder, fdv_enc_* (fdv.h:1157-1198)."""

    def __init__(self, w: int, h: int, qp: int, keyint: int, band_mbrows: int | None = None, nthreads: int = 1):
        L = lib()
        self.w, self.h = w, h
        self._e = (L.fdv_enc_open(w, h, qp, keyint) if band_mbrows is None
                   else L.fdv_enc_open_tiled(w, h, qp, keyint, band_mbrows, nthreads))
        if not self._e:
            raise FdvError(last_error() or "fdv_enc_open failed")

    def frame(self, i420) -> None:
        a = _as_frames([i420], self.w, self.h)[0]
        if lib().fdv_enc_frame(self._e, _ptr(a)) != 0:
            raise FdvError(last_error() or "fdv_enc_frame failed")

    def repeat(self) -> None:
        if lib().fdv_enc_repeat(self._e) != 0:
            raise FdvError(last_error() or "fdv_enc_repeat failed")

    def set_bitrate(self, bits_per_second: int, fps: int = 30, bufsecs: float = 1.0) -> None:
        """Average-bitrate control (fdv_enc_set_bitrate, fdv.h:1176); before the first frame."""
        if lib().fdv_enc_set_bitrate(self._e, bits_per_second, fps, bufsecs) != 0:
            raise FdvError(last_error() or "fdv_enc_set_bitrate failed")

    def count(self) -> int:
        return lib().fdv_enc_count(self._e)

    def nbytes(self) -> int:
        return lib().fdv_enc_bytes(self._e)

    def finish(self, fps: int = 25) -> bytes:
        n = C.c_size_t(0)
        p = lib().fdv_enc_finish(self._e, fps, C.byref(n))
        self._e = None
        if not p:
            raise FdvError("fdv_enc_finish returned NULL")
        data = C.string_at(p, n.value)
        C.CDLL(None).free(C.c_void_p(p))
        return data

    def close(self) -> None:
        if self._e:
            lib().fdv_enc_close(self._e)
            self._e = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """The inner engine ABI (fdvg_*): a batch of encoder units stepped together."""

    def __init__(self, sizes: Sequence[tuple[int, int]], search_range: int = 16, device: int = 0):
        n = len(sizes)
        W = (C.c_int * n)(*[s[0] for s in sizes])
        H = (C.c_int * n)(*[s[1] for s in sizes])
        self.sizes = list(sizes)
        self._g = lib().fdvg_create(n, W, H, search_range, device)
        if not self._g:
            raise FdvError(last_error() or "fdvg_create failed")

    def step(self, frames, is_intra, qp, lscale=None, force_skip=None) -> None:
        """One frame for every unit (fdvg_frame)."""
        self._call("fdvg_frame", frames, is_intra, qp, lscale, force_skip)

    def submit(self, frames, is_intra, qp, lscale=None, force_skip=None) -> None:
        """Queue one frame for every unit (fdvg_submit); collect() waits for the oldest."""
        self._call("fdvg_submit", frames, is_intra, qp, lscale, force_skip)

    def collect(self) -> None:
        if lib().fdvg_collect(self._g) != 0:
            raise FdvError(last_error())

    def max_batch(self) -> int:
        return lib().fdvg_max_batch(self._g)

    def set_tuning(self, max_batch: int, p_grid: int = 0) -> None:
        """Launch shape (fdvg_set_tuning): P-frames per launch at most and
        P-kernel blocks (0: one per SM)."""
        if lib().fdvg_set_tuning(self._g, max_batch, p_grid) != 0:
            raise FdvError(last_error())

    def tuning(self) -> dict:
        k, g, n = C.c_int(), C.c_int(), C.c_int()
        lib().fdvg_get_tuning(self._g, C.byref(k), C.byref(g), C.byref(n))
        return {"max_batch": k.value, "p_grid": g.value, "nsm": n.value}

    def submit_batch(self, frames, qp) -> None:
        """Queue consecutive P-frames as one launch (fdvg_submit_batch):
        frames[k][u] is frame k of unit u, qp[k][u] its quantiser; collect()
        then returns them one by one."""
        n, K = len(self.sizes), len(frames)
        self._keep = []
        planes = (u8p * (3 * n * K))()
        for k in range(K):
            for u, ((w, h), f) in enumerate(zip(self.sizes, frames[k])):
                a = _as_frames([f], w, h)[0]
                self._keep.append(a)
                base = a.ctypes.data
                planes[3 * (k * n + u)] = C.cast(base, u8p)
                planes[3 * (k * n + u) + 1] = C.cast(base + w * h, u8p)
                planes[3 * (k * n + u) + 2] = C.cast(base + w * h + (w // 2) * (h // 2), u8p)
        intra = (C.c_int * (n * K))(*([0] * (n * K)))
        q = (C.c_int * (n * K))(*[int(v) for row in qp for v in row])
        if lib().fdvg_submit_batch(self._g, K, planes, intra, q, None, None) != 0:
            raise FdvError(last_error())

    def _call(self, fn, frames, is_intra, qp, lscale, force_skip) -> None:
        n = len(self.sizes)
        self._keep = []
        planes = (u8p * (3 * n))()
        for u, ((w, h), f) in enumerate(zip(self.sizes, frames)):
            if f is None:
                continue
            a = _as_frames([f], w, h)[0]
            self._keep.append(a)
            base = a.ctypes.data
            planes[3 * u] = C.cast(base, u8p)
            planes[3 * u + 1] = C.cast(base + w * h, u8p)
            planes[3 * u + 2] = C.cast(base + w * h + (w // 2) * (h // 2), u8p)
        ii = (C.c_int * n)(*[int(x) for x in is_intra])
        qq = (C.c_int * n)(*[int(x) for x in qp])
        ls = (C.c_double * n)(*lscale) if lscale is not None else None
        fs = (C.c_int * n)(*[int(x) for x in force_skip]) if force_skip is not None else None
        if getattr(lib(), fn)(self._g, planes, ii, qq, ls, fs) != 0:
            raise FdvError(last_error())

    def pframe_streams(self, u: int) -> list[bytes]:
        s = (u8p * 16)()
        n = (C.c_size_t * 16)()
        if lib().fdvg_pframe_streams(self._g, u, s, n) != 0:
            raise FdvError(last_error())
        return [C.string_at(s[k], n[k]) if n[k] else b"" for k in range(16)]

    def iframe_streams(self, u: int, plane: int) -> list[bytes]:
        s = (u8p * 12)()
        n = (C.c_size_t * 12)()
        if lib().fdvg_iframe_streams(self._g, u, plane, s, n) != 0:
            raise FdvError(last_error())
        return [C.string_at(s[k], n[k]) if n[k] else b"" for k in range(12)]

    def pframe_hist(self, u: int) -> np.ndarray:
        """GPU symbol counts of the 16 P-frame streams, [16, 256]."""
        h = np.zeros((16, 256), np.uint32)
        if lib().fdvg_pframe_hist(self._g, u, h.ctypes.data_as(C.POINTER(C.c_uint32))) != 0:
            raise FdvError(last_error())
        return h

    def iframe_hist(self, u: int, plane: int) -> np.ndarray:
        """GPU symbol counts of a key-frame plane's 12 streams, [12, 256]."""
        h = np.zeros((12, 256), np.uint32)
        if lib().fdvg_iframe_hist(self._g, u, plane, h.ctypes.data_as(C.POINTER(C.c_uint32))) != 0:
            raise FdvError(last_error())
        return h

    def set_learned(self, params, conf: float = 0.8) -> None:
        """Learned proposals for later P-frames (fdvg_set_learned); None: off."""
        a = None if params is None else np.ascontiguousarray(params, np.float32)
        ptr = a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None
        if lib().fdvg_set_learned(self._g, ptr, conf) != 0:
            raise FdvError(last_error())

    def set_learned_conf(self, conf3, skip_gate: float = 0.0, inter8: bool = False) -> None:
        """Per-class thresholds (SKIP, inter, intra; above 1 keeps a class on the
        full search), the SKIP gate in units of lambda (0: none), and INTER8 in
        the confident-inter path."""
        a = (C.c_float * 5)(*[float(c) for c in conf3], float(skip_gate), float(bool(inter8)))
        if lib().fdvg_set_learned_conf(self._g, a) != 0:
            raise FdvError(last_error())

    def stats(self) -> dict:
        """Device-timed totals since creation or stats_reset() (fdvg_stats)."""
        v = [C.c_double(), C.c_double(), C.c_longlong(), C.c_double(), C.c_longlong(), C.c_longlong(),
             C.c_longlong(), C.c_longlong()]
        lib().fdvg_stats(self._g, *[C.byref(x) for x in v])
        k = ["step_ms", "p_ms", "p_launches", "i_ms", "i_launches", "launches", "steps", "d2h_bytes"]
        return {n: x.value for n, x in zip(k, v)}

    def stats_reset(self) -> None:
        lib().fdvg_stats_reset(self._g)

    def set_records(self, on: bool) -> None:
        if lib().fdvg_set_records(self._g, int(on)) != 0:
            raise FdvError(last_error())

    def mb_records(self, u: int, cost: bool = True) -> dict:
        """The last P-frame's per-macroblock mode, MV, reference (and RD cost)."""
        w, h = self.sizes[u]
        n = (w // 16) * (h // 16)
        mode = np.empty(n, np.uint8)
        mv = np.empty((n, 2), np.int16)
        ref = np.empty(n, np.uint8)
        c = np.empty(n, np.float32) if cost else None
        if lib().fdvg_mb_records(self._g, u, _ptr(mode), mv.ctypes.data_as(C.POINTER(C.c_int16)), _ptr(ref),
                                 c.ctypes.data_as(C.POINTER(C.c_float)) if cost else None) != 0:
            raise FdvError(last_error())
        return {"mode": mode, "mv": mv, "ref": ref, "cost": c}

    def recon(self, u: int) -> np.ndarray:
        w, h = self.sizes[u]
        out = np.empty(w * h * 3 // 2, np.uint8)
        if lib().fdvg_recon(self._g, u, _ptr(out)) != 0:
            raise FdvError(last_error())
        return out

    def set_refs(self, u: int, near, far=None) -> None:
        w, h = self.sizes[u]
        a = _as_frames([near], w, h)[0]
        b = _as_frames([far], w, h)[0] if far is not None else None
        if lib().fdvg_set_refs(self._g, u, _ptr(a), _ptr(b) if b is not None else None) != 0:
            raise FdvError(last_error())

    def close(self) -> None:
        if self._g:
            lib().fdvg_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TabCache:
    """The entropy state carried between P-frames (fdv.h:590-601)."""

    def __init__(self):
        self._p = lib().fdvb_tabcache_new()

    def reset(self) -> None:
        lib().fdvb_tabcache_reset(self._p)

    def __del__(self):
        try:
            lib().fdvb_tabcache_free(self._p)
        except Exception:
            pass


def _streams_arg(streams: Sequence[bytes]):
    n = len(streams)
    bufs = [np.frombuffer(s, np.uint8) if len(s) else np.zeros(1, np.uint8) for s in streams]
    ptrs = (u8p * n)(*[_ptr(b) for b in bufs])
    lens = (C.c_size_t * n)(*[len(s) for s in streams])
    return bufs, ptrs, lens


def entropy_pframe(streams: Sequence[bytes], qp: int, tc: TabCache) -> bytes:
    """A P-frame blob from its 16 symbol streams (fdv.h:6172-6426)."""
    bufs, ptrs, lens = _streams_arg(streams)
    cap = sum(len(s) for s in streams) * 3 + 65536
    out = np.empty(cap, np.uint8)
    n = lib().fdvb_entropy_pframe(ptrs, lens, qp, tc._p, _ptr(out), cap)
    if n == 0:
        raise FdvError("entropy_pframe failed")
    return out[:n].tobytes()


def entropy_image(streams: Sequence[bytes], w: int, h: int, qp: int) -> bytes:
    """An intra plane blob from its 12 symbol streams (fdv.h:4881-5032)."""
    bufs, ptrs, lens = _streams_arg(streams)
    cap = sum(len(s) for s in streams) * 3 + 65536
    out = np.empty(cap, np.uint8)
    n = lib().fdvb_entropy_image(ptrs, lens, w, h, qp, _ptr(out), cap)
    if n == 0:
        raise FdvError("entropy_image failed")
    return out[:n].tobytes()


class SceneParams(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("nframes", C.c_int), ("nrects", C.c_int),
                ("rect_min", C.c_int), ("rect_max", C.c_int), ("vmax_qpel", C.c_int),
                ("pan_qx", C.c_int), ("pan_qy", C.c_int), ("static_pct", C.c_int),
                ("seed", C.c_ulonglong)]


class Scene:
    """Seeded synthetic content (fdvb_scene_*)."""

    def __init__(self, w, h, nframes, nrects=6, rect_min=8, rect_max=64, vmax_qpel=24,
                 pan_qx=0, pan_qy=0, static_pct=0, seed=1):
        self.w, self.h = w, h
        self._prm = SceneParams(w, h, nframes, nrects, rect_min, rect_max, vmax_qpel, pan_qx, pan_qy,
                                static_pct, seed)
        self._s = lib().fdvb_scene_open(C.byref(self._prm))
        if not self._s:
            raise FdvError("bad scene parameters")

    def frame(self, f: int) -> np.ndarray:
        out = np.empty(self.w * self.h * 3 // 2, np.uint8)
        lib().fdvb_scene_frame(self._s, f, _ptr(out))
        return out

    def frames(self, n: int, start: int = 0) -> list[np.ndarray]:
        return [self.frame(start + i) for i in range(n)]

    def __del__(self):
        try:
            lib().fdvb_scene_close(self._s)
        except Exception:
            pass


class CamSceneParams(C.Structure):
    _fields_ = [("w", C.c_int), ("h", C.c_int), ("nframes", C.c_int), ("nobjects", C.c_int),
                ("obj_min", C.c_int), ("obj_max", C.c_int), ("vmax_qpel", C.c_int), ("zoom_ppm", C.c_int),
                ("pan_qx", C.c_int), ("pan_qy", C.c_int), ("noise_y_x16", C.c_int), ("noise_c_x16", C.c_int),
                ("cut_every", C.c_int), ("seed", C.c_ulonglong)]


class CamScene:
    """Camera-like stress content (fdvb_camscene_*): a 1/f^2 fractal canvas
    under a per-frame affine pan/zoom, fast textured objects, sensor noise and
    a hard cut every ``cut_every`` frames.  ``frames`` renders on several host
    threads (the library call releases the interpreter lock)."""

    def __init__(self, w, h, nframes, nobjects=200, obj_min=8, obj_max=96, vmax_qpel=96, zoom_ppm=5000,
                 pan_qx=9, pan_qy=-4, noise_y_x16=32, noise_c_x16=16, cut_every=100, seed=1):
        self.w, self.h, self.nframes = w, h, nframes
        self._prm = CamSceneParams(w, h, nframes, nobjects, obj_min, obj_max, vmax_qpel, zoom_ppm, pan_qx, pan_qy,
                                   noise_y_x16, noise_c_x16, cut_every, seed)
        self._s = lib().fdvb_camscene_open(C.byref(self._prm))
        if not self._s:
            raise FdvError("bad camera scene parameters")

    def frame(self, f: int) -> np.ndarray:
        out = np.empty(self.w * self.h * 3 // 2, np.uint8)
        if lib().fdvb_camscene_frame(self._s, f, _ptr(out)) != 0:
            raise FdvError("frame out of range")
        return out

    def frames(self, n: int, start: int = 0, threads: int | None = None) -> list[np.ndarray]:
        import concurrent.futures as cf
        with cf.ThreadPoolExecutor(max_workers=threads or min(16, os.cpu_count() or 1)) as ex:
            return list(ex.map(self.frame, range(start, start + n)))

    def __del__(self):
        try:
            lib().fdvb_camscene_close(self._s)
        except Exception:
            pass


# The benchmark workloads (synthetic, seeded).
def workload(name: str, nframes: int | None = None, seed: int = 1) -> tuple[Scene, dict]:
    """Scene and encoder settings of a named workload.

    ``cif30``   352x288, 30 frames, one key frame, QP 28, single tile, range 16, 6 rectangles.
    ``hd720``   1280x720, 120 frames, key interval 60, QP 24, 8 bands of 6 MB rows, range 32,
                40 rectangles, 2.25 px/frame pan, 40% static area.
    """
    if name == "cif30":
        n = nframes or 30
        sc = Scene(352, 288, n, nrects=6, rect_min=8, rect_max=64, vmax_qpel=24, seed=seed)
        return sc, dict(w=352, h=288, nframes=n, qp=28, keyint=0, band_mbrows=None, search_range=16)
    if name == "hd720":
        n = nframes or 120
        sc = Scene(1280, 720, n, nrects=40, rect_min=8, rect_max=64, vmax_qpel=24, pan_qx=9, pan_qy=0,
                   static_pct=40, seed=seed)
        return sc, dict(w=1280, h=720, nframes=n, qp=24, keyint=60, band_mbrows=6, search_range=32)
    raise KeyError(name)
