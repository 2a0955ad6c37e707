"""The learned proposal network: Python mirror of the fdvl_* C ABI.

``Net`` owns a network on one GPU (fp32 master weights, bf16 tensor-core
copies, Adam state) and a bank of luma planes its samples index.  Samples are
``SAMPLE`` records: bank slots of the current picture and its nearest
reference, the macroblock, the mode class (0 SKIP, 1 inter, 2 intra), an
optional quarter-pel MV target and a weight.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import FdvError, lib as _lib

SAMPLE = np.dtype([("cur", "<i4"), ("ref", "<i4"), ("mbx", "<i4"), ("mby", "<i4"), ("cls", "<i4"),
                   ("has_mv", "<i4"), ("mvx", "<i4"), ("mvy", "<i4"), ("qp", "<i4"), ("weight", "<f4")])
NOUT_PAD = 16
HINT = np.dtype([("mv", "<i2", (4, 2)), ("cls", "<i4")])
_ready = False


def lib() -> C.CDLL:
    global _ready
    L = _lib()
    if not _ready:
        i, p, f, fp = C.c_int, C.c_void_p, C.c_float, C.POINTER(C.c_float)
        L.fdvl_nparams.restype = i
        L.fdvl_create.argtypes = [i, i, i, i, i]
        L.fdvl_create.restype = p
        L.fdvl_destroy.argtypes = [p]
        L.fdvl_destroy.restype = None
        L.fdvl_set_params.argtypes = [p, fp]
        L.fdvl_get_params.argtypes = [p, fp]
        L.fdvl_bank_put.argtypes = [p, i, C.POINTER(C.c_uint8)]
        L.fdvl_features.argtypes = [p, p, i, fp]
        L.fdvl_forward.argtypes = [p, p, i, fp]
        L.fdvl_forward_fused.argtypes = [p, p, i, f, i, fp, p]
        L.fdvl_grads.argtypes = [p, p, i, fp, fp]
        L.fdvl_train_step.argtypes = [p, p, i, f, fp]
        L.fdvl_train.argtypes = [p, p, i, i, i, f, C.c_ulonglong, fp]
        L.fdvl_last_error.restype = C.c_char_p
        L.fdvl_gemm.argtypes = [i, i, i, i, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), fp, i]
        _ready = True
    return L


def last_error() -> str:
    return (lib().fdvl_last_error() or b"").decode()


def _f(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise FdvError(f"{what}: {last_error()}")


def nparams() -> int:
    return lib().fdvl_nparams()


def samples(n: int) -> np.ndarray:
    return np.zeros(n, SAMPLE)


def gemm(a_bits: np.ndarray, b_bits: np.ndarray, nsplit: int = 1, device: int = 0) -> np.ndarray:
    """D = A * B^T on the tensor cores; A [M][K], B [N][K] as bf16 bit patterns (uint16)."""
    a = np.ascontiguousarray(a_bits, np.uint16)
    b = np.ascontiguousarray(b_bits, np.uint16)
    m, k = a.shape
    n = b.shape[0]
    d = np.empty((m, n), np.float32)
    u16 = C.POINTER(C.c_uint16)
    _check(lib().fdvl_gemm(device, m, n, k, a.ctypes.data_as(u16), b.ctypes.data_as(u16), _f(d), nsplit), "gemm")
    return d


class Net:
    def __init__(self, w: int, h: int, bank_frames: int, max_batch: int = 512, device: int = 0):
        self.w, self.h = w, h
        self._n = lib().fdvl_create(device, max_batch, bank_frames, w, h)
        if not self._n:
            raise FdvError(last_error())

    def close(self) -> None:
        if self._n:
            lib().fdvl_destroy(self._n)
            self._n = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: np.ndarray) -> None:
        a = np.ascontiguousarray(p, np.float32)
        assert a.size == nparams()
        _check(lib().fdvl_set_params(self._n, _f(a)), "set_params")

    def params(self) -> np.ndarray:
        a = np.empty(nparams(), np.float32)
        _check(lib().fdvl_get_params(self._n, _f(a)), "get_params")
        return a

    def bank_put(self, slot: int, y: np.ndarray) -> None:
        a = np.ascontiguousarray(y, np.uint8).reshape(-1)[: self.w * self.h]
        _check(lib().fdvl_bank_put(self._n, slot, a.ctypes.data_as(C.POINTER(C.c_uint8))), "bank_put")

    def features(self, s: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(s, SAMPLE)
        x = np.empty((len(s), 32, 32, 4), np.float32)
        _check(lib().fdvl_features(self._n, s.ctypes.data, len(s), _f(x)), "features")
        return x

    def forward(self, s: np.ndarray) -> np.ndarray:
        s = np.ascontiguousarray(s, SAMPLE)
        o = np.empty((len(s), NOUT_PAD), np.float32)
        _check(lib().fdvl_forward(self._n, s.ctypes.data, len(s), _f(o)), "forward")
        return o

    def forward_fused(self, s: np.ndarray, conf: float = 0.8, lim: int = 64):
        """Outputs and proposals through the fused per-frame inference kernel."""
        s = np.ascontiguousarray(s, SAMPLE)
        o = np.empty((len(s), NOUT_PAD), np.float32)
        hs = np.empty(len(s), HINT)
        _check(lib().fdvl_forward_fused(self._n, s.ctypes.data, len(s), conf, lim, _f(o), hs.ctypes.data),
               "forward_fused")
        return o, hs

    def grads(self, s: np.ndarray):
        s = np.ascontiguousarray(s, SAMPLE)
        g = np.empty(nparams(), np.float32)
        loss = np.empty(3, np.float32)
        _check(lib().fdvl_grads(self._n, s.ctypes.data, len(s), _f(g), _f(loss)), "grads")
        return g, loss

    def train_step(self, s: np.ndarray, lr: float) -> np.ndarray:
        s = np.ascontiguousarray(s, SAMPLE)
        loss = np.empty(3, np.float32)
        _check(lib().fdvl_train_step(self._n, s.ctypes.data, len(s), lr, _f(loss)), "train_step")
        return loss

    def train(self, s: np.ndarray, batch: int, epochs: int, lr: float, seed: int = 1) -> np.ndarray:
        s = np.ascontiguousarray(s, SAMPLE)
        curve = np.zeros(2 * epochs, np.float32)
        _check(lib().fdvl_train(self._n, s.ctypes.data, len(s), batch, epochs, lr, seed, _f(curve)), "train")
        return curve.reshape(epochs, 2)


# ---------------------------------------------------------------------------
# Training data, training, and the learned-proposal encoder
# ---------------------------------------------------------------------------
# Content of the learned form's workload: the small workload's generator
# (band-limited noise background, 6 textured rectangles of 8-64 px moving at up
# to 6 px/frame) at 1280x720, search range 16, QPs 18-32.
CONTENT = dict(nrects=6, rect_min=8, rect_max=64, vmax_qpel=24, pan_qx=0, pan_qy=0, static_pct=0)
QPS = (18, 23, 28, 32)
W, H, RANGE = 1280, 720, 16
CLS_OF_MODE = np.array([0, 1, 2, 1], np.int32)   # SKIP, INTER16, INTRA16, INTER8 -> class


def collect(nframes: int = 2000, clip: int = 50, qps=QPS, seed0: int = 1000, skip_keep: float = 0.25,
            w: int = W, h: int = H, search_range: int = RANGE, device: int = 0, max_batch: int = 512,
            rng_seed: int = 7):
    """(block, chosen MV, chosen mode, RD cost) tuples of the plain encoder.

    Clips of ``clip`` frames (a key frame, then P-frames) of seeded content at
    the QPs in turn; every P-frame's source luma and nearest reference (the
    previous reconstruction) go into a new training network's bank, and its
    macroblocks become samples: every non-SKIP one and ``skip_keep`` of the
    SKIPs.  Returns (net, samples, info)."""
    from . import Engine, Scene
    nclips = max(1, nframes // clip)
    npf = nclips * (clip - 1)
    net = Net(w, h, 2 * npf, max_batch=max_batch, device=device)
    eng = Engine([(w, h)], search_range, device)
    eng.set_records(True)
    rng = np.random.default_rng(rng_seed)
    parts, slot = [], 0
    mbw, mbh = w // 16, h // 16
    mbx = np.tile(np.arange(mbw), mbh)
    mby = np.repeat(np.arange(mbh), mbw)
    counts = np.zeros(4, np.int64)
    for c in range(nclips):
        qp = qps[c % len(qps)]
        sc = Scene(w, h, clip, seed=seed0 + c, **CONTENT)
        prev = None
        for f in range(clip):
            fr = sc.frame(f)
            eng.step([fr], [int(f == 0)], [qp])
            if f > 0:
                net.bank_put(slot, fr[: w * h])
                net.bank_put(slot + 1, prev[: w * h])
                r = eng.mb_records(0)
                m = r["mode"]
                counts += np.bincount(m, minlength=4)[:4]
                keep = (m != 0) | (rng.random(m.size) < skip_keep)
                k = np.nonzero(keep)[0]
                s = samples(k.size)
                s["cur"], s["ref"] = slot, slot + 1
                s["mbx"], s["mby"] = mbx[k], mby[k]
                s["cls"] = CLS_OF_MODE[m[k]]
                s["has_mv"] = ((s["cls"] != 2) & (r["ref"][k] == 0)).astype(np.int32)
                s["mvx"], s["mvy"] = r["mv"][k, 0], r["mv"][k, 1]
                s["qp"] = qp
                # non-SKIP decisions are rarer and costlier to get wrong
                s["weight"] = np.where(s["cls"] == 0, 1.0, 3.0).astype(np.float32)
                parts.append(s)
                slot += 2
            prev = eng.recon(0)
    eng.close()
    smp = np.concatenate(parts)
    info = {"frames": nclips * clip, "p_frames": npf, "tuples": int(smp.size),
            "mode_counts": counts.tolist(), "class_counts": np.bincount(smp["cls"], minlength=3).tolist()}
    return net, smp, info


# fp32 parameter layout (fdv_b200/csrc/device/learned.cuh): per layer W[cout][k] then b[cout]
GEO = [(4, 32, 37), (32, 64, 288), (64, 160, 576), (160, 11, 2560)]   # cin, cout, k


def init_params(seed: int = 1) -> np.ndarray:
    """He-uniform weights, zero biases (the training run's starting point)."""
    rng = np.random.default_rng(seed)
    out = []
    for _, cout, k in GEO:
        lim = np.sqrt(6.0 / k)
        out.append(rng.uniform(-lim, lim, cout * k).astype(np.float32))
        out.append(np.zeros(cout, np.float32))
    p = np.concatenate(out)
    assert p.size == nparams()
    return p


def train(net: Net, smp: np.ndarray, epochs: int = 3, batch: int = 512, lr: float = 2e-3, seed: int = 1):
    """Adam on the GPU from a fresh He-uniform start; returns the per-epoch (mode, MV) loss curve."""
    net.set_params(init_params(seed))
    return net.train(smp, batch, epochs, lr, seed)


def save_params(path: str, p: np.ndarray) -> None:
    np.ascontiguousarray(p, np.float32).tofile(path)


def load_params(path: str) -> np.ndarray:
    p = np.fromfile(path, np.float32)
    if p.size != nparams():
        raise FdvError(f"{path}: {p.size} parameters, expected {nparams()}")
    return p


DEFAULT_WEIGHTS = __import__("os").path.join(__import__("os").path.dirname(__file__), "proposal_c4.f32")


def container(w: int, h: int, qp: int, keyint: int, blobs: list[bytes]) -> bytes:
    """The video container around per-frame blobs (fdv_video_encode's, fdv.h:6764-6805)."""
    import struct
    out = bytearray(struct.pack("<HHHBB", len(blobs), w, h, qp, keyint))
    for b in blobs:
        out += struct.pack("<I", len(b)) + b
    return bytes(out)


def encode_engine(frames, w: int, h: int, qp: int, keyint: int = 0, params=None, conf=0.8,
                  search_range: int = RANGE, device: int = 0, batch: int = 1):
    """One stream through the engine and the host entropy tail, plain or with
    learned proposals; returns (stream, reconstructions, P-frame analysis ms).
    batch > 1: runs of up to `batch` P-frames per launch (fdvg_submit_batch),
    the reconstructions then taken from decoding the stream (the decoder's
    frames equal the encoder's reconstruction)."""
    import struct
    from . import Engine, TabCache, entropy_image, entropy_pframe, video_decode
    if batch > 1:
        return _encode_engine_batched(frames, w, h, qp, keyint, params, conf, search_range, device, batch)
    eng = Engine([(w, h)], search_range, device)
    if params is not None:
        if np.ndim(conf):
            eng.set_learned(params, 0.8)
            eng.set_learned_conf(conf[:3], conf[3] if len(conf) > 3 else 0.0, bool(conf[4]) if len(conf) > 4 else False)
        else:
            eng.set_learned(params, conf)
    tc = TabCache()
    blobs, recs = [], []
    pw, ph = [w, w // 2, w // 2], [h, h // 2, h // 2]
    for f, fr in enumerate(frames):
        intra = f == 0 or (keyint > 0 and f % keyint == 0)
        eng.step([fr], [int(intra)], [qp])
        if intra:
            tc.reset()
            b = bytearray()
            for p in range(3):
                pb = entropy_image(eng.iframe_streams(0, p), pw[p], ph[p], qp)
                b += struct.pack("<I", len(pb)) + pb
            blobs.append(bytes(b))
        else:
            blobs.append(entropy_pframe(eng.pframe_streams(0), qp, tc))
        recs.append(eng.recon(0))
    st = eng.stats()
    eng.close()
    return container(w, h, qp, keyint, blobs), recs, st


def _encode_engine_batched(frames, w, h, qp, keyint, params, conf, search_range, device, batch):
    import struct
    from . import Engine, TabCache, entropy_image, entropy_pframe, video_decode
    eng = Engine([(w, h)], search_range, device)
    if params is not None:
        if np.ndim(conf):
            eng.set_learned(params, 0.8)
            eng.set_learned_conf(conf[:3], conf[3] if len(conf) > 3 else 0.0, bool(conf[4]) if len(conf) > 4 else False)
        else:
            eng.set_learned(params, conf)
    batch = min(batch, eng.max_batch())
    tc = TabCache()
    blobs = []
    pw, ph = [w, w // 2, w // 2], [h, h // 2, h // 2]
    key = lambda f: f == 0 or (keyint > 0 and f % keyint == 0)
    f = 0
    while f < len(frames):
        if key(f):
            eng.step([frames[f]], [1], [qp])
            tc.reset()
            b = bytearray()
            for p in range(3):
                pb = entropy_image(eng.iframe_streams(0, p), pw[p], ph[p], qp)
                b += struct.pack("<I", len(pb)) + pb
            blobs.append(bytes(b))
            f += 1
            continue
        n = 1
        while n < batch and f + n < len(frames) and not key(f + n):
            n += 1
        eng.submit_batch([[frames[f + k]] for k in range(n)], [[qp]] * n)
        for _ in range(n):
            eng.collect()
            blobs.append(entropy_pframe(eng.pframe_streams(0), qp, tc))
        f += n
    st = eng.stats()
    eng.close()
    stream = container(w, h, qp, keyint, blobs)
    return stream, list(video_decode(stream)), st


def device_stats(frames, w: int, h: int, qp: int, params=None, conf=0.8, search_range: int = RANGE,
                 device: int = 0) -> dict:
    """Device-timed engine statistics (fdvg_stats) of one stream coded from
    device-resident sources through fdvg_frames_device, as the product path
    runs it: one key frame, then P-frames in launches of up to thirty, the
    learned form's inference on its own stream ahead of each launch.  A
    warm-up pass runs first; the figures are the second pass's."""
    import ctypes as C
    import torch
    from . import Engine, last_error, lib as flib, u8p
    L = flib()
    nf = len(frames)
    dev = torch.from_numpy(np.stack(frames)).to(f"cuda:{device}")
    torch.cuda.synchronize(device)
    fs, cw = w * h * 3 // 2, w // 2
    planes = (u8p * (3 * nf))()
    for f in range(nf):
        fb = dev.data_ptr() + f * fs
        planes[3 * f], planes[3 * f + 1], planes[3 * f + 2] = (C.cast(fb, u8p), C.cast(fb + w * h, u8p),
                                                               C.cast(fb + w * h + (h // 2) * cw, u8p))
    qps = (C.c_int * nf)(*([qp] * nf))
    intra = (C.c_int * nf)(*[1 if f == 0 else 0 for f in range(nf)])
    g = Engine([(w, h)], search_range, device)
    try:
        if params is not None:
            if np.ndim(conf):
                g.set_learned(params, 0.8)
                g.set_learned_conf(conf[:3], conf[3], bool(conf[4]) if len(conf) > 4 else False)
            else:
                g.set_learned(params, conf)
        for k in range(2):
            if k:
                g.stats_reset()
            if L.fdvg_frames_device(g._g, nf, planes, intra, qps) != 0:
                raise RuntimeError(last_error())
        return g.stats()
    finally:
        g.close()


def psnr_y(src, rec, w: int, h: int) -> float:
    """Mean over frames of the luma PSNR (dB)."""
    vals = []
    for a, b in zip(src, rec):
        d = a[: w * h].astype(np.float64) - b[: w * h].astype(np.float64)
        mse = float((d * d).mean())
        vals.append(99.0 if mse == 0 else 10 * np.log10(255.0 ** 2 / mse))
    return float(np.mean(vals))


def frontier(pts):
    """Rate-distortion points with the dominated ones removed (a point stays
    only if it has higher PSNR than every cheaper point), as the reference's
    BD-rate tool does before fitting (tools/rd-bench.py:73-86)."""
    out, best = [], -np.inf
    for r, d in sorted(pts):
        if d > best:
            out.append((r, d))
            best = d
    return out


def bd_rate(ref_pts, new_pts):
    """Bjontegaard delta rate in percent (negative: fewer bits for the same
    PSNR): cubic fits of log10(rate) against PSNR over the overlapping PSNR
    range, integrated (tools/rd-bench.py:89-102).  None without overlap."""
    a, b = frontier(ref_pts), frontier(new_pts)
    if len(a) < 3 or len(b) < 3:
        return None

    def fit(pts):
        d = np.array([p[1] for p in pts])
        r = np.log10([p[0] for p in pts])
        return np.polyfit(d, r, min(3, len(pts) - 1)), d.min(), d.max()

    pa, la, ha = fit(a)
    pb, lb, hb = fit(b)
    lo, hi = max(la, lb), min(ha, hb)
    if hi <= lo:
        return None
    ia = np.polyval(np.polyint(pa), [lo, hi])
    ib = np.polyval(np.polyint(pb), [lo, hi])
    return float((10 ** (((ib[1] - ib[0]) - (ia[1] - ia[0])) / (hi - lo)) - 1) * 100)


def evaluate(params, conf=0.8, qps=QPS, nframes: int = 30, seeds=(1, 2), w: int = W, h: int = H,
             search_range: int = RANGE, device: int = 0, batch: int = 1) -> dict:
    """The learned form against the plain form on held-out seeds: per QP the
    bytes, luma PSNR and P-frame analysis time of both, and the BD-rate."""
    from . import Scene
    plain_pts, learn_pts, rows = [], [], []
    t_plain = t_learn = 0.0
    npf = 0
    for qp in qps:
        bp = bl = 0
        pp = pl = 0.0
        for sd in seeds:
            frames = Scene(w, h, nframes, seed=sd, **CONTENT).frames(nframes)
            s0, r0, st0 = encode_engine(frames, w, h, qp, 0, None, conf, search_range, device, batch)
            s1, r1, st1 = encode_engine(frames, w, h, qp, 0, params, conf, search_range, device, batch)
            bp += len(s0)
            bl += len(s1)
            pp += psnr_y(frames, r0, w, h) / len(seeds)
            pl += psnr_y(frames, r1, w, h) / len(seeds)
            t_plain += st0["p_ms"]
            t_learn += st1["p_ms"]
            npf += st0["p_launches"]
        plain_pts.append((bp, pp))
        learn_pts.append((bl, pl))
        rows.append({"qp": qp, "plain_bytes": bp, "learned_bytes": bl, "plain_psnr": round(pp, 4),
                     "learned_psnr": round(pl, 4)})
    mpix = w * h * npf / 1e6
    return {"bd_rate_pct": bd_rate(plain_pts, learn_pts), "points": rows, "conf": conf,
            "p_frames": npf, "plain_p_ms": t_plain / max(1, npf), "learned_p_ms": t_learn / max(1, npf),
            "plain_mpix_s": mpix / (t_plain / 1e3), "learned_mpix_s": mpix / (t_learn / 1e3),
            "speedup": t_plain / max(t_learn, 1e-9)}


def main(argv=None) -> None:
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="train / evaluate the learned proposal network")
    ap.add_argument("cmd", choices=["train", "eval", "infer-demo", "encode-demo"],
                    help="infer-demo / encode-demo: fixed small runs for profiling (fused inference over one "
                         "1280x720 frame three times plus one 512-sample training step; an 8-frame learned encode)")
    ap.add_argument("--frames", type=int, default=2000)
    ap.add_argument("--clip", type=int, default=50)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--skip-keep", type=float, default=0.25)
    ap.add_argument("--weights", default=DEFAULT_WEIGHTS)
    ap.add_argument("--out", default=None)
    ap.add_argument("--conf", type=float, default=0.8)
    ap.add_argument("--eval-frames", type=int, default=30)
    a = ap.parse_args(argv)
    if a.cmd == "train":
        t0 = time.time()
        net, smp, info = collect(a.frames, a.clip, skip_keep=a.skip_keep, max_batch=a.batch)
        t1 = time.time()
        curve = train(net, smp, a.epochs, a.batch, a.lr)
        t2 = time.time()
        p = net.params()
        save_params(a.out or a.weights, p)
        info.update({"collect_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1), "curve": curve.tolist(),
                     "samples_per_s": round(len(smp) * a.epochs / max(t2 - t1, 1e-9))})
        print(json.dumps(info))
    elif a.cmd == "eval":
        print(json.dumps(evaluate(load_params(a.weights), a.conf, nframes=a.eval_frames)))
    elif a.cmd == "infer-demo":
        net = Net(W, H, 2, max_batch=3648)
        rng = np.random.default_rng(0)
        for s in range(2):
            net.bank_put(s, rng.integers(0, 256, W * H, dtype=np.uint8))
        net.set_params(load_params(a.weights))
        s = samples((W // 16) * (H // 16))
        s["cur"], s["ref"], s["qp"] = 0, 1, 23
        s["mbx"] = np.tile(np.arange(W // 16), H // 16)
        s["mby"] = np.repeat(np.arange(H // 16), W // 16)
        for _ in range(3):
            net.forward_fused(s, a.conf, 64)
        t = samples(512)
        t["cur"], t["ref"], t["qp"], t["weight"], t["has_mv"] = 0, 1, 23, 1.0, 1
        t["mbx"], t["mby"] = rng.integers(0, W // 16, 512), rng.integers(0, H // 16, 512)
        t["cls"] = rng.integers(0, 3, 512)
        net.train_step(t, 1e-3)
        print("ok")
    else:
        from . import Scene
        frames = Scene(W, H, 8, seed=1, **CONTENT).frames(8)
        st, _, _ = encode_engine(frames, W, H, 23, 0, params=load_params(a.weights), conf=a.conf)
        print("ok", len(st))


if __name__ == "__main__":
    main()
