"""CPU restatement of the learned proposal network -- test infrastructure only.

The reference has no learned form; this numpy model is the oracle the GPU
network's features, forward pass, gradients and Adam step are checked
against.  It rounds to bf16 (round to nearest even) at the same points the GPU
path does -- input features, weights, every ReLU output, the output and
pre-activation gradients that feed a GEMM -- and sums in float64 where the
GPU sums in fp32, so the two agree to fp32 accumulation-order noise.  With
``use_bf16=False`` it is a plain float64 model, used for finite-difference
checks of the backward pass itself.

Geometry (fdv_b200/csrc/device/learned.cuh): 32 x 32 x 4 luma input, three
3x3 stride-2 pad-1 convolutions with ReLU (4->32->64->160; the first has a
37th reduction column holding the quantiser, (qp-26)/8), a 2560->11 fully
connected layer; NHWC, reduction index (ky*3+kx)*Cin + ci.
"""
from __future__ import annotations

import numpy as np

GEO = [  # sin, cin, cout, k
    (32, 4, 32, 37),
    (16, 32, 64, 288),
    (8, 64, 160, 576),
    (4, 160, 11, 2560),
]
NOUT = 11
NHYP = 4
SL1_DELTA = 0.25
WTA_EPS = 0.05


def offsets():
    offs, o = [], 0
    for _, _, cout, k in GEO:
        offs.append((o, o + cout * k))
        o += cout * k + cout
    return offs, o


OFFS, NPARAMS = offsets()


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bf16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def unpack(p: np.ndarray):
    """Flat parameters -> [(W[cout][k], b[cout])] per layer."""
    out = []
    for (wo, bo), (_, _, cout, k) in zip(OFFS, GEO):
        out.append((p[wo:wo + cout * k].reshape(cout, k), p[bo:bo + cout]))
    return out


def init_params(seed: int = 1) -> np.ndarray:
    """He-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAMS, np.float32)
    for (wo, bo), (_, _, cout, k) in zip(OFFS, GEO):
        lim = np.sqrt(6.0 / k)
        p[wo:bo] = rng.uniform(-lim, lim, cout * k).astype(np.float32)
    return p


def features(cur: np.ndarray, ref: np.ndarray, bx: int, by: int) -> np.ndarray:
    """32 x 32 x 4 input of the macroblock at (bx, by); planes are h x w luma."""
    h, w = cur.shape
    ys = np.clip(np.arange(32) + by - 8, 0, h - 1)
    xs = np.clip(np.arange(32) + bx - 8, 0, w - 1)
    c0 = cur[np.ix_(ys, xs)].astype(np.int32)
    c1 = ref[np.ix_(ys, xs)].astype(np.int32)
    gy = by - 24 + 2 * np.arange(32)
    gx = bx - 24 + 2 * np.arange(32)

    def avg(p):
        s = 0
        for dy in (0, 1):
            for dx in (0, 1):
                s = s + p[np.ix_(np.clip(gy + dy, 0, h - 1), np.clip(gx + dx, 0, w - 1))].astype(np.int32)
        return (s + 2) >> 2

    x = np.stack([c0, c1, avg(cur), avg(ref)], axis=-1).astype(np.float32)
    return bf16((x - 128.0) / 64.0)


def im2col(x: np.ndarray) -> np.ndarray:
    """x [B][S][S][C] -> [B*(S/2)^2][9C], 3x3 stride 2 pad 1."""
    b, s, _, c = x.shape
    so = s // 2
    xp = np.zeros((b, s + 2, s + 2, c), x.dtype)
    xp[:, 1:s + 1, 1:s + 1, :] = x
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(xp[:, ky:ky + 2 * so:2, kx:kx + 2 * so:2, :])
    return np.concatenate(cols, axis=-1).reshape(b * so * so, 9 * c)


def col2im(dcol: np.ndarray, b: int, s: int, c: int) -> np.ndarray:
    so = s // 2
    d = dcol.reshape(b, so, so, 9, c)
    dxp = np.zeros((b, s + 2, s + 2, c), dcol.dtype)
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + 2 * so:2, kx:kx + 2 * so:2, :] += d[:, :, :, ky * 3 + kx, :]
    return dxp[:, 1:s + 1, 1:s + 1, :]


def forward(p: np.ndarray, x: np.ndarray, qp, use_bf16: bool = True):
    """x [B][32][32][4], qp [B] -> (out [B][11], cache)."""
    r = bf16 if use_bf16 else (lambda a: a)
    acc = np.float64
    ft = np.float32 if use_bf16 else np.float64
    layers = unpack(p)
    b = x.shape[0]
    cache = {"x": x, "cols": [], "ys": []}
    a = x
    for l in range(3):
        w, bias = layers[l]
        col = im2col(a)
        if l == 0:   # the quantiser column
            col = np.concatenate([col, np.repeat((np.asarray(qp, np.float64) - 26) / 8.0, 256)[:, None]], axis=1)
        z = col.astype(acc) @ r(w).astype(acc).T + bias.astype(acc)
        y = r(np.maximum(z, 0.0).astype(ft))
        cache["cols"].append(col)
        cache["ys"].append(y)
        s = GEO[l][0] // 2
        a = y.reshape(b, s, s, GEO[l][2])
    w4, b4 = layers[3]
    flat = a.reshape(b, -1)
    out = (flat.astype(acc) @ r(w4).astype(acc).T + b4.astype(acc)).astype(ft)
    cache["flat"] = flat
    return out, cache


def _sl1(d):
    a = np.abs(d)
    val = np.where(a < SL1_DELTA, 0.5 * d * d / SL1_DELTA, a - 0.5 * SL1_DELTA)
    g = np.where(a < SL1_DELTA, d / SL1_DELTA, np.sign(d))
    return val, g


def loss_grad(out: np.ndarray, cls, has_mv, tx, ty, wgt):
    """Per-sample (ce, mv) and d(mean loss)/d(out) -- loss_kernel restated."""
    out = out.astype(np.float64)
    b = out.shape[0]
    lg = out[:, 8:11]
    mx = lg.max(axis=1, keepdims=True)
    e = np.exp(lg - mx)
    es = e.sum(axis=1, keepdims=True)
    onehot = np.eye(3)[cls]
    ce = (np.log(es[:, 0]) + mx[:, 0] - (lg * onehot).sum(axis=1)) * wgt
    g = np.zeros((b, 16))
    g[:, 8:11] = (e / es - onehot) * wgt[:, None]
    ex, gx = _sl1(out[:, 0:8:2] - tx[:, None])
    ey, gy = _sl1(out[:, 1:8:2] - ty[:, None])
    err = ex + ey
    best = np.argmin(err, axis=1)
    a = np.full((b, NHYP), WTA_EPS)
    a[np.arange(b), best] = 1.0
    a = a * wgt[:, None] * has_mv[:, None]
    mv = (a * err).sum(axis=1)
    g[:, 0:8:2] = a * gx
    g[:, 1:8:2] = a * gy
    return ce, mv, g / b


def backward(p: np.ndarray, cache, gout: np.ndarray, use_bf16: bool = True) -> np.ndarray:
    """Flat gradient of the loss whose output gradient is gout [B][16]."""
    r = bf16 if use_bf16 else (lambda a: a)
    acc = np.float64
    ft = np.float32 if use_bf16 else np.float64
    layers = unpack(p)
    grad = np.zeros(NPARAMS, np.float64)
    b = gout.shape[0]
    go = gout[:, :NOUT]
    gob = r(go.astype(ft)).astype(acc)
    w4, _ = layers[3]
    wo, bo = OFFS[3]
    grad[wo:bo] = (gob.T @ cache["flat"].astype(acc)).reshape(-1)
    grad[bo:bo + NOUT] = go.sum(axis=0)
    dy = (gob @ r(w4).astype(acc)).astype(ft)   # [B][2560]
    for l in (2, 1, 0):
        s_in, cin, cout, k = GEO[l]
        so = s_in // 2
        y = cache["ys"][l]
        dz = np.where(y > 0, dy.reshape(-1, cout), 0.0).astype(ft)
        wo, bo = OFFS[l]
        grad[bo:bo + cout] = dz.astype(acc).sum(axis=0)
        dzb = r(dz).astype(acc)
        grad[wo:bo] = (dzb.T @ cache["cols"][l].astype(acc)).reshape(-1)
        if l > 0:
            w, _ = layers[l]
            dcol = (dzb @ r(w).astype(acc)).astype(ft)
            dy = col2im(dcol, b, s_in, cin).reshape(b, -1)
    return grad


def adam(p, m, v, g, t, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (fp32 state), t counted from 1."""
    m = (b1 * m + (1 - b1) * g).astype(np.float32)
    v = (b2 * v + (1 - b2) * g * g).astype(np.float32)
    c1, c2 = 1 - b1 ** t, 1 - b2 ** t
    p = (p - lr * (m / c1) / (np.sqrt(v / c2) + eps)).astype(np.float32)
    return p, m, v
