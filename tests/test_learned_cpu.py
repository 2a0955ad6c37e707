"""CPU checks of the learned network's oracle (oracle/learned_ref.py): its
backward pass against finite differences, im2col/col2im adjointness, bf16
rounding against torch's, and the C ABI's learned entry points are exported."""
import ctypes as C

import numpy as np
import pytest

import oracle.learned_ref as R


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    x = (rng.standard_normal(20000) * np.exp(rng.uniform(-20, 20, 20000))).astype(np.float32)
    x[:4] = [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 0.0]   # ties to even
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(R.bf16(x), ref)


def test_im2col_col2im_adjoint():
    rng = np.random.default_rng(1)
    for s, c in [(32, 4), (16, 32), (8, 64)]:
        x = rng.standard_normal((2, s, s, c))
        d = rng.standard_normal((2 * (s // 2) ** 2, 9 * c))
        lhs = (R.im2col(x) * d).sum()
        rhs = (x * R.col2im(d, 2, s, c)).sum()
        assert abs(lhs - rhs) < 1e-9 * max(1.0, abs(lhs))


def _loss(p, x, t, qp=(18, 26, 35)):
    out, cache = R.forward(p, x, qp, use_bf16=False)
    ce, mv, g = R.loss_grad(out, *t)
    return (ce + mv).mean(), cache, g


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = R.init_params(2).astype(np.float64)
    p[R.OFFS[0][1]:R.OFFS[0][1] + 32] = 0.05    # biases off zero, away from ReLU kinks
    b = 3
    x = rng.uniform(-1.5, 1.5, (b, 32, 32, 4))
    t = (np.array([0, 1, 2]), np.array([1.0, 1.0, 0.0]), np.array([0.7, -1.2, 0.0]),
         np.array([0.3, 2.0, 0.0]), np.array([1.0, 0.5, 2.0]))
    _, cache, g = _loss(p, x, t)
    grad = R.backward(p, cache, g, use_bf16=False)
    eps = 1e-6
    for l in range(4):
        wo, bo = R.OFFS[l]
        cout = R.GEO[l][2]
        idx = list(rng.integers(wo, bo, 6)) + list(rng.integers(bo, bo + cout, 2))
        for i in idx:
            q = p.copy()
            q[i] += eps
            lp, _, _ = _loss(q, x, t)
            q[i] -= 2 * eps
            lm, _, _ = _loss(q, x, t)
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - grad[i]) <= 1e-5 + 1e-4 * abs(fd), (l, i, fd, grad[i])


def test_features_geometry():
    rng = np.random.default_rng(2)
    cur = rng.integers(0, 256, (48, 64), dtype=np.uint8)
    ref = rng.integers(0, 256, (48, 64), dtype=np.uint8)
    x = R.features(cur, ref, 16, 16)
    assert x.shape == (32, 32, 4)
    assert x[8, 8, 0] == (int(cur[16, 16]) - 128) / 64.0
    # coarse channel: 2x2 mean of the 64x64 window anchored 24 px up-left
    y0 = 16 - 24 + 2 * 20
    x0 = 16 - 24 + 2 * 20
    s = int(cur[y0, x0]) + int(cur[y0, x0 + 1]) + int(cur[y0 + 1, x0]) + int(cur[y0 + 1, x0 + 1])
    assert x[20, 20, 2] == ((s + 2) >> 2) / 64.0 - 2.0


def test_learned_abi_exported():
    from fdv_b200 import LIB_PATH
    L = C.CDLL(LIB_PATH)
    for name in ["fdvl_nparams", "fdvl_create", "fdvl_destroy", "fdvl_set_params", "fdvl_get_params",
                 "fdvl_bank_put", "fdvl_features", "fdvl_forward", "fdvl_grads", "fdvl_train_step", "fdvl_train",
                 "fdvl_last_error", "fdvl_gemm"]:
        assert hasattr(L, name), name
    L.fdvl_nparams.restype = C.c_int
    assert L.fdvl_nparams() == R.NPARAMS
