"""GPU parity of batched P-frames (fdvg_submit_batch): several consecutive
P-frames in one wavefront launch, each frame's rows starting while the frame
before is still being coded, its reference deblocked and prepared tile by
tile inside the wavefront.

Every frame's 16 symbol streams must equal the CPU oracle's coding the same
frames one after another (so every in-launch reference was right), and the
last frame's reconstruction must equal the oracle's.  Cases cover one and two
references, the three search ranges (the shared-memory window at 16 and 32,
direct reads at 64), units one macroblock wide or high (tiles whose borders
meet on both sides), several units of mixed sizes in one batch, and two
batches in a row (the reference ring wrapping around).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(sizes, rng, nbatch, K, qp, seed):
    import fdv_b200 as F
    import oracle as O
    nf = 1 + nbatch * K
    frames = [F.Scene(w, h, nf, nrects=max(2, w * h // 3000), pan_qx=7, pan_qy=-5, static_pct=30,
                      seed=seed + u).frames(nf) for u, (w, h) in enumerate(sizes)]
    eng = F.Engine(sizes, rng)
    assert eng.max_batch() >= K
    units = [O.OracleUnit(w, h, rng) for (w, h) in sizes]
    eng.step([frames[u][0] for u in range(len(sizes))], [1] * len(sizes), [qp] * len(sizes))
    for u, o in enumerate(units):
        o.frame(frames[u][0], 1, qp)
    f = 1
    for _ in range(nbatch):
        eng.submit_batch([[frames[u][f + k] for u in range(len(sizes))] for k in range(K)],
                         [[qp] * len(sizes) for _ in range(K)])
        for k in range(K):
            eng.collect()
            for u, o in enumerate(units):
                want, _ = o.frame(frames[u][f + k], 0, qp)
                got = eng.pframe_streams(u)
                for s in range(16):
                    assert got[s] == want[s], f"frame {f + k} unit {u} stream {s}"
        f += K
    for u, o in enumerate(units):
        assert np.array_equal(eng.recon(u), o.recon()), f"unit {u} reconstruction"
    eng.close()


@pytest.mark.parametrize("sizes,rng,nbatch,K,qp,seed", [
    ([(160, 96)], 16, 1, 6, 26, 41),
    ([(64, 48), (16, 32), (32, 16), (96, 64)], 32, 1, 5, 30, 42),
    ([(128, 64)], 64, 1, 4, 22, 43),
    ([(256, 144)], 32, 2, 6, 24, 44),
    ([(16, 16), (48, 16)], 16, 2, 3, 36, 45),
])
def test_batched_pframes_match_oracle(built, sizes, rng, nbatch, K, qp, seed):
    _run(sizes, rng, nbatch, K, qp, seed)


def test_batch_size_limits(built):
    """Batches hold P-frames only and at most fdvg_max_batch of them; decision
    records bring the limit to one."""
    import fdv_b200 as F
    w, h = 64, 48
    eng = F.Engine([(w, h)], 16)
    kmax = eng.max_batch()
    assert kmax >= 2
    fr = F.Scene(w, h, kmax + 3, nrects=3, seed=5).frames(kmax + 3)
    with pytest.raises(F.FdvError):
        eng.submit_batch([[fr[1]]], [[26]])      # no reference yet
    eng.step([fr[0]], [1], [26])
    with pytest.raises(F.FdvError):
        eng.submit_batch([[fr[k]] for k in range(1, kmax + 2)], [[26]] * (kmax + 1))
    eng.set_records(True)
    assert eng.max_batch() == 1
    with pytest.raises(F.FdvError):
        eng.submit_batch([[fr[1]], [fr[2]]], [[26], [26]])
    eng.close()


def test_learned_batch_stream(built):
    """The learned form in batches: the stream decodes; the batch's first
    P-frame (reference-based inference and SKIP pre-analysis, as one frame per
    launch) reconstructs exactly as frame-by-frame coding; the later frames
    (inference against the previous source) keep the quality within 0.3 dB."""
    import fdv_b200 as F
    import fdv_b200.learned as LN
    w, h, n = 160, 96, 9
    frames = F.Scene(w, h, n, seed=7, **LN.CONTENT).frames(n)
    p = LN.load_params(LN.DEFAULT_WEIGHTS)
    sb, rb, _ = LN.encode_engine(frames, w, h, 23, 0, p, 0.8, LN.RANGE, 0, batch=8)
    s1, r1, _ = LN.encode_engine(frames, w, h, 23, 0, p, 0.8, LN.RANGE, 0, batch=1)
    assert len(rb) == n
    assert np.array_equal(rb[0], r1[0]) and np.array_equal(rb[1], r1[1])
    assert abs(LN.psnr_y(frames, rb, w, h) - LN.psnr_y(frames, r1, w, h)) < 0.3


@pytest.mark.parametrize("kmax,nf,keyat", [(30, 76, (0, 38)), (60, 130, (0, 65))])
def test_long_batched_sequence_matches_oracle(built, kmax, nf, keyat):
    """A long sequence in launches of a given largest batch: each GOP holds a
    full launch of kmax frames and a shorter one, and the ring of reference
    slots (kmax + 2 are read or written by a launch; the ring holds 62) wraps.
    Two units of different sizes; every frame's streams (key frames: all three
    planes) and the final reconstruction equal the CPU oracle's."""
    import fdv_b200 as F
    import oracle as O
    sizes, rng, qp = [(160, 96), (64, 48)], 32, 27
    frames = [F.Scene(w, h, nf, nrects=max(2, w * h // 3000), pan_qx=9, pan_qy=-3, static_pct=25,
                      seed=61 + u).frames(nf) for u, (w, h) in enumerate(sizes)]
    eng = F.Engine(sizes, rng)
    eng.set_tuning(kmax, 0)
    assert eng.max_batch() == kmax
    units = [O.OracleUnit(w, h, rng) for (w, h) in sizes]
    nu = len(sizes)
    f, launches = 0, 0
    while f < nf:
        if f in keyat:
            eng.step([frames[u][f] for u in range(nu)], [1] * nu, [qp] * nu)
            for u, o in enumerate(units):
                want, _ = o.frame(frames[u][f], 1, qp)
                for p in range(3):
                    assert eng.iframe_streams(u, p) == list(want[p]), f"key frame {f} unit {u} plane {p}"
            f += 1
            continue
        K = 1
        while K < kmax and f + K < nf and (f + K) not in keyat:
            K += 1
        eng.submit_batch([[frames[u][f + k] for u in range(nu)] for k in range(K)], [[qp] * nu for _ in range(K)])
        launches += 1
        for k in range(K):
            eng.collect()
            for u, o in enumerate(units):
                want, _ = o.frame(frames[u][f + k], 0, qp)
                got = eng.pframe_streams(u)
                for s in range(16):
                    assert got[s] == want[s], f"frame {f + k} unit {u} stream {s}"
        f += K
    assert launches == 4
    for u, o in enumerate(units):
        assert np.array_equal(eng.recon(u), o.recon()), f"unit {u} reconstruction"
    eng.close()


@pytest.mark.parametrize("nf", [14, 11])
def test_frames_device_key_lookahead_matches_oracle(built, nf):
    """fdvg_frames_device from device-resident sources, key frames at 0, 5
    and 10: frame 5 is analysed in frame 0's launch (the key-frame lookahead)
    and reused at its own turn, frame 10 is coded at its own; the last frame's
    streams (a P-frame, or key frame 10 when the sequence ends there) and
    every unit's reconstruction equal the CPU oracle coding the frames in
    order."""
    import ctypes as C
    import torch
    import fdv_b200 as F
    import oracle as O
    sizes, rng, qp = [(160, 96), (64, 48)], 32, 26
    nu = len(sizes)
    frames = [F.Scene(w, h, nf, nrects=max(2, w * h // 3000), pan_qx=7, pan_qy=-3, static_pct=20,
                      seed=81 + u).frames(nf) for u, (w, h) in enumerate(sizes)]
    dev = [torch.from_numpy(np.stack(fr)).to("cuda:0") for fr in frames]
    torch.cuda.synchronize()
    keys = [1 if f % 5 == 0 else 0 for f in range(nf)]
    planes = (F.u8p * (3 * nu * nf))()
    for f in range(nf):
        for u, (w, h) in enumerate(sizes):
            b = dev[u].data_ptr() + f * w * h * 3 // 2
            j = 3 * (f * nu + u)
            planes[j], planes[j + 1], planes[j + 2] = (C.cast(b, F.u8p), C.cast(b + w * h, F.u8p),
                                                       C.cast(b + w * h * 5 // 4, F.u8p))
    intra = (C.c_int * (nu * nf))(*[keys[f] for f in range(nf) for _ in range(nu)])
    qps = (C.c_int * (nu * nf))(*([qp] * (nu * nf)))
    eng = F.Engine(sizes, rng)
    assert F.lib().fdvg_frames_device(eng._g, nf, planes, intra, qps) == 0, F.last_error()
    units = [O.OracleUnit(w, h, rng) for (w, h) in sizes]
    last = None
    for f in range(nf):
        last = [o.frame(frames[u][f], keys[f], qp)[0] for u, o in enumerate(units)]
    for u, o in enumerate(units):
        if keys[nf - 1]:
            for p in range(3):
                assert eng.iframe_streams(u, p) == list(last[u][p]), f"unit {u} plane {p}"
        else:
            got = eng.pframe_streams(u)
            for s in range(16):
                assert got[s] == last[u][s], f"unit {u} stream {s}"
        assert np.array_equal(eng.recon(u), o.recon()), f"unit {u} reconstruction"
    eng.close()
