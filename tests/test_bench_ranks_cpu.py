"""The multi-GPU run's host plumbing on CPU: two gloo ranks (127.0.0.1) as
torchrun starts them -- the barrier, the MAX of the per-rank step times and
the whole-job (weak-scaling) rate, a real partition of independent streams
across the ranks with the outputs gathered in stream order -- and the
reference arm under torchrun, where only rank 0 works."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks("gloo", "cpu")
    r.barrier()
    t = r.reduce_max(0.25 + 0.5 * r.rank)   # rank 1 is the slower one
    q.put((r.rank, r.world, t, bench.weak_value(r.world, 3, bench.NF, t)))
    r.close()


def test_two_gloo_ranks_max_time_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    import bench
    for rank, world, t, v in got:
        assert world == 2 and abs(t - 0.75) < 1e-12
        assert abs(v - 2 * 3 * bench.NF * bench.W * bench.H / 1e6 / 0.75) < 1e-6


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "", r.stdout


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    env0 = {k: os.environ.get(k) for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    for k in env0:
        os.environ.pop(k, None)
    try:
        r = bench.Ranks("gloo", "cpu")
        assert r.world == 1 and r.dist is None and r.reduce_max(1.5) == 1.5
        r.barrier()
        r.close()
    finally:
        for k, v in env0.items():
            if v is not None:
                os.environ[k] = v
    assert json.dumps({"v": bench.weak_value(1, 1, 1, 1.0)})


# Six independent streams of mixed sizes and QPs, as the batched workload
# mixes them (small enough for the CPU oracle).
SPECS = [dict(w=64, h=48, nframes=3, qp=22, seed=71), dict(w=96, h=64, nframes=3, qp=30, seed=72),
         dict(w=48, h=32, nframes=4, qp=18, seed=73), dict(w=128, h=64, nframes=2, qp=36, seed=74),
         dict(w=32, h=32, nframes=3, qp=26, seed=75), dict(w=64, h=64, nframes=3, qp=33, seed=76)]


def _oracle_stream(sp) -> bytes:
    import fdv_b200 as F
    import oracle as O
    fr = F.Scene(sp["w"], sp["h"], sp["nframes"], nrects=3, pan_qx=5, seed=sp["seed"]).frames(sp["nframes"])
    return O.oracle_video_stream(fr, sp["w"], sp["h"], sp["qp"], 2, 16)


def _partition_rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r = bench.Ranks("gloo", "cpu")
    mine = r.shard([sp["w"] * sp["h"] * sp["nframes"] for sp in SPECS])
    out = bench.encode_sharded(r, SPECS, _oracle_stream)
    q.put((r.rank, mine, out))
    r.close()


def test_streams_partitioned_across_two_ranks_gather_in_order():
    """Each rank codes only its share of the streams (no stream on both, none
    left out, the work balanced), and rank 0 gathers them in stream order,
    equal to one process coding all of them."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_partition_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in ps:
        p.start()
    got = dict((r, (m, o)) for r, m, o in (q.get(timeout=300) for _ in range(2)))
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    m0, m1 = got[0][0], got[1][0]
    assert sorted(m0 + m1) == list(range(len(SPECS))) and m0 and m1
    work = [sp["w"] * sp["h"] * sp["nframes"] for sp in SPECS]
    assert abs(sum(work[i] for i in m0) - sum(work[i] for i in m1)) <= max(work)
    assert got[1][1] is None
    assert got[0][1] == [_oracle_stream(sp) for sp in SPECS]
