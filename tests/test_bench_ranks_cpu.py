"""The multi-GPU run's host plumbing on CPU: two gloo ranks (127.0.0.1) as
torchrun starts them -- the barrier, the MAX of the per-rank step times and
the whole-job (weak-scaling) rate -- and the reference arm under torchrun, where
only rank 0 works."""
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
