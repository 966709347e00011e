"""The bench's multi-GPU logic on CPU ranks (gloo, world size 2): the whole-
job value takes the slowest rank's time (maximum over ranks) and the
end-to-end rate the slowest rank's rate (minimum), and under torchrun only
rank 0 runs the reference arm and prints its line."""
import datetime
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench

    slowest = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")  # this rank's total ms
    rate = bench.min_over_ranks(1e6 - 2e5 * rank, world, "cpu")     # this rank's particles/s
    value = bench.job_rate(1000, 4, world, slowest / 1e3)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, slowest, rate, value))


def test_reductions_over_two_cpu_ranks():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate, value in out:
        assert slowest == 15.0          # the slower rank's time
        assert rate == 8e5              # the slower rank's rate
        assert value == pytest.approx(1000 * 4 * 2 / 0.015)


def test_reference_arm_runs_on_rank_zero_only():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref.so")):
        pytest.skip("the reference is not built here (oracle/_ref)")
    env = dict(os.environ, RANK="1", LOCAL_RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=300, cwd=ROOT,
                       env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
