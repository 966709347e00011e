"""The batched ensemble across ranks (fmmgpu.ensemble): every system goes to
exactly one rank, the ranks' loads are balanced within the longest-
processing-time bound, and on two gloo CPU ranks each rank derives the same
partition on its own, gathers its share's particles in the layout
fmm_evaluate_batched takes, and the shares cover the ensemble exactly."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

from fmmgpu import ensemble, workloads  # noqa: E402


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_and_balances(world):
    sizes = workloads.ensemble_sizes(256, 1024, 65536, seed=4)
    shares = ensemble.partition_systems(sizes, world)
    assert len(shares) == world
    flat = sorted(i for s in shares for i in s)
    assert flat == list(range(len(sizes)))  # each system exactly once
    loads = ensemble.rank_loads(sizes, shares)
    costs = [ensemble.system_cost(n) for n in sizes]
    lower = max(sum(costs) / world, max(costs))  # no partition does better
    assert max(loads) <= 4.0 / 3.0 * lower + 1e-9
    assert max(loads) <= sum(costs) / world + max(costs) + 1e-9


def test_partition_edge_cases():
    assert ensemble.partition_systems([], 2) == [[], []]
    assert ensemble.partition_systems([10], 3) == [[0], [], []]
    # equal systems alternate between ranks
    assert ensemble.partition_systems([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        ensemble.partition_systems([1], 0)


def test_gather_systems_layout():
    pos = np.arange(30, dtype=np.float64).reshape(10, 3)
    mass = np.arange(10, dtype=np.float64)
    offsets = np.array([0, 3, 4, 10])
    p, m, loc = ensemble.gather_systems(pos, mass, offsets, [2, 0])
    np.testing.assert_array_equal(loc, [0, 6, 9])
    np.testing.assert_array_equal(m, [4, 5, 6, 7, 8, 9, 0, 1, 2])
    np.testing.assert_array_equal(p[6:], pos[:3])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.join(ROOT, "nbody-fmm_b200"))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    from fmmgpu import ensemble, workloads

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sizes = workloads.ensemble_sizes(32, 64, 512, seed=4)
    offsets = np.r_[0, np.cumsum(sizes)].astype(np.int64)
    rng = np.random.default_rng(0)
    pos = rng.random((int(offsets[-1]), 3))
    mass = np.arange(int(offsets[-1]), dtype=np.float64)  # particle ids, to check the gather
    shares = ensemble.partition_systems(sizes, world)
    p, m, loc = ensemble.gather_systems(pos, mass, offsets, shares[rank])
    mine = {"systems": shares[rank], "ids": m.astype(np.int64).tolist(), "n": int(loc[-1])}
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    # the slowest rank's time is the job's (a stand-in time proportional to the load)
    t = bench.max_over_ranks(ensemble.rank_loads(sizes, shares)[rank], world, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, gathered, t, max(ensemble.rank_loads(sizes, shares)), int(offsets[-1])))


def test_ensemble_shards_over_two_cpu_ranks():
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
    (_, g0, t0, lmax, ntot), (_, g1, t1, _, _) = out
    assert g0 == g1  # both ranks derived the same partition
    systems = sorted(s for g in g0 for s in g["systems"])
    assert systems == list(range(32))
    ids = sorted(i for g in g0 for i in g["ids"])
    assert ids == list(range(ntot))  # every particle on exactly one rank
    assert sum(g["n"] for g in g0) == ntot
    assert t0 == t1 == lmax
