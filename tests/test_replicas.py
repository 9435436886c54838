"""CPU tests of the multi-process plumbing (lbmpond_b200.replicas) with two
gloo ranks: the max over ranks that times a replicated run, the sum that
aggregates its work, and the split of a batch of independent problems."""
import os
import socket

import numpy as np


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from lbmpond_b200 import replicas
    r, local, w, dist = replicas.setup("gloo", timeout_s=60)
    try:
        assert (r, w) == (rank, world)
        times = [3.0, 7.5]
        mx = replicas.max_over_ranks(dist, times[rank])
        work = replicas.sum_over_ranks(dist, 100 * (rank + 1))
        replicas.barrier(dist)
        lengths = np.random.default_rng(0).integers(256, 4097, 101)
        mine = replicas.partition_problems(lengths, w)[rank]
        total = replicas.sum_over_ranks(dist, int(lengths[mine].sum()))
        count = replicas.sum_over_ranks(dist, mine.size)
        out.put((rank, mx, work, total, count))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    lengths = np.random.default_rng(0).integers(256, 4097, 101)
    for rank, mx, work, total, count in res:
        assert mx == 7.5                    # every rank sees the slowest rank's time
        assert work == 300                  # and the whole job's work
        assert total == lengths.sum() and count == lengths.size


def test_partition_covers_and_balances():
    from lbmpond_b200.replicas import partition_problems
    lengths = np.random.default_rng(1).integers(256, 4097, 4096)
    for world in (1, 2, 3, 8):
        parts = partition_problems(lengths, world)
        allp = np.sort(np.concatenate(parts))
        assert np.array_equal(allp, np.arange(lengths.size))
        loads = np.array([lengths[p].sum() for p in parts])
        assert loads.max() - loads.min() <= lengths.max()   # greedy longest-first bound
    assert len(partition_problems([], 4)) == 4


def test_single_process_is_a_no_op(monkeypatch):
    from lbmpond_b200 import replicas
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    r, local, w, dist = replicas.setup("gloo")
    assert (w, dist) == (1, None)
    assert replicas.max_over_ranks(None, 2.5) == 2.5
    replicas.barrier(None)
