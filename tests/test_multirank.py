"""The multi-rank host logic of bench.py, on CPU with world-size-2 gloo
process groups: rank environment, the max-over-ranks timing rule and the
bin-packing of ensemble members across ranks."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = bench.dist_env()
        got = bench.reduce_max(10.0 * (r + 1), w, device="cpu")
        nps = [500 + 37 * i for i in range(40)]
        mine = bench.binpack(nps, w)[r]
        q.put((r, w, local, got, mine))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_agree_on_timing_and_partition():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, t0, m0), (r1, w1, l1, t1, m1) = res
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    assert t0 == t1 == 20.0          # every rank reports the slowest rank's time
    assert sorted(m0 + m1) == list(range(40)) and not set(m0) & set(m1)


def test_binpack_balances_particles():
    sys.path.insert(0, str(ROOT))
    import bench
    nps = [20000, 19000, 600, 550, 800, 7000, 5000, 3000]
    bins = bench.binpack(nps, 3)
    loads = [sum(nps[i] for i in b) for b in bins]
    assert sorted(sum(bins, [])) == list(range(len(nps)))
    assert max(loads) - min(loads) <= max(nps)
    assert bench.binpack(nps, 1) == [list(range(len(nps)))]
