"""The N > 1 plumbing of bench.py on the host (gloo, world size 2): the
max-over-ranks reduction and the cost-ordered sharding of the plate batch
(every rank computes the same shards; together they cover every plate once)."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "gpu-gauntlet_b200"))
    try:
        import bench
        from plategpu.workloads import shard_lpt
        w, r, local = bench.dist_setup(None)
        bench.barrier(w)
        m = bench.max_over_ranks(w, 10.0 * (r + 1), local)
        costs = [float((k % 7) + 1) ** 2 for k in range(40)]
        sh = shard_lpt(costs, w)
        import torch.distributed as dist
        dist.destroy_process_group()
        q.put((r, w, m, sh))
    except Exception as e:  # reported to the parent
        q.put((rank, -1, repr(e), None))


@pytest.mark.timeout(120)
def test_two_rank_max_and_shards():
    pytest.importorskip("torch")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(k, 2, port, q)) for k in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=100) for _ in range(2)]
    for p in ps:
        p.join(timeout=30)
    out.sort()
    assert all(o[1] == 2 for o in out), out
    assert [o[2] for o in out] == [20.0, 20.0]  # max over ranks seen by both
    assert out[0][3] == out[1][3]  # identical shards on every rank
    covered = sorted(i for s in out[0][3] for i in s)
    assert covered == list(range(40))
