"""The multi-GPU host logic (nnm.replicas) with world size 2 over gloo on
CPU: per-rank data seeds, barrier, max over ranks of a timing, rank-0 output,
and the single-process case."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "nn-merge_b200"))
    from nnm.replicas import Replicas
    r = Replicas("gloo", timeout_s=60)
    r.barrier()
    m = r.max(1.5 + rank)  # the slower rank decides the timing
    out.put((rank, r.world, r.leader, r.data_seed(1234), m))
    r.barrier()
    r.close()


def test_two_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(i, 2, port, q)) for i in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert [r[2] for r in res] == [True, False]
    assert res[0][3] != res[1][3]  # every rank builds from its own data
    assert all(r[4] == 2.5 for r in res)


def test_single_process(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from nnm.replicas import Replicas
    r = Replicas("gloo")
    assert r.world == 1 and r.leader and r.max(3.0) == 3.0 and r.data_seed(7) == 7
    r.barrier()
    r.close()
