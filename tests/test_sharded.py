"""The leaf-sharded multi-GPU build (nnm.sharded): its partition and exchange
logic over gloo on CPU with world sizes 2 and 3 and a stand-in leaf builder
(every leaf built once, on the rank that owns it; after the one all-gather
every rank holds every leaf's graph with ids of the whole set), and on a
GPU, through the library with one rank, the graph of nnm_merge_leaves_dev."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

SIZES = [37, 50, 44, 61, 29, 58, 40]
K = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def fake_leaf_graph(rows, leaf0, k):
    """Stand-in for the engine's leaf build: a graph of block-local ids that
    names its block (ids) and leaf (distances)."""
    import torch
    n = rows
    ids = (torch.arange(n)[:, None] + torch.arange(1, k + 1)[None, :]) % n
    return ids.to(torch.int32), torch.full((n, k), float(leaf0), dtype=torch.float32)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "nn-merge_b200"))
    sys.path.insert(0, os.path.join(root, "tests"))
    import datetime
    import torch
    import torch.distributed as dist
    from nnm.sharded import ShardedBuild
    from test_sharded import K, SIZES, fake_leaf_graph
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    built = []

    def build(xb, sizes, leaf0):
        built.append((leaf0, len(sizes), xb.shape[0]))
        return fake_leaf_graph(xb.shape[0], leaf0, K)

    def merge(x, sizes, ids, dists):
        return ids.clone(), dists.clone()

    x = torch.arange(sum(SIZES) * 3, dtype=torch.float32).reshape(-1, 3)
    ids, dists = ShardedBuild(dist, build, merge, "cpu").run(x, SIZES, K)
    out.put((rank, built, ids.numpy(), dists.numpy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_exchange_over_gloo(world):
    from nnm.sharded import leaf_blocks, row_offsets
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(i, world, port, q)) for i in range(world)]
    for p in ps:
        p.start()
    res = sorted((q.get(timeout=180) for _ in ps), key=lambda r: r[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    # every leaf built once, by the rank whose block holds it
    blocks = leaf_blocks(len(SIZES), world)
    firsts = sorted(b[0] for r in res for b in r[1])
    assert firsts == sorted(a for a, b in blocks if b > a)
    assert sum(b[1] for r in res for b in r[1]) == len(SIZES)
    # the single-process expectation: each block's local ids shifted to the set
    off = row_offsets(SIZES)
    exp_i = np.zeros((int(off[-1]), K), np.int32)
    exp_d = np.zeros((int(off[-1]), K), np.float32)
    for a, b in blocks:
        if b > a:
            lo, hi = int(off[a]), int(off[b])
            i, d = fake_leaf_graph(hi - lo, a, K)
            exp_i[lo:hi] = i.numpy() + lo
            exp_d[lo:hi] = d.numpy()
    for _, _, ids, dists in res:  # every rank holds the whole graph
        assert np.array_equal(ids, exp_i) and np.array_equal(dists, exp_d)


def test_leaf_blocks_cover_every_leaf():
    from nnm.sharded import leaf_blocks
    for nleaf in (1, 2, 7, 208):
        for world in (1, 2, 3, 8):
            bl = leaf_blocks(nleaf, world)
            assert bl[0][0] == 0 and bl[-1][1] == nleaf
            assert all(bl[i][1] == bl[i + 1][0] for i in range(world - 1))
            assert max(b - a for a, b in bl) - min(b - a for a, b in bl) <= 1


@pytest.mark.gpu
def test_one_rank_sharded_build_is_merge_leaves(ctx):
    """With one rank the sharded build is the library's multi-leaf build, bit
    for bit (the leaves built, then merged); and merging the leaves of two
    half-builds gives a graph of the same quality."""
    import torch
    from nnm.datasets import gaussian_mixture_u8
    from nnm.sharded import ShardedBuild, engine_build
    x = gaussian_mixture_u8(24000, d=64, n_centres=40, seed=6)
    sizes = [6000, 5000, 7000, 6000]
    xt = torch.from_numpy(x).cuda()
    kw = dict(seed=3, rng="fast", join="tensor")
    build, merge = engine_build(ctx, 16, **kw)
    ids, ds, st = ShardedBuild(None, build, merge, "cuda").run(xt, sizes, 16)
    ref = ctx.merge_leaves(x, 16, sizes, **kw)
    assert np.array_equal(ids.cpu().numpy().view(np.uint32), ref["ids"])
    assert np.array_equal(ds.cpu().numpy(), ref["dists"])
    # two blocks built separately (as two ranks would), then merged
    i0, d0 = build(xt[:11000], sizes[:2], 0)
    i1, d1 = build(xt[11000:], sizes[2:], 2)
    mi, md, _ = merge(xt, sizes, torch.cat([i0, i1 + 11000]), torch.cat([d0, d1]))
    rows = np.arange(0, 24000, 23)
    xs = x.astype(np.float64)
    nrm = (xs * xs).sum(1)
    dd = nrm[rows][:, None] + nrm[None, :] - 2.0 * (xs[rows] @ xs.T)  # exact for integer data
    kth = np.sort(dd, axis=1)[:, 10:11]  # the 10th other row (index 0 is the row itself)
    got = md.cpu().numpy()[rows, :10]
    assert (got <= kth).mean() >= 0.95
