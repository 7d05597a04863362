"""The device recall evaluator against a CPU brute force, and the
autotuner's choice against its own contract.  All calls through the C ABI."""
import numpy as np
import pytest

from nnm.datasets import gaussian_mixture_u8

pytestmark = pytest.mark.gpu


def cpu_recall(x, ids, rows, atop):
    xi = x.astype(np.int64)
    hits = 0
    for r in rows:
        d = ((xi - xi[r]) ** 2).sum(1)
        d[r] = np.iinfo(np.int64).max
        kth = np.partition(d, atop - 1)[atop - 1]
        g = ids[r, :atop].astype(np.int64)
        hits += int((((xi[g] - xi[r]) ** 2).sum(1) <= kth).sum())
    return hits / (len(rows) * atop)


@pytest.mark.parametrize("atop", [1, 10, 16])
def test_graph_recall_matches_cpu(ctx, atop):
    x = gaussian_mixture_u8(3000, d=32, seed=71)
    g = ctx.kgraph(x, 16, seed=2, max_iter=2)  # a partial graph: recall well below 1
    rows = np.arange(0, 3000, 7, dtype=np.uint32)
    got = ctx.graph_recall(x, g["ids"], rows, atop)
    exp = cpu_recall(x, g["ids"], rows, atop)
    assert got == pytest.approx(exp, abs=1e-12), (got, exp)
    assert 0.1 < got < 1.0


def test_graph_recall_of_exact_graph_is_one(ctx):
    x = gaussian_mixture_u8(1500, d=24, seed=72)
    xi = x.astype(np.int64)
    d = ((xi[:, None, :] - xi[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d, np.iinfo(np.int64).max)
    ids = np.argsort(d, axis=1, kind="stable")[:, :10].astype(np.uint32)
    assert ctx.graph_recall(x, ids, np.arange(1500, dtype=np.uint32), 10) == 1.0


def test_graph_recall_rejects_bad_arguments(ctx):
    from nnm import NnmError
    x = gaussian_mixture_u8(100, d=8, seed=73)
    ids = np.zeros((100, 10), np.uint32)
    with pytest.raises(NnmError):
        ctx.graph_recall(x, ids, np.array([100], np.uint32), 10)
    with pytest.raises(NnmError):
        ctx.graph_recall(x, ids, np.array([1], np.uint32), 17)


def test_autotune_meets_its_target(ctx):
    import torch
    n, k = 60_000, 20
    x = gaussian_mixture_u8(n, n_centres=128, seed=74)
    sizes = [15_000] * 4
    xd = torch.from_numpy(x).cuda()
    kw = dict(seed=3, rng="fast", join="tensor", init="random")
    chosen, trials = ctx.autotune_merge_leaves_dev(xd.data_ptr(), n, 128, k, sizes, target_recall=0.93,
                                                   sample_rows=30_000, eval_rows=500, repeats=1, **kw)
    # 15 trials of sample cap x threshold, then the tile shape at the chosen pair
    assert len(trials) == 17 and all(0 < t["recall"] <= 1 and t["ms"] > 0 for t in trials)
    grid, tiles = trials[:15], trials[15:]
    ok = [t for t in grid if t["recall"] >= 0.935]
    pick = [t for t in grid if t["sample_cap"] == chosen["sample_cap"] and t["delta"] == chosen["delta"]][0]
    if ok:
        assert pick["recall"] >= 0.935 and pick["ms"] == min(t["ms"] for t in ok)
    assert [t["tile_rows"] for t in tiles] == [64, 32] and pick["tile_rows"] == 128
    assert all(t["sample_cap"] == pick["sample_cap"] and t["delta"] == pick["delta"] for t in tiles)
    assert chosen["tile_rows"] == min([pick] + tiles, key=lambda t: t["ms"])["tile_rows"]
    # the tuned build on the whole set stays near the target
    kw.update(chosen)
    g = ctx.merge_leaves(x, k, sizes, **kw)
    rows = np.arange(0, n, 60, dtype=np.uint32)
    assert ctx.graph_recall(x, g["ids"], rows, 10) >= 0.91
