"""The fast tier (counter-based random draws on the device): deterministic
under a seed, pools well formed (sorted, distinct ids, no self, exact
distances), and recall@10 against exact brute force."""
import numpy as np
import pytest

from nnm.datasets import gaussian_mixture_u8

pytestmark = pytest.mark.gpu


def exact_knn(x, k):
    import torch
    t = torch.from_numpy(x).cuda()
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        nrm = (t * t).sum(1)
        d = nrm[:, None] + nrm[None, :] - 2.0 * (t @ t.T)
        d.fill_diagonal_(float("inf"))
        return torch.topk(d, k, dim=1, largest=False).values.cpu().numpy()
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def check_pools(x, g):
    ids, ds = g["ids"], g["dists"]
    n, k = ids.shape
    assert (np.diff(ds, axis=1) >= 0).all()
    assert (ids < n).all() and (ids != np.arange(n)[:, None]).all()
    assert all(len(set(r)) == k for r in ids)
    ref = ((x[:, None, :] - x[ids]) ** 2).sum(-1)
    assert np.array_equal(ref.astype(np.float32), ds)  # integer data: exact


def recall(x, g, k=10):
    kth = exact_knn(x, k)[:, -1:]
    return float((g["dists"][:, :k] <= kth).mean())


@pytest.mark.parametrize("kind", ["kgraph", "smerge", "jmerge"])
def test_fast_tier_deterministic_and_well_formed(ctx, kind):
    x = gaussian_mixture_u8(4000, d=64, seed=9)
    a = getattr(ctx, kind)(x, 20, seed=3, rng="fast")
    b = getattr(ctx, kind)(x, 20, seed=3, rng="fast")
    assert np.array_equal(a["ids"], b["ids"]) and a["ncmps"] == b["ncmps"]
    check_pools(x, a)
    assert recall(x, a) >= 0.95


def test_fast_tier_merge_of_four_leaves(ctx):
    x = gaussian_mixture_u8(20000, d=128, n_centres=64, seed=2)
    g = ctx.merge_leaves(x, 20, [5000] * 4, seed=1, rng="fast")
    check_pools(x, g)
    assert recall(x, g) >= 0.95


def test_fast_tier_hmerge_layers(ctx):
    x = gaussian_mixture_u8(5000, d=32, seed=4)
    g = ctx.hmerge(x, 16, 16, seed=2, rng="fast")
    check_pools(x, g)
    assert [len(o) - 1 for o, _ in g["layers"]] == [64, 512, 4096, 5000]


@pytest.mark.parametrize("join", ["fp32", "tensor"])
def test_hmerge_fast_is_deterministic(ctx, join):
    x = gaussian_mixture_u8(40_000, n_centres=64, seed=91)
    a = ctx.hmerge(x, 20, 20, seed=3, rng="fast", join=join)
    b = ctx.hmerge(x, 20, 20, seed=3, rng="fast", join=join)
    diff = [g for g, ((ao, aa), (bo, ba)) in enumerate(zip(a["layers"], b["layers"]))
            if not (np.array_equal(ao, bo) and np.array_equal(aa, ba))]
    assert np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["dists"], b["dists"]), "pools differ"
    assert not diff, "layers differ: %s" % diff


@pytest.mark.parametrize("join", ["auto", "tensor"])
def test_merge_tree_of_uneven_leaves(ctx, join):
    """Bottom-up pairwise merge (NNM_MERGE_TREE) of leaves of uneven sizes and
    an odd count: deterministic, well formed, recall as the multi-way merge."""
    x = gaussian_mixture_u8(14000, d=64, n_centres=48, seed=21)
    sizes = [1200, 3300, 2500, 900, 4000, 2100]  # 6 leaves -> 3 -> 2 (one waits) -> 1
    sizes[-1] += len(x) - sum(sizes)
    a = ctx.merge_leaves(x, 16, sizes, seed=3, rng="fast", join=join, merge_order="tree")
    b = ctx.merge_leaves(x, 16, sizes, seed=3, rng="fast", join=join, merge_order="tree")
    assert np.array_equal(a["ids"], b["ids"]) and a["ncmps"] == b["ncmps"]
    check_pools(x, a)
    m = ctx.merge_leaves(x, 16, sizes, seed=3, rng="fast", join=join)
    assert recall(x, a) >= recall(x, m) - 0.02 and recall(x, a) >= 0.93
    odd = ctx.merge_leaves(x, 16, sizes[:4] + [sizes[4] + sizes[5]], seed=3, rng="fast", merge_order="tree")
    check_pools(x, odd)
    assert recall(x, odd) >= 0.93


def test_merge_tree_needs_fast_draws(ctx):
    from nnm import NnmError
    x = gaussian_mixture_u8(3000, d=16, seed=22)
    with pytest.raises(NnmError):
        ctx.merge_leaves(x, 10, [1000, 1000, 1000], seed=1, merge_order="tree")


@pytest.mark.parametrize("join", ["tensor", "fp8"])
def test_iteration_graph_matches_direct_launches(ctx, join):
    """The whole-iteration CUDA graph (one counter read per iteration,
    buffers sized ahead and checked on the device) gives the graph of direct
    launches, bit for bit, with learned and random initial graphs."""
    x = gaussian_mixture_u8(20000, d=64, n_centres=40, seed=5)
    if join == "fp8":
        x = x / 17.0 + 0.25
    for kw in (dict(init="random"), dict(init="random", merge_order="tree")):
        a = ctx.merge_leaves(x, 16, [5000] * 4, seed=2, rng="fast", join=join, **kw)
        b = ctx.merge_leaves(x, 16, [5000] * 4, seed=2, rng="fast", join=join, graph=False, **kw)
        assert np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["dists"], b["dists"])
        assert a["iterations"] == b["iterations"] and a["ncmps"] == b["ncmps"]
    k = ctx.kgraph(x[:6000], 20, seed=4, rng="fast", join=join)
    kd = ctx.kgraph(x[:6000], 20, seed=4, rng="fast", join=join, graph=False)
    assert np.array_equal(k["ids"], kd["ids"]) and k["iterations"] == kd["iterations"]
