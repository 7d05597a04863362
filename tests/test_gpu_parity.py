"""CUDA path vs the oracle (the reference restated in C, pinned bit-exact to
the reference itself): neighbour ids, distances, flags, distance-evaluation
counts and per-iteration convergence means must be identical under a fixed
seed.  All calls go through the C ABI (lib/libnnm.so)."""
import numpy as np
import pytest

import golden_lib
from nnm.datasets import gaussian_mixture_u8, queries_like, vmf_mixture

pytestmark = pytest.mark.gpu


def assert_same_graph(got, exp, check_trace=True):
    assert np.array_equal(got["ids"], exp["ids"]), "ids differ in %d rows" % int((got["ids"] != exp["ids"]).any(1).sum())
    assert np.array_equal(got["dists"].view(np.uint32), exp["dists"].view(np.uint32)), "distances differ"
    assert np.array_equal(got["flags"], exp["flags"]), "flags differ"
    assert got["ncmps"] == exp["ncmps"]
    if check_trace:
        assert np.array_equal(got["trace"], exp["trace"]), (got["trace"], exp["trace"])


@pytest.mark.parametrize("n,seed", [(600, 3), (3000, 77)])
def test_kgraph_bit_exact(ctx, oracle, n, seed):
    x = gaussian_mixture_u8(n, seed=seed)
    exp = oracle.kgraph(x, 20, seed)
    got = ctx.kgraph(x, 20, seed=seed, exact_trace=True)
    assert_same_graph(got, exp)
    assert got["iterations"] == len(exp["trace"])


def test_kgraph_float_data(ctx, oracle):
    x = vmf_mixture(2500, d=96, n_centres=32, seed=8)
    exp = oracle.kgraph(x, 16, 5)
    got = ctx.kgraph(x, 16, seed=5, exact_trace=True)
    assert_same_graph(got, exp)


@pytest.mark.parametrize("metric", ["l1", "chi2"])
def test_kgraph_other_metrics(ctx, oracle, metric):
    x = gaussian_mixture_u8(1500, d=40, seed=21)
    exp = oracle.kgraph(x, 12, 9, metric=metric)
    got = ctx.kgraph(x, 12, seed=9, metric=metric, exact_trace=True)
    assert_same_graph(got, exp)


def test_kgraph_ragged_dim(ctx, oracle):
    x = gaussian_mixture_u8(1200, d=37, seed=4)
    exp = oracle.kgraph(x, 10, 2)
    got = ctx.kgraph(x, 10, seed=2, exact_trace=True)
    assert_same_graph(got, exp)


@pytest.mark.parametrize("n", [800, 4001])
def test_smerge_bit_exact(ctx, oracle, n):
    x = gaussian_mixture_u8(n, seed=n)
    exp = oracle.smerge(x, 20, 31)
    got = ctx.smerge(x, 20, seed=31, exact_trace=True)
    assert_same_graph(got, exp)


def test_jmerge_bit_exact(ctx, oracle):
    x = gaussian_mixture_u8(3000, seed=12)
    exp = oracle.jmerge(x, 20, 8)
    got = ctx.jmerge(x, 20, seed=8, exact_trace=True)
    assert_same_graph(got, exp)


def test_merge_two_leaves_is_smerge(ctx):
    x = gaussian_mixture_u8(3001, seed=19)
    a = ctx.smerge(x, 20, seed=4)
    b = ctx.merge_leaves(x, 20, [1500, 1501], seed=4)
    assert np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["dists"], b["dists"])


_HM_CACHE = {}


def oracle_hmerge(oracle, n):
    if n not in _HM_CACHE:
        x = gaussian_mixture_u8(n, seed=5)
        _HM_CACHE[n] = (x, oracle.hmerge(x, 20, 20, 77))
    return _HM_CACHE[n]


@pytest.mark.parametrize("n", [3000, 34000])
def test_hmerge_bit_exact(ctx, oracle, n):
    x, exp = oracle_hmerge(oracle, n)
    got = ctx.hmerge(x, 20, 20, seed=77, exact_trace=True)
    assert_same_graph(got, exp)
    assert len(got["layers"]) == len(exp["layers"])
    for (go, ga), (eo, ea) in zip(got["layers"], exp["layers"]):
        assert np.array_equal(go, eo) and np.array_equal(ga, ea)


def test_search_matches_reference(ctx, oracle):
    x, h = oracle_hmerge(oracle, 34000)
    q = queries_like(1000, seed=5, query_seed=3)
    for topk in (1, 10, 60):
        exp = oracle.search(x, h["layers"], q, topk, 9)
        got = ctx.search(x, h["layers"], q, topk, seed=9)
        assert np.array_equal(got["ids"], exp["ids"]), (topk, (got["ids"] == exp["ids"]).all(1).mean())
        assert np.array_equal(got["dists"], exp["dists"])
        assert got["ncmps"] == exp["ncmps"]


@pytest.mark.parametrize("name", golden_lib.names())
def test_cuda_matches_golden(ctx, name):
    """The CUDA path against the reference's own committed outputs."""
    fx = golden_lib.load(name)
    x, k, seed, metric = fx["x"], fx["k"], fx["seed"], fx["metric"]
    if fx["cmd"] == "hmerge":
        got = ctx.hmerge(x, k, fx["m"], seed=seed, metric=metric, exact_trace=True)
        assert len(got["layers"]) == len(fx["layers"])
        for (go, ga), (eo, ea) in zip(got["layers"], fx["layers"]):
            assert np.array_equal(go, eo) and np.array_equal(ga, ea)
    else:
        got = getattr(ctx, fx["cmd"])(x, k, seed=seed, metric=metric, exact_trace=True)
    assert golden_lib.same_pools(got, fx)
    assert got["ncmps"] == fx["ncmps"]
    assert np.array_equal(got["trace"], fx["trace"])
    if "q" in fx:
        for topk in (1, 10, 40):
            s = ctx.search(x, fx["layers"], fx["q"], topk, seed=seed)
            assert np.array_equal(s["ids"], fx["search%d_ids" % topk])
            assert np.array_equal(s["dists"], fx["search%d_dists" % topk])
            assert s["ncmps"] == int(fx["search%d_ncmps" % topk])


@pytest.mark.parametrize("join", ["fp32", "auto"])
def test_kgraph_wide_vectors(ctx, oracle, join):
    """d = 600: the staged FP32 join kernels do not fit shared memory for the
    larger list sizes, whose rows take the unstaged kernel -- same sums."""
    x = gaussian_mixture_u8(1200, d=600, seed=81)
    exp = oracle.kgraph(x, 16, 9)
    got = ctx.kgraph(x, 16, seed=9, exact_trace=True, join=join)
    assert_same_graph(got, exp)
