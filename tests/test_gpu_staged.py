"""The staged merge (nnm_merge_*, AbstractMerge's steps as separate calls)
against the one-call builders and the oracle: run in the order of
Smerge::buildKGraph (smerge.cpp:46-91) and Jmerge::buildKGraph
(jmerge.cpp:43-80), the steps give the reference's graph bit for bit."""
import numpy as np
import pytest

from nnm import NnmError
from nnm.datasets import gaussian_mixture_u8

pytestmark = pytest.mark.gpu


def same(a, b):
    return (np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["dists"].view(np.uint32), b["dists"].view(np.uint32))
            and np.array_equal(a["flags"], b["flags"]))


@pytest.mark.parametrize("join", ["fp32", "tensor"])
def test_staged_smerge_is_smerge(ctx, oracle, join):
    x = gaussian_mixture_u8(3000, seed=41)
    n, k, seed = len(x), 20, 17
    pre = n * 5 // 10
    m = ctx.merge_session(x, k, seed=seed, join=join, exact_trace=True)
    try:
        g1, c1 = m.subgraph(0, pre)
        g2, c2 = m.subgraph(pre, n)
        m.init_sgraph(0, g1, 0)
        m.init_sgraph(pre, g2, 1)
        m.initial_graph("smerge", pre)
        st = m.nndescent("smerge", pre)
        m.merge2one(n)
        got = m.read()
    finally:
        m.close()
    one = ctx.smerge(x, k, seed=seed, join=join, exact_trace=True)
    exp = oracle.smerge(x, k, seed)
    assert same(got, one) and same(got, exp)
    assert c1 + c2 == one["sub_ncmps"]
    assert st["ncmps"] + n * (k // 2) == exp["ncmps"]
    # the one-call trace holds the two sub-graph loops first
    assert len(st["trace"]) and np.array_equal(st["trace"], exp["trace"][-len(st["trace"]):])


def test_staged_jmerge_is_jmerge(ctx, oracle):
    x = gaussian_mixture_u8(2500, seed=8)
    n, k, seed = len(x), 16, 5
    pre = n * 5 // 10
    m = ctx.merge_session(x, k, seed=seed)
    try:
        g1, _ = m.subgraph(0, pre)
        m.init_sgraph(0, g1, 0)
        m.initial_graph("jmerge", pre)
        m.nndescent("jmerge", pre)
        m.merge2one(pre)
        got = m.read()
    finally:
        m.close()
    assert same(got, ctx.jmerge(x, k, seed=seed))
    assert same(got, oracle.jmerge(x, k, seed))


def test_staged_subgraph_is_kgraph_of_the_range(ctx, oracle):
    """The first sub-graph of a session is KGraph::buildKGraph on cutMat(0,
    pre) in a fresh process (the std::rand() stream starts there)."""
    x = gaussian_mixture_u8(2400, seed=3)
    m = ctx.merge_session(x, 12, seed=9)
    try:
        g1, c1 = m.subgraph(0, 1200)
    finally:
        m.close()
    exp = oracle.kgraph(x[:1200], 12, 9)
    assert np.array_equal(g1, exp["ids"]) and c1 == exp["ncmps"]


def test_staged_rejects_bad_steps(ctx):
    x = gaussian_mixture_u8(500, seed=1)
    with pytest.raises(NnmError):
        ctx.merge_session(x, 10, seed=1, rng="fast")
    m = ctx.merge_session(x, 10, seed=1)
    try:
        with pytest.raises(NnmError):
            m.merge2one(500)  # no compensation lists before an initial graph
        with pytest.raises(NnmError):
            m.init_sgraph(0, np.full((250, 10), 250, np.uint32), 0)  # ids outside the range
        with pytest.raises(NnmError):
            m.initial_graph("smerge", 5)  # halves smaller than k + 2
        with pytest.raises(NnmError):
            m.subgraph(100, 105)
    finally:
        m.close()
