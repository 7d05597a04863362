"""Serving path (nnm_index_*): the resident index's exact kernel against the
oracle -- per-query beam widths, the first out_k results, learned entries --
bit for bit; the fast kernel against exact distances and the exact kernel's
recall; the entry network's kernels against the CPU oracle; training and
what the trained network changes.  All calls go through the C ABI."""
import numpy as np
import pytest

import entry_oracle as eo
from nnm import NnmError, entry_init
from nnm.datasets import gaussian_mixture_u8, queries_like

pytestmark = pytest.mark.gpu

N, NQ = 40_000, 2_000


@pytest.fixture(scope="module")
def hier(ctx):
    x = gaussian_mixture_u8(N, n_centres=64, seed=21)
    h = ctx.hmerge(x, 20, 20, seed=3, rng="fast")
    q = queries_like(NQ, n_centres=64, seed=21, query_seed=5)
    return x, h["layers"], q


@pytest.fixture(scope="module")
def index(ctx, hier):
    x, layers, _ = hier
    ix = ctx.index(x, layers, seed=9)
    yield ix
    ix.close()


def truth(x, q, k=10):
    """Exact k nearest distances of every query (float64, chunked)."""
    x64 = x.astype(np.float64)
    xn = (x64 * x64).sum(1)[None, :]
    out = []
    for i in range(0, len(q), 250):
        q64 = q[i:i + 250].astype(np.float64)
        d = (q64 * q64).sum(1)[:, None] + xn - 2.0 * q64 @ x64.T
        out.append(np.partition(d, k, axis=1)[:, :k])
    return None, np.sort(np.concatenate(out), axis=1)


def recall(ids, gt_d, x, q):
    # a result counts when its exact distance is within the true k-th
    d = ((x[ids.astype(np.int64)].astype(np.float64) - q[:, None, :]) ** 2).sum(-1)
    return float((d <= gt_d[:, -1:] * (1 + 1e-9)).mean())


def test_layers_shape(hier):
    _, layers, _ = hier
    assert [len(o) - 1 for o, _ in layers] == [64, 512, 4096, 32768, N]


@pytest.mark.parametrize("topk", [1, 10, 40])
def test_exact_index_matches_search(ctx, hier, index, topk):
    x, layers, q = hier
    exp = ctx.search(x, layers, q[:500], topk, seed=9)
    got = index.search(q[:500], out_k=topk, beam=topk, mode="exact")
    assert np.array_equal(got["ids"], exp["ids"])
    assert np.array_equal(got["dists"].view(np.uint32), exp["dists"].view(np.uint32))
    assert got["ncmps"] == exp["ncmps"]


def test_exact_per_query_beams_match_oracle(oracle, hier, index):
    x, layers, q = hier
    rng = np.random.default_rng(7)
    beams = rng.integers(10, 97, size=600).astype(np.uint32)
    exp = oracle.search_ex(x, layers, q[:600], 10, 9, beams=beams)
    got = index.search(q[:600], out_k=10, beams=beams, mode="exact")
    assert np.array_equal(got["ids"], exp["ids"])
    assert np.array_equal(got["dists"].view(np.uint32), exp["dists"].view(np.uint32))
    assert got["ncmps"] == exp["ncmps"]


def test_exact_learned_entries_match_oracle(ctx, oracle, hier, index):
    x, layers, q = hier
    layer, C = index.entry_layer()
    assert (layer, C) == (2, 4096)
    m = entry_init(128, C, seed=4)
    index.set_entry_model(m, probes=4)
    try:
        got = index.search(q[:400], out_k=10, beam=32, mode="exact", entry="learned")
    finally:
        index.set_entry_model(None)
    probes = ctx.entry_probes(m, q[:400], 4)
    exp = oracle.search_ex(x, layers, q[:400], 10, 9, beam=32, probes=probes, g0=2)
    assert np.array_equal(got["ids"], exp["ids"])
    assert np.array_equal(got["dists"].view(np.uint32), exp["dists"].view(np.uint32))
    assert got["ncmps"] == exp["ncmps"]


def test_exact_flat_search_matches_oracle(oracle, hier, index):
    x, layers, q = hier
    beams = np.random.default_rng(17).integers(10, 97, size=500).astype(np.uint32)
    exp = oracle.search_ex(x, layers, q[:500], 10, 9, beams=beams, flat=True)
    got = index.search(q[:500], out_k=10, beams=beams, mode="exact", entry="flat")
    assert np.array_equal(got["ids"], exp["ids"])
    assert np.array_equal(got["dists"].view(np.uint32), exp["dists"].view(np.uint32))
    assert got["ncmps"] == exp["ncmps"]


def test_flat_search_matches_reference_golden(ctx):
    """nndFlatSrch as the reference itself ran it (tests/golden)."""
    import golden_lib
    fx = golden_lib.load("hmerge_search")
    ix = ctx.index(fx["x"], fx["layers"], seed=int(fx["seed"]))
    try:
        for topk in (1, 10, 40):
            got = ix.search(fx["q"], out_k=topk, beam=topk, mode="exact", entry="flat")
            assert np.array_equal(got["ids"], fx["flat%d_ids" % topk])
            assert np.array_equal(got["dists"], fx["flat%d_dists" % topk])
            assert got["ncmps"] == int(fx["flat%d_ncmps" % topk])
    finally:
        ix.close()


def test_fast_flat_search(hier, index):
    x, _, q = hier
    beams = np.random.default_rng(18).integers(32, 129, size=NQ).astype(np.uint32)
    f = index.search(q, out_k=10, beams=beams, mode="fast", entry="flat")
    e = index.search(q, out_k=10, beams=beams, mode="exact", entry="flat")
    assert (np.diff(f["dists"], axis=1) >= 0).all() and all(len(set(r)) == 10 for r in f["ids"])
    _, gt_d = truth(x, q)
    rf, re = recall(f["ids"], gt_d, x, q), recall(e["ids"], gt_d, x, q)
    print("flat recall fast %.4f exact %.4f" % (rf, re))
    assert rf >= re - 0.01


def test_flat_beam_larger_than_layer_is_rejected(ctx):
    x = gaussian_mixture_u8(200, d=16, seed=3)
    off = np.arange(0, 201 * 4, 4, dtype=np.uint64)
    adj = np.random.default_rng(0).integers(0, 200, size=800).astype(np.uint32)
    ix = ctx.index(x, [(off, adj)], seed=1)
    try:
        with pytest.raises(NnmError):
            ix.search(x[:5], out_k=10, beam=300, mode="fast", entry="flat")
        r = ix.search(x[:5], out_k=10, beam=200, mode="exact", entry="flat")
        assert (r["ids"][:, 0] == np.arange(5)).all()  # every row is a seed: exact search
    finally:
        ix.close()


def test_fast_results_are_exact_distances_and_recall_holds(hier, index):
    x, _, q = hier
    rng = np.random.default_rng(8)
    beams = rng.integers(32, 129, size=NQ).astype(np.uint32)
    f = index.search(q, out_k=10, beams=beams, mode="fast")
    e = index.search(q, out_k=10, beams=beams, mode="exact")
    ids, ds = f["ids"], f["dists"]
    assert (ids < N).all()
    assert all(len(set(r)) == 10 for r in ids)
    assert (np.diff(ds, axis=1) >= 0).all()
    ref = ((x[ids.astype(np.int64)].astype(np.float64) - q[:, None, :].astype(np.float64)) ** 2).sum(-1)
    assert np.abs(ds - ref).max() <= 1e-5 * ref.max()
    _, gt_d = truth(x, q)
    rf, re = recall(ids, gt_d, x, q), recall(e["ids"], gt_d, x, q)
    print("recall fast %.4f exact %.4f" % (rf, re))
    assert rf >= re - 0.01
    assert f["expansions"] > 0 and abs(f["ncmps"] - e["ncmps"]) < 0.05 * e["ncmps"]


def test_fast_is_deterministic(hier, index):
    _, _, q = hier
    a = index.search(q[:500], out_k=10, beam=64, mode="fast")
    b = index.search(q[:500], out_k=10, beam=64, mode="fast")
    assert np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["dists"], b["dists"])


def test_device_pointer_form_matches_host(hier, index):
    import torch
    _, _, q = hier
    beams = np.random.default_rng(9).integers(16, 80, size=700).astype(np.uint32)
    h = index.search(q[:700], out_k=10, beams=beams, mode="fast")
    qd = torch.from_numpy(q[:700]).cuda()
    bd = torch.from_numpy(beams.astype(np.int32)).cuda()
    oi = torch.empty((700, 10), dtype=torch.int32, device="cuda")
    od = torch.empty((700, 10), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    st = index.search_dev(qd.data_ptr(), 700, oi.data_ptr(), od.data_ptr(), 10, beams_ptr=bd.data_ptr(),
                          beam=int(beams.max()), mode="fast")
    assert np.array_equal(oi.cpu().numpy().view(np.uint32), h["ids"])
    assert np.array_equal(od.cpu().numpy(), h["dists"])
    assert st["ncmps"] == h["ncmps"]


def test_argument_errors(hier, index):
    _, _, q = hier
    with pytest.raises(NnmError):
        index.search(q[:10], out_k=10, beam=5)
    with pytest.raises(NnmError):
        index.search(q[:10], out_k=10, beam=2000)
    with pytest.raises(NnmError):
        index.search(q[:10], out_k=10, beam=32, entry="learned")
    with pytest.raises(NnmError):
        index.set_entry_model(entry_init(128, 4096), probes=9)
    with pytest.raises(NnmError):
        index.set_entry_model(entry_init(64, 4096), probes=4)


def test_device_width_outside_bound_is_reported(hier, index):
    import torch
    _, _, q = hier
    qd = torch.from_numpy(q[:64]).cuda()
    bd = torch.full((64,), 50, dtype=torch.int32, device="cuda")
    oi = torch.empty((64, 10), dtype=torch.int32, device="cuda")
    with pytest.raises(NnmError) as e:
        index.search_dev(qd.data_ptr(), 64, oi.data_ptr(), 0, 10, beams_ptr=bd.data_ptr(), beam=40, mode="fast")
    assert e.value.status == 6
    # the index stays usable
    index.search(q[:64], out_k=10, beam=40, mode="fast")


def rel_err(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


@pytest.mark.parametrize("d,C,n", [(128, 4096, 1000), (37, 300, 77), (200, 4000, 300)])
def test_entry_inference_matches_oracle(ctx, d, C, n):
    """Tensor-core scores (BF16 h and W2, FP32 sums) against the oracle's
    float64 sums of the same BF16 operands; the probes against the oracle's
    top-4 of those scores (rows whose 4th and 5th scores are closer than the
    sums' rounding may order them differently)."""
    m = entry_init(d, C, seed=1)
    m["b2"] = np.random.default_rng(2).standard_normal(C).astype(np.float32)
    x = gaussian_mixture_u8(n, d=d, seed=3)
    os_ = eo.infer_scores(m, x)
    assert rel_err(ctx.entry_forward(m, x), os_) < 1e-3
    got, exp = ctx.entry_probes(m, x, 4), eo.probes(os_, 4)
    assert (got == exp).all(1).mean() >= 0.97
    assert (got[:, 0] == exp[:, 0]).mean() >= 0.99


@pytest.mark.parametrize("d,C,B", [(128, 4096, 512), (37, 300, 77)])
def test_entry_gradients_match_oracle(ctx, d, C, B):
    rng = np.random.default_rng(5)
    m = entry_init(d, C, seed=6)
    x = gaussian_mixture_u8(B, d=d, seed=7)
    lab = rng.integers(0, C, B).astype(np.uint32)
    loss, g = ctx.entry_grad(m, x, lab)
    oloss, og = eo.loss_and_grad(m, x, lab)
    assert abs(loss - oloss) <= 1e-4 * max(1.0, abs(oloss))
    for k in ("w1", "b1", "w2", "b2"):
        assert rel_err(g[k], og[k]) < 2e-3, k


@pytest.fixture(scope="module")
def trained(hier, index):
    _, C = index.entry_layer()
    m = entry_init(128, C, seed=11)
    loss = index.entry_train(m, steps=600, batch=2048, lr=2e-3, seed=3)
    return m, loss


def test_entry_training(ctx, hier, trained):
    x, _, q = hier
    m, loss = trained
    assert np.isfinite(loss).all()
    assert loss[-30:].mean() < 0.6 * loss[:30].mean(), (loss[:30].mean(), loss[-30:].mean())
    qlab = eo.nearest_class(np.concatenate([x[:4096], q[:1000]]), np.arange(4096, 5096), 4096)
    p = ctx.entry_probes(m, q[:1000], 4)
    hit = float((p == qlab[:, None]).any(1).mean())
    print("top-4 hit rate %.3f" % hit)
    assert hit > 0.3


def test_learned_entries_in_fast_search(hier, index, trained):
    """The trained network's entries: recall at least that of the default
    entry at equal beams, with fewer distance evaluations."""
    x, _, q = hier
    m, _ = trained
    beams = np.random.default_rng(12).integers(32, 129, size=NQ).astype(np.uint32)
    index.set_entry_model(m, probes=4)
    try:
        lr = index.search(q, out_k=10, beams=beams, mode="fast", entry="learned")
    finally:
        index.set_entry_model(None)
    df = index.search(q, out_k=10, beams=beams, mode="fast")
    _, gt_d = truth(x, q)
    rl, rd = recall(lr["ids"], gt_d, x, q), recall(df["ids"], gt_d, x, q)
    print("recall learned %.4f default %.4f; cmps %d vs %d; predict %.3f ms" % (
        rl, rd, lr["ncmps"], df["ncmps"], lr["predict_ms"]))
    assert rl >= rd - 0.005
    assert lr["ncmps"] < df["ncmps"]
    assert lr["predict_ms"] > 0


# ---- edge cases of the serving kernels -------------------------------------

def small_index(ctx, n, d, metric="l2", seed=1):
    x = gaussian_mixture_u8(n, d=d, seed=seed)
    h = ctx.hmerge(x, 10, 10, seed=3, metric=metric)
    return x, h["layers"], ctx.index(x, h["layers"], seed=5, metric=metric)


def exact_dist(x, q, ids, metric):
    a = q[:, None, :].astype(np.float64)
    b = x[ids.astype(np.int64)].astype(np.float64)
    if metric == "l2":
        return ((a - b) ** 2).sum(-1)
    if metric == "l1":
        return np.abs(a - b).sum(-1)
    s = a + b
    return np.where(s != 0, (a - b) ** 2 / np.where(s != 0, s, 1), 0).sum(-1)


def test_empty_batch(ctx):
    _, _, ix = small_index(ctx, 3000, 16)
    try:
        r = ix.search(np.zeros((0, 16), np.float32), out_k=10, beam=32)
        assert r["ids"].shape == (0, 10) and r["ncmps"] == 0
    finally:
        ix.close()


@pytest.mark.parametrize("d", [1, 13, 200, 512])
@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_dimensions(ctx, oracle, d, mode):
    x, layers, ix = small_index(ctx, 3000, d, seed=d)
    try:
        q = gaussian_mixture_u8(50, d=d, seed=d + 1)
        r = ix.search(q, out_k=5, beam=24, mode=mode)
        ids = r["ids"]
        assert (ids < 3000).all() and (np.diff(r["dists"], axis=1) >= 0).all()
        ref = exact_dist(x, q, ids, "l2")
        assert np.abs(ref - r["dists"]).max() <= 1e-5 * max(ref.max(), 1.0)
        if mode == "exact":
            e = oracle.search_ex(x, layers, q, 5, 5, beam=24)
            assert np.array_equal(ids, e["ids"])
    finally:
        ix.close()


@pytest.mark.parametrize("metric", ["l1", "chi2"])
def test_fast_kernel_other_metrics(ctx, oracle, metric):
    x, layers, ix = small_index(ctx, 4000, 32, metric=metric, seed=11)
    try:
        q = gaussian_mixture_u8(200, d=32, seed=12)
        f = ix.search(q, out_k=10, beam=64, mode="fast")
        e = ix.search(q, out_k=10, beam=64, mode="exact")
        o = oracle.search_ex(x, layers, q, 10, 5, beam=64, metric=metric)
        assert np.array_equal(e["ids"], o["ids"])
        ref = exact_dist(x, q, f["ids"], metric)
        assert np.abs(ref - f["dists"]).max() <= 1e-5 * ref.max()
        # the fast kernel finds (nearly) the exact kernel's results
        same = np.mean([len(set(a) & set(b)) / 10 for a, b in zip(f["ids"], e["ids"])])
        assert same >= 0.95, same
    finally:
        ix.close()


def test_widest_beam(ctx, oracle):
    x, layers, ix = small_index(ctx, 3000, 16, seed=13)
    try:
        q = gaussian_mixture_u8(40, d=16, seed=14)
        for mode in ("exact", "fast"):
            r = ix.search(q, out_k=16, beam=1024, mode=mode)
            ref = exact_dist(x, q, np.arange(3000)[None, :].repeat(40, 0), "l2")
            kth = np.sort(ref, axis=1)[:, 15:16]
            # a 1024-wide beam over 3,000 rows finds the exact 16 nearest
            assert (exact_dist(x, q, r["ids"], "l2") <= kth).mean() >= 0.99, mode
        e = oracle.search_ex(x, layers, q, 16, 5, beam=1024)
        assert np.array_equal(ix.search(q, out_k=16, beam=1024, mode="exact")["ids"], e["ids"])
        with pytest.raises(NnmError):
            ix.search(q, out_k=16, beam=1025, mode="fast")
    finally:
        ix.close()


def test_out_k_equal_to_small_beams(ctx):
    _, _, ix = small_index(ctx, 2000, 16, seed=15)
    try:
        q = gaussian_mixture_u8(30, d=16, seed=16)
        beams = np.full(30, 10, np.uint32)
        for mode in ("exact", "fast"):
            r = ix.search(q, out_k=10, beams=beams, mode=mode)
            assert (r["ids"] != 0xFFFFFFFF).all()
    finally:
        ix.close()


def test_width_tuner(hier, index):
    """The width autotuner times widths 1..4 and keeps the fastest; the
    search then runs at it, with the results of that width."""
    _, _, q = hier
    beams = np.random.default_rng(31).integers(32, 257, size=1000).astype(np.uint32)
    w, ms = index.tune_width(q[:1000], out_k=10, beams=beams, repeats=2)
    assert 1 <= w <= 4 and (ms > 0).all() and ms[w - 1] == ms.min()
    a = index.search(q[:300], out_k=10, beams=beams[:300], mode="fast")
    index.set_width(w)
    b = index.search(q[:300], out_k=10, beams=beams[:300], mode="fast")
    assert np.array_equal(a["ids"], b["ids"])
    index.set_width(4)
