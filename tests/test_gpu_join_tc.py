"""The tensor-core local join against the FP32 join: identical graphs, bit
for bit, for every builder, both random-draw tiers, every list-size tier and
ragged dimensions -- u8 Gram matrices for integer data, BF16 ones with the
FP32 recheck for other data; the selection rule (L2; integer components in
[0, 255] for u8; finite, bounded components and d <= 384 for BF16) and its
error when forced."""
import numpy as np
import pytest

from nnm import NnmError
from nnm.datasets import gaussian_mixture_u8

pytestmark = pytest.mark.gpu


def same(a, b):
    assert np.array_equal(a["ids"], b["ids"])
    assert np.array_equal(a["dists"].view(np.uint32), b["dists"].view(np.uint32))
    assert np.array_equal(a["flags"], b["flags"])
    assert a["ncmps"] == b["ncmps"] and a["sub_ncmps"] == b["sub_ncmps"]
    assert a["iterations"] == b["iterations"]


def both(ctx, fn, *args, tjoin="tensor", **kw):
    ctx.profile(True)
    t = fn(*args, join=tjoin, **kw)
    rows = ctx.profile_stats()["rows"]
    f = fn(*args, join="fp32", **kw)
    ctx.profile(False)
    return t, f, rows


@pytest.mark.parametrize("rng", ["exact", "fast"])
def test_kgraph(ctx, rng):
    x = gaussian_mixture_u8(6000, seed=31)
    t, f, rows = both(ctx, ctx.kgraph, x, 20, seed=3, rng=rng)
    same(t, f)
    # every joined row on the tensor cores: the tiles, and the lists longer
    # than a tile on the tensor-core pair kernel
    assert rows["tensor"] > 0 and rows["tensor"] == sum(rows["tiers"])


@pytest.mark.parametrize("rng", ["exact", "fast"])
def test_smerge_leaves(ctx, rng):
    x = gaussian_mixture_u8(8000, seed=32)
    t, f, _ = both(ctx, ctx.merge_leaves, x, 20, [2000, 2000, 2000, 2000], seed=5, rng=rng)
    same(t, f)


def test_smerge(ctx):
    x = gaussian_mixture_u8(5001, seed=33)
    t, f, _ = both(ctx, ctx.smerge, x, 16, seed=7)
    same(t, f)


def test_jmerge(ctx):
    x = gaussian_mixture_u8(5000, seed=34)
    t, f, _ = both(ctx, ctx.jmerge, x, 20, seed=8)
    same(t, f)


def test_hmerge(ctx):
    x = gaussian_mixture_u8(4000, seed=35)
    t = ctx.hmerge(x, 10, 8, seed=9, join="tensor")
    f = ctx.hmerge(x, 10, 8, seed=9, join="fp32")
    same(t, f)
    assert len(t["layers"]) == len(f["layers"])
    for a, b in zip(t["layers"], f["layers"]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("d,cap", [(128, 150), (128, 400), (160, 400), (300, 400)])
def test_all_tiers_and_big_lists(ctx, d, cap):
    # k=32 with a large sample cap gives lists of 17..128 entries and rows
    # above 128, which take the tensor-core pair kernel when two buffers of
    # their 128-slot blocks fit in shared memory (d=128, lists up
    # to 364: three blocks), else the staged u8 dp4a one (lists up to 864 at
    # d=128 and 160), or the unstaged FP32 one (d=300); k=6 gives lists of
    # <= 16
    x = gaussian_mixture_u8(4000, d=d, seed=36, n_centres=8)
    t, f, big = both(ctx, ctx.kgraph, x, 32, seed=11, sample_cap=cap)
    same(t, f)
    on_tc = d == 128 and cap == 150
    assert (big["tensor"] == sum(big["tiers"])) == on_tc, big
    t, f, small = both(ctx, ctx.kgraph, x, 6, seed=11)
    same(t, f)
    assert all(a + b > 0 for a, b in zip(big["tiers"], small["tiers"])), (big, small)
    assert big["tiers"][4] > 0 and small["tiers"][0] > 0


@pytest.mark.parametrize("cap", [150, 400])
@pytest.mark.parametrize("rng", ["exact", "fast"])
def test_big_lists_in_merges(ctx, rng, cap):
    # lists above 128 entries in the merge builders: their group and verse
    # filters on the tensor-core pair kernel (cap 150) or the staged u8 pair
    # kernel (cap 400), and the block-per-row emit
    x = gaussian_mixture_u8(4000, seed=41, n_centres=8)
    t, f, rows = both(ctx, ctx.merge_leaves, x, 32, [1000] * 4, seed=5, rng=rng, sample_cap=cap)
    same(t, f)
    assert rows["tiers"][4] > 0
    t, f, rows = both(ctx, ctx.jmerge, x, 32, seed=6, rng=rng, sample_cap=cap)
    same(t, f)
    assert rows["tiers"][4] > 0


def test_big_lists_in_hmerge(ctx):
    x = gaussian_mixture_u8(4000, seed=42, n_centres=8)
    ctx.profile(True)
    t = ctx.hmerge(x, 16, 8, seed=9, join="tensor", sample_cap=400)
    rows = ctx.profile_stats()["rows"]
    ctx.profile(False)
    f = ctx.hmerge(x, 16, 8, seed=9, join="fp32", sample_cap=400)
    same(t, f)
    assert rows["tiers"][4] > 0
    for a, b in zip(t["layers"], f["layers"]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.parametrize("d", [1, 8, 37, 96, 200])
def test_ragged_dims(ctx, d):
    x = gaussian_mixture_u8(3000, d=d, seed=37 + d)
    t, f, _ = both(ctx, ctx.kgraph, x, 12, seed=13)
    same(t, f)


def test_extreme_values(ctx):
    # components 0 or 255 only: squared distances up to 128 * 255^2,
    # near the exactness limit of the float sums
    rng = np.random.default_rng(38)
    x = (rng.integers(0, 2, size=(3000, 128)) * 255).astype(np.float32)
    t, f, _ = both(ctx, ctx.kgraph, x, 10, seed=17)
    same(t, f)


def test_auto_picks_u8_tensor_cores_for_integer_data(ctx):
    # auto: integer data -> u8 tensor cores; other data -> FP32 (the BF16
    # tier only when forced)
    x = gaussian_mixture_u8(3000, seed=39)
    for data, on_tc in ((x, True), (x + 0.5, False)):
        ctx.profile(True)
        ctx.kgraph(data, 10, seed=1)
        assert (ctx.profile_stats()["rows"]["tensor"] > 0) == on_tc
    ctx.profile(False)


def float_mixture(n, d, seed, unit=False):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((32, d))
    x = c[rng.integers(0, 32, n)] + 0.35 * rng.standard_normal((n, d))
    if unit:
        x /= np.linalg.norm(x, axis=1, keepdims=True)
    return x.astype(np.float32)


@pytest.mark.parametrize("kern", ["tensor", "fp8"])
@pytest.mark.parametrize("unit", [False, True])
@pytest.mark.parametrize("rng", ["exact", "fast"])
def test_reduced_precision_matches_fp32(ctx, kern, unit, rng):
    """BF16 (hi + lo) and FP8 (E4M3 hi + mid + lo) Gram matrices: the same
    graphs as the FP32 join, bit for bit."""
    x = float_mixture(5000, 96, 50 + unit, unit)
    t, f, rows = both(ctx, ctx.kgraph, x, 16, seed=3, rng=rng, tjoin=kern)
    same(t, f)
    assert rows["tensor"] > 0


@pytest.mark.parametrize("kern", ["tensor", "fp8"])
def test_reduced_precision_merges_match_fp32(ctx, kern):
    x = float_mixture(6000, 64, 61) * 37.0
    t, f, _ = both(ctx, ctx.merge_leaves, x, 20, [1500] * 4, seed=5, tjoin=kern)
    same(t, f)
    t, f, _ = both(ctx, ctx.merge_leaves, x, 20, [1500] * 4, seed=5, rng="fast", tjoin=kern)
    same(t, f)
    t, f, _ = both(ctx, ctx.jmerge, x[:4000], 12, seed=6, tjoin=kern)
    same(t, f)
    t = ctx.hmerge(x[:3000], 10, 8, seed=9, join=kern)
    f = ctx.hmerge(x[:3000], 10, 8, seed=9, join="fp32")
    same(t, f)


@pytest.mark.parametrize("kern", ["tensor", "fp8"])
@pytest.mark.parametrize("rng_tier", ["exact", "fast"])
def test_reduced_precision_ties_and_scales(ctx, kern, rng_tier):
    """Many exact ties (few distinct values) and mixed magnitudes.  In the
    fast tier a proposal at exactly the K-th distance and of a smaller id
    would displace the K-th entry; the FP32 join never proposes it (its
    filter is strict), so neither may the reduced-precision join's merge."""
    rng = np.random.default_rng(62)
    x = (rng.integers(-3, 4, size=(4000, 40)) * 0.25).astype(np.float32)
    x[::7] *= 1e3
    t, f, _ = both(ctx, ctx.kgraph, x, 12, seed=7, rng=rng_tier, tjoin=kern)
    same(t, f)
    y = (rng.integers(0, 3, size=(6000, 24)) * 0.5).astype(np.float32)  # every distance a multiple of 0.25
    t, f, _ = both(ctx, ctx.merge_leaves, y, 16, [1500] * 4, seed=8, rng=rng_tier, tjoin=kern)
    same(t, f)


def test_fp8_on_integer_data_matches_fp32(ctx):
    # FP8 when asked for, even where the u8 join would be exact
    x = gaussian_mixture_u8(5000, seed=71)
    t, f, rows = both(ctx, ctx.kgraph, x, 20, seed=3, tjoin="fp8")
    same(t, f)
    assert rows["tensor"] > 0


@pytest.mark.parametrize("kern", ["tensor", "fp8"])
@pytest.mark.parametrize("data", ["unit", "scaled", "ties", "spread", "sparse"])
def test_reduced_precision_bound_holds(ctx, kern, data):
    """Every joined pair's d~ within err_c (|a|^2 + |b|^2) of its exact FP32
    distance (the audit computes them all and fails the call otherwise)."""
    rng = np.random.default_rng(80)
    if data == "unit":
        x = float_mixture(3000, 96, 81, True)
    elif data == "scaled":
        x = float_mixture(3000, 128, 82) * 1e-3
    elif data == "ties":
        x = (rng.integers(-3, 4, size=(3000, 40)) * 0.25).astype(np.float32)
    elif data == "spread":  # components over many binades within a row
        x = (rng.standard_normal((3000, 64)) * np.exp2(rng.integers(-20, 20, size=(3000, 64)))).astype(np.float32)
    else:  # mostly zeros, a few large components
        x = np.zeros((3000, 96), np.float32)
        m = rng.random((3000, 96)) < 0.05
        x[m] = rng.standard_normal(int(m.sum())).astype(np.float32) * 100
    ctx.kgraph(x, 12, seed=4, join=kern, audit=True)
    ctx.kgraph(x, 12, seed=4, join=kern, audit=True, rng="fast")


@pytest.mark.parametrize("bad", ["nan", "inf", "huge", "tiny", "wide"])
def test_forced_tensor_rejects_uncovered_data(ctx, bad):
    x = float_mixture(2000, 64, 40)
    if bad == "nan":
        x[5, 3] = np.nan
    elif bad == "inf":
        x[7, 1] = np.inf
    elif bad == "huge":
        x[9, 0] = 2.0 ** 60
    elif bad == "tiny":
        x[9, 0] = 2.0 ** -70
    else:
        x = float_mixture(2000, 400, 41)  # BF16 tier: d <= 192
    with pytest.raises(NnmError) as e:
        ctx.kgraph(x, 10, seed=1, join="tensor")
    assert e.value.status == 1


def test_forced_tensor_rejects_other_metrics(ctx):
    x = gaussian_mixture_u8(2000, d=32, seed=41)
    with pytest.raises(NnmError):
        ctx.kgraph(x, 10, seed=1, metric="l1", join="tensor")


@pytest.mark.parametrize("rng", ["exact", "fast"])
def test_tile_rows_give_the_same_graph(ctx, rng):
    """Lists longer than tile_rows go from the tensor-core tiles to the
    tensor-core pair kernel: both exact, the same graph for every boundary."""
    x = gaussian_mixture_u8(6000, seed=91)
    ref = ctx.kgraph(x, 20, seed=3, rng=rng, join="tensor")
    for tr in (32, 64):
        ctx.profile(True)
        g = ctx.kgraph(x, 20, seed=3, rng=rng, join="tensor", tile_rows=tr)
        rows = ctx.profile_stats()["rows"]
        ctx.profile(False)
        same(g, ref)
        assert rows["tensor"] > 0 and rows["tiers"][4] > 0
    with pytest.raises(NnmError):
        ctx.kgraph(x, 20, seed=3, join="tensor", tile_rows=48)
