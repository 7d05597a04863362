"""The tensor-core local join (u8 Gram matrices on tcgen05) against the FP32
join: identical graphs, bit for bit, for every builder, both random-draw
tiers, every list-size tier and ragged dimensions; the selection rule
(integer components in [0, 255], L2) and its error when forced."""
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


def both(ctx, fn, *args, **kw):
    ctx.profile(True)
    t = fn(*args, join="tensor", **kw)
    rows = ctx.profile_stats()["rows"]
    f = fn(*args, join="fp32", **kw)
    ctx.profile(False)
    return t, f, rows


@pytest.mark.parametrize("rng", ["exact", "fast"])
def test_kgraph(ctx, rng):
    x = gaussian_mixture_u8(6000, seed=31)
    t, f, rows = both(ctx, ctx.kgraph, x, 20, seed=3, rng=rng)
    same(t, f)
    assert rows["tensor"] > 0 and rows["tensor"] == sum(rows["tiers"][:4])


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


def test_all_tiers_and_big_lists(ctx):
    # k=32 with a large sample cap gives lists of 17..128 entries and rows
    # above 128 that stay on the FP32 kernel; k=6 gives lists of <= 16
    x = gaussian_mixture_u8(4000, seed=36, n_centres=8)
    t, f, big = both(ctx, ctx.kgraph, x, 32, seed=11, sample_cap=400)
    same(t, f)
    t, f, small = both(ctx, ctx.kgraph, x, 6, seed=11)
    same(t, f)
    assert all(a + b > 0 for a, b in zip(big["tiers"], small["tiers"])), (big, small)
    assert big["tiers"][4] > 0 and small["tiers"][0] > 0


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


def test_auto_picks_tensor_only_when_exact(ctx):
    x = gaussian_mixture_u8(3000, seed=39)
    ctx.profile(True)
    a = ctx.kgraph(x, 10, seed=1)
    assert ctx.profile_stats()["rows"]["tensor"] > 0
    ctx.profile(True)
    xf = x + 0.5
    b = ctx.kgraph(xf, 10, seed=1)
    assert ctx.profile_stats()["rows"]["tensor"] == 0
    ctx.profile(False)
    assert a["ids"].shape == b["ids"].shape


@pytest.mark.parametrize("bad", ["fraction", "negative", "big", "norm"])
def test_forced_tensor_rejects_inexact_data(ctx, bad):
    x = gaussian_mixture_u8(2000, d=64, seed=40)
    if bad == "fraction":
        x[5, 3] += 0.25
    elif bad == "negative":
        x[7, 1] = -1.0
    elif bad == "big":
        x[9, 0] = 256.0
    else:
        x = np.full((2000, 300), 255.0, np.float32)  # 2 * |x|^2 >= 2^24
        x[:, 0] = np.arange(2000) % 256
    with pytest.raises(NnmError) as e:
        ctx.kgraph(x, 10, seed=1, join="tensor")
    assert e.value.status == 1


def test_forced_tensor_rejects_other_metrics(ctx):
    x = gaussian_mixture_u8(2000, d=32, seed=41)
    with pytest.raises(NnmError):
        ctx.kgraph(x, 10, seed=1, metric="l1", join="tensor")
