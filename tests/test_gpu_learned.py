"""Learned initialisation on the device: the MLP kernels against the CPU
oracle (forward, codes, gradients), training, and what the trained network
gains over the method without it (random initial graphs)."""
import numpy as np
import pytest

import mlp_oracle as mo
from nnm import NnmError, mlp_init
from nnm.datasets import gaussian_mixture_u8

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def recall10(x, ids):
    import torch
    t = torch.from_numpy(x).cuda()
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        nrm = (t * t).sum(1)
        d = nrm[:, None] + nrm[None, :] - 2.0 * (t @ t.T)
        d.fill_diagonal_(float("inf"))
        kth = torch.topk(d, 10, dim=1, largest=False).values[:, -1:]
        g = torch.as_tensor(ids[:, :10].astype(np.int64)).cuda()
        return float((torch.gather(d, 1, g) <= kth).float().mean())
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


@pytest.mark.parametrize("d", [128, 37])
def test_forward_and_codes_match_oracle(ctx, d):
    m = mlp_init(d, seed=1)
    x = gaussian_mixture_u8(3000, d=d, seed=2)
    codes, z = ctx.mlp_codes(m, x, want_z=True)
    oc, oz = mo.codes(m, x)
    assert rel_err(z, oz) < 1e-5
    flip = (((codes ^ oc)[:, None] >> np.arange(32, dtype=np.uint32)) & 1).astype(bool)
    # a code bit can differ only where z is within rounding of 0
    assert flip.sum() == 0 or np.abs(oz[flip]).max() < 1e-4 * np.abs(oz).max()


@pytest.mark.parametrize("margin", [2.0, 16.0])
def test_gradients_match_oracle(ctx, margin):
    rng = np.random.default_rng(4)
    d = 128
    m = mlp_init(d, seed=7)
    x = gaussian_mixture_u8(2000, d=d, seed=8)
    tr = rng.integers(0, 2000, size=(512, 3)).astype(np.uint32)
    loss, g = ctx.mlp_grad(m, x, tr, margin=margin)
    oloss, og = mo.loss_and_grad(m, x, tr, margin=margin)
    assert abs(loss - oloss) <= 1e-4 * max(1.0, abs(oloss))
    for k in ("w1", "b1", "w2", "b2"):
        assert rel_err(g[k], og[k]) < 2e-3, k


def test_grad_rejects_bad_input(ctx):
    m = mlp_init(16, seed=0)
    x = np.zeros((10, 16), np.float32)
    with pytest.raises(NnmError):
        ctx.mlp_grad(m, x, np.array([[0, 1, 10]], np.uint32))
    with pytest.raises(NnmError):
        ctx.mlp_codes(m, np.zeros((10, 17), np.float32))


@pytest.fixture(scope="module")
def trained(ctx):
    """A model trained on the graph the method builds for a 50k set of the
    same generator (256 centres), as the learned initialisation is meant
    to be used: trained once, applied to fresh data."""
    x = gaussian_mixture_u8(50_000, n_centres=256, seed=101)
    g = ctx.kgraph(x, 20, seed=1, rng="fast", join="tensor")
    m = mlp_init(128, seed=3)
    loss = ctx.mlp_train(x, g["ids"], m, steps=300, batch=2048, lr=2e-3, margin=16.0, seed=9)
    return m, loss


def test_training_reduces_loss(trained):
    _, loss = trained
    assert np.isfinite(loss).all()
    assert loss[-20:].mean() < 0.7 * loss[:20].mean(), (loss[:20].mean(), loss[-20:].mean())


def test_training_is_deterministic(ctx):
    x = gaussian_mixture_u8(5000, seed=12)
    g = ctx.kgraph(x, 10, seed=1, rng="fast")
    a, b = mlp_init(128, seed=1), mlp_init(128, seed=1)
    la = ctx.mlp_train(x, g["ids"], a, steps=20, batch=512, seed=3)
    lb = ctx.mlp_train(x, g["ids"], b, steps=20, batch=512, seed=3)
    assert np.array_equal(la, lb) and np.array_equal(a["w1"], b["w1"]) and np.array_equal(a["w2"], b["w2"])


def test_learned_init_needs_model_and_fast_rng(ctx):
    x = gaussian_mixture_u8(2000, seed=13)
    ctx.set_init_model(None)
    with pytest.raises(NnmError):
        ctx.kgraph(x, 10, seed=1, rng="fast", init="learned")
    ctx.set_init_model(mlp_init(128, seed=1))
    with pytest.raises(NnmError):
        ctx.kgraph(x, 10, seed=1, rng="exact", init="learned")
    ctx.set_init_model(None)


def test_learned_builds_are_deterministic_and_well_formed(ctx, trained):
    m, _ = trained
    ctx.set_init_model(m)
    x = gaussian_mixture_u8(20_000, n_centres=256, seed=202)
    a = ctx.merge_leaves(x, 20, [5000] * 4, seed=4, rng="fast", init="learned")
    b = ctx.merge_leaves(x, 20, [5000] * 4, seed=4, rng="fast", init="learned")
    ctx.set_init_model(None)
    assert np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["dists"], b["dists"])
    ids, ds = a["ids"], a["dists"]
    assert (np.diff(ds, axis=1) >= 0).all()
    assert (ids != np.arange(len(x))[:, None]).all()
    assert all(len(set(r)) == 20 for r in ids[:2000])
    ref = ((x[:, None, :] - x[ids]) ** 2).sum(-1).astype(np.float32)
    assert np.array_equal(ref, ds)


def test_trained_network_gains_over_random_init(ctx, trained):
    """Fresh data (another seed): the initial graph from the trained codes
    is far closer to the exact graph than a random one, and after the same
    small number of NN-Descent iterations the learned start keeps a clear
    recall lead; an untrained network of the same shape gains less."""
    m, _ = trained
    x = gaussian_mixture_u8(30_000, n_centres=256, seed=303)
    res = {}
    for name, model in (("random", None), ("untrained", mlp_init(128, seed=3)), ("trained", m)):
        ctx.set_init_model(model)
        init = "random" if model is None else "learned"
        g0 = ctx.kgraph(x, 20, seed=5, rng="fast", init=init, max_iter=1)
        g2 = ctx.kgraph(x, 20, seed=5, rng="fast", init=init, max_iter=3)
        gf = ctx.kgraph(x, 20, seed=5, rng="fast", init=init)
        res[name] = dict(r1=recall10(x, g0["ids"]), r3=recall10(x, g2["ids"]), rf=recall10(x, gf["ids"]),
                         iters=gf["iterations"])
    ctx.set_init_model(None)
    print(res)
    assert res["trained"]["r1"] > res["random"]["r1"] + 0.2
    assert res["trained"]["r3"] > res["random"]["r3"] + 0.02
    assert res["trained"]["r1"] > res["untrained"]["r1"]
    assert res["trained"]["rf"] >= res["random"]["rf"] - 0.005
    assert res["trained"]["iters"] <= res["random"]["iters"]
