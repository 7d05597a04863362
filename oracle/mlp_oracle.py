"""CPU oracle of the learned-initialisation code MLP -- test infrastructure.

Only the tests (and nothing on the product path) use this module: it is the
checker for the device kernels in nn-merge_b200/csrc/learned.cu.  The
reference has no learned part, so this restates the model as the library
documents it (include/nnm.h, "Learned initialisation"):

    u = x * in_scale + in_shift
    h = relu(W1 u + b1),  z = W2 h + b2,  t = tanh(z),  code bit o = z_o > 0
    loss = mean_b max(0, margin + |t_a - t_p|^2 - |t_a - t_n|^2)

in float64 over the BF16-rounded weights (round to nearest even), with the
analytic gradients of the loss with respect to those weights.
"""
import numpy as np


def bf16_round(a):
    """float32 values rounded to the nearest bfloat16 (ties to even)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _weights(model, rounded=True):
    f = bf16_round if rounded else (lambda a: np.asarray(a, np.float64))
    return (f(model["w1"]).astype(np.float64), np.asarray(model["b1"], np.float64),
            f(model["w2"]).astype(np.float64), np.asarray(model["b2"], np.float64))


def forward(model, x, rounded=True):
    w1, b1, w2, b2 = _weights(model, rounded)
    u = np.asarray(x, np.float64) * model["in_scale"] + model["in_shift"]
    hp = u @ w1.T + b1
    h = np.maximum(hp, 0.0)
    z = h @ w2.T + b2
    return u, hp, h, z


def codes(model, x):
    z = forward(model, x)[3]
    bits = (z > 0).astype(np.uint64) << np.arange(z.shape[1], dtype=np.uint64)
    return bits.sum(axis=1).astype(np.uint32), z


def loss_and_grad(model, x, triplets, margin=16.0, rounded=True):
    """Loss and gradient dict (w1, b1, w2, b2) over triplets (B x 3 rows)."""
    tr = np.asarray(triplets, np.int64)
    B = tr.shape[0]
    rows = np.concatenate([tr[:, 0], tr[:, 1], tr[:, 2]])
    u, hp, h, z = forward(model, np.asarray(x)[rows], rounded)
    t = np.tanh(z)
    ta, tp, tn = t[:B], t[B:2 * B], t[2 * B:]
    dp = ((ta - tp) ** 2).sum(1)
    dn = ((ta - tn) ** 2).sum(1)
    l = np.maximum(margin + dp - dn, 0.0)
    sc = np.where(l > 0, 2.0 / B, 0.0)[:, None]
    dt = np.concatenate([sc * (tn - tp), -sc * (ta - tp), sc * (ta - tn)])
    dz = dt * (1.0 - t * t)
    _, _, w2, _ = _weights(model, rounded)
    dh = (dz @ w2) * (hp > 0)
    grad = dict(w1=dh.T @ u, b1=dh.sum(0), w2=dz.T @ h, b2=dz.sum(0))
    return float(l.mean()), grad
