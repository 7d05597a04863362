"""CPU oracle of the serving path's entry-point network -- test infrastructure.

Only the tests (and nothing on the product path) use this module: it is the
checker for the device kernels in nn-merge_b200/csrc/entry.cu.  The
reference has no learned part (its LySearch starts every query at one
random node, lysearch.cpp:382), so this restates the network as the library
documents it (include/nnm.h, "Entry-point network"):

    u = x * in_scale + in_shift
    h = relu(W1 u + b1),  s = W2 h + b2          (d -> 256 -> C)
    inference rounds h to BF16 (the tensor-core operand) before W2
    loss = mean_b [ log sum_c exp(s_bc) - s_b,label_b ]
    label of a row = its nearest class row (rows 0..C-1), squared L2,
                     ties to the lower class
    probes of a query = the classes of its P largest scores, ties to the
                     lower class, in descending order

in float64 over the BF16-rounded weights, with the analytic gradients of the
loss with respect to those weights.
"""
import numpy as np

from mlp_oracle import bf16_round


def _weights(model, rounded=True):
    f = bf16_round if rounded else (lambda a: np.asarray(a, np.float64))
    return (f(model["w1"]).astype(np.float64), np.asarray(model["b1"], np.float64),
            f(model["w2"]).astype(np.float64), np.asarray(model["b2"], np.float64))


def forward(model, x, rounded=True):
    w1, b1, w2, b2 = _weights(model, rounded)
    u = np.asarray(x, np.float64) * model["in_scale"] + model["in_shift"]
    hp = u @ w1.T + b1
    h = np.maximum(hp, 0.0)
    s = h @ w2.T + b2
    return u, hp, h, s


def scores(model, x):
    """Scores with h in full precision (the training forward)."""
    return forward(model, x)[3]


def infer_scores(model, x):
    """Scores as inference computes them: h rounded to BF16 (after rounding
    to float32, where the device accumulates it), s = W2 h + b2."""
    _, _, w2, b2 = _weights(model)
    h = bf16_round(forward(model, x)[2].astype(np.float32)).astype(np.float64)
    return h @ w2.T + b2


def loss_and_grad(model, x, labels, rounded=True):
    """Mean cross-entropy and its gradient dict (w1, b1, w2, b2)."""
    lab = np.asarray(labels, np.int64)
    u, hp, h, s = forward(model, x, rounded)
    B = s.shape[0]
    m = s.max(axis=1, keepdims=True)
    e = np.exp(s - m)
    se = e.sum(axis=1, keepdims=True)
    loss = float(np.mean(np.log(se[:, 0]) + m[:, 0] - s[np.arange(B), lab]))
    g = e / se
    g[np.arange(B), lab] -= 1.0
    g /= B
    _, _, w2, _ = _weights(model, rounded)
    gw2 = g.T @ h
    gb2 = g.sum(axis=0)
    dh = (g @ w2) * (hp > 0)
    gw1 = dh.T @ u
    gb1 = dh.sum(axis=0)
    return loss, dict(w1=gw1, b1=gb1, w2=gw2, b2=gb2)


def nearest_class(x, rows, n_classes):
    """Label of each row index in `rows`: the nearest of x[0..C-1]."""
    xr = np.asarray(x, np.float64)[np.asarray(rows, np.int64)]
    cls = np.asarray(x, np.float64)[:n_classes]
    d = (xr * xr).sum(1)[:, None] + (cls * cls).sum(1)[None, :] - 2.0 * xr @ cls.T
    return np.argmin(d, axis=1).astype(np.uint32)


def probes(s, p):
    """Classes of the p largest scores per row, ties to the lower class."""
    s = np.asarray(s)
    order = np.lexsort((np.broadcast_to(np.arange(s.shape[1]), s.shape), -s), axis=1)
    return order[:, :p].astype(np.uint32)
