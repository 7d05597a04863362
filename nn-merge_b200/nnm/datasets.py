"""Seeded synthetic inputs standing in for the reference's SIFT-style data.

The reference's own inputs (sift100k.txt and its ground truth) are not
shipped, so every workload here is generated from a seed:

- ``gaussian_mixture_u8``: integer-valued float32 vectors in [0, 255] from a
  mixture of isotropic Gaussians with centres uniform in [0, centre_hi)
  (the 128-d, 0-255 integer shape of SIFT descriptors).
- ``vmf_mixture``: unit-norm float32 vectors from a von Mises-Fisher-like
  mixture (a centre direction plus Gaussian noise of scale 1/sqrt(kappa),
  renormalised).
- ``queries_like``: fresh draws from the same mixture as a base set.
"""
import numpy as np


def _mixture_int(rng, n, d, centres, sigma):
    lab = rng.integers(0, centres.shape[0], n)
    out = np.empty((n, d), np.float32)
    step = 1 << 16
    for b in range(0, n, step):
        e = min(n, b + step)
        v = centres[lab[b:e]] + rng.normal(0.0, sigma, (e - b, d))
        out[b:e] = np.clip(np.rint(v), 0, 255)
    return out


def gaussian_mixture_u8(n, d=128, n_centres=64, sigma=20.0, centre_hi=120.0, seed=1234):
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, centre_hi, (n_centres, d))
    return _mixture_int(rng, n, d, centres, sigma)


def queries_like(nq, d=128, n_centres=64, sigma=20.0, centre_hi=120.0, seed=1234, query_seed=99):
    """Queries from the same mixture as gaussian_mixture_u8(seed=seed), drawn
    with an independent seed."""
    centres = np.random.default_rng(seed).uniform(0.0, centre_hi, (n_centres, d))
    return _mixture_int(np.random.default_rng(query_seed), nq, d, centres, sigma)


def vmf_mixture(n, d=96, n_centres=1024, kappa=50.0, seed=4321):
    rng = np.random.default_rng(seed)
    mu = rng.normal(size=(n_centres, d))
    mu /= np.linalg.norm(mu, axis=1, keepdims=True)
    out = np.empty((n, d), np.float32)
    step = 1 << 16
    for b in range(0, n, step):
        e = min(n, b + step)
        lab = rng.integers(0, n_centres, e - b)
        v = mu[lab] + rng.normal(0.0, 1.0 / np.sqrt(kappa), (e - b, d))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        out[b:e] = v
    return out
