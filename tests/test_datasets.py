import numpy as np

from nnm.datasets import gaussian_mixture_u8, queries_like, vmf_mixture


def test_mixture_is_integer_valued_and_seeded():
    a = gaussian_mixture_u8(5000, seed=3)
    b = gaussian_mixture_u8(5000, seed=3)
    assert a.dtype == np.float32 and a.shape == (5000, 128)
    assert np.array_equal(a, b)
    assert a.min() >= 0 and a.max() <= 255 and np.array_equal(a, np.rint(a))
    assert 0.0 < (a == 0).mean() < 0.3


def test_queries_come_from_the_same_mixture():
    q = queries_like(100, seed=3, query_seed=4)
    assert q.shape == (100, 128) and not np.array_equal(q, gaussian_mixture_u8(100, seed=3))


def test_vmf_rows_are_unit_norm():
    v = vmf_mixture(1000, d=96, n_centres=16, seed=1)
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0, atol=1e-5)
