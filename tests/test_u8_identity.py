"""The identity behind the u8 join kernels (the tcgen05 kind::i8 tiles and
the staged dp4a kernel for lists over 128 entries): when every component is
an integer in [0, 255] and 2 * max |x|^2 < 2^24 (the gate checked on upload),
|a|^2 + |b|^2 - 2 a.b computed in integers equals, bit for bit, the
reference's sequential float sum of squared differences (vmath.cpp:56-88,
restated by the oracle)."""
import numpy as np
import pytest

from oracle_lib import Oracle


def integer_form(x, i, j):
    a = x[i].astype(np.int64)
    b = x[j].astype(np.int64)
    return np.float32(int(a @ a) + int(b @ b) - 2 * int(a @ b))


def gate(x):
    n2 = (x.astype(np.int64) ** 2).sum(1)
    return 2 * int(n2.max()) < (1 << 24)


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.mark.parametrize("d", [1, 8, 37, 96, 128, 200, 256])
def test_integer_form_equals_reference_sum(oracle, d):
    rng = np.random.default_rng(d)
    hi = 256 if 2 * d * 255 * 255 < (1 << 24) else int(np.sqrt((1 << 23) / d))
    x = rng.integers(0, hi, size=(64, d)).astype(np.float32)
    assert gate(x)
    for i in range(0, 64, 3):
        for j in range(i + 1, 64, 5):
            ref = np.float32(oracle.dist(x, i, j))
            assert integer_form(x, i, j).view(np.uint32) == ref.view(np.uint32), (d, i, j)


def test_extremes_at_the_gate(oracle):
    # components 0 or 255 at d = 128: distances up to 128 * 255^2, just
    # below 2^24, where every partial sum is still exact
    rng = np.random.default_rng(7)
    x = (rng.integers(0, 2, size=(48, 128)) * 255).astype(np.float32)
    x[0] = 0.0
    x[1] = 255.0
    assert gate(x)
    for i in range(48):
        for j in range(i + 1, 48, 7):
            assert integer_form(x, i, j) == np.float32(oracle.dist(x, i, j)), (i, j)
    assert integer_form(x, 0, 1) == np.float32(128 * 255 * 255)
