"""The oracle (oracle/nnm_oracle.c, the reference restated in C) against the
reference's own outputs: the committed fixtures in tests/golden/ and, where
oracle/_ref/nnm_ref is built, live runs on fresh seeds."""
import ctypes
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import golden_lib
from oracle_lib import ref_available, run_ref
from nnm.datasets import gaussian_mixture_u8, queries_like


def run_oracle(oracle, fx):
    cmd, x, k, seed, metric = fx["cmd"], fx["x"], fx["k"], fx["seed"], fx["metric"]
    if cmd == "hmerge":
        return oracle.hmerge(x, k, fx["m"], seed, metric=metric)
    return getattr(oracle, cmd)(x, k, seed, metric=metric)


@pytest.mark.parametrize("name", golden_lib.names())
def test_oracle_matches_golden(oracle, name):
    fx = golden_lib.load(name)
    got = run_oracle(oracle, fx)
    assert golden_lib.same_pools(got, fx)
    assert got["ncmps"] == fx["ncmps"]
    assert np.array_equal(got["trace"], fx["trace"])
    if "layers" in fx:
        assert len(got["layers"]) == len(fx["layers"])
        for (go, ga), (eo, ea) in zip(got["layers"], fx["layers"]):
            assert np.array_equal(go, eo) and np.array_equal(ga, ea)


def test_oracle_search_matches_golden(oracle):
    fx = golden_lib.load("hmerge_search")
    for topk in (1, 10, 40):
        got = oracle.search(fx["x"], fx["layers"], fx["q"], topk, fx["seed"])
        assert np.array_equal(got["ids"], fx["search%d_ids" % topk])
        assert np.array_equal(got["dists"], fx["search%d_dists" % topk])
        assert got["ncmps"] == int(fx["search%d_ncmps" % topk])
        assert got["entry"] == int(fx["search%d_entry" % topk])


def test_oracle_flat_search_matches_golden(oracle):
    """nndFlatSrch: the reference's own flat search (random seeds of the
    last layer, no descent) against the oracle's restatement."""
    fx = golden_lib.load("hmerge_search")
    for topk in (1, 10, 40):
        got = oracle.search_ex(fx["x"], fx["layers"], fx["q"], topk, fx["seed"], beam=topk, flat=True)
        assert np.array_equal(got["ids"], fx["flat%d_ids" % topk])
        assert np.array_equal(got["dists"], fx["flat%d_dists" % topk])
        assert got["ncmps"] == int(fx["flat%d_ncmps" % topk])


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cmd,n,k,seed", [("kgraph", 1500, 20, 1), ("kgraph", 900, 16, 123456),
                                          ("smerge", 1200, 20, 7), ("jmerge", 1300, 12, 99),
                                          ("hmerge", 2500, 16, 5)])
def test_oracle_matches_live_reference(oracle, cmd, n, k, seed):
    x = gaussian_mixture_u8(n, d=48, seed=n + k)
    with tempfile.TemporaryDirectory() as td:
        exp = run_ref(cmd, x, k, seed, td, m=16)
    got = oracle.hmerge(x, k, 16, seed) if cmd == "hmerge" else getattr(oracle, cmd)(x, k, seed)
    for key in ("ids", "dists", "flags", "trace"):
        assert np.array_equal(got[key], exp[key]), key
    assert got["ncmps"] == exp["ncmps"]


def test_glibc_rand_restatement_matches_libc(oracle):
    libc = ctypes.CDLL(None)
    for seed in (1, 2, 12345, 4000000000):
        libc.srand(ctypes.c_uint(seed))
        ref = [libc.rand() for _ in range(2000)]
        assert list(oracle.glibc_rand(seed, 2000)) == ref
    libc.srand(ctypes.c_uint(0))  # srand(0) behaves as srand(1)
    assert [libc.rand() for _ in range(10)] == list(oracle.glibc_rand(1, 10))


def test_mt19937_known_answer(oracle):
    # The C++ standard pins the 10000th output of default-seeded mt19937.
    assert int(oracle.mt19937(5489, 10000)[-1]) == 4123659995


def test_rnd_seeds_distinct_and_in_range(oracle):
    for n, k in ((100, 21), (21, 21), (22, 21), (1000, 40)):
        s = oracle.rnd_seeds(3, 50, k, n)
        assert (s < n).all()
        assert all(len(set(r)) == k for r in s)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_sort_port_matches_libstdcxx(oracle):
    """The restated std::sort must order ties exactly as libstdc++ does."""
    src = r"""
    #include <algorithm>
    #include <cstdio>
    #include <vector>
    struct E { unsigned id; float d; };
    int main() {
        unsigned n, t; std::vector<E> v;
        while (scanf("%u", &n) == 1) {
            v.resize(n);
            for (unsigned i = 0; i < n; i++) { scanf("%u", &t); v[i].id = i; v[i].d = (float)t; }
            std::sort(v.begin(), v.end(), [](const E &a, const E &b) { return a.d < b.d; });
            for (unsigned i = 0; i < n; i++) printf("%u ", v[i].id);
            printf("\n");
        }
    }"""
    rng = np.random.default_rng(0)
    cases = [rng.integers(0, m, size) for size in (1, 2, 5, 16, 17, 20, 24, 25, 31, 40, 64, 200)
             for m in (1, 2, 3, 50) for _ in range(3)]
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "s")
        subprocess.run(["g++", "-O2", "-x", "c++", "-", "-o", exe], input=src, text=True, check=True)
        inp = "".join("%d %s\n" % (len(c), " ".join(map(str, c))) for c in cases)
        out = subprocess.run([exe], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    for c, line in zip(cases, out):
        exp = [int(t) for t in line.split()]
        ids, _, _ = oracle.sort_pool(np.arange(len(c)), c.astype(np.float32), np.zeros(len(c), np.uint8))
        assert list(ids) == exp, (len(c), c)
