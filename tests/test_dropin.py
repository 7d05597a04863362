"""The C++ drop-in classes (nn-merge_b200/cpp/nnm_dropin.hpp) used the way the
reference's own test() functions use its classes."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from nnm.datasets import gaussian_mixture_u8
from oracle_lib import ref_available, run_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_gxx = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def build(td):
    exe = os.path.join(td, "dropin_main")
    subprocess.run(["g++", "-O2", "-std=c++11", "-I", os.path.join(ROOT, "nn-merge_b200", "cpp"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"), "-o", exe,
                    "-L", os.path.join(ROOT, "nn-merge_b200", "lib"), "-lnnm",
                    "-Wl,-rpath," + os.path.join(ROOT, "nn-merge_b200", "lib")], check=True)
    return exe


def write_fvecs(path, x):
    with open(path, "wb") as f:
        for row in x:
            f.write(np.int32(x.shape[1]).tobytes())
            f.write(row.astype(np.float32).tobytes())


def read_knn(path):
    lines = open(path).read().split("\n")
    n, k = map(int, lines[0].split())
    ids = np.array([[int(t) for t in lines[1 + i].split()[2:2 + k]] for i in range(n)], np.uint32)
    return ids


@needs_gxx
def test_dropin_compiles_against_the_reference_interface():
    with tempfile.TemporaryDirectory() as td:
        assert os.path.exists(build(td))


@needs_gxx
@pytest.mark.gpu
@pytest.mark.parametrize("cmd", ["kgraph", "smerge", "jmerge"])
def test_dropin_matches_oracle(oracle, cmd):
    x = gaussian_mixture_u8(2000, d=64, seed=3)
    with tempfile.TemporaryDirectory() as td:
        exe = build(td)
        src, dst = os.path.join(td, "x.fvecs"), os.path.join(td, "g.txt")
        write_fvecs(src, x)
        env = dict(os.environ, NNM_SEED="4242")
        subprocess.run([exe, cmd, src, "20", dst], check=True, env=env, capture_output=True)
        got = read_knn(dst)
    exp = getattr(oracle, cmd)(x, 20, 4242)
    assert np.array_equal(got, exp["ids"])


@needs_gxx
@pytest.mark.gpu
@pytest.mark.parametrize("cmd", ["search", "flatsearch"])
def test_dropin_search_matches_oracle(oracle, cmd):
    """LyNNDescent::buildhgraph then LySearch::knnSearch / singleknnSearch
    through the drop-in classes: the last beam of the sweep (2, with no
    ground truth) against the oracle's search at that beam."""
    from nnm.datasets import queries_like
    x = gaussian_mixture_u8(34000, d=16, seed=9)
    q = queries_like(300, d=16, seed=9, query_seed=4)
    with tempfile.TemporaryDirectory() as td:
        exe = build(td)
        src, qp = os.path.join(td, "x.fvecs"), os.path.join(td, "q.fvecs")
        write_fvecs(src, x)
        write_fvecs(qp, q)
        env = dict(os.environ, NNM_SEED="77")
        pre = os.path.join(td, "h")
        subprocess.run([exe, "hmerge", src, "10", "10", pre], check=True, env=env, capture_output=True)
        out, rec = os.path.join(td, "s.txt"), os.path.join(td, "r.txt")
        subprocess.run([exe, cmd, src, pre + ".txt", qp, out, rec], check=True, env=env, capture_output=True)
        got = np.array([int(l.split()[1]) for l in open(out).read().strip().split("\n")], np.uint32)
        assert len(open(rec).read().strip().split("\n")) == 17
    h = oracle.hmerge(x, 10, 10, 77)
    exp = oracle.search_ex(x, h["layers"], q, 2, 77, beam=2, flat=(cmd == "flatsearch"))
    assert np.array_equal(got, exp["ids"][:, 0])


@needs_gxx
@pytest.mark.gpu
@pytest.mark.skipif(not ref_available(), reason="oracle/_ref/nnm_ref (the reference compiled from its sources) not built")
def test_reference_reads_the_dropin_hierarchy(oracle):
    """LyNNDescent::buildhgraph of the drop-in writes <dst>.txt; the
    reference's own LySearch::loadGraphs (lysearch.cpp:112-186) reads it and
    searches: its results equal the oracle's search on the layers as this
    package parses them (so both read the file alike), and those layers are
    the reference's own H-Merge hierarchy.  The reference's search walks
    five layers (lysearch.cpp:393-421), so the set has more than 32,768
    rows."""
    from nnm import io as nio
    from nnm.datasets import queries_like
    x = gaussian_mixture_u8(34000, d=16, seed=12)
    q = queries_like(200, d=16, seed=12, query_seed=5)
    with tempfile.TemporaryDirectory() as td:
        exe = build(td)
        src = os.path.join(td, "x.fvecs")
        write_fvecs(src, x)
        pre = os.path.join(td, "h")
        subprocess.run([exe, "hmerge", src, "10", "10", pre], check=True, capture_output=True,
                       env=dict(os.environ, NNM_SEED="31"))
        layers = nio.read_layers_text(pre + ".txt")
        ref = run_ref("search", x, 10, 31, td, layers_txt=pre + ".txt", queries=q, topk=10)
    exp = oracle.search(x, layers, q, 10, 31)
    assert np.array_equal(ref["ids"], exp["ids"]) and np.array_equal(ref["dists"], exp["dists"])
    assert ref["ncmps"] == exp["ncmps"]
    h = oracle.hmerge(x, 10, 10, 31)
    assert len(h["layers"]) == len(layers)
    for (a, b), (c, e) in zip(h["layers"], layers):
        assert np.array_equal(a, c) and np.array_equal(b, e)
