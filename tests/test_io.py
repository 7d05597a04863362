"""File formats on the CPU: what the drop-in (nn-merge_b200/cpp) and the
Python host side (nnm.io) write, the reference's own readers read the same
way -- IODelegator::load_refSet for vectors (iodelegator.cpp:159-182) and
IODelegator::loadKNNGraph for k-NN graphs (:65-102), run from the reference
compiled from its sources (oracle/_ref) -- and the binary graph form round
trips through both."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from nnm import io as nio
from oracle_lib import REF_BIN, ref_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_io(td):
    exe = os.path.join(td, "io_main")
    subprocess.run(["g++", "-O2", "-std=c++11", "-I", os.path.join(ROOT, "nn-merge_b200", "cpp"),
                    os.path.join(ROOT, "tests", "cpp", "io_main.cpp"), "-o", exe,
                    "-L", os.path.join(ROOT, "nn-merge_b200", "lib"), "-lnnm",
                    "-Wl,-rpath," + os.path.join(ROOT, "nn-merge_b200", "lib")], check=True)
    return exe


def read_mat(path):
    b = open(path, "rb").read()
    n, d = np.frombuffer(b[:8], np.uint32)
    return np.frombuffer(b[8:], np.float32, int(n) * int(d)).reshape(int(n), int(d))


def read_ids(path):
    b = open(path, "rb").read()
    n, k = np.frombuffer(b[:8], np.uint32)
    return np.frombuffer(b[8:], np.uint32, int(n) * int(k)).reshape(int(n), int(k))


@pytest.fixture(scope="module")
def io_exe():
    if shutil.which("g++") is None:
        pytest.skip("needs g++")
    td = tempfile.mkdtemp()
    yield build_io(td)
    shutil.rmtree(td)


@pytest.mark.parametrize("ext", [".fvecs", ".bvecs", ".txt"])
def test_vectors_read_alike(io_exe, ext):
    rng = np.random.default_rng(3)
    x = rng.integers(0, 256, size=(300, 24)).astype(np.float32)
    if ext == ".fvecs":
        x = x + rng.random(x.shape, np.float32) * (x < 128)  # non-integer values too
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "x" + ext)
        if ext == ".fvecs":
            nio.write_fvecs(src, x)
        elif ext == ".bvecs":
            nio.write_bvecs(src, x)
        else:
            with open(src, "w") as f:
                f.write("%d %d\n" % x.shape)
                for row in x:
                    f.write(" ".join(repr(float(v)) for v in row) + "\n")
        mine = os.path.join(td, "mine.mat")
        subprocess.run([io_exe, "vecs", src, mine], check=True)
        got_py = nio.read_vecs(src)
        assert np.array_equal(read_mat(mine), x) and np.array_equal(got_py, x)
        if ref_available():
            ref = os.path.join(td, "ref.mat")
            subprocess.run([REF_BIN, "loadvecs", src, ref], check=True, capture_output=True)
            assert np.array_equal(read_mat(ref), x)


def test_knn_graph_formats_round_trip(io_exe):
    rng = np.random.default_rng(5)
    ids = rng.integers(0, 5000, size=(5000, 20)).astype(np.uint32)
    with tempfile.TemporaryDirectory() as td:
        txt, binf = os.path.join(td, "g.txt"), os.path.join(td, "g.knng")
        nio.write_knn_text(txt, ids)
        subprocess.run([io_exe, "knn", txt, binf], check=True)  # text -> binary (drop-in)
        assert np.array_equal(nio.read_knn(binf), ids)
        back = os.path.join(td, "back.txt")
        subprocess.run([io_exe, "knn", binf, back], check=True)  # binary -> text (drop-in)
        assert np.array_equal(nio.read_knn(back), ids)
        nio.write_knn_bin(os.path.join(td, "py.knng"), ids)
        assert open(os.path.join(td, "py.knng"), "rb").read() == open(binf, "rb").read()
        assert nio.file_size(binf) == 16 + ids.size * 4
        if ref_available():
            for f in (txt, back):
                out = os.path.join(td, "ref.ids")
                subprocess.run([REF_BIN, "loadknn", f, "20", out], check=True, capture_output=True)
                assert np.array_equal(read_ids(out), ids)
                subprocess.run([REF_BIN, "loadknn", f, "10", out], check=True, capture_output=True)
                assert np.array_equal(read_ids(out), ids[:, :10])


def test_hierarchy_text_round_trip():
    rng = np.random.default_rng(9)
    layers = []
    for rows in (64, 512, 3000):
        deg = rng.integers(1, 12, size=rows)
        off = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint64)
        layers.append((off, rng.integers(0, rows, size=int(off[-1])).astype(np.uint32)))
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "h.txt")
        nio.write_layers_text(p, layers)
        got = nio.read_layers_text(p)
    assert len(got) == 3
    for (a, b), (c, e) in zip(got, layers):
        assert np.array_equal(a, c) and np.array_equal(b, e)
