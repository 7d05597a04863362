"""Test-side bindings to the checker in oracle/ (never used by the product).

- ``Oracle``: ctypes wrapper of oracle/libnnm_oracle.so, the C restatement of
  the reference hot path.
- ``run_ref``: runs oracle/_ref/nnm_ref, the reference itself compiled from
  its sources, where that binary exists.
"""
import ctypes
import os
import struct
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "libnnm_oracle.so")
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "nnm_ref")
METRICS = {"l2": 0, "l1": 1, "chi2": 2}


class Stats(ctypes.Structure):
    _fields_ = [("ncmps", ctypes.c_uint64), ("trace_len", ctypes.c_uint32),
                ("trace_cap", ctypes.c_uint32), ("trace", ctypes.POINTER(ctypes.c_float))]


class Layers(ctypes.Structure):
    _fields_ = [("nlayers", ctypes.c_uint32), ("nrows", ctypes.c_uint32 * 16),
                ("off", ctypes.POINTER(ctypes.c_uint64) * 16),
                ("adj", ctypes.POINTER(ctypes.c_uint32) * 16)]


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                           capture_output=True)
        self.lib = ctypes.CDLL(ORACLE_SO)

    def _graph(self, fn, x, k, seed, metric, extra=()):
        x = np.ascontiguousarray(x, dtype=np.float32)
        n, d = x.shape
        ids = np.zeros((n, k), np.uint32)
        dists = np.zeros((n, k), np.float32)
        flags = np.zeros((n, k), np.uint8)
        trace = np.zeros(4096, np.float32)
        st = Stats(0, 0, 4096, _p(trace, ctypes.c_float))
        args = [_p(x, ctypes.c_float), ctypes.c_uint32(n), ctypes.c_uint32(d), ctypes.c_uint32(k)]
        args += [ctypes.c_uint32(e) for e in extra]
        args += [ctypes.c_int(METRICS[metric]), ctypes.c_uint32(seed), _p(ids, ctypes.c_uint32),
                 _p(dists, ctypes.c_float), _p(flags, ctypes.c_uint8), ctypes.byref(st)]
        return args, dict(ids=ids, dists=dists, flags=flags, trace=trace, st=st)

    def _finish(self, rc, out):
        if rc != 0:
            raise RuntimeError("oracle call failed: %d" % rc)
        st = out.pop("st")
        out["ncmps"] = int(st.ncmps)
        out["trace"] = out["trace"][: min(st.trace_len, 4096)].copy()
        return out

    def kgraph(self, x, k, seed, metric="l2"):
        args, out = self._graph(self.lib.nno_kgraph, x, k, seed, metric)
        return self._finish(self.lib.nno_kgraph(*args), out)

    def smerge(self, x, k, seed, metric="l2"):
        args, out = self._graph(self.lib.nno_smerge, x, k, seed, metric)
        return self._finish(self.lib.nno_smerge(*args), out)

    def jmerge(self, x, k, seed, metric="l2"):
        args, out = self._graph(self.lib.nno_jmerge, x, k, seed, metric)
        return self._finish(self.lib.nno_jmerge(*args), out)

    def hmerge(self, x, k, m, seed, metric="l2"):
        args, out = self._graph(self.lib.nno_hmerge, x, k, seed, metric, extra=(m,))
        lay = Layers()
        rc = self.lib.nno_hmerge(*args, ctypes.byref(lay))
        out = self._finish(rc, out)
        layers = []
        for g in range(lay.nlayers):
            nr = lay.nrows[g]
            off = np.ctypeslib.as_array(lay.off[g], shape=(nr + 1,)).copy()
            adj = np.ctypeslib.as_array(lay.adj[g], shape=(max(int(off[-1]), 1),))[: int(off[-1])].copy()
            layers.append((off, adj))
        self.lib.nno_free_layers(ctypes.byref(lay))
        out["layers"] = layers
        return out

    def search(self, x, layers, q, topk, seed, metric="l2"):
        x = np.ascontiguousarray(x, dtype=np.float32)
        q = np.ascontiguousarray(q, dtype=np.float32)
        lay = Layers()
        lay.nlayers = len(layers)
        keep = []
        for g, (off, adj) in enumerate(layers):
            off = np.ascontiguousarray(off, np.uint64)
            adj = np.ascontiguousarray(adj if len(adj) else np.zeros(1, np.uint32), np.uint32)
            keep += [off, adj]
            lay.nrows[g] = len(off) - 1
            lay.off[g] = _p(off, ctypes.c_uint64)
            lay.adj[g] = _p(adj, ctypes.c_uint32)
        nq = q.shape[0]
        ids = np.zeros((nq, topk), np.uint32)
        ds = np.zeros((nq, topk), np.float32)
        nc = ctypes.c_uint64(0)
        ent = ctypes.c_uint32(0)
        rc = self.lib.nno_search(_p(x, ctypes.c_float), ctypes.c_uint32(x.shape[0]),
                                 ctypes.c_uint32(x.shape[1]), ctypes.byref(lay),
                                 _p(q, ctypes.c_float), ctypes.c_uint32(nq), ctypes.c_uint32(topk),
                                 ctypes.c_int(METRICS[metric]), ctypes.c_uint32(seed),
                                 _p(ids, ctypes.c_uint32), _p(ds, ctypes.c_float),
                                 ctypes.byref(nc), ctypes.byref(ent))
        if rc:
            raise RuntimeError("oracle search failed")
        return dict(ids=ids, dists=ds, ncmps=int(nc.value), entry=int(ent.value))

    def search_ex(self, x, layers, q, out_k, seed, beams=None, beam=None, probes=None, g0=0, flat=False,
                  metric="l2"):
        """Serving form: per-query beams, the first out_k results, optional
        learned entries (probes: nq x P rows of layer g0) or the reference's
        flat search (random seeds on the last layer, no descent)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        q = np.ascontiguousarray(q, dtype=np.float32)
        lay = Layers()
        lay.nlayers = len(layers)
        keep = []
        for g, (off, adj) in enumerate(layers):
            off = np.ascontiguousarray(off, np.uint64)
            adj = np.ascontiguousarray(adj if len(adj) else np.zeros(1, np.uint32), np.uint32)
            keep += [off, adj]
            lay.nrows[g] = len(off) - 1
            lay.off[g] = _p(off, ctypes.c_uint64)
            lay.adj[g] = _p(adj, ctypes.c_uint32)
        nq = q.shape[0]
        b = None if beams is None else np.ascontiguousarray(beams, np.uint32)
        pr = None if probes is None else np.ascontiguousarray(probes, np.uint32)
        if beam is None:
            beam = out_k if b is None else int(b.max())
        ids = np.zeros((nq, out_k), np.uint32)
        ds = np.zeros((nq, out_k), np.float32)
        nc = ctypes.c_uint64(0)
        ent = ctypes.c_uint32(0)
        nul = ctypes.POINTER(ctypes.c_uint32)()
        rc = self.lib.nno_search_ex(_p(x, ctypes.c_float), ctypes.c_uint32(x.shape[0]),
                                    ctypes.c_uint32(x.shape[1]), ctypes.byref(lay),
                                    _p(q, ctypes.c_float), ctypes.c_uint32(nq),
                                    nul if b is None else _p(b, ctypes.c_uint32), ctypes.c_uint32(beam),
                                    ctypes.c_uint32(out_k), nul if pr is None else _p(pr, ctypes.c_uint32),
                                    ctypes.c_uint32(0 if pr is None else pr.shape[1]), ctypes.c_uint32(g0),
                                    ctypes.c_int(1 if flat else 0), ctypes.c_int(METRICS[metric]),
                                    ctypes.c_uint32(seed),
                                    _p(ids, ctypes.c_uint32), _p(ds, ctypes.c_float),
                                    ctypes.byref(nc), ctypes.byref(ent))
        if rc:
            raise RuntimeError("oracle search failed")
        return dict(ids=ids, dists=ds, ncmps=int(nc.value), entry=int(ent.value))

    def glibc_rand(self, seed, count):
        out = np.zeros(count, np.int32)
        self.lib.nno_glibc_rand(ctypes.c_uint32(seed), ctypes.c_uint32(count), _p(out, ctypes.c_int32))
        return out

    def mt19937(self, seed, count):
        out = np.zeros(count, np.uint32)
        self.lib.nno_mt19937(ctypes.c_uint32(seed), ctypes.c_uint32(count), _p(out, ctypes.c_uint32))
        return out

    def rnd_seeds(self, seed, rows, k, n):
        out = np.zeros((rows, k), np.uint32)
        self.lib.nno_rnd_seeds(ctypes.c_uint32(seed), ctypes.c_uint32(rows), ctypes.c_uint32(k),
                               ctypes.c_uint32(n), _p(out, ctypes.c_uint32))
        return out

    def dist(self, x, i, j, metric="l2"):
        """The reference's distance of rows i and j of x (its sequential float sum)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        self.lib.nno_dist.restype = ctypes.c_float
        return self.lib.nno_dist(_p(x, ctypes.c_float), ctypes.c_uint64(i), _p(x, ctypes.c_float),
                                 ctypes.c_uint64(j), ctypes.c_uint32(x.shape[1]), ctypes.c_int(METRICS[metric]))

    def sort_pool(self, ids, dists, flags):
        ids = np.ascontiguousarray(ids, np.uint32).copy()
        dists = np.ascontiguousarray(dists, np.float32).copy()
        flags = np.ascontiguousarray(flags, np.uint8).copy()
        self.lib.nno_sort_pool(_p(ids, ctypes.c_uint32), _p(dists, ctypes.c_float),
                               _p(flags, ctypes.c_uint8), ctypes.c_uint32(len(ids)))
        return ids, dists, flags


def ref_available():
    return os.path.exists(REF_BIN)


def write_mat(path, x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    with open(path, "wb") as f:
        f.write(struct.pack("<II", *x.shape))
        f.write(x.tobytes())


def read_graph(path):
    b = open(path, "rb").read()
    n, k = struct.unpack("<II", b[:8])
    off = 8
    ids = np.frombuffer(b, np.uint32, n * k, off).reshape(n, k).copy(); off += 4 * n * k
    dists = np.frombuffer(b, np.float32, n * k, off).reshape(n, k).copy(); off += 4 * n * k
    flags = np.frombuffer(b, np.uint8, n * k, off).reshape(n, k).copy(); off += n * k
    ncmps, = struct.unpack("<Q", b[off:off + 8]); off += 8
    t, = struct.unpack("<I", b[off:off + 4]); off += 4
    trace = np.frombuffer(b, np.float32, t, off).copy()
    return dict(ids=ids, dists=dists, flags=flags, ncmps=ncmps, trace=trace)


def read_layers_text(path):
    """Parses the H-Merge hierarchy text file (lynndescent.cpp:625-638 per
    layer, read back by lysearch.cpp:112-186) into (offsets, ids) per layer."""
    toks = open(path).read().split()
    pos = 0
    layers = []
    while pos < len(toks):
        rows = int(toks[pos]); pos += 1
        off = np.zeros(rows + 1, np.uint64)
        adj = []
        for i in range(rows):
            _idx, num = int(toks[pos]), int(toks[pos + 1]); pos += 2
            adj.extend(int(t) for t in toks[pos:pos + num]); pos += num
            off[i + 1] = off[i] + num
        layers.append((off, np.array(adj, np.uint32)))
    return layers


def run_ref(cmd, x, k, seed, tmpdir, metric="l2", m=None, layers_txt=None, queries=None, topk=None):
    """Runs the compiled reference; returns its outputs as numpy arrays."""
    mat = os.path.join(tmpdir, "in.mat")
    write_mat(mat, x)
    out = os.path.join(tmpdir, "out.bin")
    if cmd in ("kgraph", "smerge", "jmerge"):
        argv = [REF_BIN, cmd, metric, mat, str(k), str(seed), out]
    elif cmd == "hmerge":
        prefix = os.path.join(tmpdir, "hier")
        argv = [REF_BIN, cmd, metric, mat, str(k), str(m), str(seed), out, prefix]
    else:
        qp = os.path.join(tmpdir, "q.mat")
        write_mat(qp, queries)
        argv = [REF_BIN, cmd, metric, mat, layers_txt, qp, str(topk), str(seed), out]
    r = subprocess.run(argv, capture_output=True, text=True, cwd=tmpdir)
    if r.returncode != 0:
        raise RuntimeError("reference failed: %s %s" % (r.stdout[-2000:], r.stderr[-2000:]))
    if cmd in ("search", "flatsearch"):
        b = open(out, "rb").read()
        nq, tk, entry = struct.unpack("<III", b[:12])
        nc, = struct.unpack("<Q", b[12:20])
        ids = np.frombuffer(b, np.uint32, nq * tk, 20).reshape(nq, tk).copy()
        ds = np.frombuffer(b, np.float32, nq * tk, 20 + 4 * nq * tk).reshape(nq, tk).copy()
        return dict(ids=ids, dists=ds, ncmps=nc, entry=entry)
    res = read_graph(out)
    if cmd == "hmerge":
        res["layers"] = read_layers_text(os.path.join(tmpdir, "hier.txt"))
    return res
