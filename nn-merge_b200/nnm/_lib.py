"""ctypes binding of the C ABI in include/nnm.h (lib/libnnm.so).

There is no fallback: if the shared library is missing or no CUDA device is
present, the calls raise.
"""
import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libnnm.so")

METRICS = {"l2": 0, "l1": 1, "chi2": 2}
EXPORTED = (
    "nnm_opts_default", "nnm_status_string", "nnm_last_error", "nnm_ctx_create", "nnm_ctx_destroy",
    "nnm_kgraph_build", "nnm_kgraph_build_dev", "nnm_smerge", "nnm_jmerge", "nnm_merge_leaves",
    "nnm_merge_leaves_dev", "nnm_hmerge_build", "nnm_layers_free", "nnm_search",
    "nnm_profile_enable", "nnm_profile_get", "nnm_launch_count",
    "nnm_train_opts_default", "nnm_mlp_train", "nnm_mlp_grad", "nnm_mlp_codes", "nnm_set_init_model",
    "nnm_merge_create", "nnm_merge_subgraph", "nnm_merge_init_sgraph", "nnm_merge_initial_graph",
    "nnm_merge_nndescent", "nnm_merge_merge2one", "nnm_merge_read", "nnm_merge_free",
    "nnm_build_leaves_dev", "nnm_merge_prebuilt_dev",
)
MLP_HIDDEN, MLP_OUT = 256, 32


class NnmError(RuntimeError):
    """A non-zero nnm_status from the library."""

    def __init__(self, status, message):
        super().__init__("nnm status %d: %s" % (status, message))
        self.status = status


class Opts(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint32), ("rng_mode", ctypes.c_uint32), ("metric", ctypes.c_uint32),
                ("sample_cap", ctypes.c_uint32), ("delta", ctypes.c_float), ("max_iter", ctypes.c_uint32),
                ("exact_trace", ctypes.c_uint32), ("join_kernel", ctypes.c_uint32),
                ("init", ctypes.c_uint32), ("audit", ctypes.c_uint32), ("merge_order", ctypes.c_uint32),
                ("no_graph", ctypes.c_uint32), ("tile_rows", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


class Mlp(ctypes.Structure):
    _fields_ = [("d_in", ctypes.c_uint32), ("in_scale", ctypes.c_float), ("in_shift", ctypes.c_float),
                ("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p), ("w2", ctypes.c_void_p), ("b2", ctypes.c_void_p)]


class TrainOpts(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint32), ("batch", ctypes.c_uint32), ("lr", ctypes.c_float),
                ("margin", ctypes.c_float), ("seed", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 7)]


def mlp_init(d, seed=0, in_scale=1.0 / 64.0, in_shift=-1.0):
    """A fresh code model (He-initialised weights, zero biases) as a dict of
    float32 arrays: w1 (256 x d), b1 (256), w2 (32 x 256), b2 (32)."""
    rng = np.random.default_rng(seed)
    return dict(w1=(rng.standard_normal((MLP_HIDDEN, d)) * np.sqrt(2.0 / d)).astype(np.float32),
                b1=np.zeros(MLP_HIDDEN, np.float32),
                w2=(rng.standard_normal((MLP_OUT, MLP_HIDDEN)) * np.sqrt(1.0 / MLP_HIDDEN)).astype(np.float32),
                b2=np.zeros(MLP_OUT, np.float32), in_scale=float(in_scale), in_shift=float(in_shift))


def _mlp_struct(m):
    """C view of a model dict; the dict's arrays must stay alive (and are
    made contiguous float32 in place)."""
    for k in ("w1", "b1", "w2", "b2"):
        m[k] = np.ascontiguousarray(m[k], np.float32)
    return Mlp(m["w1"].shape[1], m["in_scale"], m["in_shift"], m["w1"].ctypes.data, m["b1"].ctypes.data,
               m["w2"].ctypes.data, m["b2"].ctypes.data)


class EntryMlp(ctypes.Structure):
    _fields_ = [("d_in", ctypes.c_uint32), ("n_classes", ctypes.c_uint32), ("in_scale", ctypes.c_float),
                ("in_shift", ctypes.c_float), ("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p),
                ("w2", ctypes.c_void_p), ("b2", ctypes.c_void_p)]


class SearchStats(ctypes.Structure):
    _fields_ = [("ncmps", ctypes.c_uint64), ("expansions", ctypes.c_uint64), ("device_ms", ctypes.c_double),
                ("predict_ms", ctypes.c_double)]


def entry_init(d, n_classes, seed=0, in_scale=1.0 / 64.0, in_shift=-1.0):
    """A fresh entry-point network (He-initialised weights, zero biases) as a
    dict of float32 arrays: w1 (256 x d), b1 (256), w2 (C x 256), b2 (C)."""
    rng = np.random.default_rng(seed)
    return dict(w1=(rng.standard_normal((MLP_HIDDEN, d)) * np.sqrt(2.0 / d)).astype(np.float32),
                b1=np.zeros(MLP_HIDDEN, np.float32),
                w2=(rng.standard_normal((n_classes, MLP_HIDDEN)) * np.sqrt(1.0 / MLP_HIDDEN)).astype(np.float32),
                b2=np.zeros(n_classes, np.float32), in_scale=float(in_scale), in_shift=float(in_shift))


def _entry_struct(m):
    for k in ("w1", "b1", "w2", "b2"):
        m[k] = np.ascontiguousarray(m[k], np.float32)
    return EntryMlp(m["w1"].shape[1], m["w2"].shape[0], m["in_scale"], m["in_shift"], m["w1"].ctypes.data,
                    m["b1"].ctypes.data, m["w2"].ctypes.data, m["b2"].ctypes.data)


class TuneOpts(ctypes.Structure):
    _fields_ = [("target_recall", ctypes.c_float), ("margin", ctypes.c_float), ("sample_rows", ctypes.c_uint32),
                ("eval_rows", ctypes.c_uint32), ("repeats", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 7)]


class TuneTrial(ctypes.Structure):
    _fields_ = [("sample_cap", ctypes.c_uint32), ("delta", ctypes.c_float), ("recall", ctypes.c_float),
                ("tile_rows", ctypes.c_uint32), ("ms", ctypes.c_double)]


class TuneResult(ctypes.Structure):
    _fields_ = [("ntrials", ctypes.c_uint32), ("chosen", ctypes.c_uint32), ("trials", TuneTrial * 32)]


class Stats(ctypes.Structure):
    _fields_ = [("ncmps", ctypes.c_uint64), ("sub_ncmps", ctypes.c_uint64), ("iterations", ctypes.c_uint32),
                ("n_trace", ctypes.c_uint32), ("trace", ctypes.c_float * 256), ("device_ms", ctypes.c_double)]


class Layers(ctypes.Structure):
    _fields_ = [("nlayers", ctypes.c_uint32), ("nrows", ctypes.c_uint32 * 16),
                ("off", ctypes.POINTER(ctypes.c_uint64) * 16), ("adj", ctypes.POINTER(ctypes.c_uint32) * 16)]


_lib = None


def load():
    """Loads lib/libnnm.so once; raises if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("nnm: %s not built (run make -C nn-merge_b200)" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        lib.nnm_status_string.restype = ctypes.c_char_p
        lib.nnm_last_error.restype = ctypes.c_char_p
        lib.nnm_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        lib.nnm_ctx_destroy.argtypes = [ctypes.c_void_p]
        lib.nnm_last_error.argtypes = [ctypes.c_void_p]
        vp, u64, u32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32
        build_args = [vp, vp, u64, u32, u32, vp, vp, vp, vp, vp]
        for name in ("nnm_kgraph_build", "nnm_kgraph_build_dev", "nnm_smerge", "nnm_jmerge"):
            getattr(lib, name).argtypes = build_args
        for name in ("nnm_merge_leaves", "nnm_merge_leaves_dev"):
            getattr(lib, name).argtypes = [vp, vp, u64, u32, u32, vp, u32, vp, vp, vp, vp, vp]
        lib.nnm_hmerge_build.argtypes = [vp, vp, u64, u32, u32, u32, vp, vp, vp, vp, vp, vp]
        lib.nnm_layers_free.argtypes = [vp]
        lib.nnm_search.argtypes = [vp, vp, u64, u32, vp, vp, u64, u32, vp, vp, vp, vp]
        lib.nnm_profile_enable.argtypes = [vp, ctypes.c_int]
        lib.nnm_profile_get.argtypes = [vp, ctypes.c_char_p, u64]
        lib.nnm_launch_count.restype = ctypes.c_uint64
        lib.nnm_train_opts_default.argtypes = [vp]
        lib.nnm_mlp_train.argtypes = [vp, vp, u64, u32, vp, u32, vp, vp, vp]
        lib.nnm_mlp_grad.argtypes = [vp, vp, vp, u64, u32, vp, u32, ctypes.c_float, vp, vp]
        lib.nnm_mlp_codes.argtypes = [vp, vp, vp, u64, u32, vp, vp]
        lib.nnm_set_init_model.argtypes = [vp, vp]
        lib.nnm_graph_recall.argtypes = [vp, vp, u64, u32, vp, u32, vp, u32, u32, vp]
        lib.nnm_tune_opts_default.argtypes = [vp]
        lib.nnm_autotune_merge_leaves.argtypes = [vp, vp, u64, u32, u32, vp, u32, vp, vp, vp, vp]
        lib.nnm_index_create.argtypes = [vp, vp, u64, u32, vp, u32, u32, ctypes.POINTER(ctypes.c_void_p)]
        lib.nnm_index_free.argtypes = [vp]
        for name in ("nnm_index_search", "nnm_index_search_dev"):
            getattr(lib, name).argtypes = [vp, vp, u64, vp, u32, u32, u32, u32, vp, vp, vp]
        lib.nnm_index_entry_layer.argtypes = [vp, vp, vp]
        lib.nnm_index_set_width.argtypes = [vp, u32]
        lib.nnm_index_tune_width.argtypes = [vp, vp, u64, vp, u32, u32, u32, u32, vp, vp]
        lib.nnm_entry_forward.argtypes = [vp, vp, vp, u64, u32, vp]
        lib.nnm_entry_probes.argtypes = [vp, vp, vp, u64, u32, u32, vp]
        lib.nnm_entry_grad.argtypes = [vp, vp, vp, u64, u32, vp, vp, vp]
        lib.nnm_entry_train.argtypes = [vp, vp, vp, vp]
        lib.nnm_index_set_entry_model.argtypes = [vp, vp, u32]
        lib.nnm_merge_create.argtypes = [vp, vp, u64, u32, u32, vp, ctypes.POINTER(ctypes.c_void_p)]
        lib.nnm_merge_subgraph.argtypes = [vp, u32, u32, vp, vp]
        lib.nnm_merge_init_sgraph.argtypes = [vp, u32, vp, u32, u32]
        lib.nnm_merge_initial_graph.argtypes = [vp, u32, u32]
        lib.nnm_merge_nndescent.argtypes = [vp, u32, u32, vp]
        lib.nnm_merge_merge2one.argtypes = [vp, u32]
        lib.nnm_merge_read.argtypes = [vp, vp, vp, vp]
        lib.nnm_merge_free.argtypes = [vp]
        lib.nnm_build_leaves_dev.argtypes = [vp, vp, u64, u32, u32, vp, u32, u32, vp, vp, vp, vp]
        lib.nnm_merge_prebuilt_dev.argtypes = [vp, vp, u64, u32, u32, vp, u32, vp, vp, vp, vp, vp, vp, vp]
        _lib = lib
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


RNG_MODES = {"exact": 0, "fast": 1}


JOIN_KERNELS = {"auto": 0, "fp32": 1, "tensor": 2, "bf16": 2, "fp8": 3}
INITS = {"random": 0, "learned": 1}


def make_opts(seed=0, metric="l2", sample_cap=100, delta=0.002, max_iter=0, exact_trace=False, rng="exact",
              join="auto", init="random", audit=False, merge_order="all", graph=True, tile_rows=0):
    lib = load()
    o = Opts()
    lib.nnm_opts_default(ctypes.byref(o))
    o.seed = seed
    o.rng_mode = RNG_MODES[rng]
    o.metric = METRICS[metric] if isinstance(metric, str) else int(metric)
    o.sample_cap = sample_cap
    o.delta = delta
    o.max_iter = max_iter
    o.exact_trace = 1 if exact_trace else 0
    o.join_kernel = JOIN_KERNELS[join]
    o.init = INITS[init]
    o.audit = 1 if audit else 0
    o.merge_order = {"all": 0, "tree": 1}[merge_order]
    o.no_graph = 0 if graph else 1
    o.tile_rows = tile_rows
    return o


def _stats_dict(st):
    return dict(ncmps=int(st.ncmps), sub_ncmps=int(st.sub_ncmps), iterations=int(st.iterations),
                trace=np.array(st.trace[: st.n_trace], np.float32), device_ms=float(st.device_ms))


class Context:
    """One CUDA device + stream (nnm_ctx)."""

    def __init__(self, device=0):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.nnm_ctx_create(device, ctypes.byref(h))
        if rc != 0:
            raise NnmError(rc, self.lib.nnm_status_string(rc).decode())
        self.h = h

    def close(self):
        if self.h:
            self.lib.nnm_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.nnm_last_error(self.h).decode()
            raise NnmError(rc, "%s: %s" % (self.lib.nnm_status_string(rc).decode(), msg))

    def _build(self, fn, x, k, opts, extra=()):
        x = np.ascontiguousarray(x, np.float32)
        n, d = x.shape
        ids = np.empty((n, k), np.uint32)
        dists = np.empty((n, k), np.float32)
        flags = np.empty((n, k), np.uint8)
        st = Stats()
        head = [self.h, _ptr(x), n, d, k]
        tail = [ctypes.byref(opts), _ptr(ids), _ptr(dists), _ptr(flags), ctypes.byref(st)]
        self._check(fn(*(head + list(extra) + tail)))
        return dict(ids=ids, dists=dists, flags=flags, **_stats_dict(st))

    def profile(self, on=True):
        self._check(self.lib.nnm_profile_enable(self.h, 1 if on else 0))

    def profile_stats(self):
        import json
        buf = ctypes.create_string_buffer(1 << 20)
        self._check(self.lib.nnm_profile_get(self.h, buf, 1 << 20))
        return json.loads(buf.value.decode())

    def launch_count(self):
        return int(self.lib.nnm_launch_count())

    # -- learned initialisation ------------------------------------------
    def mlp_train(self, x, graph, model, steps=400, batch=2048, lr=2e-3, margin=16.0, seed=0):
        """Trains `model` (dict from mlp_init) in place on triplets of the
        k-NN graph `graph` (n x k ids of x); returns the per-step losses."""
        x = np.ascontiguousarray(x, np.float32)
        graph = np.ascontiguousarray(graph, np.uint32)
        n, d = x.shape
        o = TrainOpts()
        self.lib.nnm_train_opts_default(ctypes.byref(o))
        o.steps, o.batch, o.lr, o.margin, o.seed = steps, batch, lr, margin, seed
        ms = _mlp_struct(model)
        loss = np.empty(steps, np.float32)
        self._check(self.lib.nnm_mlp_train(self.h, _ptr(x), n, d, _ptr(graph), graph.shape[1], ctypes.byref(o),
                                           ctypes.byref(ms), _ptr(loss)))
        return loss

    def mlp_grad(self, model, x, triplets, margin=16.0):
        """(loss, gradient dict) of the triplet loss over `triplets`
        (t x 3 row indices: anchor, positive, negative)."""
        x = np.ascontiguousarray(x, np.float32)
        tr = np.ascontiguousarray(triplets, np.uint32)
        n, d = x.shape
        grad = {k: np.zeros_like(np.asarray(model[k], np.float32)) for k in ("w1", "b1", "w2", "b2")}
        grad.update(in_scale=model["in_scale"], in_shift=model["in_shift"])
        ms, gs = _mlp_struct(model), _mlp_struct(grad)
        loss = ctypes.c_float()
        self._check(self.lib.nnm_mlp_grad(self.h, ctypes.byref(ms), _ptr(x), n, d, _ptr(tr), tr.shape[0], margin,
                                          ctypes.byref(loss), ctypes.byref(gs)))
        return float(loss.value), grad

    def mlp_codes(self, model, x, want_z=False):
        x = np.ascontiguousarray(x, np.float32)
        n, d = x.shape
        codes = np.empty(n, np.uint32)
        z = np.empty((n, MLP_OUT), np.float32) if want_z else None
        ms = _mlp_struct(model)
        self._check(self.lib.nnm_mlp_codes(self.h, ctypes.byref(ms), _ptr(x), n, d, _ptr(codes), _ptr(z)))
        return (codes, z) if want_z else codes

    def set_init_model(self, model):
        """The model init="learned" builds use (None clears it)."""
        if model is None:
            self._check(self.lib.nnm_set_init_model(self.h, None))
            return
        ms = _mlp_struct(model)
        self._check(self.lib.nnm_set_init_model(self.h, ctypes.byref(ms)))

    def merge_leaves_dev(self, x_ptr, n, d, k, leaf_sizes, ids_ptr=0, dists_ptr=0, flags_ptr=0, **kw):
        """Device-pointer build (inputs resident in HBM, outputs on the device)."""
        sizes = np.ascontiguousarray(leaf_sizes, np.uint32)
        st = Stats()
        o = make_opts(**kw)
        self._check(self.lib.nnm_merge_leaves_dev(self.h, ctypes.c_void_p(x_ptr), n, d, k, _ptr(sizes), len(sizes),
                                                  ctypes.byref(o), ctypes.c_void_p(ids_ptr),
                                                  ctypes.c_void_p(dists_ptr), ctypes.c_void_p(flags_ptr),
                                                  ctypes.byref(st)))
        return _stats_dict(st)

    def build_leaves_dev(self, x_ptr, n, d, k, leaf_sizes, ids_ptr, dists_ptr, leaf0=0, **kw):
        """The leaf builds of merge_leaves_dev alone (fast tier): ids local
        to the rows at x_ptr; leaf0 = index of the first leaf in the build."""
        sizes = np.ascontiguousarray(leaf_sizes, np.uint32)
        st = Stats()
        o = make_opts(**kw)
        self._check(self.lib.nnm_build_leaves_dev(self.h, ctypes.c_void_p(x_ptr), n, d, k, _ptr(sizes), len(sizes),
                                                  leaf0, ctypes.byref(o), ctypes.c_void_p(ids_ptr),
                                                  ctypes.c_void_p(dists_ptr), ctypes.byref(st)))
        return _stats_dict(st)

    def merge_prebuilt_dev(self, x_ptr, n, d, k, leaf_sizes, ids_in_ptr, dists_in_ptr, ids_ptr, dists_ptr,
                           flags_ptr=0, **kw):
        """The merge of merge_leaves_dev over leaves whose graphs are given."""
        sizes = np.ascontiguousarray(leaf_sizes, np.uint32)
        st = Stats()
        o = make_opts(**kw)
        self._check(self.lib.nnm_merge_prebuilt_dev(self.h, ctypes.c_void_p(x_ptr), n, d, k, _ptr(sizes), len(sizes),
                                                    ctypes.byref(o), ctypes.c_void_p(ids_in_ptr),
                                                    ctypes.c_void_p(dists_in_ptr), ctypes.c_void_p(ids_ptr),
                                                    ctypes.c_void_p(dists_ptr), ctypes.c_void_p(flags_ptr),
                                                    ctypes.byref(st)))
        return _stats_dict(st)

    def merge_leaves_into(self, x, k, leaf_sizes, ids, dists=None, flags=None, **kw):
        """Host-pointer build writing into caller-provided (e.g. pinned) arrays."""
        sizes = np.ascontiguousarray(leaf_sizes, np.uint32)
        st = Stats()
        o = make_opts(**kw)
        self._check(self.lib.nnm_merge_leaves(self.h, _ptr(x), x.shape[0], x.shape[1], k, _ptr(sizes), len(sizes),
                                              ctypes.byref(o), _ptr(ids), _ptr(dists), _ptr(flags),
                                              ctypes.byref(st)))
        return _stats_dict(st)

    def kgraph(self, x, k, **kw):
        return self._build(self.lib.nnm_kgraph_build, x, k, make_opts(**kw))

    def smerge(self, x, k, **kw):
        return self._build(self.lib.nnm_smerge, x, k, make_opts(**kw))

    def jmerge(self, x, k, **kw):
        return self._build(self.lib.nnm_jmerge, x, k, make_opts(**kw))

    def merge_leaves(self, x, k, leaf_sizes, **kw):
        sizes = np.ascontiguousarray(leaf_sizes, np.uint32)
        return self._build(self.lib.nnm_merge_leaves, x, k, make_opts(**kw), extra=(_ptr(sizes), len(sizes)))

    def hmerge(self, x, k, m, **kw):
        x = np.ascontiguousarray(x, np.float32)
        n, d = x.shape
        ids = np.empty((n, k), np.uint32)
        dists = np.empty((n, k), np.float32)
        flags = np.empty((n, k), np.uint8)
        st = Stats()
        lay = Layers()
        o = make_opts(**kw)
        self._check(self.lib.nnm_hmerge_build(self.h, _ptr(x), n, d, k, m, ctypes.byref(o), _ptr(ids),
                                              _ptr(dists), _ptr(flags), ctypes.byref(lay), ctypes.byref(st)))
        layers = []
        for g in range(lay.nlayers):
            nr = lay.nrows[g]
            off = np.ctypeslib.as_array(lay.off[g], shape=(nr + 1,)).copy()
            tot = int(off[-1])
            adj = np.ctypeslib.as_array(lay.adj[g], shape=(max(tot, 1),))[:tot].copy()
            layers.append((off, adj))
        self.lib.nnm_layers_free(ctypes.byref(lay))
        return dict(ids=ids, dists=dists, flags=flags, layers=layers, **_stats_dict(st))

    def merge_session(self, x, k, **kw):
        """A staged merge (nnm_merge_*): AbstractMerge's steps as calls."""
        return Merge(self, x, k, **kw)

    def search(self, x, layers, q, topk, seed=0, metric="l2"):
        x = np.ascontiguousarray(x, np.float32)
        q = np.ascontiguousarray(q, np.float32)
        lay, keep = _layers_struct(layers)
        nq = q.shape[0]
        ids = np.empty((nq, topk), np.uint32)
        ds = np.empty((nq, topk), np.float32)
        nc = ctypes.c_uint64(0)
        o = make_opts(seed=seed, metric=metric)
        self._check(self.lib.nnm_search(self.h, _ptr(x), x.shape[0], x.shape[1], ctypes.byref(lay), _ptr(q), nq,
                                        topk, ctypes.byref(o), _ptr(ids), _ptr(ds), ctypes.byref(nc)))
        return dict(ids=ids, dists=ds, ncmps=int(nc.value))

    # -- evaluation and tuning -----------------------------------------------
    def graph_recall(self, x, ids, rows, atop=10):
        """Recall@atop of the graph `ids` (n x k) on the listed rows against
        exact brute force on the device (ties at the atop-th distance count)."""
        x = np.ascontiguousarray(x, np.float32)
        ids = np.ascontiguousarray(ids, np.uint32)
        rows = np.ascontiguousarray(rows, np.uint32)
        r = ctypes.c_double()
        self._check(self.lib.nnm_graph_recall(self.h, _ptr(x), x.shape[0], x.shape[1], _ptr(ids), ids.shape[1],
                                              _ptr(rows), len(rows), atop, ctypes.byref(r)))
        return float(r.value)

    def autotune_merge_leaves_dev(self, x_ptr, n, d, k, leaf_sizes, target_recall=0.95, margin=0.005,
                                  sample_rows=200_000, eval_rows=1000, repeats=2, **kw):
        """Chooses sample_cap and delta for nnm_merge_leaves_dev on the
        device-resident x; returns (options for merge_leaves*, trials)."""
        sizes = np.ascontiguousarray(leaf_sizes, np.uint32)
        o = make_opts(**kw)
        t = TuneOpts()
        self.lib.nnm_tune_opts_default(ctypes.byref(t))
        t.target_recall, t.margin, t.sample_rows, t.eval_rows, t.repeats = (target_recall, margin, sample_rows,
                                                                           eval_rows, repeats)
        tuned = Opts()
        res = TuneResult()
        self._check(self.lib.nnm_autotune_merge_leaves(self.h, ctypes.c_void_p(x_ptr), n, d, k, _ptr(sizes),
                                                       len(sizes), ctypes.byref(o), ctypes.byref(t),
                                                       ctypes.byref(tuned), ctypes.byref(res)))
        trials = [dict(sample_cap=int(res.trials[i].sample_cap), delta=float(res.trials[i].delta),
                       recall=float(res.trials[i].recall), tile_rows=int(res.trials[i].tile_rows),
                       ms=float(res.trials[i].ms)) for i in range(res.ntrials)]
        chosen = trials[res.chosen]
        return dict(sample_cap=chosen["sample_cap"], delta=chosen["delta"], tile_rows=chosen["tile_rows"]), trials

    # -- serving ------------------------------------------------------------
    def index(self, x, layers, seed=0, metric="l2"):
        """A resident search index over x and its hierarchy (list of (off, adj))."""
        return Index(self, x, layers, seed, metric)

    def entry_forward(self, model, x):
        x = np.ascontiguousarray(x, np.float32)
        n, d = x.shape
        ms = _entry_struct(model)
        s = np.empty((n, ms.n_classes), np.float32)
        self._check(self.lib.nnm_entry_forward(self.h, ctypes.byref(ms), _ptr(x), n, d, _ptr(s)))
        return s

    def entry_probes(self, model, x, probes=4):
        """The probes a learned search takes for the rows of x (n x probes)."""
        x = np.ascontiguousarray(x, np.float32)
        n, d = x.shape
        ms = _entry_struct(model)
        out = np.empty((n, probes), np.uint32)
        self._check(self.lib.nnm_entry_probes(self.h, ctypes.byref(ms), _ptr(x), n, d, probes, _ptr(out)))
        return out

    def entry_grad(self, model, x, labels):
        x = np.ascontiguousarray(x, np.float32)
        lab = np.ascontiguousarray(labels, np.uint32)
        n, d = x.shape
        grad = {k: np.zeros_like(np.asarray(model[k], np.float32)) for k in ("w1", "b1", "w2", "b2")}
        grad.update(in_scale=model["in_scale"], in_shift=model["in_shift"])
        ms, gs = _entry_struct(model), _entry_struct(grad)
        loss = ctypes.c_float()
        self._check(self.lib.nnm_entry_grad(self.h, ctypes.byref(ms), _ptr(x), n, d, _ptr(lab), ctypes.byref(loss),
                                            ctypes.byref(gs)))
        return float(loss.value), grad


MERGE_KINDS = {"smerge": 1, "jmerge": 2}


class Merge:
    """AbstractMerge (abstractmerge.h:16-40) step by step on the device:
    InitialMemory at construction, then subgraph (KGraph::buildKGraph on a
    row range, continuing the merge's std::rand() stream), init_sgraph
    (InitSGraph), initial_graph (Smerge/Jmerge::InitialGraph), nndescent
    (nnDescent with that class's localJoin), merge2one and read (the
    pools).  Reference streams only."""

    def __init__(self, ctx, x, k, **kw):
        self.ctx, self.k = ctx, k
        x = np.ascontiguousarray(x, np.float32)
        self.n, self.d = x.shape
        self.h = ctypes.c_void_p()
        o = make_opts(**kw)
        ctx._check(ctx.lib.nnm_merge_create(ctx.h, _ptr(x), self.n, self.d, k, ctypes.byref(o), ctypes.byref(self.h)))

    def close(self):
        if self.h:
            self.ctx.lib.nnm_merge_free(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def subgraph(self, b, e):
        g = np.empty((e - b, self.k), np.uint32)
        c = ctypes.c_uint64()
        self.ctx._check(self.ctx.lib.nnm_merge_subgraph(self.h, b, e, _ptr(g), ctypes.byref(c)))
        return g, int(c.value)

    def init_sgraph(self, b, graph, gid):
        graph = np.ascontiguousarray(graph, np.uint32)
        self.ctx._check(self.ctx.lib.nnm_merge_init_sgraph(self.h, b, _ptr(graph), gid, graph.shape[0]))

    def initial_graph(self, kind, pre):
        self.ctx._check(self.ctx.lib.nnm_merge_initial_graph(self.h, MERGE_KINDS[kind], pre))

    def nndescent(self, kind, pre):
        st = Stats()
        self.ctx._check(self.ctx.lib.nnm_merge_nndescent(self.h, MERGE_KINDS[kind], pre, ctypes.byref(st)))
        return _stats_dict(st)

    def merge2one(self, sz):
        self.ctx._check(self.ctx.lib.nnm_merge_merge2one(self.h, sz))

    def read(self):
        ids = np.empty((self.n, self.k), np.uint32)
        dists = np.empty((self.n, self.k), np.float32)
        flags = np.empty((self.n, self.k), np.uint8)
        self.ctx._check(self.ctx.lib.nnm_merge_read(self.h, _ptr(ids), _ptr(dists), _ptr(flags)))
        return dict(ids=ids, dists=dists, flags=flags)


def _layers_struct(layers):
    lay = Layers()
    lay.nlayers = len(layers)
    keep = []
    for g, (off, adj) in enumerate(layers):
        off = np.ascontiguousarray(off, np.uint64)
        adj = np.ascontiguousarray(adj if len(adj) else np.zeros(1, np.uint32), np.uint32)
        keep += [off, adj]
        lay.nrows[g] = len(off) - 1
        lay.off[g] = off.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
        lay.adj[g] = adj.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    return lay, keep


SERVE_MODES = {"exact": 0, "fast": 1}
ENTRY_MODES = {"default": 0, "learned": 1, "flat": 2}


class Index:
    """nnm_index: vectors and hierarchy resident on the device, batched
    LySearch with per-query beam widths and default or learned entries."""

    def __init__(self, ctx, x, layers, seed=0, metric="l2"):
        self.ctx = ctx
        x = np.ascontiguousarray(x, np.float32)
        self.n, self.d = x.shape
        lay, keep = _layers_struct(layers)
        h = ctypes.c_void_p()
        ctx._check(ctx.lib.nnm_index_create(ctx.h, _ptr(x), self.n, self.d, ctypes.byref(lay), seed,
                                            METRICS[metric], ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.ctx.lib.nnm_index_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def search(self, q, out_k=10, beams=None, beam=None, mode="fast", entry="default"):
        q = np.ascontiguousarray(q, np.float32)
        nq = q.shape[0]
        b = None if beams is None else np.ascontiguousarray(beams, np.uint32)
        if beam is None:
            beam = out_k if b is None else int(b.max())
        ids = np.empty((nq, out_k), np.uint32)
        ds = np.empty((nq, out_k), np.float32)
        st = SearchStats()
        self.ctx._check(self.ctx.lib.nnm_index_search(self.h, _ptr(q), nq, _ptr(b), beam, out_k, SERVE_MODES[mode],
                                                      ENTRY_MODES[entry], _ptr(ids), _ptr(ds), ctypes.byref(st)))
        return dict(ids=ids, dists=ds, ncmps=int(st.ncmps), expansions=int(st.expansions),
                    device_ms=float(st.device_ms), predict_ms=float(st.predict_ms))

    def search_dev(self, q_ptr, nq, out_ids_ptr, out_d_ptr, out_k, beams_ptr=0, beam=None, mode="fast",
                   entry="default"):
        """Device-pointer form: q (nq x d float32), beams (nq uint32, `beam`
        >= every width), out_ids / out_d (nq x out_k)."""
        st = SearchStats()
        self.ctx._check(self.ctx.lib.nnm_index_search_dev(self.h, ctypes.c_void_p(q_ptr), nq,
                                                          ctypes.c_void_p(beams_ptr), beam, out_k, SERVE_MODES[mode],
                                                          ENTRY_MODES[entry], ctypes.c_void_p(out_ids_ptr),
                                                          ctypes.c_void_p(out_d_ptr), ctypes.byref(st)))
        return dict(ncmps=int(st.ncmps), expansions=int(st.expansions), device_ms=float(st.device_ms),
                    predict_ms=float(st.predict_ms))

    def set_width(self, width):
        self.ctx._check(self.ctx.lib.nnm_index_set_width(self.h, width))

    def tune_width(self, q, out_k=10, beams=None, beam=None, entry="default", repeats=2):
        """Times the fast kernel at widths 1..4 on these queries, keeps the
        fastest; returns (width, ms per width)."""
        q = np.ascontiguousarray(q, np.float32)
        b = None if beams is None else np.ascontiguousarray(beams, np.uint32)
        if beam is None:
            beam = out_k if b is None else int(b.max())
        w = ctypes.c_uint32()
        ms = np.zeros(4, np.float64)
        self.ctx._check(self.ctx.lib.nnm_index_tune_width(self.h, _ptr(q), q.shape[0], _ptr(b), beam, out_k,
                                                          ENTRY_MODES[entry], repeats, ctypes.byref(w), _ptr(ms)))
        return int(w.value), ms

    def entry_layer(self):
        layer, nc = ctypes.c_uint32(), ctypes.c_uint32()
        self.ctx._check(self.ctx.lib.nnm_index_entry_layer(self.h, ctypes.byref(layer), ctypes.byref(nc)))
        return int(layer.value), int(nc.value)

    def entry_train(self, model, steps=1000, batch=2048, lr=2e-3, seed=0):
        """Trains the entry network `model` (dict from entry_init) in place on
        the index's rows; returns the per-step losses."""
        o = TrainOpts()
        self.ctx.lib.nnm_train_opts_default(ctypes.byref(o))
        o.steps, o.batch, o.lr, o.seed = steps, batch, lr, seed
        ms = _entry_struct(model)
        loss = np.empty(steps, np.float32)
        self.ctx._check(self.ctx.lib.nnm_entry_train(self.h, ctypes.byref(ms), ctypes.byref(o), _ptr(loss)))
        return loss

    def set_entry_model(self, model, probes=4):
        if model is None:
            self.ctx._check(self.ctx.lib.nnm_index_set_entry_model(self.h, None, 0))
            return
        ms = _entry_struct(model)
        self.ctx._check(self.ctx.lib.nnm_index_set_entry_model(self.h, ctypes.byref(ms), probes))
