"""nnm_search_noalloc: the search entry point for callers that cannot
allocate device memory (a pool owned by another framework, a fixed serving
budget, a latency path that must avoid cudaMalloc's synchronisation).

Called through the C ABI with every input and output already in device
memory, it must return exactly what nnm_search returns, on two calls in a
row (its scratch array keeps the previous call's contents).  This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import golden_lib
import nnm
from nnm import _lib

pytestmark = pytest.mark.gpu


class DevLayers(ctypes.Structure):
    _fields_ = [("nlayers", ctypes.c_uint32), ("nrows", ctypes.c_uint32 * 16),
                ("off", ctypes.c_void_p * 16), ("adj", ctypes.c_void_p * 16)]


def test_noalloc_search_matches_search():
    import torch
    lib = nnm.load()
    lib.nnm_search_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
    fx = golden_lib.load("hmerge_search")
    x, q, seed = fx["x"], fx["q"], fx["seed"]
    ctx = nnm.Context(0)
    try:
        x_d = torch.from_numpy(x).cuda()
        q_d = torch.from_numpy(q).cuda()
        lay = DevLayers()
        lay.nlayers = len(fx["layers"])
        keep = []
        for g, (off, adj) in enumerate(fx["layers"]):
            o = torch.from_numpy(off.astype(np.int64)).cuda()
            a = torch.from_numpy(adj.astype(np.int32)).cuda()
            keep += [o, a]
            lay.nrows[g] = len(off) - 1
            lay.off[g] = o.data_ptr()
            lay.adj[g] = a.data_ptr()
        for topk in (10, 40):
            exp = ctx.search(x, fx["layers"], q, topk, seed=seed)
            for call in range(2):  # the second call reuses the scratch left by the first
                ids = torch.full((len(q), topk), -7, dtype=torch.int32, device="cuda")
                ds = torch.zeros((len(q), topk), dtype=torch.float32, device="cuda")
                nc = ctypes.c_uint64(0)
                rc = lib.nnm_search_noalloc(x_d.data_ptr(), x.shape[0], x.shape[1], ctypes.byref(lay),
                                            q_d.data_ptr(), len(q), topk, seed, 0, ids.data_ptr(), ds.data_ptr(),
                                            ctypes.byref(nc), None)
                assert rc == 0, lib.nnm_status_string(rc)
                got_ids = ids.cpu().numpy().view(np.uint32)
                assert np.array_equal(got_ids, exp["ids"]), (topk, call)
                assert np.array_equal(ds.cpu().numpy(), exp["dists"]), (topk, call)
                assert nc.value == exp["ncmps"], (topk, call)
        # sizes beyond the stated maximum are rejected before any device work
        lay.nrows[lay.nlayers - 1] = (1 << 20) + 1
        ids = torch.empty((len(q), 10), dtype=torch.int32, device="cuda")
        rc = lib.nnm_search_noalloc(x_d.data_ptr(), (1 << 20) + 1, x.shape[1], ctypes.byref(lay), q_d.data_ptr(),
                                    len(q), 10, seed, 0, ids.data_ptr(), None, None, None)
        assert rc == 1
    finally:
        ctx.close()
