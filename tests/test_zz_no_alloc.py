"""nnm_search_noalloc: the search entry point for callers that cannot
allocate device memory (a pool owned by another framework, a fixed serving
budget, a latency path that must avoid cudaMalloc's synchronisation).

Called through the C ABI with every input and output already in device
memory, it must return exactly what nnm_search returns -- and, for the
reference's metric, what the reference itself returned on the golden
hierarchy -- on two calls in a row (its scratch array keeps the previous
call's contents), without the device's free memory changing.  This file is
collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import golden_lib
import nnm

pytestmark = pytest.mark.gpu


class DevLayers(ctypes.Structure):
    _fields_ = [("nlayers", ctypes.c_uint32), ("nrows", ctypes.c_uint32 * 16),
                ("off", ctypes.c_void_p * 16), ("adj", ctypes.c_void_p * 16)]


METRIC_IDS = {"l2": 0, "l1": 1, "chi2": 2}


def bind():
    lib = nnm.load()
    lib.nnm_search_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
    return lib


def device_layers(torch, layers):
    lay = DevLayers()
    lay.nlayers = len(layers)
    keep = []
    for g, (off, adj) in enumerate(layers):
        o = torch.from_numpy(off.astype(np.int64)).cuda()
        a = torch.from_numpy(adj.astype(np.int32)).cuda()
        keep += [o, a]
        lay.nrows[g] = len(off) - 1
        lay.off[g] = o.data_ptr()
        lay.adj[g] = a.data_ptr()
    return lay, keep


@pytest.mark.parametrize("metric", ["l2", "l1", "chi2"])
def test_noalloc_search_matches_search(metric):
    import torch
    lib = bind()
    fx = golden_lib.load("hmerge_search")
    x, q, seed = fx["x"], fx["q"], fx["seed"]
    ctx = nnm.Context(0)
    stream = torch.cuda.Stream()
    try:
        x_d = torch.from_numpy(x).cuda()
        q_d = torch.from_numpy(q).cuda()
        lay, keep = device_layers(torch, fx["layers"])
        for topk in (10, 40):
            exp = ctx.search(x, fx["layers"], q, topk, seed=seed, metric=metric)
            if metric == "l2":  # the reference's own output on this hierarchy
                assert np.array_equal(exp["ids"], fx["search%d_ids" % topk])
            ids = torch.full((len(q), topk), -7, dtype=torch.int32, device="cuda")
            ds = torch.zeros((len(q), topk), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            for call in range(2):  # the second call reuses the scratch left by the first
                free0 = torch.cuda.mem_get_info()[0]
                used0 = torch.cuda.memory_allocated()
                nc = ctypes.c_uint64(0)
                rc = lib.nnm_search_noalloc(x_d.data_ptr(), x.shape[0], x.shape[1], ctypes.byref(lay),
                                            q_d.data_ptr(), len(q), topk, seed, METRIC_IDS[metric],
                                            ids.data_ptr(), ds.data_ptr(), ctypes.byref(nc),
                                            ctypes.c_void_p(stream.cuda_stream))
                assert rc == 0, lib.nnm_status_string(rc)
                if call == 1:  # after the first call's one-time set-up, nothing is allocated
                    assert torch.cuda.mem_get_info()[0] == free0
                    assert torch.cuda.memory_allocated() == used0
                got_ids = ids.cpu().numpy().view(np.uint32)
                assert np.array_equal(got_ids, exp["ids"]), (topk, call)
                assert np.array_equal(ds.cpu().numpy(), exp["dists"]), (topk, call)
                assert nc.value == exp["ncmps"], (topk, call)
                if metric == "l2":
                    assert np.array_equal(got_ids, fx["search%d_ids" % topk])
                    assert nc.value == int(fx["search%d_ncmps" % topk])
                ids.fill_(-7)
                ds.zero_()
                torch.cuda.synchronize()
        del keep
    finally:
        ctx.close()


def test_noalloc_rejects_sizes_beyond_its_maximum():
    import torch
    lib = bind()
    fx = golden_lib.load("hmerge_search")
    x, q, seed = fx["x"], fx["q"], fx["seed"]
    x_d = torch.from_numpy(x).cuda()
    q_d = torch.from_numpy(q).cuda()
    lay, keep = device_layers(torch, fx["layers"])
    ids = torch.empty((len(q), 10), dtype=torch.int32, device="cuda")
    # last layer above 2^20 rows, topk above 1024, d above 4096: rejected before any device work
    lay.nrows[lay.nlayers - 1] = (1 << 20) + 1
    assert lib.nnm_search_noalloc(x_d.data_ptr(), (1 << 20) + 1, x.shape[1], ctypes.byref(lay), q_d.data_ptr(),
                                  len(q), 10, seed, 0, ids.data_ptr(), None, None, None) == 1
    lay.nrows[lay.nlayers - 1] = x.shape[0]
    assert lib.nnm_search_noalloc(x_d.data_ptr(), x.shape[0], x.shape[1], ctypes.byref(lay), q_d.data_ptr(),
                                  len(q), 1025, seed, 0, ids.data_ptr(), None, None, None) == 1
    assert lib.nnm_search_noalloc(x_d.data_ptr(), x.shape[0], 4097, ctypes.byref(lay), q_d.data_ptr(),
                                  len(q), 10, seed, 0, ids.data_ptr(), None, None, None) == 1
    del keep


def test_noalloc_after_a_failed_call():
    """A call that the kernel's own id checks fail (adjacency ids past the
    last layer) returns an error; the next call on well-formed layers still
    returns exactly nnm_search's result (the visited bitmaps are cleared only
    when a call may have left bits set, so this checks that a failed call
    leaves none)."""
    import torch
    lib = bind()
    fx = golden_lib.load("hmerge_search")
    x, q, seed = fx["x"], fx["q"], fx["seed"]
    ctx = nnm.Context(0)
    try:
        exp = ctx.search(x, fx["layers"], q, 10, seed=seed)
    finally:
        ctx.close()
    x_d = torch.from_numpy(x).cuda()
    q_d = torch.from_numpy(q).cuda()
    good, keep = device_layers(torch, fx["layers"])
    off, adj = fx["layers"][-1]
    nlast = len(off) - 1
    bad_adj = adj.astype(np.int64).copy()
    bad_adj[::7] = nlast + 3  # every 7th neighbour out of range: the kernel skips it and records the error
    bad, keep2 = device_layers(torch, fx["layers"][:-1] + [(off, bad_adj)])
    ids = torch.empty((len(q), 10), dtype=torch.int32, device="cuda")
    for lay, want_ok in ((good, True), (bad, False), (good, True), (bad, False), (bad, False), (good, True)):
        ids.fill_(-7)
        rc = lib.nnm_search_noalloc(x_d.data_ptr(), x.shape[0], x.shape[1], ctypes.byref(lay), q_d.data_ptr(),
                                    len(q), 10, seed, 0, ids.data_ptr(), None, None, None)
        if want_ok:
            assert rc == 0, lib.nnm_status_string(rc)
            assert np.array_equal(ids.cpu().numpy().view(np.uint32), exp["ids"])
        else:
            assert rc != 0
    del keep, keep2
