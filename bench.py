#!/usr/bin/env python
"""Headline benchmark: build time of a 1M x 128, k=20 k-NN graph.

Workload (one step = one complete build): 1,000,000 x 128 float32 vectors
from a seeded 256-centre Gaussian mixture (integer values 0-255, the shape of
SIFT-like descriptors), split into 4 leaves of 250,000 rows; every leaf is
built with NN-Descent and the leaves are S-Merged (each row keeps its best
k - k/2 entries, samples k/2 ids from the other leaves, cross-leaf
NN-Descent, merge2one).

Default path (the headline): learned initialisation (a code MLP trained,
untimed, on the graph of a separate 50,000-row set of the same generator),
counter-based random draws and the tensor-core local join.  The plain FP32
path -- the reference's random streams and FP32 join, bit-exact with
Smerge::buildKGraph for two leaves -- is timed in the same run
(`plain_fp32`, `speedup_vs_plain_fp32`); --path exact --join fp32 --init
random makes it the measured path.

Printed JSON (one line, rank 0):
  value       seconds per build with the vectors already resident in HBM
              (nnm_merge_leaves_dev), max over ranks;
  e2e         the same through the host C ABI (nnm_merge_leaves): pinned
              host vectors copied in, the graph (ids) copied back, per step;
  roofline    the dominant kernel (the local join) from the library's own
              CUDA-event timing and algorithmic byte count, over a second
              run of the same K steps with those events on (the timed
              steps run without them);
  cpu_baseline the reference itself (oracle/_ref, built from its sources) on
              the first 40,000 and 100,000 rows of the same set,
              extrapolated to 1M rows by the power law through both times;
  cfg1        the 100,000-row plain S-Merge (64-centre mixture): the
              reference and the plain FP32 and exact u8 device paths on the
              same rows (same configuration, same graphs);
  search      the serving workload below, measured in the same run.

--workload search measures batched LySearch serving instead (one step = a
batch of 100,000 queries, top-10, beam widths drawn from 32..512, through
nnm_index_search_dev on the 1M-row H-Merge hierarchy): `value` is queries/s
with the learned entry, beside the default entry and the learned entry at
narrower beams down to the default's recall@10.

--impl reference times the reference's CPU path instead (rank 0 only).
Multi-GPU (torchrun, N > 1): every rank builds its own 1M graph from its own
seeded data (independent replicas, weak scaling), timed as the max over ranks.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "nn-merge_b200"))

METRIC = "1M×128 k=20 build s at recall@10≥0.95: learned+BF16 vs plain FP32 GPU"
HBM_FALLBACK = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="nnm", choices=["nnm", "reference"])
    p.add_argument("--n", type=int, default=1_000_000)
    p.add_argument("--d", type=int, default=128)
    p.add_argument("--k", type=int, default=20)
    p.add_argument("--leaves", type=int, default=4)
    p.add_argument("--centres", type=int, default=256)
    p.add_argument("--seed", type=int, default=1234)
    p.add_argument("--recall-rows", type=int, default=2000)
    p.add_argument("--cpu-sample", type=int, default=40_000)
    p.add_argument("--fit-rows", type=int, default=100_000,
                   help="second size of the reference's timing, for the exponent of its extrapolation")
    p.add_argument("--no-cfg1", action="store_true",
                   help="skip the 100,000-row plain S-Merge timed on the reference and the GPU")
    p.add_argument("--no-search", action="store_true", help="build workload: skip the embedded serving measurement")
    p.add_argument("--dump-iters", default=None, help="write the profiled steps' per-iteration counters (JSON)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--path", default="fast", choices=["exact", "fast"],
                   help="exact: the reference's random streams, bit-exact (plain FP32); "
                        "fast: counter-based draws on the device")
    p.add_argument("--delta", type=float, default=None, help="convergence threshold (default: the reference's 0.002)")
    p.add_argument("--smpl", type=int, default=100, help="reverse-sample cap smplNum (reference: 100)")
    p.add_argument("--join", default="tensor", choices=["auto", "fp32", "tensor"],
                   help="local-join kernel: FP32 CUDA cores, or u8 Gram matrices on the tensor cores "
                        "(bit-identical for integer data)")
    p.add_argument("--init", default="learned", choices=["random", "learned"],
                   help="initial graphs: random, or from the codes of a trained MLP (needs --path fast)")
    p.add_argument("--train-steps", type=int, default=400)
    p.add_argument("--no-plain", action="store_true", help="skip timing the plain FP32 path beside")
    p.add_argument("--no-tune", action="store_true",
                   help="skip the autotuner (sample cap and convergence threshold from --smpl/--delta)")
    p.add_argument("--workload", default="build", choices=["build", "search", "vmf"],
                   help="build: the headline 1M graph build; search: batched LySearch serving on a 1M hierarchy; "
                        "vmf: 10M x 96 unit vectors, log-uniform leaves merged, FP32 / BF16 / FP8 joins")
    p.add_argument("--vmf-n", type=int, default=10_000_000)
    p.add_argument("--vmf-tiers", default="fp32,tensor,fp8")
    p.add_argument("--vmf-tree-tiers", default="tensor,fp8",
                   help="vmf: join tiers also timed with the bottom-up pairwise merge of the leaves")
    p.add_argument("--queries", type=int, default=100_000)
    p.add_argument("--probes", type=int, default=4)
    p.add_argument("--entry-steps", type=int, default=1500)
    p.add_argument("--no-flat", action="store_true", help="search: skip the flat k-NN graph measurement")
    return p.parse_args()


BF16_FALLBACK = 1590.0  # TFLOP/s


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def tensor_peak():
    """Dense BF16 tensor TFLOP/s as measured (burst), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return BF16_FALLBACK, "fallback"


# DRAM bytes measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum,
# one pass, every launch of the class) over whole builds of this workload
# (1,000,000 x 128, four leaves, the untuned sample cap), as a ratio to the
# library's algorithmic bytes of the same launches; the bench reports that
# ratio times the live run's algorithmic bytes per launch.  Keyed by (kernel
# class, tensor join).  Per build, measured against algorithmic: join
# (k_join_tc<0> + k_pairs_tc) 21.80 / 41.33 GB, emit (k_join_tc<1> +
# k_emit_rows) 44.03 / 49.03 GB, merge (k_merge_fast) 9.68 / 11.00 GB.
NCU_TRAFFIC_RATIO = {("join", True): 0.527, ("emit", True): 0.898, ("merge", True): 0.880}


def traffic_per_launch(kind, stat, a):
    r = NCU_TRAFFIC_RATIO.get((kind, a.join != "fp32"))
    if r is None or not stat["launches"]:
        return None
    return r * stat["bytes"] / stat["launches"]


def leaf_sizes(n, leaves):
    base = n // leaves
    sizes = [base] * leaves
    sizes[-1] += n - base * leaves
    return sizes


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def recall_at(ids, x_t, rows, atop, torch, both=False):
    """Recall@atop of the graph rows `rows` against exact brute force
    (FP32 squared L2 without TF32: exact for integer data).  The first
    figure counts an entry as a hit when its exact distance is within the
    atop-th exact distance (ties counted as hits); with both=True the second
    is Evaluator::getKGraphRecall's (evaluator.cpp:258-295): the graph's
    first atop ids intersected with the atop exact neighbours, ties at the
    atop-th distance broken by id."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        q = x_t[rows]
        qn = (q * q).sum(1, keepdim=True)
        xn = (x_t * x_t).sum(1)
        hits = ihits = 0
        for b in range(0, len(rows), 256):
            qb, qnb = q[b:b + 256], qn[b:b + 256]
            d = qnb + xn[None, :] - 2.0 * (qb @ x_t.T)
            d[torch.arange(len(qb)), torch.as_tensor(rows[b:b + 256], device=d.device)] = float("inf")
            kth = torch.topk(d, atop, dim=1, largest=False).values[:, -1:]
            g = torch.as_tensor(ids[b:b + 256, :atop].astype(np.int64), device=d.device)
            hits += int((torch.gather(d, 1, g) <= kth).sum())
            if both:
                # exact neighbours with ties by id: the atop smallest of (distance, id)
                cand = torch.topk(d, atop + 16, dim=1, largest=False)
                cd, ci = cand.values.cpu().numpy(), cand.indices.cpu().numpy()
                for r in range(len(qb)):
                    order = np.lexsort((ci[r], cd[r]))[:atop]
                    ihits += len(np.intersect1d(ci[r][order], ids[b + r, :atop].astype(np.int64)))
        rec = hits / (len(rows) * atop)
        return (rec, ihits / (len(rows) * atop)) if both else rec
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def reference_cpu(x, k, seed, sample, want_graph=False):
    """Times the reference on the first `sample` rows: S-Merge with its own
    split (smerge.cpp:53), one thread (the reference has no threading).
    Returns (seconds, kind, cores) -- and the graph's ids with want_graph.
    The time includes the reference process reading its input."""
    ref = os.path.join(ROOT, "oracle", "_ref", "nnm_ref")
    xs = np.ascontiguousarray(x[:sample])
    if os.path.exists(ref):
        with tempfile.TemporaryDirectory() as td:
            mat = os.path.join(td, "in.mat")
            with open(mat, "wb") as f:
                f.write(np.array(xs.shape, np.uint32).tobytes())
                f.write(xs.tobytes())
            out = os.path.join(td, "out")
            t0 = time.perf_counter()
            subprocess.run([ref, "smerge", "l2", mat, str(k), str(seed), out], check=True, capture_output=True, cwd=td)
            t = time.perf_counter() - t0
            ids = None
            if want_graph:
                b = open(out, "rb").read()
                n, kk = np.frombuffer(b, np.uint32, 2)
                ids = np.frombuffer(b, np.uint32, int(n) * int(kk), 8).reshape(int(n), int(kk)).copy()
            return (t, "reference", 1, ids) if want_graph else (t, "reference", 1)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle()
    t0 = time.perf_counter()
    r = o.smerge(xs, k, seed)
    t = time.perf_counter() - t0
    return (t, "port", 1, r["ids"]) if want_graph else (t, "port", 1)


def cpu_fit(x, k, seed, s1, s2, n):
    """The reference's S-Merge timed at two sizes of the same rows; the
    power law t = t1 (m / s1)^alpha through both points extrapolates it to
    n rows (NN-Descent is slightly super-linear in the row count)."""
    t1, kind, cores = reference_cpu(x, k, seed, s1)
    t2, _, _ = reference_cpu(x, k, seed, s2)
    alpha = float(np.log(t2 / t1) / np.log(s2 / s1))
    return {"t_small": t1, "t_large": t2, "rows": [s1, s2], "alpha": alpha,
            "value": t2 * (n / s2) ** alpha, "kind": kind, "cores": cores}


def run_reference_arm(a, rank):
    """The reference's S-Merge (oracle/_ref: its own sources) on the first
    cpu_sample rows of the same 1M set the GPU arm builds, each step one
    run; one run on the first fit_rows rows fixes the power-law exponent
    that scales the per-step median to the full row count."""
    if rank != 0:
        return
    from nnm.datasets import gaussian_mixture_u8
    x = gaussian_mixture_u8(a.n, d=a.d, n_centres=a.centres, seed=a.seed)
    times = []
    kind = "reference"
    for step in range(min(a.warmup, 1) + a.steps):
        t, kind, cores = reference_cpu(x, a.k, a.seed, a.cpu_sample)
        if step >= min(a.warmup, 1):
            times.append(t)
    t_med = statistics.median(times)
    t_fit, _, _ = reference_cpu(x, a.k, a.seed, a.fit_rows)
    alpha = float(np.log(t_fit / t_med) / np.log(a.fit_rows / a.cpu_sample))
    v = t_fit * (a.n / a.fit_rows) ** alpha
    line = {
        "metric": METRIC, "impl": "reference", "value": v, "unit": "s", "n_gpus": a.gpus, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": t_med * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded %d-centre Gaussian mixture, integers 0-255 (the GPU arm's rows)" % a.centres,
        "config": {"workload": "S-Merge (smerge.cpp:46-91) of the first %d rows per step; seconds extrapolated to "
                               "%d rows by t = t(%d) (n / %d)^alpha, alpha = %.3f from the %d- and %d-row times"
                               % (a.cpu_sample, a.n, a.fit_rows, a.fit_rows, alpha, a.cpu_sample, a.fit_rows),
                   "n": a.n, "d": a.d, "k": a.k, "t_sample_s": t_med, "t_fit_rows_s": t_fit, "alpha": alpha,
                   "fit_rows": a.fit_rows, "sample_rows": a.cpu_sample},
        "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": kind,
                         "sample": "%d rows per step (%d for the exponent), S-Merge, single thread (the reference "
                                   "has no threading)" % (a.cpu_sample, a.fit_rows)},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


SEARCH_METRIC = ("LySearch queries/s, 1M×128 k=20 H-Merge hierarchy, 100K queries, top-10, beams U{32..512}: "
                 "learned vs default entry at equal recall@10")


def search_truth(x_t, q, torch, k=10):
    """k-th exact neighbour distance of every query: FP32 GEMM candidates
    (top 16, no TF32) re-ranked in float64."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        xn = (x_t * x_t).sum(1)
        x_np = x_t.cpu().numpy()
        kth = np.empty(len(q))
        for i in range(0, len(q), 500):
            qt = torch.from_numpy(q[i:i + 500]).cuda()
            d = (qt * qt).sum(1)[:, None] + xn[None, :] - 2.0 * (qt @ x_t.T)
            cand = torch.topk(d, 16, dim=1, largest=False).indices.cpu().numpy()
            ex = ((x_np[cand].astype(np.float64) - q[i:i + 500, None, :]) ** 2).sum(-1)
            kth[i:i + 500] = np.sort(ex, axis=1)[:, k - 1]
        return kth
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def search_recall(ids, x, q, kth):
    """Results whose exact distance is within the query's k-th exact distance."""
    d = ((x[ids.astype(np.int64)].astype(np.float64) - q[:, None, :].astype(np.float64)) ** 2).sum(-1)
    return float((d <= kth[:, None] + 1e-6).mean())


def search_cpu(x, layers, q, beams, seed, sample):
    """The oracle's restatement of LySearch (nno_search_ex: the reference's
    heaps and float sums, one thread) on the first `sample` queries."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import Oracle
    o = Oracle()
    t0 = time.perf_counter()
    o.search_ex(x, layers, q[:sample], 10, seed, beams=beams[:sample])
    return time.perf_counter() - t0


def run_search(a, rank, world, local, reps=None, embedded=False):
    """Serving workload (one step = one batch of `queries` queries through
    nnm_index_search_dev with the vectors, hierarchy and queries resident).
    embedded: measured inside the build bench -- returns the line's fields
    (rank 0) instead of printing, and skips the flat-graph comparison."""
    import torch
    import nnm
    from nnm.datasets import gaussian_mixture_u8, queries_like
    from nnm.replicas import Replicas

    torch.cuda.set_device(local)
    own_reps = reps is None
    if own_reps:
        reps = Replicas("nccl")
    n, d, k, nq = a.n, a.d, a.k, a.queries
    seed = reps.data_seed(a.seed)
    x = gaussian_mixture_u8(n, d=d, n_centres=a.centres, seed=seed)
    q = queries_like(nq, d=d, n_centres=a.centres, seed=seed, query_seed=seed + 77)
    beams = np.random.default_rng(seed + 5).integers(32, 513, size=nq).astype(np.uint32)
    ctx = nnm.Context(local)
    t0 = time.perf_counter()
    h = ctx.hmerge(x, k, 20, seed=a.seed, rng="fast", join="tensor")
    ix = ctx.index(x, h["layers"], seed=a.seed)
    layer, C = ix.entry_layer()
    model = nnm.entry_init(d, C, seed=11)
    losses = ix.entry_train(model, steps=a.entry_steps, batch=2048, lr=2e-3, seed=3)
    ix.set_entry_model(model, probes=a.probes)
    # autotuner (untimed): the fast kernel's width, timed on 10,000 of the queries
    width, width_ms = ix.tune_width(q[:10_000], out_k=10, beams=beams[:10_000], entry="learned")
    prep_s = time.perf_counter() - t0
    x_t = torch.from_numpy(x).cuda()
    q_dev = torch.from_numpy(q).cuda()
    oi = torch.empty((nq, 10), dtype=torch.int32, device="cuda")
    od = torch.empty((nq, 10), dtype=torch.float32, device="cuda")
    nrec = min(nq, 10_000)
    kth = search_truth(x_t, q[:nrec], torch)

    def timed(entry, scale=1.0, steps=a.steps, warm=a.warmup):
        b = np.maximum(10, np.round(beams * scale)).astype(np.uint32)
        b_dev = torch.from_numpy(b.astype(np.int32)).cuda()
        kw = dict(beams_ptr=b_dev.data_ptr(), beam=int(b.max()), mode="fast", entry=entry)
        for _ in range(warm):
            ix.search_dev(q_dev.data_ptr(), nq, oi.data_ptr(), od.data_ptr(), 10, **kw)
        torch.cuda.synchronize()
        tot = pred = 0.0
        cm = ex = 0
        l0 = ctx.launch_count()
        reps.barrier()
        for _ in range(steps):
            st = ix.search_dev(q_dev.data_ptr(), nq, oi.data_ptr(), od.data_ptr(), 10, **kw)
            tot += st["device_ms"]
            pred += st["predict_ms"]
            cm += st["ncmps"]
            ex += st["expansions"]
        reps.barrier()
        ids = oi[:nrec].cpu().numpy().view(np.uint32)
        return dict(ms=tot / steps, predict_ms=pred / steps, ncmps=cm / steps, expansions=ex / steps,
                    launches=ctx.launch_count() - l0, recall=search_recall(ids, x, q[:nrec], kth), scale=scale)

    with ClockSampler(local) as clocks:
        learned = timed("learned")
    default = timed("default")
    # equal recall: the learned entry at narrower beams, down to the default's recall
    sweep = []
    for sc in (0.7, 0.5, 0.3, 0.2, 0.15, 0.1, 0.07, 0.05):
        r = timed("learned", sc, steps=1, warm=1)
        sweep.append({"scale": sc, "recall": r["recall"], "qps": nq / r["ms"] * 1e3})
        if r["recall"] < default["recall"]:
            break
    eq = [s for s in sweep if s["recall"] >= default["recall"]]
    ms = reps.max(learned["ms"])
    value = world * nq / (ms / 1e3)

    # end to end through the host C ABI: pinned queries and beams in, ids and distances out
    e2e = None
    if not a.no_e2e:
        q_pin = torch.from_numpy(q).pin_memory().numpy()
        b_pin = torch.from_numpy(beams.astype(np.int32)).pin_memory().numpy().view(np.uint32)
        ix.search(q_pin, out_k=10, beams=b_pin, mode="fast", entry="learned")
        reps.barrier()
        t1 = time.perf_counter()
        for _ in range(a.steps):
            ix.search(q_pin, out_k=10, beams=b_pin, mode="fast", entry="learned")
        e2e_s = reps.max((time.perf_counter() - t1) / a.steps)
        e2e = {"value": world * nq / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(q.nbytes + beams.nbytes),
               "d2h_bytes_per_step": int(nq * 10 * 8)}

    # the same queries against the flat 1M k-NN graph of the headline build
    # (one layer): the reference's flat search (random seeds) vs the
    # learned entry
    flat = None
    if not a.no_flat and not embedded:
        k_ids = torch.empty((n, k), dtype=torch.int32, device="cuda")
        k_ds = torch.empty((n, k), dtype=torch.float32, device="cuda")
        ctx.merge_leaves_dev(x_t.data_ptr(), n, d, k, leaf_sizes(n, a.leaves), k_ids.data_ptr(), k_ds.data_ptr(), 0,
                             seed=a.seed, rng="fast", join="tensor", init="random")
        adj = k_ids.cpu().numpy().view(np.uint32).reshape(-1)
        fx = ctx.index(x, [(np.arange(0, n * k + 1, k, dtype=np.uint64), adj)], seed=a.seed)
        fl, fc = fx.entry_layer()
        fm = nnm.entry_init(d, fc, seed=11)
        fx.entry_train(fm, steps=a.entry_steps, batch=2048, lr=2e-3, seed=3)
        fx.set_entry_model(fm, probes=a.probes)
        flat = {}
        for entry in ("flat", "learned"):
            fx.search(q, out_k=10, beams=beams, mode="fast", entry=entry)
            r = fx.search(q, out_k=10, beams=beams, mode="fast", entry=entry)
            flat[entry] = {"qps": nq / r["device_ms"] * 1e3, "ms": r["device_ms"],
                           "recall": search_recall(r["ids"][:nrec], x, q[:nrec], kth),
                           "ncmps": r["ncmps"] / nq, "expansions": r["expansions"] / nq}
        fx.close()

    hbm, peak_kind = peaks()
    kern_ms = learned["ms"] - learned["predict_ms"]
    row_bytes = ((d + 3) // 4) * 16
    achieved = learned["ncmps"] * row_bytes / (kern_ms * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": "k_serve<L2,1> (warp-per-query beam search, fast kernel)",
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
            "traffic": None,
            "algorithmic_bytes": "distance evaluations x %d B (one vector row each) per step" % row_bytes,
            "kernel_ms": kern_ms, "predict_ms": learned["predict_ms"]}
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        sample = 2000
        t = search_cpu(x, h["layers"], q, beams, a.seed, sample)
        cpu = {"value": sample / t, "unit": "queries/s", "cores": 1, "kind": "port",
               "sample": "the oracle's LySearch (nno_search_ex, reference heaps and sums) on the first %d queries "
                         "with their beams, default entry, single thread (%.1f s)" % (sample, t)}
    if rank == 0:
        line = {
            "metric": SEARCH_METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded %d-centre Gaussian mixture, integers 0-255; queries from the same mixture "
                    "(fresh seed)" % a.centres,
            "config": {"workload": "LySearch batch of %d queries, top-10, beams U{32..512}, fast kernel (tuned width), "
                                   "learned entry (probes %d), on the H-Merge hierarchy of %dx%d k=%d"
                                   % (nq, a.probes, n, d, k),
                       "n": n, "d": d, "k": k, "queries": nq, "layers": [len(o) - 1 for o, _ in h["layers"]],
                       "entry_layer": layer, "classes": C, "entry_train_steps": a.entry_steps,
                       "width": width, "width_ms_10k": [round(float(v), 3) for v in width_ms],
                       "entry_loss_first": float(losses[:20].mean()), "entry_loss_last": float(losses[-20:].mean()),
                       "prep_s": prep_s, "recall@10": learned["recall"], "recall_rows": nrec,
                       "learned": learned, "default": default,
                       "qps_default": nq / default["ms"] * 1e3,
                       "equal_recall": {"default_recall": default["recall"], "sweep": sweep,
                                        "learned_qps_at_default_recall": eq[-1]["qps"] if eq else None,
                                        "speedup": (eq[-1]["qps"] / (nq / default["ms"] * 1e3)) if eq else None},
                       "flat_graph": flat,
                       "l2": "vectors (%d MB) larger than L2 (126 MB)" % (x.nbytes >> 20),
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": learned["launches"],
            "clocks": clocks.summary(),
        }
        if not embedded:
            print(json.dumps(line), flush=True)
    ix.close()
    ctx.close()
    if own_reps:
        reps.close()
    if embedded and rank == 0:
        return {key: line[key] for key in ("metric", "value", "unit", "ms_per_step", "config", "roofline",
                                           "cpu_baseline", "e2e", "gpu_launches", "clocks")}
    return None


def run_search_reference_arm(a, rank):
    """The oracle's LySearch (the reference's steps, one thread) on a bounded
    sample of the serving workload; the hierarchy is built by the library
    (a CPU H-Merge of 1M rows does not fit the run)."""
    if rank != 0:
        return
    import nnm
    from nnm.datasets import gaussian_mixture_u8, queries_like
    x = gaussian_mixture_u8(a.n, d=a.d, n_centres=a.centres, seed=a.seed)
    q = queries_like(2000, d=a.d, n_centres=a.centres, seed=a.seed, query_seed=a.seed + 77)
    beams = np.random.default_rng(a.seed + 5).integers(32, 513, size=len(q)).astype(np.uint32)
    ctx = nnm.Context(0)
    h = ctx.hmerge(x, a.k, 20, seed=a.seed, rng="fast", join="tensor")
    ctx.close()
    times = [search_cpu(x, h["layers"], q, beams, a.seed, 500) for _ in range(max(1, a.steps))]
    v = 500 / statistics.median(times)
    line = {"metric": SEARCH_METRIC, "impl": "reference", "value": v, "unit": "queries/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": statistics.median(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic, as the nnm arm", "config": {"workload": "500 queries per step, default entry",
                                                           "n": a.n, "d": a.d, "k": a.k},
            "cpu_baseline": {"value": v, "unit": "queries/s", "cores": 1, "kind": "port",
                             "sample": "500 queries with their beams, single thread"},
            "e2e": {"value": v, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


VMF_METRIC = "10M×96 k=16 vMF build s, log-uniform leaves merged: FP32 vs BF16 vs FP8 join"


def loguniform_leaves(n, lo, hi, seed):
    """Leaf sizes drawn log-uniformly from [lo, hi] until they cover n rows
    (the last leaf takes the rest, or joins its predecessor when below lo)."""
    rng = np.random.default_rng(seed)
    sizes, tot = [], 0
    while tot < n:
        sz = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        sz = min(sz, n - tot)
        if sz < lo and sizes:
            sizes[-1] += sz
        else:
            sizes.append(sz)
        tot += sz
    return sizes


def run_vmf(a, rank, world, local):
    """10M x 96 unit-norm vectors from the 1024-centre vMF-like mixture
    (kappa 50), leaves of log-uniform sizes in [5,000, 200,000], k = 16, all
    leaves built and merged in one multi-way merge (fast draws, random
    initial graphs), once per join tier: FP32 (the reference's sums), BF16
    (hi + lo) and FP8 (E4M3 hi + mid + lo).  The reduced-precision tiers
    give the FP32 tier's graph bit for bit; value = the BF16 tier's seconds."""
    import torch
    import nnm
    from nnm.datasets import vmf_mixture
    from nnm.replicas import Replicas

    torch.cuda.set_device(local)
    reps = Replicas("nccl")
    n, d, k = a.vmf_n, 96, 16
    t0 = time.perf_counter()
    x = vmf_mixture(n, d=d, n_centres=1024, kappa=50.0, seed=reps.data_seed(4321))
    gen_s = time.perf_counter() - t0
    sizes = loguniform_leaves(n, 5_000, 200_000, 17)
    x_dev = torch.from_numpy(x).cuda()
    ids_dev = torch.empty((n, k), dtype=torch.int32, device="cuda")
    dists_dev = torch.empty((n, k), dtype=torch.float32, device="cuda")
    ctx = nnm.Context(local)
    rows = np.sort(np.random.default_rng(7).choice(n, 2000, replace=False))
    tiers, ref_ids = {}, None
    runs = [(t, "all") for t in a.vmf_tiers.split(",") if t] + [(t, "tree") for t in a.vmf_tree_tiers.split(",") if t]
    for tier, order in runs:
        kw = dict(seed=a.seed, rng="fast", join=tier, init="random", merge_order=order)
        ctx.merge_leaves_dev(x_dev.data_ptr(), n, d, k, sizes, ids_dev.data_ptr(), dists_dev.data_ptr(), 0, **kw)
        ctx.profile(True)
        times = []
        for _ in range(max(1, a.steps)):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            st = ctx.merge_leaves_dev(x_dev.data_ptr(), n, d, k, sizes, ids_dev.data_ptr(), dists_dev.data_ptr(), 0,
                                      **kw)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        prof = ctx.profile_stats()
        ctx.profile(False)
        ids = ids_dev.cpu().numpy().view(np.uint32)
        rec, rec_ids = recall_at(ids[rows], x_dev, rows, 10, torch, both=True)
        ids_s = ids[rows].astype(np.int64)
        ds_s = dists_dev[torch.as_tensor(rows, device="cuda")].cpu().numpy().astype(np.float64)
        ref_s = ((x[rows][:, None, :].astype(np.float64) - x[ids_s].astype(np.float64)) ** 2).sum(-1)
        rel = np.abs(ds_s - ref_s) / np.maximum(ref_s, 1e-30)
        same = None
        if order == "all":
            if ref_ids is None:
                ref_ids = ids.copy()
            else:
                same = bool(np.array_equal(ids, ref_ids))
        tiers[tier if order == "all" else tier + "/tree"] = {
                       "s": statistics.median(times), "times": times, "iterations": st["iterations"],
                       "merge_order": order,
                       "recall@10": rec, "recall@10_ids": rec_ids,
                       "dist_err_vs_fp64": {"max_rel": float(rel.max()), "mean_rel": float(rel.mean())},
                       "same_graph_as_first_tier": same,
                       "join_ms": prof["join"]["ms"], "emit_ms": prof["emit"]["ms"], "merge_ms": prof["merge"]["ms"],
                       "proposals": int(sum(L[3] for L in prof["iters"])),
                       # reduced precision: proposals carrying d~, and the share the merge recomputed exactly
                       "approx_proposals": prof["approx"]["proposals"],
                       "recheck_rate": (prof["approx"]["rechecks"] / prof["approx"]["proposals"]
                                        if prof["approx"]["proposals"] else None)}
    ms = reps.max(tiers.get("tensor", next(iter(tiers.values())))["s"] * 1e3)
    if rank == 0:
        line = {"metric": VMF_METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": a.steps,
                "warmup": 1, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "bf16", "data": "synthetic: seeded 1024-centre vMF-like mixture (kappa 50), unit norm",
                "config": {"workload": "%dx%d k=%d, %d log-uniform leaves (%d..%d rows) built and merged, fast draws, "
                                       "random init" % (n, d, k, len(sizes), min(sizes), max(sizes)),
                           "n": n, "d": d, "k": k, "leaves": len(sizes), "gen_s": gen_s, "tiers": tiers},
                "cpu_baseline": None, "e2e": None}
        print(json.dumps(line), flush=True)
    ctx.close()
    reps.close()


def run_cfg1(ctx, torch, seed):
    """100,000 x 128 from the 64-centre mixture, S-Merge of the halves, k=20
    (Smerge::buildKGraph, smerge.cpp:46-91): the reference's own process on
    one host core, and the plain FP32 and exact u8 device paths (reference
    streams) through the host C ABI on the same rows.  Returns the times,
    whether the device graphs equal the reference's, and recall@10 of both."""
    from nnm.datasets import gaussian_mixture_u8
    x = gaussian_mixture_u8(100_000, d=128, n_centres=64, seed=1234)
    t_ref, kind, cores, ref_ids = reference_cpu(x, 20, seed, len(x), want_graph=True)
    out = {"workload": "100000x128 (64-centre mixture) S-Merge of the halves, k=20, reference streams",
           "reference_s": t_ref, "reference_kind": kind, "reference_cores": cores, "host_cpus": os.cpu_count()}
    for name, join in (("plain_fp32", "fp32"), ("exact_u8", "tensor")):
        ctx.smerge(x, 20, seed=seed, join=join)  # warm-up
        t0 = time.perf_counter()
        r = ctx.smerge(x, 20, seed=seed, join=join)
        t = time.perf_counter() - t0
        out[name] = {"s_host_api": t, "device_ms": r["device_ms"], "iterations": r["iterations"],
                     "same_graph_as_reference": bool(np.array_equal(r["ids"], ref_ids)),
                     "ratio_reference_over_device": t_ref / t}
    x_t = torch.from_numpy(x).cuda()
    rows = np.sort(np.random.default_rng(7).choice(len(x), 2000, replace=False))
    out["recall@10_reference"] = recall_at(ref_ids[rows], x_t, rows, 10, torch, both=True)
    out["recall@10_device"] = recall_at(r["ids"][rows], x_t, rows, 10, torch, both=True)
    return out


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        if a.workload == "search":
            run_search_reference_arm(a, rank)
        else:
            run_reference_arm(a, rank)
        return
    if a.workload == "search":
        run_search(a, rank, world, local)
        return
    if a.workload == "vmf":
        run_vmf(a, rank, world, local)
        return

    import torch
    import nnm
    from nnm.datasets import gaussian_mixture_u8
    from nnm.replicas import Replicas

    torch.cuda.set_device(local)
    reps = Replicas("nccl")
    barrier, max_over_ranks = reps.barrier, reps.max

    n, d, k = a.n, a.d, a.k
    sizes = leaf_sizes(n, a.leaves)
    x = gaussian_mixture_u8(n, d=d, n_centres=a.centres, seed=reps.data_seed(a.seed))
    x_dev = torch.from_numpy(x).cuda()
    ids_dev = torch.empty((n, k), dtype=torch.int32, device="cuda")
    dists_dev = torch.empty((n, k), dtype=torch.float32, device="cuda")
    ctx = nnm.Context(local)
    build_seed = a.seed

    bkw = dict(seed=build_seed, rng=a.path, sample_cap=a.smpl, join=a.join, init=a.init,
               delta=a.delta if a.delta is not None else 0.002)

    def build_dev(**kw):
        return ctx.merge_leaves_dev(x_dev.data_ptr(), n, d, k, sizes, ids_dev.data_ptr(), dists_dev.data_ptr(), 0,
                                    **(kw or bkw))

    # learned initialisation: the model is trained once (untimed) on the
    # graph the method builds for another 50,000-row set of the generator
    train = None
    if a.init == "learned":
        xt = gaussian_mixture_u8(50_000, d=d, n_centres=a.centres, seed=a.seed + 10_000 + rank)
        t0 = time.perf_counter()
        gt = ctx.kgraph(xt, k, seed=1, rng="fast", join=a.join)
        model = nnm.mlp_init(d, seed=3)
        losses = ctx.mlp_train(xt, gt["ids"], model, steps=a.train_steps, batch=2048, seed=9)
        train = {"rows": 50_000, "steps": a.train_steps, "s": time.perf_counter() - t0,
                 "loss_first": float(losses[:10].mean()), "loss_last": float(losses[-10:].mean())}
        ctx.set_init_model(model)

    # autotuner (untimed, like the training): sample cap and convergence
    # threshold from trial builds on the whole set (a smaller sample reads a
    # higher recall than the full build), scored on the device on 2,000 rows
    # against recall@10 >= 0.95 + 0.005
    tune = None
    if not a.no_tune and a.path == "fast":
        # tuned on a held-out set of the same generator and size (another
        # seed), so that the timed set's recall is measured, not fitted
        t0 = time.perf_counter()
        xh = torch.from_numpy(gaussian_mixture_u8(n, d=d, n_centres=a.centres,
                                                  seed=reps.data_seed(a.seed) + 50_000)).cuda()
        chosen, trials = ctx.autotune_merge_leaves_dev(xh.data_ptr(), n, d, k, sizes, sample_rows=n,
                                                       eval_rows=2000, repeats=2, **bkw)
        del xh
        bkw.update(chosen)
        tune = {"chosen": chosen, "s": time.perf_counter() - t0, "sample_rows": n, "eval_rows": 2000,
                "held_out_seed": reps.data_seed(a.seed) + 50_000, "trials": trials}

    rng_rows = np.random.default_rng(7)
    rows = np.sort(rng_rows.choice(n, min(a.recall_rows, n), replace=False))

    def recall_now(both=False):
        ids_np = ids_dev[torch.as_tensor(rows, device="cuda")].cpu().numpy().view(np.uint32)
        return recall_at(ids_np, x_dev, rows, 10, torch, both=both)

    # the plain FP32 GPU path (reference streams, FP32 join, random init),
    # timed the same way, for the speed-up of the default path
    plain = None
    if not a.no_plain and not (a.path == "exact" and a.join == "fp32" and a.init == "random"):
        pkw = dict(seed=build_seed, rng="exact", sample_cap=a.smpl, join="fp32", init="random",
                   delta=a.delta if a.delta is not None else 0.002)
        build_dev(**pkw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(2):
            pst = build_dev(**pkw)
        e1.record()
        torch.cuda.synchronize()
        prec, pirec = recall_now(both=True)
        plain = {"s": e0.elapsed_time(e1) / 2 / 1e3, "recall@10": prec, "recall@10_ids": pirec,
                 "iterations": pst["iterations"], "steps": 2}

    for _ in range(a.warmup):
        st = build_dev()
    torch.cuda.synchronize()
    l0 = ctx.launch_count()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(a.steps):
            st = build_dev()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    launches = ctx.launch_count() - l0
    # the same K steps again with the library's per-kernel CUDA events on
    # (the roofline's kernel times and byte counts come from this run)
    ctx.profile(True)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(a.steps):
        build_dev()
    p1.record(stream)
    torch.cuda.synchronize()
    prof = ctx.profile_stats()
    ctx.profile(False)
    prof_ms = p0.elapsed_time(p1) / a.steps
    if a.dump_iters:
        with open(a.dump_iters, "w") as f:
            json.dump({"iters": prof["iters"], "kq": (d + 31) // 32 * 32, "steps": a.steps,
                       "columns": ["n", "rows_per_tier", "pairs", "proposals", "flags", "ncmps", "sum_s",
                                   "ms_join", "ms_emit", "ms_merge"]}, f)
    # the same build with every kernel launched directly (no iteration graphs)
    direct = None
    if a.path == "fast":
        build_dev(**dict(bkw, graph=False))
        torch.cuda.synchronize()
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        d0.record(stream)
        for _ in range(3):
            build_dev(**dict(bkw, graph=False))
        d1.record(stream)
        torch.cuda.synchronize()
        direct = {"s": d0.elapsed_time(d1) / 3 / 1e3, "steps": 3}
    # builds run on the library's stream and synchronize before returning, so
    # the events on torch's stream bracket them
    ms = ev0.elapsed_time(ev1) / a.steps
    ms = max_over_ranks(ms)

    # end to end through the host C ABI: pinned host input, graph ids back
    e2e = None
    if not a.no_e2e:
        x_pin = torch.from_numpy(x).pin_memory()
        ids_pin = torch.empty((n, k), dtype=torch.int32).pin_memory()
        xh, ih = x_pin.numpy(), ids_pin.numpy().view(np.uint32)
        ctx.merge_leaves_into(xh, k, sizes, ih, **bkw)
        barrier()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            ctx.merge_leaves_into(xh, k, sizes, ih, **bkw)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / a.steps)
        e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(x.nbytes),
               "d2h_bytes_per_step": int(n * k * 4)}

    # quality: recall@10 on a seeded row sample vs exact brute force
    build_dev()
    rec, rec_ids = recall_now(both=True)
    # distance error of the returned distances against FP64 on the same rows
    ids_s = ids_dev[torch.as_tensor(rows, device="cuda")].cpu().numpy().view(np.uint32).astype(np.int64)
    ds_s = dists_dev[torch.as_tensor(rows, device="cuda")].cpu().numpy().astype(np.float64)
    ref_s = ((x[rows][:, None, :].astype(np.float64) - x[ids_s].astype(np.float64)) ** 2).sum(-1)
    rel = np.abs(ds_s - ref_s) / np.maximum(ref_s, 1e-30)
    dist_err = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()), "rows": len(rows)}

    hbm, peak_kind = peaks()
    names = {"join": ("local-join count pass: k_join_tc<0> (u8 Gram tiles on tcgen05) + k_pairs_tc (lists > 128, "
                      "128-slot blocks on tcgen05)"
                      if a.join != "fp32" else "local-join pair distances (FP32 k_pairs, all tiers)"),
             "emit": ("local-join emit pass: k_join_tc<1> + k_emit_rows" if a.join != "fp32" else "proposal emit (k_emit)"),
             "merge": "top-K merge (k_merge)"}
    dom = max(("join", "emit", "merge"), key=lambda c: prof[c]["ms"])
    j = prof[dom]
    roof = None
    if j["launches"]:
        per_ms = j["ms"] / j["launches"]
        per_bytes = j["bytes"] / j["launches"]
        achieved = per_bytes / (per_ms * 1e-3) / 1e9
        # tensor pipe: the 8-bit MMAs run at twice the BF16 rate, so their
        # peak is twice the measured BF16 figure
        tpk, tpk_kind = tensor_peak()
        t_ops = j.get("tensor_ops", 0.0) / j["launches"]
        tpeak = tpk * (2.0 if a.join != "fp32" else 1.0)
        roof = {"bound": "hbm", "kernel": names[dom],
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "peak_kind": peak_kind, "traffic": traffic_per_launch(dom, j, a),
                "tensor_tflops": t_ops / (per_ms * 1e-3) / 1e12,
                "tensor_frac": (t_ops / (per_ms * 1e-3) / 1e12) / tpeak,
                "tensor_peak": tpeak, "tensor_peak_kind": tpk_kind + " (bf16, x2 for 8-bit operands)",
                "join_share_of_step": prof["join"]["ms"] / (prof_ms * a.steps),
                "emit_share_of_step": prof["emit"]["ms"] / (prof_ms * a.steps),
                "merge_share_of_step": prof["merge"]["ms"] / (prof_ms * a.steps),
                "profiled_ms_per_step": prof_ms,
                # per class and step: launches, device ms, algorithmic bytes (the ncu
                # traffic ratios are measured against these)
                "classes": {c: {"launches": prof[c]["launches"] / a.steps, "ms": prof[c]["ms"] / a.steps,
                                "bytes": prof[c]["bytes"] / a.steps} for c in ("join", "emit", "merge")}}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        f = cpu_fit(x, k, build_seed, a.cpu_sample, a.fit_rows, n)
        cpu = {"value": f["value"], "unit": "s", "cores": f["cores"], "kind": f["kind"], "host_cpus": os.cpu_count(),
               "sample": "S-Merge of the first %d and %d rows of this set (%.1f s, %.1f s), extrapolated to %d rows "
                         "by the power law through both (exponent %.3f)"
                         % (f["rows"][0], f["rows"][1], f["t_small"], f["t_large"], n, f["alpha"]),
               "fit": f}

    # the 100,000-row plain S-Merge (the reference's CPU-runnable workload):
    # the reference on the host next to the plain FP32 and exact u8 device
    # paths on the same rows -- a same-configuration ratio
    cfg1 = None
    if rank == 0 and world == 1 and not a.no_cfg1:
        cfg1 = run_cfg1(ctx, torch, build_seed)

    # serving on the same kind of data (LySearch on a 1M hierarchy)
    search = None
    if not a.no_search:
        ctx.close()
        ctx = None
        search = run_search(a, rank, world, local, reps=reps, embedded=True)

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8" if a.join != "fp32" else "f32",
            "data": "synthetic: seeded %d-centre Gaussian mixture, integers 0-255 (stand-in for SIFT-like data)"
                    % a.centres,
            "config": {"workload": "%dx%d k=%d: NN-Descent on %d leaves of %d rows + S-Merge of the leaves (%s)"
                                   % (n, d, k, a.leaves, sizes[0],
                                      "plain FP32, reference-exact"
                                      if (a.path, a.join, a.init) == ("exact", "fp32", "random")
                                      else "%s init, %s draws, %s join" % (a.init, a.path, a.join)),
                       "n": n, "d": d, "k": k, "leaves": a.leaves,
                       "path": a.path, "init": a.init, "train": train, "tune": tune,
                       "delta": bkw["delta"], "smpl": bkw["sample_cap"], "join": a.join,
                       "join_rows": prof["rows"],
                       "recall@10": rec, "recall@10_ids": rec_ids,
                       "recall_note": "recall@10 counts ties at the 10th exact distance; recall@10_ids intersects ids "
                                      "(Evaluator::getKGraphRecall)",
                       "dist_err_vs_fp64": dist_err, "iterations": st["iterations"],
                       "ncmps_merge": st["ncmps"],
                       "ncmps_leaves": st["sub_ncmps"],
                       "l2": "inputs (%d MB) larger than L2 (126 MB)" % (x.nbytes >> 20),
                       "parallelism": "replicas" if world > 1 else "single"},
            "plain_fp32": plain,
            "direct_launches": direct,
            "speedup_vs_plain_fp32": (plain["s"] / (ms / 1e3)) if plain else None,
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clocks.summary(), "cfg1": cfg1, "search": search,
        }
        print(json.dumps(line), flush=True)
    if ctx is not None:
        ctx.close()
    reps.close()


if __name__ == "__main__":
    main()
