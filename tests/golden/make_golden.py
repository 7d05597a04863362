"""Generates the golden fixtures in this directory by running the reference
itself (oracle/_ref/nnm_ref: the reference sources compiled by
oracle/Makefile, seeded through a frozen clock and srand(seed)).

Run from the repository root after `make -C oracle ref`:

    python tests/golden/make_golden.py

Each fixture stores its input, the parameters and the reference's outputs
(pool ids, distances, flags, distance-evaluation count, per-iteration
convergence means; DPG layers and search results where applicable).
Inputs are small integer-valued float32 matrices stored as uint8, several
with duplicated rows so that exactly equal distances (and with them the
reference's sort and insert tie order) are exercised.
"""
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "nn-merge_b200"))

from oracle_lib import ref_available, run_ref  # noqa: E402
from nnm.datasets import gaussian_mixture_u8  # noqa: E402


def with_duplicates(x, frac, seed):
    """Replaces a fraction of rows by copies of other rows."""
    rng = np.random.default_rng(seed)
    x = x.copy()
    n = x.shape[0]
    dst = rng.choice(n, int(frac * n), replace=False)
    src = rng.integers(0, n, len(dst))
    x[dst] = x[src]
    return x


def coarse(n, d, seed):
    """Few distinct values per coordinate: many exactly equal distances."""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, 3, (n, d)) * 10).astype(np.float32)


CASES = [
    # name, command, data builder, K, extra
    ("kgraph_mix", "kgraph", lambda: gaussian_mixture_u8(400, d=32, n_centres=8, seed=101), 10, {}),
    ("kgraph_dup", "kgraph", lambda: with_duplicates(gaussian_mixture_u8(300, d=24, seed=102), 0.3, 1), 8, {}),
    ("kgraph_coarse", "kgraph", lambda: coarse(200, 6, 103), 8, {}),
    ("kgraph_l1", "kgraph", lambda: gaussian_mixture_u8(300, d=20, seed=104), 8, {"metric": "l1"}),
    ("kgraph_chi2", "kgraph", lambda: gaussian_mixture_u8(300, d=20, seed=105), 8, {"metric": "chi2"}),
    ("kgraph_ragged", "kgraph", lambda: gaussian_mixture_u8(250, d=13, seed=106), 6, {}),
    ("kgraph_min", "kgraph", lambda: gaussian_mixture_u8(12, d=8, seed=107), 10, {}),
    ("smerge_mix", "smerge", lambda: gaussian_mixture_u8(500, d=32, seed=111), 10, {}),
    ("smerge_dup", "smerge", lambda: with_duplicates(gaussian_mixture_u8(401, d=16, seed=112), 0.25, 2), 8, {}),
    ("jmerge_mix", "jmerge", lambda: gaussian_mixture_u8(500, d=32, seed=121), 10, {}),
    ("jmerge_coarse", "jmerge", lambda: coarse(300, 8, 122), 8, {}),
    ("hmerge_small", "hmerge", lambda: gaussian_mixture_u8(1000, d=16, seed=131), 8, {"m": 8}),
    ("hmerge_search", "hmerge", lambda: gaussian_mixture_u8(33000, d=8, n_centres=64, seed=132), 8,
     {"m": 8, "queries": 200, "topk": (1, 10, 40), "hash_pools": True}),
]

SEED = 20240601


def main():
    if not ref_available():
        sys.exit("oracle/_ref/nnm_ref is missing: run `make -C oracle ref` first")
    only = set(sys.argv[1:])  # optional: regenerate just these fixtures
    for name, cmd, make, k, extra in CASES:
        if only and name not in only:
            continue
        x = make()
        out = {"x_u8": x.astype(np.uint8), "k": k, "seed": SEED, "cmd": cmd,
               "metric": extra.get("metric", "l2")}
        assert np.array_equal(out["x_u8"].astype(np.float32), x)
        with tempfile.TemporaryDirectory() as td:
            r = run_ref(cmd, x, k, SEED, td, metric=out["metric"], m=extra.get("m"))
            for key in ("ids", "dists", "flags", "trace"):
                out[key] = r[key]
            if extra.get("hash_pools"):  # large case: keep digests of the pools only
                for key in ("ids", "dists", "flags"):
                    out[key + "_sha256"] = hashlib.sha256(np.ascontiguousarray(out.pop(key)).tobytes()).hexdigest()
            out["ncmps"] = r["ncmps"]
            if cmd == "hmerge":
                out["m"] = extra["m"]
                out["n_layers"] = len(r["layers"])
                for g, (off, adj) in enumerate(r["layers"]):
                    out["layer%d_off" % g] = off
                    out["layer%d_adj" % g] = adj
                if "queries" in extra:
                    q = gaussian_mixture_u8(extra["queries"], d=x.shape[1], n_centres=64, seed=999)
                    out["q_u8"] = q.astype(np.uint8)
                    for topk in extra["topk"]:
                        s = run_ref("search", x, None, SEED, td, metric=out["metric"],
                                    layers_txt=os.path.join(td, "hier.txt"), queries=q, topk=topk)
                        out["search%d_ids" % topk] = s["ids"]
                        out["search%d_dists" % topk] = s["dists"]
                        out["search%d_ncmps" % topk] = s["ncmps"]
                        out["search%d_entry" % topk] = s["entry"]
                        f = run_ref("flatsearch", x, None, SEED, td, metric=out["metric"],
                                    layers_txt=os.path.join(td, "hier.txt"), queries=q, topk=topk)
                        out["flat%d_ids" % topk] = f["ids"]
                        out["flat%d_dists" % topk] = f["dists"]
                        out["flat%d_ncmps" % topk] = f["ncmps"]
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **out)
        print("%-16s %-7s n=%-6d d=%-3d k=%-3d iters=%-3d ncmps=%d  %d bytes"
              % (name, cmd, x.shape[0], x.shape[1], k, len(out["trace"]), out["ncmps"], os.path.getsize(path)))


if __name__ == "__main__":
    main()
