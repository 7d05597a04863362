"""Loads the fixtures in tests/golden/ (outputs of the reference itself)."""
import glob
import hashlib
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names(cmd=None):
    out = []
    for p in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        with np.load(p) as z:
            if cmd is None or str(z["cmd"]) == cmd:
                out.append(os.path.basename(p)[:-4])
    return out


def load(name):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        f = {k: z[k] for k in z.files}
    f["x"] = f["x_u8"].astype(np.float32)
    if "q_u8" in f:
        f["q"] = f["q_u8"].astype(np.float32)
    for key in ("k", "seed", "ncmps", "m", "n_layers"):
        if key in f:
            f[key] = int(f[key])
    f["cmd"] = str(f["cmd"])
    f["metric"] = str(f["metric"])
    if "n_layers" in f:
        f["layers"] = [(f["layer%d_off" % g], f["layer%d_adj" % g]) for g in range(f["n_layers"])]
    return f


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def same_pools(got, fx):
    """True when a result's pools equal the fixture's (full arrays or digests)."""
    for key in ("ids", "dists", "flags"):
        if key in fx:
            if not np.array_equal(np.ascontiguousarray(got[key]).view(np.uint8), np.ascontiguousarray(fx[key]).view(np.uint8)):
                return False
        elif sha(got[key]) != str(fx[key + "_sha256"]):
            return False
    return True
