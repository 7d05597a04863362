"""Readers and writers of the reference's file formats, plus binary forms.

- Vectors: ``.fvecs`` (per row: int32 d, d float32), ``.bvecs`` (int32 d, d
  bytes; at most 10^7 rows, as IODelegator::loadBvec10m reads,
  iodelegator.cpp:319-385) and ``.txt`` ("rows cols" then the values,
  IODelegator::loadMatrix, :186-220), dispatched by extension as
  IODelegator::load_refSet (:159-182).  The binary forms are memory-mapped.
- k-NN graphs: the text format "n k" then "i k id..." per row
  (abstractmerge.cpp:278-291, read by IODelegator::loadKNNGraph,
  iodelegator.cpp:65-102) and a binary form ("NNMK", u32 version 1, u32 n,
  u32 k, n x k u32 ids) that loads by memory map.
- H-Merge hierarchies: the text format of lynndescent.cpp:625-638 ("rows"
  then "i n ids..." per row, layer after layer), read by
  LySearch::loadGraphs (lysearch.cpp:112-186); layers as (offsets, ids).
"""
import os

import numpy as np

KNN_MAGIC = b"NNMK"


def read_vecs(path):
    """float32 matrix of a .fvecs, .bvecs or .txt file."""
    if path.endswith(".txt"):
        toks = open(path).read().split()
        r, c = int(round(float(toks[0]))), int(round(float(toks[1])))
        return np.array(toks[2:2 + r * c], np.float32).reshape(r, c)
    if path.endswith(".fvecs"):
        raw = np.memmap(path, np.int32, "r")
        d = int(raw[0])
        rows = raw.reshape(-1, d + 1)
        return np.ascontiguousarray(rows[:, 1:]).view(np.float32)
    if path.endswith(".bvecs"):
        raw = np.memmap(path, np.uint8, "r")
        d = int(raw[:4].view(np.int32)[0])
        rows = raw.reshape(-1, d + 4)[:10_000_000]
        return rows[:, 4:].astype(np.float32)
    raise ValueError("unknown vector format: " + path)


def write_fvecs(path, x):
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty((x.shape[0], x.shape[1] + 1), np.int32)
    out[:, 0] = x.shape[1]
    out[:, 1:] = x.view(np.int32)
    out.tofile(path)


def write_bvecs(path, x):
    x = np.asarray(x)
    out = np.empty((x.shape[0], x.shape[1] + 4), np.uint8)
    out[:, :4] = np.frombuffer(np.int32(x.shape[1]).tobytes(), np.uint8)
    out[:, 4:] = x.astype(np.uint8)
    out.tofile(path)


def write_knn_text(path, ids):
    n, k = ids.shape
    with open(path, "w") as f:
        f.write("%d %d\n" % (n, k))
        for i in range(n):
            f.write("%d %d %s \n" % (i, k, " ".join(str(int(v)) for v in ids[i])))


def write_knn_bin(path, ids):
    ids = np.ascontiguousarray(ids, np.uint32)
    with open(path, "wb") as f:
        f.write(KNN_MAGIC)
        f.write(np.array([1, ids.shape[0], ids.shape[1]], np.uint32).tobytes())
        f.write(ids.tobytes())


def read_knn(path):
    """n x k uint32 ids of a k-NN graph file, text or binary."""
    with open(path, "rb") as f:
        head = f.read(16)
    if head[:4] == KNN_MAGIC:
        ver, n, k = np.frombuffer(head[4:16], np.uint32)
        if ver != 1:
            raise ValueError("unknown graph version %d" % ver)
        return np.array(np.memmap(path, np.uint32, "r", 16, (int(n), int(k))))
    toks = open(path).read().split()
    n, k = int(toks[0]), int(toks[1])
    ids = np.zeros((n, k), np.uint32)
    pos = 2
    for i in range(n):
        num = int(toks[pos + 1])
        row = toks[pos + 2:pos + 2 + num]
        ids[i, :min(k, num)] = np.array(row[:k], np.uint32)
        pos += 2 + num
    return ids


def write_layers_text(path, layers):
    with open(path, "w") as f:
        for off, adj in layers:
            rows = len(off) - 1
            f.write("%d\n" % rows)
            for i in range(rows):
                nb = adj[int(off[i]):int(off[i + 1])]
                f.write("%d %d %s\n" % (i, len(nb), " ".join(str(int(v)) for v in nb)))


def read_layers_text(path):
    toks = open(path).read().split()
    pos, layers = 0, []
    while pos < len(toks):
        rows = int(toks[pos])
        pos += 1
        off = np.zeros(rows + 1, np.uint64)
        adj = []
        for i in range(rows):
            num = int(toks[pos + 1])
            adj.extend(int(t) for t in toks[pos + 2:pos + 2 + num])
            pos += 2 + num
            off[i + 1] = off[i] + num
        layers.append((off, np.array(adj, np.uint32)))
    return layers


def file_size(path):
    return os.path.getsize(path)
