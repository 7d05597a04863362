"""Leaf-sharded multi-GPU build of one k-NN graph (fast tier): one process
per GPU under torchrun, ranks over torch.distributed (NCCL on GPUs, gloo in
the CPU tests).

The reference's merges build independent sub-graphs and then merge them
(Smerge::buildKGraph, smerge.cpp:46-91).  Here the leaves of a multi-leaf
build are split over the ranks in contiguous blocks; each rank builds its
block's leaves (nnm_build_leaves_dev, no communication); one all-gather
then gives every rank every leaf's graph -- the one data-path exchange --
and every rank runs the merge of the prebuilt leaves
(nnm_merge_prebuilt_dev).  The merge is deterministic, so all ranks hold the
same graph; it is not split over ranks (its NN-Descent iterations would
need an exchange of pools and proposals per iteration).  With one rank this
is exactly nnm_merge_leaves_dev.

The engine calls are injected (`build`, `merge`) so that the partition and
exchange logic runs on CPU with a stand-in builder.
"""
import numpy as np


def leaf_blocks(nleaf, world):
    """Contiguous blocks of leaves per rank, sizes differing by at most one:
    [(first leaf, end leaf)] for ranks 0 .. world-1 (empty for ranks beyond
    the leaf count)."""
    out = []
    for r in range(world):
        a = (nleaf * r) // world
        b = (nleaf * (r + 1)) // world
        out.append((a, b))
    return out


def row_offsets(leaf_sizes):
    off = np.zeros(len(leaf_sizes) + 1, np.int64)
    off[1:] = np.cumsum(leaf_sizes)
    return off


class ShardedBuild:
    """One multi-leaf build over the ranks of `dist` (torch.distributed,
    initialised by the caller; rank/world from it).

    build(x_block, sizes_block, leaf0) -> (ids, dists): the leaf graphs of a
        block (ids local to the block's rows), as torch tensors on `device`;
    merge(x, sizes, ids, dists) -> result of merging prebuilt leaves.
    """

    def __init__(self, dist, build, merge, device):
        self.dist, self.build, self.merge, self.device = dist, build, merge, device
        self.rank = dist.get_rank() if dist is not None else 0
        self.world = dist.get_world_size() if dist is not None else 1

    def run(self, x, leaf_sizes, k):
        import torch
        sizes = [int(s) for s in leaf_sizes]
        off = row_offsets(sizes)
        blocks = leaf_blocks(len(sizes), self.world)
        a, b = blocks[self.rank]
        r0, r1 = int(off[a]), int(off[b])
        ids = torch.empty((int(off[-1]), k), dtype=torch.int32, device=self.device)
        dists = torch.empty((int(off[-1]), k), dtype=torch.float32, device=self.device)
        if b > a:
            bi, bd = self.build(x[r0:r1], sizes[a:b], a)
            ids[r0:r1] = bi + r0  # block-local ids -> ids of the whole set
            dists[r0:r1] = bd
        if self.world > 1:
            # the exchange: every rank's block to every rank (blocks differ in
            # size, so each is sent as a padded slice of the largest)
            rows = [int(off[bb] - off[aa]) for aa, bb in blocks]
            m = max(rows)
            send_i = torch.zeros((m, k), dtype=torch.int32, device=self.device)
            send_d = torch.zeros((m, k), dtype=torch.float32, device=self.device)
            send_i[: r1 - r0] = ids[r0:r1]
            send_d[: r1 - r0] = dists[r0:r1]
            got_i = [torch.empty_like(send_i) for _ in range(self.world)]
            got_d = [torch.empty_like(send_d) for _ in range(self.world)]
            self.dist.all_gather(got_i, send_i)
            self.dist.all_gather(got_d, send_d)
            for r, (aa, bb) in enumerate(blocks):
                lo, hi = int(off[aa]), int(off[bb])
                ids[lo:hi] = got_i[r][: hi - lo]
                dists[lo:hi] = got_d[r][: hi - lo]
        return self.merge(x, sizes, ids, dists)


def engine_build(ctx, k, **kw):
    """build/merge functions over the library (device tensors)."""
    import torch

    def build(xb, sizes, leaf0):
        xb = xb.contiguous()
        n, d = xb.shape
        ids = torch.empty((n, k), dtype=torch.int32, device=xb.device)
        ds = torch.empty((n, k), dtype=torch.float32, device=xb.device)
        ctx.build_leaves_dev(xb.data_ptr(), n, d, k, sizes, ids.data_ptr(), ds.data_ptr(), leaf0=leaf0, **kw)
        return ids, ds

    def merge(x, sizes, ids, ds):
        n, d = x.shape
        oi = torch.empty((n, k), dtype=torch.int32, device=x.device)
        od = torch.empty((n, k), dtype=torch.float32, device=x.device)
        st = ctx.merge_prebuilt_dev(x.data_ptr(), n, d, k, sizes, ids.contiguous().data_ptr(),
                                    ds.contiguous().data_ptr(), oi.data_ptr(), od.data_ptr(), **kw)
        return oi, od, st

    return build, merge
