"""Row-sharded operator apply over several ranks (one process per GPU).

The apply shards by observation rows: rank r owns a contiguous range of
observation triangles -- its rows of y, its farfield observation tiles and
its BSR block rows -- and needs the whole input x.  One exchange per apply:
an all-gather of the ranks' slices of x (NCCL over NVLink between GPUs; any
torch.distributed backend works, gloo on CPU in the tests), no reduction
(the outputs are disjoint).  The reference is single-device; this is the
natural multi-GPU layout of its `RegularizedSparseIntegralOp.dot`
(ops/sparse_integral_op.py:35-55).

A shard is the full operator's rows, not an operator over the shard's
triangles: ``RegularizedSparseIntegralOp(..., row_range=(r0, r1))`` runs the
near-pair search over all observation triangles and keeps the pairs of its
rows, so every rank holds exactly the blocks of the one global operator (the
reference's leaf test reads radii by octree position, so a search over the
shard's triangles alone could move pairs at the threshold across the
near/far line).  An FMM farfield shard likewise keeps the whole observation
set's trees and interaction lists and evaluates only the observation nodes
that hold its rows (their P2P and M2L/M2P entries, L2L chain and L2P); every
rank computes all source moments (P2M, M2M: a few per cent of an apply), so
the only exchange stays the all-gather of x, and the shard's rows are the
unsharded FMM's bit for bit.
"""
import numpy as np


def row_ranges(n_rows, world):
    """Contiguous, balanced [start, end) row ranges of n_rows over world ranks."""
    edges = np.linspace(0, n_rows, world + 1).round().astype(np.int64)
    return [(int(edges[r]), int(edges[r + 1])) for r in range(world)]


class RowShardedOp:
    """This rank's rows of y = A x.

    op_factory(row_range) builds block rows [r0, r1) of the global operator
    (all sources), e.g.
    ``lambda rr: RegularizedSparseIntegralOp(..., row_range=rr)``; its
    ``dot`` takes the full x (9 n_tris values).  ``dot(x_local)`` takes this
    rank's slice of x and returns this rank's slice of y."""

    def __init__(self, op_factory, n_tris, rank, world, group=None, dofs_per_tri=9):
        self.rank, self.world, self.group = rank, world, group
        self.k = dofs_per_tri
        self.ranges = row_ranges(n_tris, world)
        self.r0, self.r1 = self.ranges[rank]
        self.n_tris = n_tris
        self.max_rows = max(e - s for s, e in self.ranges)
        self.op = op_factory((self.r0, self.r1))

    def gather_x(self, x_local):
        """All-gather the ranks' slices into the full x (padded equal-size
        all_gather_into_tensor, then the padding is dropped)."""
        import torch
        import torch.distributed as dist
        pad = torch.zeros(self.max_rows * self.k, dtype=x_local.dtype, device=x_local.device)
        pad[: x_local.numel()] = x_local
        out = torch.empty(self.world * self.max_rows * self.k, dtype=x_local.dtype,
                          device=x_local.device)
        dist.all_gather_into_tensor(out, pad, group=self.group)
        parts = [out[r * self.max_rows * self.k:(r * self.max_rows + e - s) * self.k]
                 for r, (s, e) in enumerate(self.ranges)]
        return torch.cat(parts)

    def dot(self, x_local):
        return self.op.dot(self.gather_x(x_local))
