"""Row-sharded apply over world_size 2 gloo ranks on CPU: the partition,
the all-gather of x and the assembled y against the unsharded product."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tectosaur_b200.sharded import RowShardedOp, row_ranges


class DenseRows:
    """Stand-in operator: block rows [r0, r1) of a dense matrix (the GPU
    operator's row_range restriction), applied on CPU tensors."""

    def __init__(self, A, row_range, k=9):
        r0, r1 = row_range
        self.A = torch.from_numpy(A[r0 * k:r1 * k])

    def dot(self, x):
        return self.A @ x


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_tris, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(0)
        A = rng.standard_normal((9 * n_tris, 9 * n_tris))
        x = rng.standard_normal(9 * n_tris)
        op = RowShardedOp(lambda rr: DenseRows(A, rr), n_tris, rank, world)
        x_local = torch.from_numpy(x[op.r0 * 9:op.r1 * 9].copy())
        y_local = op.dot(x_local)
        ys = [None] * world
        dist.all_gather_object(ys, (op.r0, op.r1, y_local.numpy()))
        if rank == 0:
            y = np.concatenate([v for _, _, v in sorted(ys, key=lambda t: t[0])])
            out_q.put(float(np.abs(y - A @ x).max() / np.abs(A @ x).max()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_tris", [10, 7])
def test_row_sharded_apply_two_ranks(n_tris):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n_tris, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) < 1e-13


def test_row_ranges():
    assert row_ranges(10, 3) == [(0, 3), (3, 7), (7, 10)]
    r = row_ranges(59858, 8)
    assert r[0][0] == 0 and r[-1][1] == 59858
    sizes = [e - s for s, e in r]
    assert max(sizes) - min(sizes) <= 1


def _pairs_worker(rank, world, port, out_q):
    """Each rank finds its row shard's near pairs the way the row_range
    operator does (search over all observation triangles, keep its rows);
    rank 0 checks that the shards stack up to the full operator's pairs."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from helpers import bumpy_mesh
        from tectosaur_b200.nearfield.nearfield_op import nearfield_pairs
        pts, tris = bumpy_mesh(13, seed=4)
        n = tris.shape[0]
        r0, r1 = row_ranges(n, world)[rank]
        idx = np.arange(n)
        mine = nearfield_pairs(pts, tris, idx, idx, 2.5, row_range=(r0, r1))
        got = [None] * world
        dist.all_gather_object(got, (r0, mine))
        if rank == 0:
            full = nearfield_pairs(pts, tris, idx, idx, 2.5)
            ok = True
            for c in full:
                recs = np.concatenate([m[c][0] for _, m in sorted(got, key=lambda t: t[0])])
                dofs = np.concatenate([m[c][1] + [r, 0] for r, m in sorted(got, key=lambda t: t[0])])
                ok = ok and np.array_equal(recs, full[c][0]) and np.array_equal(dofs, full[c][1])
            out_q.put(bool(ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_row_shards_hold_the_full_operators_pairs(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_pairs_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True
