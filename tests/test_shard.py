"""Row-sharded SpMV (XAMG's NODE layer, softx-d-21-00014_b200/shard.py) with
gloo ranks on the CPU (spawned processes, rendezvous on 127.0.0.1) and the
oracle computing the block products: the halo exchange and the block plan
must give, bit for bit, what one process computes with the same split
(diagonal block first, then each remote rank's block in rank order), and the
unsplit product to rounding."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def matrix(n, seed):
    """Banded rows (3-D 7-point pattern) plus a few far-off columns."""
    rng = np.random.default_rng(seed)
    nx, ny = 11, 9
    row, cols, vals = [0], [], []
    for i in range(n):
        c = {i}
        for o in (1, nx, nx * ny):
            if i - o >= 0:
                c.add(i - o)
            if i + o < n:
                c.add(i + o)
        if i % 7 == 0:
            c.update(int(v) for v in rng.integers(0, n, 3))
        c = sorted(c)
        cols += c
        vals += rng.standard_normal(len(c)).tolist()
        row.append(len(cols))
    return np.array(row, np.uint32), np.array(cols, np.uint32), np.array(vals)


class OracleCompute:
    def __init__(self):
        import oracle_py as O
        self.O = O

    def ax_y(self, blk, x, nrows, nv):
        import torch
        y = self.O.csr_ax_y(blk[0], blk[1], blk[2], x.numpy().ravel(), nv, ncols=x.shape[0])
        return torch.from_numpy(y).reshape(nrows, nv)

    def axpy(self, blk, x, y, nrows, nv):
        import torch
        out = self.O.csr_ax_y(blk[0], blk[1], blk[2], x.numpy().ravel(), nv, ncols=x.shape[0],
                              axpy_y=y.numpy().ravel())
        return torch.from_numpy(out).reshape(nrows, nv)


def split_reference(row, col, val, x, nv, world):
    """One process, the same split and order."""
    import shard
    O = OracleCompute()
    out = []
    for r in range(world):
        p = shard.ShardPlan(row, col, val, world, r)
        xr = x[p.r0:p.r0 + p.nl]
        import torch
        y = O.ax_y(p.diag, torch.from_numpy(xr), p.nl, nv)
        for j in sorted(p.offd):
            y = O.axpy(p.offd[j], torch.from_numpy(x[p.halo[j]]), y, p.nl, nv)
        out.append(y.numpy())
    return np.concatenate(out)


def _rank_main(rank, world, port, n, nv, seed, out_dir):
    sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import torch
    import torch.distributed as dist
    import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    row, col, val = matrix(n, seed)
    x = np.random.default_rng(seed + 1).standard_normal((n, nv))
    plan = shard.ShardPlan(row, col, val, world, rank).exchange_lists(dist)
    xl = torch.from_numpy(np.ascontiguousarray(x[plan.r0:plan.r0 + plan.nl]))
    y = shard.spmv(plan, xl, nv, OracleCompute(), dist, torch)
    parts = [None] * world
    dist.all_gather_object(parts, y.numpy())
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        np.save(os.path.join(out_dir, "y.npy"), np.concatenate(parts))


def test_row_blocks_follow_xamg():
    import shard
    assert shard.row_blocks(10, 3).tolist() == [0, 3, 6, 10]
    assert shard.row_blocks(7, 1).tolist() == [0, 7]


@pytest.mark.parametrize("world,nv", [(2, 1), (3, 4)])
def test_sharded_spmv_gloo(tmp_path, world, nv):
    import torch.multiprocessing as mp
    n, seed = 1500, 11
    mp.start_processes(_rank_main, args=(world, _free_port(), n, nv, seed, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    y = np.load(tmp_path / "y.npy")
    row, col, val = matrix(n, seed)
    x = np.random.default_rng(seed + 1).standard_normal((n, nv))
    ref = split_reference(row, col, val, x, nv, world)
    assert y.tobytes() == ref.tobytes()
    import scipy.sparse as sp
    full = sp.csr_matrix((val, col, row), shape=(n, n)) @ x
    assert np.abs(y - full).max() <= 1e-12 * np.abs(full).max()
