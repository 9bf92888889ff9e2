"""The row-sharded path on the GPU (one GPU here): every rank's diagonal and
off-diagonal blocks (shard.ShardPlan) multiplied in one process through
XAMG_b200_spmv, the halo rows taken directly from x, must equal the oracle's
split product bit for bit; the sharded BiCGStab on one rank must equal its
one-process replay."""
import os
import sys

import numpy as np
import pytest

from test_shard import matrix, split_reference

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world,nv", [(1, 2), (3, 4), (4, 8)])
def test_shard_blocks_on_gpu(gpu, world, nv):
    import torch
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "softx-d-21-00014_b200"))
    import shard
    n, seed = 2000, 5
    row, col, val = matrix(n, seed)
    x = np.random.default_rng(seed + 1).standard_normal((n, nv))
    st = torch.cuda.ExternalStream(gpu.stream())
    comp = shard.LibraryCompute(gpu, torch)
    out = []
    with torch.cuda.stream(st):
        for r in range(world):
            p = shard.ShardPlan(row, col, val, world, r)
            xr = torch.from_numpy(np.ascontiguousarray(x[p.r0:p.r0 + p.nl])).cuda()
            y = comp.ax_y(p.diag, xr, p.nl, nv)
            for j in sorted(p.offd):
                xh = torch.from_numpy(np.ascontiguousarray(x[p.halo[j]])).cuda()
                y = comp.axpy(p.offd[j], xh, y, p.nl, nv)
            torch.cuda.synchronize()
            out.append(y.cpu().numpy())
    got = np.concatenate(out)
    assert got.tobytes() == split_reference(row, col, val, x, nv, world).tobytes()


def test_sharded_bicgstab_one_rank_gpu(gpu, oracle):
    """shard.bicgstab on the GPU (block products and dot products through the
    library, vector updates in torch on the library's stream), one rank:
    equal bit for bit to the one-process replay with the oracle in the
    kernels' reduction order."""
    import torch
    import shard
    from test_shard import laplacian, replay_bicgstab
    row, col, val = laplacian(10, 9, 8, 5)
    n, nv = len(row) - 1, 4
    b = np.random.default_rng(6).uniform(-1, 1, (n, nv))
    plan = shard.ShardPlan(row, col, val, 1, 0)
    d = np.array([val[row[i]:row[i + 1]][col[row[i]:row[i + 1]] == i][0] for i in range(n)])
    st = torch.cuda.ExternalStream(gpu.stream())
    with torch.cuda.stream(st):
        bl = torch.from_numpy(b).cuda()
        x, it, rel = shard.bicgstab(plan, bl, torch.zeros_like(bl), nv,
                                    shard.LibraryCompute(gpu, torch), None, torch,
                                    torch.from_numpy(1.0 / d).cuda(), 1e-8, 500)
        torch.cuda.synchronize()
    oracle.set_reduction(1)
    try:
        xr, itr = replay_bicgstab(row, col, val, b, nv, 1, 1e-8, 500)
    finally:
        oracle.set_reduction(0)
    assert it == itr
    assert x.cpu().numpy().tobytes() == xr.tobytes()
