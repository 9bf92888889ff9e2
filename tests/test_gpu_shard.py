"""The row-sharded SpMV's block products on the GPU: every rank's diagonal
and off-diagonal blocks (shard.ShardPlan) multiplied in one process through
XAMG_b200_spmv, the halo rows taken directly from x (no exchange: one GPU),
must equal the oracle's split product bit for bit."""
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
