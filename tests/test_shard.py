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


# --- the distributed BiCGStab over row shards --------------------------------

def laplacian(nx, ny, nz, seed):
    """7-point variable-coefficient diffusion (diagonally dominant), sorted rows."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    kap = np.exp(rng.standard_normal(n) * 0.5)
    row, cols, vals = [0], [], []
    for i in range(n):
        x, y, z = i % nx, (i // nx) % ny, i // (nx * ny)
        nb = []
        for d, ok in ((-nx * ny, z > 0), (-nx, y > 0), (-1, x > 0), (1, x < nx - 1),
                      (nx, y < ny - 1), (nx * ny, z < nz - 1)):
            if ok:
                nb.append(i + d)
        ent = {j: -0.5 * (kap[i] + kap[j]) for j in nb}
        ent[i] = -sum(ent.values()) + 0.1 * kap[i]
        for j in sorted(ent):
            cols.append(j)
            vals.append(ent[j])
        row.append(len(cols))
    return np.array(row, np.uint32), np.array(cols, np.uint32), np.array(vals)


class OracleDotCompute(OracleCompute):
    def dot(self, a, c, nv):
        import torch
        return torch.from_numpy(self.O.dot(a.numpy().ravel(), c.numpy().ravel(), nv))


def replay_bicgstab(row, col, val, b, nv, world, tol, max_iters):
    """One process playing every rank in turn: the split SpMV, per-rank
    partial dots added in rank order, and the same recurrences as
    shard.bicgstab."""
    import torch
    import shard
    O = OracleDotCompute()
    plans = [shard.ShardPlan(row, col, val, world, r) for r in range(world)]
    n = len(row) - 1
    dg = np.array([val[row[i]:row[i + 1]][col[row[i]:row[i + 1]] == i][0] for i in range(n)])
    dinv = [torch.from_numpy(1.0 / dg[p.r0:p.r0 + p.nl]) for p in plans]

    def A(vs):
        full = torch.cat(vs).numpy()
        out = []
        for p in plans:
            y = O.ax_y(p.diag, torch.from_numpy(full[p.r0:p.r0 + p.nl]), p.nl, nv)
            for j in sorted(p.offd):
                y = O.axpy(p.offd[j], torch.from_numpy(full[p.halo[j]]), y, p.nl, nv)
            out.append(y)
        return out

    def gdot(a, c):
        s = O.dot(a[0], c[0], nv)
        for r in range(1, world):
            s = s + O.dot(a[r], c[r], nv)
        return s

    def lin(f, *vs):
        return [f(*z) for z in zip(*vs)]

    bs = [torch.from_numpy(np.ascontiguousarray(b[p.r0:p.r0 + p.nl])) for p in plans]
    xs = [torch.zeros_like(t) for t in bs]
    Ax = A(xs)
    r0 = lin(lambda bb, ax: bb - ax, bs, Ax)
    r = [t.clone() for t in r0]
    p = [t.clone() for t in r0]
    rho = gdot(r0, r0)
    res0 = rho.clone()
    iconv = torch.ones(nv, dtype=torch.float64)
    it = 0
    while it < max_iters:
        it += 1
        p_ = [pp * d[:, None] for pp, d in zip(p, dinv)]
        v = A(p_)
        alpha = rho / gdot(r0, v) * iconv
        s = lin(lambda rr, vv: rr - alpha * vv, r, v)
        s_ = [ss * d[:, None] for ss, d in zip(s, dinv)]
        t = A(s_)
        omega = gdot(t, s) / gdot(t, t) * iconv
        xs = lin(lambda xx, pp, ss: xx + alpha * pp + omega * ss, xs, p_, s_)
        r = lin(lambda ss, tt: ss - omega * tt, s, t)
        rel = torch.sqrt(gdot(r, r) / res0)
        conv = (rel <= tol) | (res0 == 0)
        iconv = iconv * (~conv).to(iconv.dtype)
        if bool(conv.all()):
            break
        rho_new = gdot(r0, r)
        beta = (rho_new / rho) * (alpha / omega)
        beta = torch.where(iconv > 0, beta, torch.zeros_like(beta))
        p = lin(lambda rr, pp, vv: rr + beta * (pp - omega * vv), r, p, v)
        rho = rho_new
    return torch.cat(xs).numpy(), it


def _solve_main(rank, world, port, grid, nv, seed, out_dir):
    sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import torch
    import torch.distributed as dist
    import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    row, col, val = laplacian(*grid, seed)
    n = len(row) - 1
    b = np.random.default_rng(seed + 1).uniform(-1, 1, (n, nv))
    plan = shard.ShardPlan(row, col, val, world, rank).exchange_lists(dist)
    d = np.array([val[row[i]:row[i + 1]][col[row[i]:row[i + 1]] == i][0]
                  for i in range(plan.r0, plan.r0 + plan.nl)])
    bl = torch.from_numpy(np.ascontiguousarray(b[plan.r0:plan.r0 + plan.nl]))
    x, it, rel = shard.bicgstab(plan, bl, torch.zeros_like(bl), nv, OracleDotCompute(), dist,
                                torch, torch.from_numpy(1.0 / d), 1e-8, 500)
    parts = [None] * world
    dist.all_gather_object(parts, (x.numpy(), it, rel.numpy()))
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        np.save(os.path.join(out_dir, "x.npy"), np.concatenate([q[0] for q in parts]))
        np.save(os.path.join(out_dir, "it.npy"), np.array([q[1] for q in parts]))


@pytest.mark.parametrize("world,nv", [(2, 1), (3, 4)])
def test_sharded_bicgstab_gloo(tmp_path, world, nv):
    """Every rank ends after the same iterations; the gathered solution
    equals the one-process replay of the same split bit for bit and solves
    the system to the tolerance."""
    import torch.multiprocessing as mp
    grid, seed = (9, 8, 7), 21
    mp.start_processes(_solve_main, args=(world, _free_port(), grid, nv, seed, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    x = np.load(tmp_path / "x.npy")
    its = np.load(tmp_path / "it.npy")
    assert len(set(its.tolist())) == 1
    row, col, val = laplacian(*grid, seed)
    n = len(row) - 1
    b = np.random.default_rng(seed + 1).uniform(-1, 1, (n, nv))
    xr, itr = replay_bicgstab(row, col, val, b, nv, world, 1e-8, 500)
    assert itr == its[0]
    assert x.tobytes() == xr.tobytes()
    import scipy.sparse as sp
    Am = sp.csr_matrix((val, col, row), shape=(n, n))
    rel = np.linalg.norm(b - Am @ x, axis=0) / np.linalg.norm(b, axis=0)
    assert rel.max() <= 2e-8
