"""Row-sharded SpMV across ranks (one process per GPU): XAMG's NODE layer.

A square matrix is split into contiguous row blocks, one per rank, by XAMG's
rule (part.h:98-110: n/world rows each, the last rank takes the remainder).
Each rank keeps its rows as a diagonal block (its own columns, renumbered
from 0) and one off-diagonal block per other rank that owns some of its
columns (columns renumbered into that rank's halo: the sorted distinct remote
columns, XAMG's compress, csr_matrix.inl:87-170). One SpMV is

    y = A_diag x_own            (Ax_y)
    y += A_offd[j] x_halo[j]    (Axpy, for each other rank j in rank order)

after a halo exchange of the needed x rows (nv values each), as
blas2.h:46-147 orders it, so every row is summed diagonal entries first, then
each remote block's entries, each in CSR order.

The plan is host logic (numpy); the exchange runs over torch.distributed (NCCL
between GPUs, gloo on the CPU) and the block products run on a `compute`
object: the library's XAMG_b200_spmv on device arrays, or the CPU oracle in
the tests.
"""
import numpy as np


def row_blocks(n, world):
    """Start row of each rank and n at the end (part.h:98-110)."""
    b = n // world
    starts = [r * b for r in range(world)]
    return np.array(starts + [n], dtype=np.int64)


def _csr(rows, cols, vals, nrows):
    row = np.zeros(nrows + 1, np.uint32)
    np.add.at(row, rows + 1, 1)
    return np.cumsum(row, dtype=np.uint32), cols.astype(np.uint32), vals.astype(np.float64)


class ShardPlan:
    """This rank's diagonal and off-diagonal blocks and its halo lists."""

    def __init__(self, row, col, val, world, rank):
        row = np.asarray(row, np.int64)
        col = np.asarray(col, np.int64)
        val = np.asarray(val, np.float64)
        n = len(row) - 1
        self.world, self.rank, self.n = world, rank, n
        self.starts = row_blocks(n, world)
        r0, r1 = int(self.starts[rank]), int(self.starts[rank + 1])
        self.r0, self.nl = r0, r1 - r0
        e0, e1 = int(row[r0]), int(row[r1])
        lrow = np.repeat(np.arange(self.nl), np.diff(row[r0:r1 + 1]))
        c, v = col[e0:e1], val[e0:e1]
        owner = np.searchsorted(self.starts, c, side="right") - 1
        mine = owner == rank
        self.diag = _csr(lrow[mine], c[mine] - r0, v[mine], self.nl)
        self.offd, self.halo = {}, {}
        for j in range(world):
            if j == rank:
                continue
            sel = owner == j
            if not sel.any():
                continue
            h = np.unique(c[sel])
            self.halo[j] = h  # global columns received from rank j
            self.offd[j] = _csr(lrow[sel], np.searchsorted(h, c[sel]), v[sel], self.nl)
        self.send = {}  # filled by exchange_lists: local rows each rank needs

    def exchange_lists(self, dist):
        """Tell every rank which of its rows this rank needs (all_gather)."""
        lists = [None] * self.world
        dist.all_gather_object(lists, {j: h.tolist() for j, h in self.halo.items()})
        for j in range(self.world):
            if j != self.rank and self.rank in lists[j]:
                self.send[j] = np.asarray(lists[j][self.rank], np.int64) - self.r0
        return self


def spmv(plan, x_local, nv, compute, dist, torch):
    """y = A x for this rank's rows; x_local is a [nl][nv] tensor of this
    rank's x rows on the device the process group uses."""
    reqs, bufs = [], {}
    for j, h in plan.halo.items():
        bufs[j] = torch.empty(len(h), nv, dtype=x_local.dtype, device=x_local.device)
        reqs.append(dist.irecv(bufs[j], src=j))
    for j, idx in plan.send.items():
        out = x_local[torch.as_tensor(idx, device=x_local.device)].contiguous()
        reqs.append(dist.isend(out, dst=j))
    y = compute.ax_y(plan.diag, x_local, plan.nl, nv)
    for r in reqs:
        r.wait()
    for j in sorted(plan.offd):
        y = compute.axpy(plan.offd[j], bufs[j], y, plan.nl, nv)
    return y


class LibraryCompute:
    """Block products on the GPU through XAMG_b200_spmv (FP64, 32-bit
    columns) on device copies of the blocks, on the library's stream (make it
    torch's current stream around spmv)."""

    def __init__(self, X, torch):
        self.X, self.torch, self.keep = X, torch, {}

    def _desc(self, blk, ncols):
        # keyed by the block's identity; the entry keeps the block alive so
        # that its id is not reused by another block
        key = id(blk)
        if key not in self.keep:
            t = self.torch
            r, c, v = (t.from_numpy(a).cuda() for a in blk)
            d = self.X.Csr(len(blk[0]) - 1, ncols, len(blk[1]), r.data_ptr(), c.data_ptr(),
                           v.data_ptr(), 4, 0)
            self.keep[key] = (d, r, c, v, blk)
        return self.keep[key][0]

    def ax_y(self, blk, x, nrows, nv):
        import ctypes as C
        y = self.torch.empty(nrows, nv, dtype=self.torch.float64, device=x.device)
        d = self._desc(blk, x.shape[0])
        self.X.call("XAMG_b200_spmv", C.byref(d), x.data_ptr(), y.data_ptr(), nv, 0,
                    self.X.stream())
        return y

    def axpy(self, blk, x, y, nrows, nv):
        import ctypes as C
        d = self._desc(blk, x.shape[0])
        self.X.call("XAMG_b200_spmv", C.byref(d), x.data_ptr(), y.data_ptr(), nv, 1,
                    self.X.stream())
        return y

    def dot(self, a, c, nv):
        """Partial (a, c) per right-hand side over this rank's rows
        (XAMG_b200_dot, the library's fixed reduction order), as a device
        tensor."""
        import numpy as np
        a, c = a.contiguous(), c.contiguous()
        out = np.zeros(nv)
        self.X.call("XAMG_b200_dot", a.shape[0], nv, a.data_ptr(), c.data_ptr(),
                    out.ctypes.data, self.X.stream())
        return self.torch.from_numpy(out).to(a.device)


def rank_sum(dist, torch, local, world):
    """The global sum of every rank's partial values (nv of them), added in
    rank order on every rank, so that all ranks hold the same bits (XAMG's
    allreduce also hands every rank one result, shm_allreduce.h:37-164)."""
    if world == 1:
        return local
    parts = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(parts, local.contiguous())
    s = parts[0].clone()
    for p in parts[1:]:
        s = s + p
    return s


def bicgstab(plan, b, x, nv, compute, dist, torch, dinv, rel_tol=1e-8, max_iters=1000):
    """Jacobi-preconditioned BiCGStab (the iteration of
    merged_pbicgstab.inl:44-225 with M = D^-1) on this rank's rows: one halo
    exchange per SpMV, and the dot products as per-rank partial sums (the
    compute object's `dot`) added in rank order (rank_sum). b, x: [nl][nv]
    tensors of this rank's rows; dinv: [nl] inverse diagonal. Converged
    right-hand sides are frozen (their alpha and omega set to zero), as XAMG's
    per-RHS iconv mask does (merged_bicgstab.inl:173-174,198-199). Returns x,
    the iteration count and the final relative residuals."""
    W = plan.world

    def gdot(a, c):
        return rank_sum(dist, torch, compute.dot(a, c, nv), W)

    def A(v):
        return spmv(plan, v, nv, compute, dist, torch)

    def M(v):
        return v * dinv[:, None]

    r0 = b - A(x)
    r, p = r0.clone(), r0.clone()
    rho = gdot(r0, r0)
    res0 = rho.clone()
    iconv = torch.ones(nv, dtype=b.dtype, device=b.device)
    it = 0
    rel = torch.ones_like(rho)
    while it < max_iters:
        it += 1
        p_ = M(p)
        v = A(p_)
        alpha = rho / gdot(r0, v) * iconv
        s = r - alpha * v
        s_ = M(s)
        t = A(s_)
        omega = gdot(t, s) / gdot(t, t) * iconv
        x = x + alpha * p_ + omega * s_
        r = s - omega * t
        rr = gdot(r, r)
        rel = torch.sqrt(rr / res0)
        conv = (rel <= rel_tol) | (res0 == 0)
        iconv = iconv * (~conv).to(iconv.dtype)
        if bool(conv.all()):
            break
        rho_new = gdot(r0, r)
        beta = (rho_new / rho) * (alpha / omega)
        beta = torch.where(iconv > 0, beta, torch.zeros_like(beta))
        p = r + beta * (p - omega * v)
        rho = rho_new
    return x, it, rel

