"""Learned coarse initial guess (the benchmark description's configuration 4).

For a fixed matrix, a small MLP (the library's XAMG_b200_mlp_*, BF16 on the
tcgen05 GEMM) maps a right-hand side restricted to a coarse AMG level to coarse
coefficients of the solution; prolongated to the fine grid they are the
initial guess of the Krylov solve. Training pairs come from the solver
itself. A guess is kept per right-hand side only if its initial residual is
below that of the zero guess (which stays the fallback).

Data plumbing (right-hand-side generation, norms, column selection) uses torch
tensors on the device; the restriction/prolongation SpMVs, the MLP and the
solves are the library's own kernels.
"""
import time

import numpy as np
import torch

import xamg_b200 as X


def gaussian_rhs(n_edge, nv, gen, nsrc=8):
    """[n][nv] float64 device tensor: each column a sum of nsrc Gaussian
    sources, centres uniform in the unit cube, widths uniform in [0.02, 0.1],
    amplitudes N(0, 1), on the grid points ((i+1)/(n+1), ...) ordered
    i + n*(j + n*k)."""
    dev = "cuda"
    c = torch.rand(nv, nsrc, 3, generator=gen, dtype=torch.float64).to(dev)
    w = (0.02 + 0.08 * torch.rand(nv, nsrc, generator=gen, dtype=torch.float64)).to(dev)
    a = torch.randn(nv, nsrc, generator=gen, dtype=torch.float64).to(dev)
    t = (torch.arange(n_edge, dtype=torch.float64, device=dev) + 1.0) / (n_edge + 1.0)
    inv = 1.0 / (2.0 * w * w)  # [nv, nsrc]
    # separable: exp(-|p - c|^2 / 2w^2) = ex(x) ey(y) ez(z)
    e = [torch.exp(-((t[None, None, :] - c[:, :, d, None]) ** 2) * inv[:, :, None])
         for d in range(3)]  # each [nv, nsrc, n]
    b = torch.einsum("gsk,gsj,gsi,gs->kjig", e[2], e[1], e[0], a)  # [z][y][x][nv]
    return b.reshape(-1, nv).contiguous()


class Transfer:
    """Composite restriction to / prolongation from level `level` with the
    FP64 transfer operators of a multigrid solver (XAMG_b200_solver_level_spmv
    with which = 1 for R_l, 2 for P_l)."""

    def __init__(self, S, level):
        self.S, self.level = S, level
        self.n = [S.level_info(l, 0)["nrows"] for l in range(level + 1)]

    def restrict(self, v, nv):
        for l in range(self.level):
            out = torch.empty(self.n[l + 1] * nv, dtype=torch.float64, device="cuda")
            self.S.level_spmv(l, 1, v.data_ptr(), out.data_ptr(), nv)
            v = out
        return v

    def prolong(self, v, nv):
        for l in range(self.level - 1, -1, -1):
            out = torch.empty(self.n[l] * nv, dtype=torch.float64, device="cuda")
            self.S.level_spmv(l, 2, v.data_ptr(), out.data_ptr(), nv)
            v = out
        return v


def pad128(n):
    return (n + 127) // 128 * 128


class LearnedGuess:
    """Training data, MLP and guess for one matrix."""

    def __init__(self, S64, level, hidden=1024, seed=0):
        self.T = Transfer(S64, level)
        self.nc = self.T.n[-1]
        self.np_ = pad128(self.nc)
        self.mlp = X.Mlp(self.np_, hidden, self.np_, seed)
        ones = torch.ones(self.T.n[0], dtype=torch.float64, device="cuda")
        self.w = self.T.restrict(ones, 1)  # row sums of the composite restriction

    def features(self, b, nv):
        """Scaled coarse right-hand sides [nv][np] (FP32) and the scales."""
        bc = self.T.restrict(b.reshape(-1), nv).reshape(self.nc, nv)
        s = bc.norm(dim=0).clamp_min(1e-300)
        F = torch.zeros(nv, self.np_, dtype=torch.float32, device="cuda")
        F[:, :self.nc] = (bc / s).T.float()
        return F, s

    def targets(self, x, s, nv):
        """Coarse coefficients of the solution: the composite restriction of x
        weighted to an average, scaled like the features."""
        xc = self.T.restrict(x.reshape(-1), nv).reshape(self.nc, nv) / self.w[:, None]
        Tt = torch.zeros(nv, self.np_, dtype=torch.float32, device="cuda")
        Tt[:, :self.nc] = (xc / s).T.float()
        return Tt

    def train(self, F, Tt, steps, batch=512, lr=1e-3, gen=None):
        n = F.shape[0]
        losses = []
        for _ in range(steps):
            idx = torch.randperm(n, generator=gen)[:batch].cuda()
            Fb, Tb = F[idx].contiguous(), Tt[idx].contiguous()
            losses.append(self.mlp.train_step(Fb.data_ptr(), Tb.data_ptr(), batch, lr))
        return losses

    def guess(self, b, nv, smooth=None):
        """Fine-grid initial guess [n][nv] for the right-hand sides b; with
        smooth (a callable taking and returning the guess) the prolongated
        guess is smoothed before use."""
        F, s = self.features(b, nv)
        rows = pad128(nv)
        Fp = torch.zeros(rows, self.np_, dtype=torch.float32, device="cuda")
        Fp[:nv] = F
        Y = torch.empty(rows, self.np_, dtype=torch.float32, device="cuda")
        self.mlp.predict(Fp.data_ptr(), Y.data_ptr(), rows)
        yc = (Y[:nv, :self.nc].double().T * s).contiguous()  # [nc][nv]
        x0 = self.T.prolong(yc.reshape(-1), nv).reshape(-1, nv)
        return smooth(x0) if smooth else x0


def residual_norms(S, x, b, nv):
    """||b - A x|| per column with the solver's own FP64 SpMV."""
    Ax = torch.empty_like(x)
    S.level_spmv(0, 0, x.data_ptr(), Ax.data_ptr(), nv)
    torch.cuda.synchronize()
    return (b - Ax).norm(dim=0)


def solver_params(tol, smoother="Chebyshev"):
    """The chosen form of the solve: MergedPBiCGStab with an FP32 AMG V(1,1)
    preconditioner (PMIS, strength 0.25, ext+i)."""
    sm = {"method": smoother, "polynomial_order": 2}
    return {"solver": {"method": "MergedPBiCGStab", "max_iters": 500, "rel_tolerance": tol,
                       "abs_tolerance": 0, "gpu_index_compress": 2},
            "preconditioner": {"method": "MultiGrid", "max_iters": 1, "mg_agg_num_levels": 0,
                               "mg_strength_threshold": 0.25, "mg_coarsening_type": 8,
                               "mg_interpolation_type": 6, "mg_coarse_matrix_size": 500,
                               "gpu_precond_f32": 1, "gpu_index_compress": 2},
            "pre_smoother": sm, "post_smoother": dict(sm)}


def fp64_transfer_params(tol):
    p = solver_params(tol)
    p["preconditioner"] = dict(p["preconditioner"], gpu_precond_f32=0, gpu_index_compress=1)
    p["solver"]["gpu_index_compress"] = 1
    return p


def vcycle_params(reduced=1):
    """One V(1,1) cycle of the same hierarchy as a stationary step from the
    given x: x + M^-1 (b - A x) with the multigrid cycle M (levels below the
    finest in FP32 with reduced = 1, XAMG's mg_reduced_precision)."""
    sm = {"method": "Chebyshev", "polynomial_order": 2}
    return {"solver": {"method": "MultiGrid", "max_iters": 1, "convergence_check": 0,
                       "mg_agg_num_levels": 0, "mg_strength_threshold": 0.25,
                       "mg_coarsening_type": 8, "mg_interpolation_type": 6,
                       "mg_coarse_matrix_size": 500, "mg_reduced_precision": reduced,
                       "gpu_index_compress": 2},
            "pre_smoother": sm, "post_smoother": dict(sm),
            "coarse_grid_solver": {"method": "Direct"}}


def run(n_edge=96, n_train=4096, n_eval=1024, nv=32, steps=400, level=3, hidden=1024,
        sigma=1.0, seed=0, train_tol=1e-10, tol=1e-8, lr=1e-3, batch=512, log=print,
        smoothing="vcycle"):
    """Trains the guess on n_train solved right-hand sides and compares it with
    the zero guess on n_eval held-out ones (all in blocks of nv). smoothing:
    what is applied to the prolongated guess before it is tested: "vcycle"
    (one multigrid V-cycle step x0 + M^-1 (b - A x0), which removes the
    high-frequency error the coarse coefficients leave) or "jacobi" (two
    damped Jacobi sweeps). Returns a dict of iterations, ms per right-hand
    side and initial residuals."""
    st = torch.cuda.ExternalStream(X.stream())
    with torch.cuda.stream(st):
        return _run(n_edge, n_train, n_eval, nv, steps, level, hidden, sigma, seed, train_tol,
                    tol, lr, batch, log, st, smoothing)


def _run(n_edge, n_train, n_eval, nv, steps, level, hidden, sigma, seed, train_tol, tol, lr,
         batch, log, st, smoothing):
    t_setup = time.time()
    row, col, val = X.generate_diffusion(7, n_edge, n_edge, n_edge, sigma, 1.0, seed)
    n = len(row) - 1
    M = X.Matrix(row, col, val)
    xv, bv = X.Vector(n, nv), X.Vector(n, nv)
    xv.set(0.0)
    bv.set(1.0)
    S_train = X.Solver(M, X.Params(solver_params(train_tol)), xv, bv)
    S_eval = X.Solver(M, X.Params(solver_params(tol)), xv, bv)
    x1, b1 = X.Vector(n, 1), X.Vector(n, 1)
    x1.set(0.0)
    b1.set(1.0)
    S64 = X.Solver(M, X.Params(fp64_transfer_params(tol)), x1, b1)
    # the prolongated guess is smoothed before its residual is tested: the
    # coarse coefficients leave high-frequency error that the multigrid
    # cycle (or, more weakly, two damped Jacobi sweeps) removes
    xs, bs = X.Vector(n, nv), X.Vector(n, nv)
    if smoothing == "jacobi":
        S_smooth = X.Solver(M, X.Params({"solver": {"method": "Jacobi", "max_iters": 2,
                                                    "convergence_check": 0,
                                                    "relax_factor": 0.8}}), xs, bs)
    else:
        S_smooth = X.Solver(M, X.Params(vcycle_params(0 if smoothing == "vcycle64" else 1)),
                            xs, bs)
    nl = S64.nlevels()
    level = min(level, nl - 1)
    LG = LearnedGuess(S64, level, hidden, seed)
    gen = torch.Generator().manual_seed(seed + 1)
    setup_s = time.time() - t_setup
    log(f"levels {[S64.level_info(l, 0)['nrows'] for l in range(nl)]}, guess level {level} "
        f"({LG.nc} unknowns), setup {setup_s:.1f} s")

    def upload(v, t):
        X.call("XAMG_vector_upload_d", t.data_ptr(), n, 0, nv, v.h)

    def download(v):
        out = torch.empty(n, nv, dtype=torch.float64, device="cuda")
        X.call("XAMG_vector_download_d", out.data_ptr(), n, 0, nv, v.h)
        return out

    cur_b = {}

    def smooth(x0):
        upload(xs, x0.contiguous())
        upload(bs, cur_b["b"])
        S_smooth.solve()
        return download(xs)

    # training pairs from the solver itself
    t0 = time.time()
    F, T = [], []
    for _ in range(n_train // nv):
        b = gaussian_rhs(n_edge, nv, gen)
        upload(bv, b)
        xv.set(0.0)
        S_train.solve()
        x = download(xv)
        f, s = LG.features(b, nv)
        F.append(f)
        T.append(LG.targets(x, s, nv))
    F, T = torch.cat(F), torch.cat(T)
    data_s = time.time() - t0
    t0 = time.time()
    losses = LG.train(F, T, steps, batch=batch, lr=lr, gen=gen)
    train_s = time.time() - t0
    log(f"training data {data_s:.1f} s, {steps} Adam steps {train_s:.1f} s, "
        f"loss {losses[0]:.3e} -> {losses[-1]:.3e}")

    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    res = dict(zero_iters=[], learned_iters=[], zero_ms=0.0, learned_ms=0.0, r0_ratio=[],
               kept=0, total=0)
    for _ in range(n_eval // nv):
        b = gaussian_rhs(n_edge, nv, gen)
        bnorm = b.norm(dim=0)
        upload(bv, b)
        torch.cuda.synchronize()
        ev[0].record(st)
        xv.set(0.0)
        S_eval.solve()
        ev[1].record(st)
        res["zero_iters"].append(S_eval.stats()["iters"])
        ev[2].record(st)
        cur_b["b"] = b
        x0 = LG.guess(b, nv, smooth)
        r0 = residual_norms(S_eval, x0, b, nv)
        keep = r0 < bnorm
        x0 = x0 * keep.to(x0.dtype)[None, :]
        upload(xv, x0.contiguous())
        S_eval.solve()
        ev[3].record(st)
        ev[3].synchronize()
        res["learned_iters"].append(S_eval.stats()["iters"])
        res["zero_ms"] += ev[0].elapsed_time(ev[1])
        res["learned_ms"] += ev[2].elapsed_time(ev[3])
        res["r0_ratio"] += (torch.where(keep, r0, bnorm) / bnorm).tolist()
        res["kept"] += int(keep.sum())
        res["total"] += nv
    nrhs = res["total"]
    out = dict(rows=n, nnz=len(col), levels=nl, guess_level=level, coarse=LG.nc,
               train_rhs=F.shape[0], eval_rhs=nrhs, steps=steps, first_loss=losses[0],
               final_loss=losses[-1], setup_s=setup_s, data_s=data_s, train_s=train_s,
               zero_iters=float(np.mean(res["zero_iters"])),
               learned_iters=float(np.mean(res["learned_iters"])),
               zero_ms_per_rhs=res["zero_ms"] / nrhs, learned_ms_per_rhs=res["learned_ms"] / nrhs,
               initial_residual_ratio=float(np.median(res["r0_ratio"])),
               guesses_kept=res["kept"] / nrhs, smoothing=smoothing)
    log(out)
    return out
