"""The persistent BiCGStab (gpu_persistent, default 1): PBiCGStab and
MergedPBiCGStab with no preconditioner or a Jacobi preconditioner run every
iteration, the convergence test and the final update in one cooperative
launch with bounded grid barriers. It must give the iteration-by-iteration
path's results bit for bit (iterations, convergence flags, residuals,
solution), whether the solve converges or stops at max_iters, and a grid
barrier that can never complete must end in a reported timeout with the GPU
context still usable."""
import ctypes as C

import numpy as np
import pytest

from test_gpu_solve import gpu_solve, true_rel_res

pytestmark = pytest.mark.gpu


def params(method, prec, persistent, max_iters=1000, sweeps=None, tol=1e-8):
    p = {"solver": {"method": method, "max_iters": max_iters, "rel_tolerance": tol,
                    "abs_tolerance": 0, "gpu_persistent": persistent}}
    if prec:
        p["preconditioner"] = {"method": "Jacobi"}
        if sweeps:
            p["preconditioner"]["max_iters"] = sweeps
    return p


@pytest.mark.parametrize("method,prec,nv,sweeps,grid,cap",
                         [("MergedPBiCGStab", True, 1, None, (32, 32, 32), 1000),
                          ("MergedPBiCGStab", True, 2, 3, (20, 19, 18), 1000),
                          ("PBiCGStab", True, 8, 1, (16, 16, 16), 1000),
                          ("PBiCGStab", False, 4, None, (17, 16, 15), 1000),
                          ("MergedPBiCGStab", True, 1, None, (32, 32, 32), 7)])
@pytest.mark.parametrize("share", [1, 3, 4])
def test_persistent_equals_stepwise(gpu, method, prec, nv, sweeps, grid, cap, share):
    """share (gpu_persistent): canonical blocks each block of the launch plays;
    the reductions stay per canonical block, so every share gives the same
    bits as the step-by-step solve."""
    row, col, val = gpu.generate_cube(*grid)
    n = len(row) - 1
    b = np.random.default_rng(nv + grid[0]).uniform(-1, 1, n * nv)
    out = {}
    for persistent in (0, share):
        k0 = gpu.kernel_launches()
        x, st, S = gpu_solve(gpu, row, col, val, nv, params(method, prec, persistent, cap, sweeps),
                             b)
        out[persistent] = (x, st, gpu.kernel_launches() - k0)
    (x0, s0, l0), (x1, s1, l1) = out[0], out[share]
    assert s0["iters"] == s1["iters"]
    assert s0["conv"].tolist() == s1["conv"].tolist()
    assert s0["rel_res"].tobytes() == s1["rel_res"].tobytes()
    assert s0["abs_res"].tobytes() == s1["abs_res"].tobytes()
    assert x0.tobytes() == x1.tobytes()
    assert l1 < l0 and l1 <= 3  # start, the persistent launch (a converged solve: no more)
    if cap < 1000:
        assert s1["iters"] == cap and not s1["conv"].any()
    else:
        assert s1["conv"].all()
        assert true_rel_res(row, col, val, x1, b, nv).max() <= 1e-7


def test_grid_barrier_wait_runs_out(gpu):
    t = C.c_int(-1)
    gpu.call("XAMG_b200_grid_selftest", 0.05, C.byref(t))
    assert t.value == 1
    # the context is still usable: a persistent solve right after
    row, col, val = gpu.generate_cube(12, 12, 12)
    b = np.ones(len(row) - 1)
    x, st, S = gpu_solve(gpu, row, col, val, 1, params("MergedPBiCGStab", True, 1), b)
    assert st["conv"].all()
