"""Whole solves as one graph launch (gpu_solve_graph, default 1): from the
third solve with the same x and b on, a merged BiCGStab solve runs as one
graph whose device-side loop (conditional WHILE and IF nodes, set by the
convergence test kernels of csrc/loop.cu) replaces the host round trip of
every iteration. Every such solve must equal the same solve run by steps
(gpu_solve_graph = 0) bit for bit: solution, iteration count, per-RHS
convergence flags and residual statistics; also when the solve stops at
max_iters, when b = 0 passes the test before the first iteration, and in a
batch of systems solved together."""
import numpy as np
import pytest

from test_gpu_batch import config3_params, systems
from test_gpu_solve import MG_BASE

pytestmark = pytest.mark.gpu

CHEB = {"method": "Chebyshev", "polynomial_order": 2}


def params(kind, loop, max_iters=200):
    solver = {"method": "MergedPBiCGStab", "max_iters": max_iters, "rel_tolerance": 1e-8,
              "abs_tolerance": 0, "gpu_solve_graph": loop, "gpu_persistent": 0}
    if kind == "mg64":
        return {"solver": solver, "preconditioner": dict(MG_BASE, method="MultiGrid"),
                "pre_smoother": CHEB, "post_smoother": dict(CHEB),
                "coarse_grid_solver": {"method": "Direct"}}
    if kind == "mg32":
        solver["gpu_index_compress"] = 2
        return {"solver": solver,
                "preconditioner": dict(MG_BASE, method="MultiGrid", gpu_precond_f32=1,
                                       gpu_index_compress=3, gpu_level_bf16=1),
                "pre_smoother": CHEB, "post_smoother": dict(CHEB),
                "coarse_grid_solver": {"method": "Direct"}}
    if kind == "jacobi":
        return {"solver": solver, "preconditioner": {"method": "Jacobi"}}
    if kind == "merged_plain":
        solver["method"] = "MergedBiCGStab"
        return {"solver": solver}
    raise ValueError(kind)


def solves(gpu, row, col, val, nv, p, b, reps):
    M = gpu.Matrix(row, col, val)
    xv, bv = gpu.Vector(M.n, nv), gpu.Vector(M.n, nv)
    bv.upload(b)
    S = gpu.Solver(M, gpu.Params(p), xv, bv)
    out = []
    for _ in range(reps):
        xv.set(0.0)
        S.solve()
        st = S.stats()
        out.append((xv.download(), st["iters"], st["conv"].tolist(), st["abs_res"].tobytes(),
                    st["rel_res"].tobytes()))
    return out


@pytest.mark.parametrize("kind", ["mg64", "mg32", "jacobi", "merged_plain"])
@pytest.mark.parametrize("nv", [1, 4])
def test_loop_graph_equals_steps(gpu, kind, nv):
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 5)
    n = len(row) - 1
    b = np.random.default_rng(31).uniform(-1, 1, n * nv)
    ref = solves(gpu, row, col, val, nv, params(kind, 0), b, 4)
    got = solves(gpu, row, col, val, nv, params(kind, 1), b, 4)
    for a, g in zip(ref, got):
        assert a[0].tobytes() == g[0].tobytes()
        assert a[1:] == g[1:]
    assert all(c == 1 for c in got[-1][2])


@pytest.mark.parametrize("kind", ["mg32", "jacobi"])
def test_loop_graph_max_iters(gpu, kind):
    """A solve cut at max_iters runs the rest of its last iteration too."""
    row, col, val = gpu.generate_diffusion(7, 16, 15, 14, 1.5, 1.0, 6)
    n, nv = len(row) - 1, 2
    b = np.random.default_rng(32).uniform(-1, 1, n * nv)
    ref = solves(gpu, row, col, val, nv, params(kind, 0, max_iters=2), b, 3)
    got = solves(gpu, row, col, val, nv, params(kind, 1, max_iters=2), b, 3)
    for a, g in zip(ref, got):
        assert a[0].tobytes() == g[0].tobytes()
        assert a[1:] == g[1:]
    assert got[-1][1] == 2


def test_loop_graph_zero_rhs(gpu):
    """b = 0: rho0 passes the test, no iteration runs, x stays zero."""
    row, col, val = gpu.generate_diffusion(7, 12, 11, 10, 1.0, 1.0, 7)
    n, nv = len(row) - 1, 4
    b = np.zeros(n * nv)
    ref = solves(gpu, row, col, val, nv, params("mg32", 0), b, 3)
    got = solves(gpu, row, col, val, nv, params("mg32", 1), b, 3)
    for a, g in zip(ref, got):
        assert a[0].tobytes() == g[0].tobytes()
        assert a[1:] == g[1:]
    assert got[-1][1] == 0 and not got[-1][0].any()


def test_batch_with_loop_graphs(gpu):
    """A batch solved three times (the third with every system as one graph
    launch) equals each system's own solve run by steps."""
    specs = []
    for i, (edge, nv) in enumerate([(16, 1), (24, 4), (12, 16), (20, 4)]):
        p = config3_params()
        specs.append((edge, nv, 40 + i, p))
    sys_ = systems(gpu, specs)
    ref = []
    # references: the same systems with gpu_solve_graph = 0, one solve each
    ref_specs = []
    for edge, nv, seed, p in specs:
        q = {k: dict(v) for k, v in p.items()}
        q["solver"]["gpu_solve_graph"] = 0
        ref_specs.append((edge, nv, seed, q))
    ref_sys = systems(gpu, ref_specs)
    for _, xv, bv, S in ref_sys:
        xv.set(0.0)
        S.solve(xv, bv)
        ref.append((xv.download(), S.stats()))
    for _ in range(3):
        for _, xv, _, _ in sys_:
            xv.set(0.0)
        gpu.solve_batch([s[3] for s in sys_], [s[1] for s in sys_], [s[2] for s in sys_])
        for (xr, sr), (_, xv, _, S) in zip(ref, sys_):
            st = S.stats()
            assert xv.download().tobytes() == xr.tobytes()
            assert st["iters"] == sr["iters"]
            assert st["conv"].tolist() == sr["conv"].tolist()
            assert st["rel_res"].tobytes() == sr["rel_res"].tobytes()


def test_renew_params_after_graphs(gpu):
    """XAMG_solver_renew_params after the solve has been recorded as a graph:
    the recorded graphs are dropped, and the next solves use the new
    parameters (here max_iters and the tolerance) as the step-by-step solve
    does."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 9)
    n, nv = len(row) - 1, 2
    b = np.random.default_rng(34).uniform(-1, 1, n * nv)
    out = {}
    for loop in (0, 1):
        M = gpu.Matrix(row, col, val)
        xv, bv = gpu.Vector(M.n, nv), gpu.Vector(M.n, nv)
        bv.upload(b)
        S = gpu.Solver(M, gpu.Params(params("mg32", loop)), xv, bv)
        for _ in range(4):
            xv.set(0.0)
            S.solve()
        full = S.stats()["iters"]
        S.renew(gpu.Params({"solver": {"max_iters": 2, "rel_tolerance": 1e-4}},
                           set_default=False))
        res = []
        for _ in range(4):
            xv.set(0.0)
            S.solve()
            st = S.stats()
            res.append((xv.download().tobytes(), st["iters"], st["rel_res"].tobytes()))
        out[loop] = (full, res)
    assert out[0] == out[1]
    assert out[1][1][-1][1] <= 2 < out[1][0]
