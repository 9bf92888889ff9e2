"""The batch solve (XAMG_b200_solver_solve_batch): independent systems of
uneven size and nv, each on its own stream, the merged BiCGStab forms in
lockstep. Every system's solution, iteration count and residuals must equal
its own XAMG_solver_solve2 call bit for bit (those are checked against the
oracle in test_gpu_solve / test_gpu_configs), on the first call and on later
ones, where the preconditioner runs from CUDA graphs recorded per stream."""
import numpy as np
import pytest

from test_gpu_solve import MG_BASE
from xamg_b200 import XamgError

pytestmark = pytest.mark.gpu

HSGS = {"method": "HSGS", "max_iters": 1}


def config3_params(method="MergedPBiCGStab"):
    return {"solver": {"method": method, "max_iters": 200, "rel_tolerance": 1e-8,
                       "abs_tolerance": 0, "gpu_index_compress": 2},
            "preconditioner": dict(MG_BASE, method="MultiGrid", gpu_precond_f32=1,
                                   gpu_index_compress=2),
            "pre_smoother": HSGS, "post_smoother": dict(HSGS),
            "coarse_grid_solver": {"method": "Direct"}}


def systems(gpu, specs):
    out = []
    for edge, nv, seed, params in specs:
        row, col, val = gpu.generate_diffusion(7, edge, edge, edge, 1.5, 1.0, seed)
        M = gpu.Matrix(row, col, val)
        xv, bv = gpu.Vector(M.n, nv), gpu.Vector(M.n, nv)
        bv.upload(np.random.default_rng(seed).uniform(-1, 1, M.n * nv))
        xv.set(0.0)
        S = gpu.Solver(M, gpu.Params(params), xv, bv)
        out.append((M, xv, bv, S))
    return out


def run_each(sys_):
    res = []
    for _, xv, bv, S in sys_:
        xv.set(0.0)
        S.solve(xv, bv)
        res.append((xv.download(), S.stats()))
    return res


def run_batch(gpu, sys_):
    for _, xv, _, _ in sys_:
        xv.set(0.0)
    gpu.solve_batch([s[3] for s in sys_], [s[1] for s in sys_], [s[2] for s in sys_])
    return [(xv.download(), S.stats()) for _, xv, _, S in sys_]


def same(a, b):
    for (xa, sa), (xb, sb) in zip(a, b):
        assert xa.tobytes() == xb.tobytes()
        assert sa["iters"] == sb["iters"]
        assert sa["conv"].tolist() == sb["conv"].tolist()
        assert sa["rel_res"].tobytes() == sb["rel_res"].tobytes()


def test_batch_equals_single_solves(gpu):
    """Configuration 3 in small: 7-point kappa = exp(N(0, 1.5^2)) systems of
    edges 12..28 with nv in {1, 4, 16}, AMG V(1,1) HSGS in FP32."""
    rng = np.random.default_rng(3)
    specs = [(int(e), int(v), 100 + i, config3_params())
             for i, (e, v) in enumerate(zip(rng.choice([12, 16, 20, 24, 28], 9),
                                            rng.choice([1, 4, 16], 9)))]
    sys_ = systems(gpu, specs)
    want = run_each(sys_)
    for _ in range(3):  # first call, graph recording, graph replay
        same(run_batch(gpu, sys_), want)
    for (x, st), (M, _, _, _) in zip(want, sys_):
        assert st["conv"].all()


def test_batch_mixed_methods(gpu):
    """Lockstep systems beside ones that run to the end on their lane (PCG,
    a multigrid solver), and an unpreconditioned merged BiCGStab."""
    mg_solver = dict(config3_params())
    mg_solver["solver"] = dict(MG_BASE, method="MultiGrid", max_iters=30, rel_tolerance=1e-8,
                               abs_tolerance=0)
    del mg_solver["preconditioner"]
    specs = [(16, 4, 7, config3_params()),
             (12, 1, 8, config3_params("PCG")),
             (14, 2, 9, {"solver": {"method": "MergedBiCGStab", "max_iters": 400,
                                    "rel_tolerance": 1e-8, "abs_tolerance": 0}}),
             (10, 8, 10, mg_solver),
             (18, 16, 11, config3_params("PBiCGStab"))]
    sys_ = systems(gpu, specs)
    want = run_each(sys_)
    for _ in range(2):
        same(run_batch(gpu, sys_), want)


def test_batch_argument_errors(gpu):
    sys_ = systems(gpu, [(8, 1, 1, config3_params()), (8, 4, 2, config3_params())])
    (M0, x0, b0, S0), (M1, x1, b1, S1) = sys_
    gpu.solve_batch([], [], [])
    with pytest.raises(XamgError):
        gpu.solve_batch([S0, S0], [x0, x1], [b0, b1])  # one solver twice
    with pytest.raises(XamgError):
        gpu.solve_batch([S0, S1], [x0, x0], [b0, b1])  # one solution vector twice
    with pytest.raises(XamgError):
        gpu.solve_batch([S0], [x1], [b0])  # nv of x differs from b's
    # the library is still usable afterwards
    same(run_batch(gpu, sys_), run_each(sys_))


def test_repeated_solves_equal(gpu):
    """A multigrid solver with HSGS smoothing whose right-hand sides converge
    at different iterations (per-RHS relaxation factors frozen to zero) gives
    the same result on its next solve: the smoothers' device factors are
    reset when a solve starts with every right-hand side active."""
    p = {"solver": dict(MG_BASE, method="MultiGrid", max_iters=30, rel_tolerance=1e-8,
                        abs_tolerance=0),
         "pre_smoother": HSGS, "post_smoother": dict(HSGS),
         "coarse_grid_solver": {"method": "Direct"}}
    sys_ = systems(gpu, [(10, 8, 10, p)])
    first = run_each(sys_)
    same(run_each(sys_), first)
    same(run_batch(gpu, sys_), first)


@pytest.mark.parametrize("method", ["MergedPBiCGStab", "MergedBiCGStab"])
def test_batch_stopped_at_max_iters(gpu, method):
    """Systems that stop at max_iters before converging, beside one that
    converges: the rest of each system's last iteration (its x update) still
    runs, so every result equals its single solve bit for bit, on the first
    call and once the iterations replay as graphs."""
    specs = []
    for i, (edge, nv, cap) in enumerate([(20, 4, 7), (16, 1, 5), (12, 2, 2000)]):
        p = config3_params(method)
        p["solver"]["max_iters"] = cap
        if method == "MergedBiCGStab":
            p = {"solver": p["solver"]}
        specs.append((edge, nv, 40 + i, p))
    sys_ = systems(gpu, specs)
    want = run_each(sys_)
    assert not want[0][1]["conv"].all() and want[0][1]["iters"] == 7
    assert want[2][1]["conv"].all()
    for _ in range(4):
        same(run_batch(gpu, sys_), want)
