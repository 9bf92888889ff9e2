"""The CPU oracle against the reference itself: XAMG's own C API and solve
phase compiled unmodified from the reference sources (with the
single-process stand-ins of oracle/ref_shim for MPI, argsparser's parameter
dictionary and hypre; oracle/Makefile target `ref`), run on one rank. With
XAMG's reduction order on one core (mode 0, ncores = 1) the oracle must give
the reference's solution bit for bit: every Krylov method, the multigrid
cycles (V, W and the F-cycle as the reference runs it), every smoother, the
direct coarse solve, reduced precision and per-level overrides. The
multigrid hierarchy (hypre's part) is the one the library's host setup builds
(oracle/liboracle_setup.so), registered with the hypre stand-in.

Skipped where the reference sources (and so oracle/_ref) are not present."""
import numpy as np
import pytest

import ref_capi

pytestmark = pytest.mark.skipif(not ref_capi.available(1), reason="reference not built here")

MG = {"mg_agg_num_levels": 0, "mg_strength_threshold": 0.25, "mg_coarsening_type": 8,
      "mg_interpolation_type": 6, "mg_coarse_matrix_size": 60, "max_iters": 1}


def compare(oracle, row, col, val, nv, params, seed=3, overrides=None, oracle_params=None):
    n = len(row) - 1
    mg_role = next((r for r, kv in params.items() if kv.get("method") == "MultiGrid"), None)
    H = oracle.setup_hierarchy(row, col, val, params[mg_role]) if mg_role else None
    b = np.random.default_rng(seed).uniform(-1, 1, n * nv)
    R = ref_capi.Solve(row, col, val, nv, params, overrides=overrides, hierarchy=H)
    try:
        xr, conv = R.solve(b)
    finally:
        R.close()
    sysm = oracle.System(nv)
    sysm.set_params(oracle_params or params)
    sysm.hsgs_cores(1)   # the reference's one core is one Gauss-Seidel block
    if H is None:
        sysm.add_level(row, col, val)
    else:
        for lv in H:
            sysm.add_level(*lv["A"], lv["min_eig"], lv["max_eig"])
            if lv["P"] is not None:
                sysm.add_interp(*lv["P"])
    sysm.setup()
    oracle.set_reduction(0, 1)
    try:
        xo, so = sysm.solve(b)
    finally:
        oracle.set_reduction(0)
    assert conv.tolist() == so["conv"].tolist()
    assert xr.tobytes() == xo.tobytes(), np.abs(xr - xo).max()
    return so


def test_config1_poisson32_merged_pbicgstab_jacobi(oracle):
    row, col, val = oracle.generate_cube(32, 32, 32)
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 1000, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": {"method": "Jacobi"}}
    so = compare(oracle, row, col, val, 1, params, seed=0)
    assert so["conv"].all() and 30 < so["iters"] < 80


@pytest.mark.parametrize("method", ["BiCGStab", "PBiCGStab", "MergedBiCGStab",
                                    "MergedPBiCGStab", "PCG", "RBiCGStab", "MergedRBiCGStab"])
@pytest.mark.parametrize("nv", [1, 4])
def test_krylov_methods(oracle, method, nv):
    row, col, val = oracle.setup_generate_diffusion(7, 12, 11, 10, 1.0, 1.0, 4)
    params = {"solver": {"method": method, "max_iters": 300, "rel_tolerance": 1e-9,
                         "abs_tolerance": 0}}
    if method not in ("BiCGStab", "MergedBiCGStab"):
        params["preconditioner"] = {"method": "Jacobi", "max_iters": 3}
    compare(oracle, row, col, val, nv, params, seed=nv)


@pytest.mark.parametrize("smoother", ["Jacobi", "Chebyshev", "HSGS"])
@pytest.mark.parametrize("cycle", [0, 1, 2])
def test_multigrid_cycles_and_smoothers(oracle, smoother, cycle):
    row, col, val = oracle.setup_generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 21)
    sm = {"method": smoother}
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 40, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": dict(MG, method="MultiGrid", mg_cycle=cycle),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    compare(oracle, row, col, val, 4, params, seed=cycle)


@pytest.mark.parametrize("nv", [2, 8])
def test_multigrid_reduced_precision(oracle, nv):
    """mg_reduced_precision = 1: levels below the finest, R and P in float
    (mg.inl:114-132)."""
    row, col, val = oracle.setup_generate_diffusion(27, 16, 15, 14, 1.0, 1.0, 8)
    sm = {"method": "Chebyshev", "polynomial_order": 3}
    params = {"solver": {"method": "PBiCGStab", "max_iters": 100, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": dict(MG, method="MultiGrid", mg_reduced_precision=1),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    so = compare(oracle, row, col, val, nv, params, seed=nv)
    assert so["conv"].all()


def test_multigrid_as_solver_with_level_overrides(oracle):
    """MultiGrid as the solver, smoother settings overridden per level
    ("value@levA-B", xamg_params_details.h layer prefix "lev")."""
    row, col, val = oracle.setup_generate_diffusion(7, 16, 16, 16, 1.5, 1.0, 9)
    params = {"solver": dict(MG, method="MultiGrid", max_iters=25, rel_tolerance=1e-8,
                             abs_tolerance=0, convergence_check=1),
              "pre_smoother": {"method": "Jacobi", "max_iters": 2},
              "post_smoother": {"method": "Jacobi", "max_iters": 2},
              "coarse_grid_solver": {"method": "Direct"}}
    overrides = {"pre_smoother": {"max_iters": "3@lev1-2", "relax_factor": "0.8@lev0"}}
    oracle_params = {k: dict(v) for k, v in params.items()}
    oracle_params["pre_smoother"].update({"max_iters@1": 3, "max_iters@2": 3,
                                          "relax_factor@0": 0.8})
    compare(oracle, row, col, val, 2, params, seed=5, overrides=overrides,
            oracle_params=oracle_params)


def test_headline_workload_small(oracle):
    """The benchmark's plain-FP64 method (PMIS, strength 0.25, ext+i, AMG
    V(1,1) Chebyshev-2, MergedPBiCGStab, 1e-8) on the 27-point
    variable-kappa matrix at 32^3, nv = 8."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    w = dict(bench.WORKLOADS["amg27"], grid=32)
    row, col, val = oracle.setup_generate_diffusion(27, 32, 32, 32, 1.0, 1.0, 0)
    so = compare(oracle, row, col, val, 8, bench.params_for(w, False), seed=1000)
    assert so["conv"].all()
