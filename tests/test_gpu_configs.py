"""The benchmark description's other configurations as parity cases, at sizes
the oracle solves in seconds (the 128^3 configuration is the bench workload):

* configuration 3: uneven 7-point variable-coefficient systems
  (kappa = exp(N(0, 1.5^2))), each with its own nv in {1, 4, 16}, AMG V(1,1)
  with hybrid Gauss-Seidel smoothing applied in FP32;
* configuration 5: 27-point variable-coefficient diffusion with
  kappa = exp(N(0, 2^2)) and 4:1 anisotropy in z, nv = 32, BiCGStab with an
  AMG V(2,2) Chebyshev degree-3 preconditioner in FP32 (2-byte relative
  columns), FP64 outer iteration.

Every solve must equal the oracle's replay bit for bit and XAMG's own order to
1e-6 relative, with true residuals at the tolerance."""
import numpy as np
import pytest

from test_gpu_solve import MG_BASE, check, gpu_solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("edge,nv,seed", [(16, 1, 31), (24, 4, 32), (32, 16, 33), (20, 16, 34),
                                          (28, 1, 35)])
def test_config3_uneven_systems_hsgs_fp32(gpu, oracle, edge, nv, seed):
    row, col, val = gpu.generate_diffusion(7, edge, edge, edge, 1.5, 1.0, seed)
    sm = {"method": "HSGS", "max_iters": 1}
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 200, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0, "gpu_index_compress": 2},
              "preconditioner": dict(MG_BASE, method="MultiGrid", gpu_precond_f32=1,
                                     gpu_index_compress=2),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    st, S = check(gpu, oracle, row, col, val, nv, params, seed=seed)
    assert st["iters"] < 60


def test_config5_anisotropic_27pt_vcycle22_cheby3(gpu, oracle):
    row, col, val = gpu.generate_diffusion(27, 20, 20, 20, 2.0, 4.0, 5)
    nv = 32
    sm = {"method": "Chebyshev", "polynomial_order": 3, "max_iters": 2}
    params = {"solver": {"method": "PBiCGStab", "max_iters": 200, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0, "gpu_index_compress": 2},
              "preconditioner": dict(MG_BASE, method="MultiGrid", gpu_precond_f32=1,
                                     gpu_index_compress=2),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    st, S = check(gpu, oracle, row, col, val, nv, params, seed=5)
    assert st["iters"] < 80


@pytest.mark.parametrize("levels,smoother,half", [(1, "Chebyshev", "bf16"),
                                                   (2, "Chebyshev", "bf16"), (2, "Jacobi", "bf16"),
                                                   (2, "HSGS", "bf16"), (2, "Chebyshev", "fp16"),
                                                   (2, "HSGS", "fp16")])
def test_config5_bf16_levels(gpu, oracle, levels, smoother, half):
    """Configuration 5's 16-bit level values (gpu_level_bf16: the finest FP32
    cycle operators store BF16 values, or with gpu_level_fp16 = 1 FP16 values
    scaled by a per-level power of two; float arithmetic; smoother diagonals,
    hybrid Gauss-Seidel blocks and transfers from the float values). The
    oracle given the same setup replays the solve bit for bit, XAMG's order
    agrees to 1e-6, and the true residuals reach the tolerance."""
    if smoother == "Chebyshev":
        row, col, val = gpu.generate_diffusion(27, 20, 20, 20, 2.0, 4.0, 5)
        sm = {"method": smoother, "max_iters": 2, "polynomial_order": 3}
    else:
        # Jacobi and hybrid Gauss-Seidel smoothing on the isotropic matrix
        row, col, val = gpu.generate_diffusion(27, 18, 18, 18, 1.0, 1.0, 5)
        sm = {"method": smoother, "max_iters": 2}
    nv = 4
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 200, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0, "gpu_index_compress": 2},
              "preconditioner": dict(MG_BASE, method="MultiGrid", gpu_precond_f32=1,
                                     gpu_index_compress=2, gpu_level_bf16=levels,
                                     gpu_level_fp16=1 if half == "fp16" else 0),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    st, S = check(gpu, oracle, row, col, val, nv, params, seed=5, tol=1.5e-9)
    assert S.level_info(levels - 1, 3)[half] and not S.level_info(levels, 3)[half]
