"""Files on the GPU path: a system read from XAMG's binary format solves like
the same arrays given directly, and a multigrid hierarchy written by one
solver and attached to a new matrix object gives a solver whose solves are
bit-identical to the first one's (its setup is skipped)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MG = {"solver": {"method": "PBiCGStab", "rel_tolerance": 1e-8, "max_iters": 100},
      "preconditioner": {"method": "MultiGrid", "mg_agg_num_levels": 0,
                         "mg_strength_threshold": 0.25, "mg_coarsening_type": 8,
                         "mg_interpolation_type": 6, "mg_coarse_matrix_size": 60,
                         "max_iters": 1},
      "pre_smoother": {"method": "Chebyshev"}, "post_smoother": {"method": "Chebyshev"}}


def solve(gpu, M, params, b, nv):
    X, B = gpu.Vector(M.n, nv), gpu.Vector(M.n, nv)
    B.upload(b)
    X.set(0.0)
    S = gpu.Solver(M, gpu.Params(params), X, B)
    S.solve()
    return X.download(), S.stats(), S


def test_system_file_solve(gpu, tmp_path):
    row, col, val = gpu.generate_diffusion(7, 14, 13, 12, 1.0, 1.0, 4)
    nv = 2
    b = np.random.default_rng(1).uniform(-1, 1, (len(row) - 1) * nv)
    path = tmp_path / "sys.bin"
    gpu.write_system(path, row, col, val, nv, b)
    r, c, v, bb, xx, found = gpu.read_system(path, nv)
    assert found == 1
    x1, s1, _ = solve(gpu, gpu.Matrix(r, c, v), MG, bb, nv)
    x0, s0, _ = solve(gpu, gpu.Matrix(row, col, val), MG, b, nv)
    assert s1["iters"] == s0["iters"] and x1.tobytes() == x0.tobytes()


def test_hierarchy_file_round_trip(gpu, tmp_path):
    row, col, val = gpu.generate_diffusion(27, 16, 15, 14, 1.0, 1.0, 5)
    nv = 4
    b = np.random.default_rng(2).uniform(-1, 1, (len(row) - 1) * nv)
    x0, s0, S0 = solve(gpu, gpu.Matrix(row, col, val), MG, b, nv)
    path = tmp_path / "h.bin"
    S0.save_hierarchy(path)
    M1 = gpu.Matrix(row, col, val)
    M1.load_hierarchy(path)
    x1, s1, S1 = solve(gpu, M1, MG, b, nv)
    assert S1.nlevels() == S0.nlevels()
    assert s1["iters"] == s0["iters"] and x1.tobytes() == x0.tobytes()
    # another matrix (one value changed) is refused
    val2 = val.copy()
    val2[7] *= 1.5
    M2 = gpu.Matrix(row, col, val2)
    with pytest.raises(gpu.XamgError):
        M2.load_hierarchy(path)
