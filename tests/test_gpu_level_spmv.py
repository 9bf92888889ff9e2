"""The SpMV on a solver's own level matrices (XAMG_b200_solver_level_spmv),
as its solves run it: the library's uploaded copy with XAMG's narrowing or
2-byte relative columns, FP64 on the Krylov level and FP32 on the cycle's
level 0 with gpu_precond_f32. Every element must equal
the oracle's sequential row sum bit for bit, for y = A x and y += A x. The
matrices mix banded rows with rows of far-off random columns, with row counts
that leave ragged last tiles, and rows stored sorted or diagonal first."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def banded_plus_random(n, far_from, n_far, seed, diag_first=False):
    """7-point band of a 3-D grid of n rows (plus-minus 1, nx, nx*ny), and
    from row far_from on n_far extra random columns per row; diag_first
    stores each row's diagonal first, as hypre does."""
    rng = np.random.default_rng(seed)
    nx, ny = 13, 11
    row, cols, vals = [0], [], []
    for i in range(n):
        c = {i}
        for o in (1, nx, nx * ny):
            if i - o >= 0:
                c.add(i - o)
            if i + o < n:
                c.add(i + o)
        if i >= far_from:
            c.update(int(v) for v in rng.integers(0, n, n_far))
        c = sorted(c)
        if diag_first:
            c = [i] + [v for v in c if v != i]
        cols.extend(c)
        vals.extend((rng.standard_normal(len(c)) + np.where(np.array(c) == i, 8.0, 0.0)).tolist())
        row.append(len(cols))
    return np.array(row, np.uint32), np.array(cols, np.uint32), np.array(vals, np.float64)


def solver_on(gpu, row, col, val, nv, params):
    M = gpu.Matrix(row, col, val)
    xv, bv = gpu.Vector(M.n, nv), gpu.Vector(M.n, nv)
    xv.set(0.0)
    bv.set(1.0)
    return M, xv, bv, gpu.Solver(M, gpu.Params(params), xv, bv)


def run_level_spmv(gpu, S, level, which, row, col, val, nv, f32, seed):
    import torch
    n = len(row) - 1
    dt = torch.float32 if f32 else torch.float64
    rng = np.random.default_rng(seed)
    xh = rng.uniform(-1, 1, n * nv).astype(np.float32 if f32 else np.float64)
    y0 = rng.uniform(-1, 1, n * nv).astype(xh.dtype)
    x = torch.from_numpy(xh).cuda()
    y = torch.empty(n * nv, dtype=dt, device="cuda")
    S.level_spmv(level, which, x.data_ptr(), y.data_ptr(), nv, 0)
    ya = torch.from_numpy(y0).cuda()
    S.level_spmv(level, which, x.data_ptr(), ya.data_ptr(), nv, 1)
    torch.cuda.synchronize()
    return xh, y0, y.cpu().numpy(), ya.cpu().numpy()


def krylov(tune=1):
    return {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 10,
                       "gpu_spmv_tune": tune},
            "preconditioner": {"method": "Jacobi"}}


@pytest.mark.parametrize("nv", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("n,far_from,diag_first", [(3001, 2400, False), (2000, 2000, True),
                                                   (257, 200, False), (1003, 1003, True)])
@pytest.mark.parametrize("tune", [0, 1])
def test_fp64_level_spmv_bit_exact(gpu, oracle, nv, n, far_from, diag_first, tune):
    row, col, val = banded_plus_random(n, far_from, 9, seed=n + nv, diag_first=diag_first)
    _, _, _, S = solver_on(gpu, row, col, val, nv, krylov(tune))
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, 0, row, col, val, nv, False, seed=nv)
    want = oracle.csr_ax_y(row, col, val, xh, nv)
    assert y.tobytes() == want.tobytes()
    want_a = oracle.csr_ax_y(row, col, val, xh, nv, axpy_y=y0)
    assert ya.tobytes() == want_a.tobytes()


@pytest.mark.parametrize("nv", [1, 4, 8, 32])
@pytest.mark.parametrize("tune", [0, 1])
def test_fp32_cycle_operator_bit_exact(gpu, oracle, nv, tune):
    """Level 0 of an FP32 multigrid preconditioner (gpu_precond_f32 = 1),
    with 2-byte relative columns, on a 27-point FE matrix."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 3)
    params = {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 5,
                         "gpu_index_compress": 2},
              "preconditioner": {"method": "MultiGrid", "mg_max_levels": 3,
                                 "mg_coarsening_type": 8, "mg_interpolation_type": 6,
                                 "mg_agg_num_levels": 0, "gpu_spmv_tune": tune,
                                 "gpu_precond_f32": 1, "gpu_index_compress": 2},
              "pre_smoother": {"method": "Chebyshev"}, "post_smoother": {"method": "Chebyshev"}}
    _, _, _, S = solver_on(gpu, row, col, val, nv, params)
    info = S.level_info(0, 3)
    assert info["f32"]
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, 3, row, col, val, nv, True, seed=nv)
    v32 = val.astype(np.float32)
    assert y.tobytes() == oracle.csr_ax_y(row, col, v32, xh, nv).tobytes()
    assert ya.tobytes() == oracle.csr_ax_y(row, col, v32, xh, nv, axpy_y=y0).tobytes()


@pytest.mark.parametrize("nv", [1, 8, 32])
@pytest.mark.parametrize("tune", [0, 1])
def test_fp64_27pt_diag_first(gpu, oracle, nv, tune):
    """27-point FE rows stored diagonal first (hypre's order)."""
    row, col, val = gpu.generate_diffusion(27, 13, 12, 11, 1.0, 1.0, 5)
    col, val = col.copy(), val.copy()
    for i in range(len(row) - 1):
        a, b = int(row[i]), int(row[i + 1])
        d = a + int(np.nonzero(col[a:b] == i)[0][0])
        order = [d] + [j for j in range(a, b) if j != d]
        col[a:b], val[a:b] = col[order], val[order]
    _, _, _, S = solver_on(gpu, row, col, val, nv, krylov(tune))
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, 0, row, col, val, nv, False, seed=nv)
    assert y.tobytes() == oracle.csr_ax_y(row, col, val, xh, nv).tobytes()
    assert ya.tobytes() == oracle.csr_ax_y(row, col, val, xh, nv, axpy_y=y0).tobytes()


def bf16_round(v):
    """float64 values rounded to float32 and then to BF16 (round to nearest
    even), returned as float32: what an FP32 level stored in BF16 holds."""
    b = np.asarray(v, np.float64).astype(np.float32).view(np.uint32)
    b = (b + (((b >> 16) & 1) + 0x7FFF)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("nv", [1, 8, 32])
@pytest.mark.parametrize("tune", [0, 1])
def test_bf16_cycle_operators_bit_exact(gpu, oracle, nv, tune):
    """gpu_level_bf16 = 2: the two finest FP32 cycle operators store BF16
    values and compute in float. Their SpMVs must equal the oracle's float
    row sums over the BF16-rounded values bit for bit."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 3)
    params = {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 5,
                         "gpu_index_compress": 2},
              "preconditioner": {"method": "MultiGrid", "mg_max_levels": 3,
                                 "mg_coarsening_type": 8, "mg_interpolation_type": 6,
                                 "mg_agg_num_levels": 0, "gpu_spmv_tune": tune,
                                 "gpu_precond_f32": 1, "gpu_index_compress": 2,
                                 "gpu_level_bf16": 2},
              "pre_smoother": {"method": "Chebyshev"}, "post_smoother": {"method": "Chebyshev"}}
    _, _, _, S = solver_on(gpu, row, col, val, nv, params)
    assert S.level_info(0, 3)["bf16"] and S.level_info(1, 3)["bf16"]
    assert not S.level_info(2, 3)["bf16"]
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, 3, row, col, val, nv, True, seed=nv)
    vb = bf16_round(val)
    assert y.tobytes() == oracle.csr_ax_y(row, col, vb, xh, nv).tobytes()
    assert ya.tobytes() == oracle.csr_ax_y(row, col, vb, xh, nv, axpy_y=y0).tobytes()
    r1, c1, v1, info = S.level_download(1, 3)
    x1, y01, y1, ya1 = run_level_spmv(gpu, S, 1, 3, r1, c1, v1, nv, True, seed=nv + 1)
    assert y1.tobytes() == oracle.csr_ax_y(r1, c1.astype(np.uint32), v1, x1, nv).tobytes()


def fp16_round(v):
    """float64 values rounded to float32, divided by the level's power-of-two
    scale (2^(E-15) for the largest magnitude m * 2^E, m in [0.5, 1)),
    rounded to FP16 (nearest even) and multiplied back, as float32: what an
    FP32 level stored in FP16 holds."""
    f = np.asarray(v, np.float64).astype(np.float32)
    mx = float(np.abs(f).max())
    s = np.float32(2.0 ** max(np.frexp(mx)[1] - 15, -126)) if mx > 0 else np.float32(1.0)
    return ((f / s).astype(np.float16).astype(np.float32) * s).astype(np.float32)


@pytest.mark.parametrize("nv", [1, 8, 32])
@pytest.mark.parametrize("tune", [0, 1])
def test_fp16_cycle_operators_bit_exact(gpu, oracle, nv, tune):
    """gpu_level_bf16 = 2 with gpu_level_fp16 = 1: the two finest FP32 cycle
    operators store FP16 values scaled by a per-level power of two and
    compute in float. Their SpMVs must equal the oracle's float row sums over
    the values rounded that way bit for bit; the levels below keep float."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 3)
    params = {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 5,
                         "gpu_index_compress": 2},
              "preconditioner": {"method": "MultiGrid", "mg_max_levels": 3,
                                 "mg_coarsening_type": 8, "mg_interpolation_type": 6,
                                 "mg_agg_num_levels": 0, "gpu_spmv_tune": tune,
                                 "gpu_precond_f32": 1, "gpu_index_compress": 2,
                                 "gpu_level_bf16": 2, "gpu_level_fp16": 1},
              "pre_smoother": {"method": "Chebyshev"}, "post_smoother": {"method": "Chebyshev"}}
    _, _, _, S = solver_on(gpu, row, col, val, nv, params)
    assert S.level_info(0, 3)["fp16"] and S.level_info(1, 3)["fp16"]
    assert not S.level_info(0, 3)["bf16"]
    assert not S.level_info(2, 3)["fp16"]
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, 3, row, col, val, nv, True, seed=nv)
    vh = fp16_round(val)
    assert not np.array_equal(vh, val.astype(np.float32))  # the rounding is real
    assert y.tobytes() == oracle.csr_ax_y(row, col, vh, xh, nv).tobytes()
    assert ya.tobytes() == oracle.csr_ax_y(row, col, vh, xh, nv, axpy_y=y0).tobytes()
    r1, c1, v1, info = S.level_download(1, 3)
    x1, y01, y1, ya1 = run_level_spmv(gpu, S, 1, 3, r1, c1, v1, nv, True, seed=nv + 1)
    assert y1.tobytes() == oracle.csr_ax_y(r1, c1.astype(np.uint32), v1, x1, nv).tobytes()
    # the downloaded level-0 values are the FP16 values times the level's scale
    _, _, v0, _ = S.level_download(0, 3)
    assert v0.tobytes() == vh.tobytes()


@pytest.mark.parametrize("nv", [1, 2, 8, 32])
@pytest.mark.parametrize("f32", [False, True])
def test_warp_per_row_kernel_bit_exact(gpu, oracle, nv, f32):
    """The warp-per-row SpMV (gpu_spmv_tune = 3; an autotuner candidate for
    small matrices) on rows long enough to span several chunks of its
    shared-memory product buffer: every element equals the oracle's
    sequential row sum, for y = A x and y += A x."""
    row, col, val = banded_plus_random(1500, 700, 300, seed=nv + 50)
    krylov = {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 5,
              "gpu_spmv_tune": 3}
    params = {"solver": krylov}
    if f32:
        params = {"solver": dict(krylov, gpu_index_compress=2),
                  "preconditioner": {"method": "MultiGrid", "mg_max_levels": 2,
                                     "mg_coarsening_type": 8, "mg_interpolation_type": 6,
                                     "mg_agg_num_levels": 0, "gpu_precond_f32": 1,
                                     "gpu_spmv_tune": 3},
                  "pre_smoother": {"method": "Jacobi"}, "post_smoother": {"method": "Jacobi"}}
    _, _, _, S = solver_on(gpu, row, col, val, nv, params)
    which = 3 if f32 else 0
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, which, row, col, val, nv, f32, seed=nv)
    v = val.astype(np.float32) if f32 else val
    assert y.tobytes() == oracle.csr_ax_y(row, col, v, xh, nv).tobytes()
    assert ya.tobytes() == oracle.csr_ax_y(row, col, v, xh, nv, axpy_y=y0).tobytes()


@pytest.mark.parametrize("nv", [1, 2, 8, 32])
@pytest.mark.parametrize("bf16", [False, True])
def test_x_staged_kernel_bit_exact(gpu, oracle, nv, bf16):
    """The x-staged SpMV (gpu_spmv_tune = 4; an autotuner candidate on
    multigrid levels with long rows): each tile's x rows copied once into
    shared memory by unique column, each row summed from there in entry
    order. Every element equals the oracle's sequential row sum, for y = A x
    and y += A x, on the FP32 cycle operator (FP32 or BF16 values) of a
    27-point matrix (8,000 rows, diagonal first)."""
    row, col, val = gpu.generate_diffusion(27, 20, 20, 20, 1.0, 1.0, nv + 70)
    params = {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 5,
                         "gpu_index_compress": 2},
              "preconditioner": {"method": "MultiGrid", "mg_max_levels": 2,
                                 "mg_coarsening_type": 8, "mg_interpolation_type": 6,
                                 "mg_agg_num_levels": 0, "gpu_precond_f32": 1,
                                 "gpu_index_compress": 2, "gpu_spmv_tune": 4,
                                 "gpu_level_bf16": 1 if bf16 else 0},
              "pre_smoother": {"method": "Jacobi"}, "post_smoother": {"method": "Jacobi"}}
    _, _, _, S = solver_on(gpu, row, col, val, nv, params)
    assert S.level_xstaged(0, 3) == nv
    xh, y0, y, ya = run_level_spmv(gpu, S, 0, 3, row, col, val, nv, True, seed=nv)
    v = bf16_round(val) if bf16 else val.astype(np.float32)
    assert y.tobytes() == oracle.csr_ax_y(row, col, v, xh, nv).tobytes()
    assert ya.tobytes() == oracle.csr_ax_y(row, col, v, xh, nv, axpy_y=y0).tobytes()


def test_x_staged_solves_same_bits(gpu):
    """Whole FP32-preconditioned solves on a 27-point matrix whose first two
    levels get an x-staged copy (gpu_spmv_tune = 4): the same bits and
    iterations as the CSR kernel."""
    row, col, val = gpu.generate_diffusion(27, 40, 40, 40, 1.0, 1.0, 8)
    nv = 8
    n = len(row) - 1
    b = np.random.default_rng(33).uniform(-1, 1, n * nv)
    out = {}
    for t in (0, 4):
        params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 100,
                             "rel_tolerance": 1e-8, "abs_tolerance": 0,
                             "gpu_index_compress": 2},
                  "preconditioner": {"method": "MultiGrid", "mg_coarsening_type": 8,
                                     "mg_interpolation_type": 6, "mg_agg_num_levels": 0,
                                     "mg_coarse_matrix_size": 500, "gpu_precond_f32": 1,
                                     "gpu_index_compress": 2, "gpu_spmv_tune": t},
                  "pre_smoother": {"method": "Chebyshev"},
                  "post_smoother": {"method": "Chebyshev"},
                  "coarse_grid_solver": {"method": "Direct"}}
        M, xv, bv, S = solver_on(gpu, row, col, val, nv, params)
        bv.upload(b)
        for _ in range(2):
            xv.set(0.0)
            S.solve()
        assert S.level_xstaged(1, 3) == (nv if t else 0)
        out[t] = (xv.download(), S.stats()["iters"])
    assert out[0][0].tobytes() == out[4][0].tobytes()
    assert out[0][1] == out[4][1]
