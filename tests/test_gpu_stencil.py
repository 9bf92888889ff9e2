"""The grid-stencil SpMV (gpu_index_compress = 3, csrc/stencil.cuh) against
the CSR SpMV it stands in for: a multigrid solver built with the stencil
copy of its level-0 operator must give, for y = A x and y += A x and for
whole solves, the same bits as the same solver on the CSR form (itself
bit-exact against the oracle's row sums). Matrices: 27-point FE diffusion,
7-point finite-volume diffusion and the reference's 7-point cube generator
(all three store each row's diagonal first) and the 27-point matrix with
its rows sorted, on grids whose edges differ and leave partial groups of
lines; FP64, FP32 and BF16 level values; nv 1..32."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

def sorted_rows(m):
    row, col, val = m
    col, val = col.copy(), val.copy()
    for i in range(len(row) - 1):
        a, b = int(row[i]), int(row[i + 1])
        o = np.argsort(col[a:b], kind="stable")
        col[a:b], val[a:b] = col[a:b][o], val[a:b][o]
    return row, col, val


MATS = {
    "fe27": lambda X: X.generate_diffusion(27, 13, 11, 10, 1.0, 1.0, 2),
    "fe27s": lambda X: sorted_rows(X.generate_diffusion(27, 11, 13, 9, 1.0, 1.0, 4)),
    "fv7": lambda X: X.generate_diffusion(7, 12, 9, 11, 1.5, 1.0, 3),
    "cube": lambda X: X.generate_cube(10, 13, 9),
}


def params(compress, f32, bf16, smoother="Chebyshev", tune=0):
    """tune: gpu_spmv_tune (0: the stencil kernel's 64-register form, 2: its
    128-register form, 1: whichever of those and the CSR kernel measured
    fastest)."""
    prec = {"method": "MultiGrid", "mg_max_levels": 3, "mg_coarsening_type": 8,
            "mg_interpolation_type": 6, "mg_agg_num_levels": 0, "gpu_index_compress": compress,
            "gpu_precond_f32": 1 if f32 else 0, "gpu_level_bf16": 1 if bf16 else 0,
            "gpu_spmv_tune": tune}
    return {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 100,
                       "abs_tolerance": 0, "gpu_index_compress": compress, "gpu_spmv_tune": tune},
            "preconditioner": prec, "pre_smoother": {"method": smoother},
            "post_smoother": {"method": smoother}, "coarse_grid_solver": {"method": "Direct"}}


def build(gpu, row, col, val, nv, p):
    M = gpu.Matrix(row, col, val)
    xv, bv = gpu.Vector(M.n, nv), gpu.Vector(M.n, nv)
    xv.set(0.0)
    bv.set(1.0)
    return M, xv, bv, gpu.Solver(M, gpu.Params(p), xv, bv)


def level0_spmv(S, nv, f32, seed):
    import torch
    n = S.level_info(0, 3)["nrows"]
    dt = torch.float32 if f32 else torch.float64
    g = torch.Generator().manual_seed(seed)
    x = (torch.rand(n * nv, generator=g, dtype=torch.float64) * 2 - 1).to(dt).cuda()
    y0 = (torch.rand(n * nv, generator=g, dtype=torch.float64) * 2 - 1).to(dt).cuda()
    y = torch.empty_like(x)
    ya = y0.clone()
    S.level_spmv(0, 3, x.data_ptr(), y.data_ptr(), nv, 0)
    S.level_spmv(0, 3, x.data_ptr(), ya.data_ptr(), nv, 1)
    torch.cuda.synchronize()
    return x.cpu().numpy(), y0.cpu().numpy(), y.cpu().numpy(), ya.cpu().numpy()


@pytest.mark.parametrize("mat", list(MATS))
@pytest.mark.parametrize("form", ["f64", "f32", "bf16"])
@pytest.mark.parametrize("nv", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("tune", [0, 2])
def test_level0_spmv_same_bits(gpu, oracle, mat, form, nv, tune):
    row, col, val = MATS[mat](gpu)
    f32, bf16 = form != "f64", form == "bf16"
    out = {}
    for compress in (2, 3):
        _, _, _, S = build(gpu, row, col, val, nv, params(compress, f32, bf16, tune=tune))
        pat = S.level_stencil(0, 3)
        if compress == 3:
            assert pat[0] == (0 if mat.startswith("fe27") else 1), pat
            assert pat[3] == (0 if mat == "fe27s" else 1), pat
        else:
            assert pat[0] == -1
        out[compress] = level0_spmv(S, nv, f32, seed=nv)
    for a, b in zip(out[2], out[3]):
        assert a.tobytes() == b.tobytes()
    if form == "f64":
        xh, y0, y, ya = out[3]
        assert y.tobytes() == oracle.csr_ax_y(row, col, val, xh, nv).tobytes()
        assert ya.tobytes() == oracle.csr_ax_y(row, col, val, xh, nv, axpy_y=y0).tobytes()


@pytest.mark.parametrize("mat", list(MATS))
@pytest.mark.parametrize("form,smoother", [("f64", "Chebyshev"), ("f32", "Chebyshev"),
                                           ("bf16", "Chebyshev"), ("f32", "Jacobi")])
@pytest.mark.parametrize("tune", [0, 1])
def test_solves_same_bits(gpu, mat, form, smoother, tune):
    """Whole preconditioned solves: same iterations and solution bits (with
    the autotuner on, the stencil and CSR kernels give the same bits
    whichever it picks)."""
    row, col, val = MATS[mat](gpu)
    nv = 4
    n = len(row) - 1
    b = np.random.default_rng(7).uniform(-1, 1, n * nv)
    res = {}
    for compress in (2, 3):
        _, xv, bv, S = build(gpu, row, col, val, nv,
                             params(compress, form != "f64", form == "bf16", smoother, tune))
        bv.upload(b)
        for _ in range(2):  # the second solve replays the recorded graphs
            xv.set(0.0)
            S.solve()
        st = S.stats()
        res[compress] = (st["iters"], xv.download())
        assert st["conv"].all()
    assert res[2][0] == res[3][0]
    assert res[2][1].tobytes() == res[3][1].tobytes()
