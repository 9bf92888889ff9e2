"""Whole solves through the public XAMG C API on the GPU, checked against the
oracle. With the oracle replaying the kernels' fixed reduction order (mode 1)
the GPU solution, iteration count and residuals must be identical bit for
bit; against XAMG's own sequential order (mode 0) they must agree to 1e-6
relative with both true residuals at the tolerance."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

MG_BASE = {"mg_agg_num_levels": 0, "mg_strength_threshold": 0.25, "mg_coarsening_type": 8,
           "mg_interpolation_type": 6, "mg_coarse_matrix_size": 60, "max_iters": 1}


def gpu_solve(xamg, row, col, val, nv, params, b, x0=None, overrides=None):
    M = xamg.Matrix(row, col, val)
    X = xamg.Vector(M.n, nv, M.part)
    B = xamg.Vector(M.n, nv, M.part)
    B.upload(b)
    if x0 is None:
        X.set(0.0)
    else:
        X.upload(x0)
    P = xamg.Params(params, overrides=overrides)
    S = xamg.Solver(M, P, X, B)
    S.solve()
    return X.download(), S.stats(), S


def oracle_solve(oracle, S_gpu, row, col, val, nv, params, b, mode, x0=None, hsgs_rows=32):
    sysm = oracle.System(nv)
    sysm.set_params(params)
    sysm.hsgs_cores(-hsgs_rows)
    mg = "MultiGrid" in (params.get("solver", {}).get("method"),
                         params.get("preconditioner", {}).get("method"))
    if mg:
        for lv in S_gpu.hierarchy():
            sysm.add_level(*lv["A"], lv["min_eig"], lv["max_eig"])
            if lv["P"] is not None:
                sysm.add_interp(*lv["P"])
    else:
        sysm.add_level(row, col, val)
    sysm.setup()
    oracle.set_reduction(mode)
    try:
        x, st = sysm.solve(b, x0)
    finally:
        oracle.set_reduction(0)
    return x, st, sysm


def true_rel_res(row, col, val, x, b, nv):
    A = sp.csr_matrix((val.copy(), col.copy(), row.copy()))
    X, Bm = x.reshape(-1, nv), b.reshape(-1, nv)
    return np.linalg.norm(Bm - A @ X, axis=0) / np.linalg.norm(Bm, axis=0)


def check(xamg, oracle, row, col, val, nv, params, seed=0, tol=1e-8, overrides=None,
          hsgs_rows=32):
    n = len(row) - 1
    b = np.random.default_rng(seed).uniform(-1, 1, n * nv)
    xg, sg, S = gpu_solve(xamg, row, col, val, nv, params, b, overrides=overrides)
    # bit-exact against the replay of the kernels' order
    xo, so, _ = oracle_solve(oracle, S, row, col, val, nv, params, b, 1, hsgs_rows=hsgs_rows)
    assert sg["iters"] == so["iters"]
    assert sg["conv"].tolist() == so["conv"].tolist()
    assert sg["rel_res"].tobytes() == so["rel_res"].tobytes()
    assert xg.tobytes() == xo.tobytes(), np.abs(xg - xo).max()
    # against XAMG's sequential order
    xs, ss, _ = oracle_solve(oracle, S, row, col, val, nv, params, b, 0, hsgs_rows=hsgs_rows)
    assert all(sg["conv"]) and all(ss["conv"])
    # the convergence test uses the recursive residual (res = theta - omega*phi,
    # merged_bicgstab.inl:170-171); the true residual may drift a little above it
    rg = true_rel_res(row, col, val, xg, b, nv)
    rs = true_rel_res(row, col, val, xs, b, nv)
    assert rg.max() <= 10 * tol and rs.max() <= 10 * tol, (rg, rs)
    dx = np.linalg.norm((xg - xs).reshape(-1, nv), axis=0) / np.linalg.norm(xs.reshape(-1, nv),
                                                                             axis=0)
    assert dx.max() <= 1e-6, dx
    return sg, S


def test_config1_merged_pbicgstab_jacobi(gpu, oracle):
    """32^3 Poisson, nv = 1, MergedPBiCGStab + Jacobi, FP64, 1e-8."""
    row, col, val = gpu.generate_cube(32, 32, 32)
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 1000, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": {"method": "Jacobi"}}
    st, S = check(gpu, oracle, row, col, val, 1, params)
    assert 30 < st["iters"] < 80
    # XAMG narrowing: 32768 columns -> 2-byte column indices on the device
    assert S.level_info(0, 0)["col_bytes"] == 2


@pytest.mark.parametrize("method", ["PBiCGStab", "BiCGStab", "MergedBiCGStab", "PCG",
                                    "RBiCGStab", "MergedRBiCGStab"])
@pytest.mark.parametrize("nv", [2, 8])
def test_krylov_variants(gpu, oracle, method, nv):
    row, col, val = gpu.generate_cube(14, 13, 12)
    params = {"solver": {"method": method, "max_iters": 500, "rel_tolerance": 1e-9,
                         "abs_tolerance": 0}}
    if method in ("PBiCGStab", "PCG", "RBiCGStab", "MergedRBiCGStab"):
        params["preconditioner"] = {"method": "Jacobi", "max_iters": 3}
    check(gpu, oracle, row, col, val, nv, params, seed=nv, tol=1e-9)


@pytest.mark.parametrize("precond", [None, "MultiGrid"])
def test_pcg(gpu, oracle, precond):
    """PCG (pcg.inl:44-162): unpreconditioned (the identity) and with an AMG
    V-cycle (Jacobi smoothing keeps the preconditioner symmetric)."""
    row, col, val = gpu.generate_diffusion(7, 15, 14, 13, 1.0, 1.0, 6)
    nv = 4
    params = {"solver": {"method": "PCG", "max_iters": 400, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0}}
    if precond:
        params["preconditioner"] = dict(MG_BASE, method="MultiGrid")
        params["pre_smoother"] = {"method": "Jacobi"}
        params["post_smoother"] = {"method": "Jacobi"}
        params["coarse_grid_solver"] = {"method": "Direct"}
    st, S = check(gpu, oracle, row, col, val, nv, params, seed=3)
    assert st["iters"] < (40 if precond else 400)


@pytest.mark.parametrize("smoother,reduced", [("Jacobi", 0), ("Chebyshev", 0), ("HSGS", 0),
                                              ("Chebyshev", 1), ("HSGS", 1), ("Jacobi", 1),
                                              ("Chebyshev", "full32"), ("HSGS", "full32")])
def test_amg_preconditioner(gpu, oracle, smoother, reduced):
    """reduced: 0 FP64 (XAMG), 1 XAMG's mg_reduced_precision (levels >= 1 in
    float), "full32" every level in float with 2-byte relative columns."""
    row, col, val = gpu.generate_diffusion(7, 18, 17, 16, 1.0, 1.0, 0)
    nv = 4
    sm = {"method": smoother}
    if smoother == "Chebyshev":
        sm["polynomial_order"] = 2
    if smoother == "HSGS":
        sm["max_iters"] = 1
    prec = dict(MG_BASE, method="MultiGrid", mg_reduced_precision=int(reduced == 1))
    solver = {"method": "MergedPBiCGStab", "max_iters": 300, "rel_tolerance": 1e-8,
              "abs_tolerance": 0}
    if reduced == "full32":
        prec.update(gpu_precond_f32=1, gpu_index_compress=2)
        solver["gpu_index_compress"] = 2
    params = {"solver": solver, "preconditioner": prec,
              "pre_smoother": sm, "post_smoother": dict(sm), "coarse_grid_solver": {"method": "Direct"}}
    st, S = check(gpu, oracle, row, col, val, nv, params, seed=5)
    assert S.nlevels() >= 3
    assert st["iters"] < 60


def test_uploaded_levels_match_oracle_narrowing(gpu, oracle):
    """Every uploaded level matrix equals, bit for bit, what XAMG's parse of the
    same hierarchy produces: values converted to float when reduced, columns
    narrowed to define_int_type(ncols), R = transpose(P)."""
    row, col, val = gpu.generate_diffusion(27, 12, 12, 12, 1.0, 1.0, 1)
    nv = 2
    params = {"solver": {"method": "PBiCGStab", "max_iters": 100},
              "preconditioner": dict(MG_BASE, method="MultiGrid", mg_reduced_precision=1),
              "pre_smoother": {"method": "Chebyshev"}, "post_smoother": {"method": "Chebyshev"}}
    b = np.random.default_rng(0).uniform(-1, 1, (len(row) - 1) * nv)
    _, _, S = gpu_solve(gpu, row, col, val, nv, params, b)
    _, _, sysm = oracle_solve(oracle, S, row, col, val, nv, params, b, 1)
    nl = S.nlevels()
    assert nl >= 3
    for l in range(nl):
        for which in ((0, 1, 2) if l + 1 < nl else (0,)):
            r, c, v, info = S.level_download(l, which)
            orow, ocol, oval, oncols = sysm.level_matrix(l, which)
            assert info["col_bytes"] == {0: 1, 1: 2, 2: 4}[oracle.define_int_type(info["ncols"])]
            assert info["hash"] == oracle.encode_hash(info["nnz"], info["ncols"], info["nrows"],
                                                      info["ncols"], reduced=info["f32"])
            assert r.tobytes() == orow.tobytes()
            assert c.astype(np.uint32).tobytes() == ocol.tobytes()
            assert v.dtype == oval.dtype and v.tobytes() == oval.tobytes()


def test_multigrid_as_solver(gpu, oracle):
    row, col, val = gpu.generate_diffusion(7, 16, 16, 16, 1.0, 1.0, 2)
    params = {"solver": dict(MG_BASE, method="MultiGrid", max_iters=100, rel_tolerance=1e-8,
                             abs_tolerance=0),
              "pre_smoother": {"method": "Jacobi"}, "post_smoother": {"method": "Jacobi"}}
    check(gpu, oracle, row, col, val, 2, params, seed=9)


def test_jacobi_as_solver(gpu, oracle):
    row, col, val = gpu.generate_cube(8, 8, 8)
    params = {"solver": {"method": "Jacobi", "max_iters": 2000, "rel_tolerance": 1e-6,
                         "abs_tolerance": 0}}
    check(gpu, oracle, row, col, val, 1, params, tol=1e-6)


def test_zero_rhs_converges_at_once(gpu):
    row, col, val = gpu.generate_cube(6, 6, 6)
    params = {"solver": {"method": "MergedPBiCGStab"}, "preconditioner": {"method": "Jacobi"}}
    x, st, S = gpu_solve(gpu, row, col, val, 4, params, np.zeros(216 * 4))
    assert st["iters"] == 0 and all(st["conv"])
    assert not x.any()


def test_renew_params_and_solve2(gpu):
    row, col, val = gpu.generate_cube(12, 12, 12)
    n, nv = len(row) - 1, 2
    params = {"solver": {"method": "PBiCGStab", "max_iters": 500, "rel_tolerance": 1e-4,
                         "abs_tolerance": 0},
              "preconditioner": {"method": "Jacobi"}}
    b = np.random.default_rng(0).uniform(-1, 1, n * nv)
    x, st1, S = gpu_solve(gpu, row, col, val, nv, params, b)
    P2 = gpu.Params({"solver": {"rel_tolerance": 1e-10}}, set_default=False)
    S.renew(P2)
    M = gpu.Matrix(row, col, val)
    X = gpu.Vector(n, nv)
    B = gpu.Vector(n, nv)
    X.set(0.0)
    B.upload(b)
    S.solve(X, B)
    st2 = S.stats()
    assert st2["iters"] > st1["iters"]
    assert true_rel_res(row, col, val, X.download(), b, nv).max() < 1e-9
    assert S.convergence_info().tolist() == [1, 1]


def test_nv_mismatch_is_an_error(gpu):
    row, col, val = gpu.generate_cube(4, 4, 4)
    M = gpu.Matrix(row, col, val)
    X = gpu.Vector(64, 2)
    B = gpu.Vector(64, 2)
    X.set(0.0)
    B.set(1.0)
    S = gpu.Solver(M, gpu.Params({"solver": {"method": "BiCGStab"}}), X, B)
    with pytest.raises(gpu.XamgError) as e:
        gpu.call("XAMG_solver_solve1", 4, S.h)
    assert e.value.code == -3
    with pytest.raises(gpu.XamgError):
        gpu.call("XAMG_vector_alloc_d", 10, 3, X.h)


@pytest.mark.parametrize("smoother", ["Chebyshev", "HSGS"])
def test_graph_replay_matches_direct_launches(gpu, smoother):
    """gpu_graph = 1 (default) records each preconditioner application as a
    CUDA graph on its second call and replays it; gpu_graph = 0 launches every
    kernel directly. Both must give the same solution bit for bit, with the
    same iterations and the same kernel count."""
    row, col, val = gpu.generate_diffusion(27, 20, 19, 18, 1.0, 1.0, 2)
    nv = 8
    sm = {"method": smoother}
    if smoother == "HSGS":
        sm["max_iters"] = 1
    prec = dict(MG_BASE, method="MultiGrid", gpu_precond_f32=1, gpu_index_compress=2)
    b = np.random.default_rng(9).uniform(-1, 1, (len(row) - 1) * nv)
    out = []
    for graph in (0, 1):
        params = {"solver": {"method": "PBiCGStab", "max_iters": 100, "rel_tolerance": 1e-8,
                             "gpu_graph": graph, "gpu_index_compress": 2},
                  "preconditioner": prec, "pre_smoother": sm, "post_smoother": dict(sm)}
        k0 = gpu.kernel_launches()
        x, st, S = gpu_solve(gpu, row, col, val, nv, params, b)
        out.append((x, st, gpu.kernel_launches() - k0))
    (x0, s0, l0), (x1, s1, l1) = out
    assert s0["iters"] == s1["iters"] and s0["iters"] >= 3
    assert x0.tobytes() == x1.tobytes()
    assert l0 == l1


@pytest.mark.parametrize("method,prec,cap", [("MergedPBiCGStab", "Jacobi", 200),
                                             ("MergedPBiCGStab", "Jacobi", 9),
                                             ("PBiCGStab", "MultiGrid", 200),
                                             ("MergedBiCGStab", None, 200),
                                             ("MergedBiCGStab", None, 11),
                                             ("PCG", "MultiGrid", 200),
                                             ("PCG", None, 12),
                                             ("RBiCGStab", "MultiGrid", 200),
                                             ("MergedRBiCGStab", "Jacobi", 200),
                                             ("MergedRBiCGStab", "Jacobi", 10)])
def test_step_graph_matches_direct_launches(gpu, oracle, method, prec, cap):
    """gpu_graph = 1 also records each BiCGStab iteration (the previous
    iteration's x, r and p updates, then the iteration up to its residual),
    and each PCG or RBiCGStab iteration, as a CUDA graph on its third call
    and replays it from then on. Over a solve
    of many iterations, converged or stopped at max_iters (cap), the replayed
    form must give the direct launches' solution, iterations and kernel count
    bit for bit, and match the oracle."""
    row, col, val = gpu.generate_cube(24, 24, 24)
    nv = 2
    b = np.random.default_rng(5).uniform(-1, 1, (len(row) - 1) * nv)
    out = []
    for graph in (0, 1):
        params = {"solver": {"method": method, "max_iters": cap, "rel_tolerance": 1e-8,
                             "abs_tolerance": 0, "gpu_graph": graph}}
        if prec == "Jacobi":
            params["preconditioner"] = {"method": "Jacobi"}
        elif prec == "MultiGrid":
            params.update(preconditioner=dict(MG_BASE, method="MultiGrid"),
                          pre_smoother={"method": "Jacobi"}, post_smoother={"method": "Jacobi"},
                          coarse_grid_solver={"method": "Direct"})
        k0 = gpu.kernel_launches()
        x, st, S = gpu_solve(gpu, row, col, val, nv, params, b)
        out.append((x, st, gpu.kernel_launches() - k0))
    (x0, s0, l0), (x1, s1, l1) = out
    assert s0["iters"] == s1["iters"] and s0["iters"] >= 5
    assert (s0["iters"] == cap) == (cap < 100)
    assert x0.tobytes() == x1.tobytes()
    assert l0 == l1
    xo, so, _ = oracle_solve(oracle, S, row, col, val, nv, params, b, 1)
    assert s1["iters"] == so["iters"]
    assert s1["conv"].tolist() == so["conv"].tolist()
    assert x1.tobytes() == xo.tobytes()


@pytest.mark.parametrize("method", ["RBiCGStab", "MergedRBiCGStab"])
@pytest.mark.parametrize("f32", [0, 1])
def test_rbicgstab_with_amg(gpu, oracle, method, f32):
    """Reordered BiCGStab (rbicgstab.inl, merged_rbicgstab.inl) with an AMG
    V-cycle as the preconditioner (FP64, or FP32 with 2-byte relative
    columns), its three applications graph-replayed. The GPU must match the
    oracle bit for bit whether or not the recurrence converges."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 7)
    nv = 8
    params = {"solver": {"method": method, "max_iters": 60, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": dict(MG_BASE, method="MultiGrid"),
              "pre_smoother": {"method": "Chebyshev"}, "post_smoother": {"method": "Chebyshev"},
              "coarse_grid_solver": {"method": "Direct"}}
    if f32:
        params["solver"]["gpu_index_compress"] = 2
        params["preconditioner"].update(gpu_precond_f32=1, gpu_index_compress=2)
    b = np.random.default_rng(8).uniform(-1, 1, (len(row) - 1) * nv)
    xg, sg, S = gpu_solve(gpu, row, col, val, nv, params, b)
    xo, so, _ = oracle_solve(oracle, S, row, col, val, nv, params, b, 1)
    assert sg["iters"] == so["iters"]
    assert sg["conv"].tolist() == so["conv"].tolist()
    assert sg["rel_res"].tobytes() == so["rel_res"].tobytes()
    assert xg.tobytes() == xo.tobytes()


@pytest.mark.parametrize("stencil,edge,nv,f32", [(27, 14, 8, True), (27, 12, 4, False),
                                                 (7, 20, 16, True), (7, 18, 32, False)])
def test_autotuned_spmv_same_results(gpu, stencil, edge, nv, f32):
    """The SpMV autotuner (gpu_spmv_tune) only picks launch shapes: a solve
    with it equals the solve without it bit for bit, and it has recorded a
    choice for the matrices the preconditioner's SpMVs ran on."""
    row, col, val = gpu.generate_diffusion(stencil, edge, edge, edge, 1.0, 1.0, 4)
    n = len(row) - 1
    b = np.random.default_rng(9).uniform(-1, 1, n * nv)
    sm = {"method": "Chebyshev", "polynomial_order": 2}
    out = {}
    for tune in (0, 1):
        params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 100,
                             "rel_tolerance": 1e-8, "abs_tolerance": 0, "gpu_spmv_tune": tune},
                  "preconditioner": dict(MG_BASE, method="MultiGrid",
                                         gpu_precond_f32=1 if f32 else 0, gpu_spmv_tune=tune),
                  "pre_smoother": sm, "post_smoother": dict(sm),
                  "coarse_grid_solver": {"method": "Direct"}}
        x, st, S = gpu_solve(gpu, row, col, val, nv, params, b)
        out[tune] = (x, st)
        codes = S.level_tuned(1, 3)
        assert (codes.any()) == bool(tune)
    assert out[0][0].tobytes() == out[1][0].tobytes()
    assert out[0][1]["iters"] == out[1][1]["iters"]


@pytest.mark.parametrize("stencil,edge,nv,f32", [(27, 20, 8, True), (27, 18, 4, False),
                                                 (7, 22, 16, True), (27, 17, 2, False)])
def test_plane_walk_spmv_same_results(gpu, oracle, stencil, edge, nv, f32):
    """gpu_spmv_tune = 5 runs every SpMV without dot products on a matrix
    with a plane-walk distance in the walk order (each block taking tiles one
    grid plane apart; the grids leave tiles past the last whole plane, which
    keep their order). Only the order in which tiles are visited changes, so
    the solve equals the untuned one and the oracle in the kernels' order bit
    for bit."""
    row, col, val = gpu.generate_diffusion(stencil, edge, edge, edge, 1.0, 1.0, 5)
    n = len(row) - 1
    b = np.random.default_rng(10).uniform(-1, 1, n * nv)
    sm = {"method": "Chebyshev", "polynomial_order": 2}
    out = {}
    for tune in (0, 5):
        params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 100,
                             "rel_tolerance": 1e-8, "abs_tolerance": 0, "gpu_spmv_tune": tune},
                  "preconditioner": dict(MG_BASE, method="MultiGrid",
                                         gpu_precond_f32=1 if f32 else 0, gpu_spmv_tune=tune),
                  "pre_smoother": sm, "post_smoother": dict(sm),
                  "coarse_grid_solver": {"method": "Direct"}}
        if f32:
            params["solver"]["gpu_index_compress"] = 2
            params["preconditioner"]["gpu_index_compress"] = 2
        out[tune] = gpu_solve(gpu, row, col, val, nv, params, b)
    x5, s5, S5 = out[5]
    assert out[0][0].tobytes() == x5.tobytes()
    assert out[0][1]["iters"] == s5["iters"]
    xo, so, _ = oracle_solve(oracle, S5, row, col, val, nv, params, b, 1)
    assert s5["iters"] == so["iters"]
    assert x5.tobytes() == xo.tobytes()


@pytest.mark.parametrize("method", ["PCG", "MergedRBiCGStab"])
def test_graph_fallback_keeps_zero_flag(gpu, method):
    """A preconditioner that reads back its residual (Jacobi with
    convergence_check) cannot be recorded into an iteration graph. The
    recording attempt changes the host-side flags as if the iteration had
    run; the direct run that follows must start from the flags it was called
    with. Each solve writes into a fresh, zero-flagged x placed at the address
    of the previous one (so its memory holds the previous solution): the
    iteration graph key (lane, x zero, x) repeats, and the third solve is the
    one whose recording fails. Every solve must equal the same solve without
    graphs bit for bit."""
    row, col, val = gpu.generate_diffusion(7, 16, 15, 14, 1.0, 1.0, 11)
    n, nv = len(row) - 1, 2
    M = gpu.Matrix(row, col, val)
    B = gpu.Vector(n, nv, M.part)
    b = np.random.default_rng(12).uniform(-1, 1, n * nv)
    B.upload(b)
    results = {}
    for graph in (0, 1):
        params = {"solver": {"method": method, "max_iters": 200, "rel_tolerance": 1e-8,
                             "abs_tolerance": 0, "gpu_graph": graph},
                  "preconditioner": {"method": "Jacobi", "max_iters": 2,
                                     "convergence_check": 1, "rel_tolerance": 1e-12,
                                     "abs_tolerance": 0}}
        P = gpu.Params(params)
        X = gpu.Vector(n, nv, M.part)
        S = gpu.Solver(M, P, X, B)
        addr, out = None, []
        for i in range(4):
            if i:
                # a fresh vector where the last one was: zero-flagged, its
                # memory still holding the previous solution
                gpu.call("XAMG_vector_destroy", X.h)
                X = gpu.Vector(n, nv, M.part)
                assert X.device_ptr() == addr, "allocator did not reuse the address"
            addr = X.device_ptr()
            gpu.call("XAMG_solver_solve2", nv, X.h, B.h, S.h)
            out.append((X.download(), S.stats()["iters"]))
        results[graph] = out
        gpu.call("XAMG_vector_destroy", X.h)
    for (x0, i0), (x1, i1) in zip(results[0], results[1]):
        assert i0 == i1
        assert x0.tobytes() == x1.tobytes()
    r = true_rel_res(row, col, val, results[1][-1][0], b, nv)
    assert r.max() < 1e-7


@pytest.mark.parametrize("f32", [0, 1])
def test_w_cycle(gpu, oracle, f32):
    """mg_cycle = 2 (W-cycle, mg.inl:229-232) as the preconditioner, FP64 or
    FP32, against the oracle bit for bit and XAMG's order to 1e-6."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 21)
    sm = {"method": "Chebyshev", "polynomial_order": 2}
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 100, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": dict(MG_BASE, method="MultiGrid", mg_cycle=2,
                                     mg_coarse_matrix_size=20),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    if f32:
        params["solver"]["gpu_index_compress"] = 2
        params["preconditioner"].update(gpu_precond_f32=1, gpu_index_compress=2)
    st, S = check(gpu, oracle, row, col, val, 4, params, seed=2)
    assert S.nlevels() >= 4


@pytest.mark.parametrize("f32", [0, 1])
def test_f_cycle_as_the_reference_runs_it(gpu, oracle, f32):
    """mg_cycle = 1 (F-cycle, mg.inl:198,233-234). Its first visit of a level
    skips pre-smoothing, and the prolongation then adds P x_H to whatever the
    zero-flagged x holds from the previous cycle (blas2 Axpy accumulates into
    the vector's memory). The reference built from its own sources does
    exactly this (oracle pinned to it in tests/test_ref_pins.py), and on this
    matrix the preconditioner it gives stalls the iteration. The GPU must
    reproduce the same iterates bit for bit, solve after solve."""
    row, col, val = gpu.generate_diffusion(27, 14, 13, 12, 1.0, 1.0, 21)
    nv = 4
    sm = {"method": "Chebyshev", "polynomial_order": 2}
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 30, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": dict(MG_BASE, method="MultiGrid", mg_cycle=1,
                                     mg_coarse_matrix_size=20),
              "pre_smoother": sm, "post_smoother": dict(sm),
              "coarse_grid_solver": {"method": "Direct"}}
    if f32:
        params["solver"]["gpu_index_compress"] = 2
        params["preconditioner"].update(gpu_precond_f32=1, gpu_index_compress=2)
    n = len(row) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n * nv)
    M = gpu.Matrix(row, col, val)
    X, B = gpu.Vector(n, nv, M.part), gpu.Vector(n, nv, M.part)
    B.upload(b)
    X.set(0.0)
    S = gpu.Solver(M, gpu.Params(params), X, B)
    sysm = oracle.System(nv)
    sysm.set_params(params)
    for lv in S.hierarchy():
        sysm.add_level(*lv["A"], lv["min_eig"], lv["max_eig"])
        if lv["P"] is not None:
            sysm.add_interp(*lv["P"])
    sysm.setup()
    for _ in range(2):   # the second solve starts from the buffers the first left
        X.set(0.0)
        S.solve()
        xg, sg = X.download(), S.stats()
        oracle.set_reduction(1)
        try:
            xo, so = sysm.solve(b)
        finally:
            oracle.set_reduction(0)
        assert sg["iters"] == so["iters"]
        assert sg["conv"].tolist() == so["conv"].tolist()
        assert xg.tobytes() == xo.tobytes()


def test_max_levels_truncation(gpu, oracle):
    """mg_max_levels stops the hierarchy early: the Direct coarse solve then
    inverts a larger coarsest level (inverse.inl:31-106)."""
    row, col, val = gpu.generate_diffusion(7, 18, 17, 16, 1.0, 1.0, 22)
    params = {"solver": {"method": "PBiCGStab", "max_iters": 100, "rel_tolerance": 1e-8,
                         "abs_tolerance": 0},
              "preconditioner": dict(MG_BASE, method="MultiGrid", mg_max_levels=2),
              "pre_smoother": {"method": "Jacobi"}, "post_smoother": {"method": "Jacobi"},
              "coarse_grid_solver": {"method": "Direct"}}
    st, S = check(gpu, oracle, row, col, val, 2, params, seed=3)
    assert S.nlevels() == 2
    assert S.level_info(1, 0)["nrows"] > 300


@pytest.mark.parametrize("key,value", [("mg_coarsening_type", 10), ("mg_coarsening_type", 6),
                                       ("mg_interpolation_type", 0),
                                       ("mg_agg_num_levels", 2)])
def test_unsupported_hierarchy_options_are_refused(gpu, key, value):
    """The host setup implements PMIS with extended+i and no aggressive
    levels; other choices (hypre_base.h:155-163) are refused with
    XAMG_ERR_UNSUPPORTED instead of being replaced, also when given as a
    per-level override."""
    row, col, val = gpu.generate_cube(10, 10, 10)
    n = len(row) - 1
    for as_override in (False, True):
        pre = dict(MG_BASE, method="MultiGrid")
        overrides = None
        if as_override:
            overrides = {"preconditioner": {key: f"{value}@lev1"}}
        else:
            pre[key] = value
        params = {"solver": {"method": "PBiCGStab", "max_iters": 10},
                  "preconditioner": pre}
        M = gpu.Matrix(row, col, val)
        X, B = gpu.Vector(n, 1, M.part), gpu.Vector(n, 1, M.part)
        X.set(0.0)
        B.set(1.0)
        with pytest.raises(gpu.XamgError) as e:
            gpu.Solver(M, gpu.Params(params, overrides=overrides), X, B)
        assert e.value.code == -8, (key, value, as_override)
        assert key in gpu.last_error()


@pytest.mark.parametrize("case", ["config1", "amg27"])
def test_gpu_against_the_reference_itself(gpu, case):
    """The GPU solve against XAMG's own solve phase built from the reference
    sources (oracle/_ref, one rank) on the same inputs and hierarchy: the
    solutions agree to 1e-6 relative and both converge."""
    import ref_capi
    if not ref_capi.available(1):
        pytest.skip("reference not built here")
    if case == "config1":
        row, col, val = gpu.generate_cube(32, 32, 32)
        nv = 1
        params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 1000,
                             "rel_tolerance": 1e-8, "abs_tolerance": 0},
                  "preconditioner": {"method": "Jacobi"}}
    else:
        row, col, val = gpu.generate_diffusion(27, 24, 24, 24, 1.0, 1.0, 0)
        nv = 8
        sm = {"method": "Chebyshev", "polynomial_order": 2}
        params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 200,
                             "rel_tolerance": 1e-8, "abs_tolerance": 0},
                  "preconditioner": dict(MG_BASE, method="MultiGrid"),
                  "pre_smoother": sm, "post_smoother": dict(sm),
                  "coarse_grid_solver": {"method": "Direct"}}
    n = len(row) - 1
    b = np.random.default_rng(77).uniform(-1, 1, n * nv)
    xg, sg, S = gpu_solve(gpu, row, col, val, nv, params, b)
    H = S.hierarchy() if case != "config1" else None
    R = ref_capi.Solve(row, col, val, nv, params, hierarchy=H)
    try:
        xr, conv = R.solve(b)
    finally:
        R.close()
    assert conv.all() and sg["conv"].all()
    X, Xr = xg.reshape(-1, nv), xr.reshape(-1, nv)
    err = np.linalg.norm(X - Xr, axis=0) / np.linalg.norm(Xr, axis=0)
    assert err.max() <= 1e-6, err
    assert true_rel_res(row, col, val, xg, b, nv).max() <= 1e-8 * 1.5
