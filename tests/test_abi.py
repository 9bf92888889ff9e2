"""The C-ABI library: it loads, exports every symbol the headers declare, and
its host-only logic (parameters, generators, narrowing) behaves like the
reference. CPU only: nothing here launches a kernel."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import ref_pins

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("xamg_c_api.h", "xamg_b200.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(XAMG_\w+)\s*\(", text):
            if not text[m.start() - 8:m.start()].strip().endswith("define"):
                names.add(m.group(1))
    names.discard("XAMG_id_get_comm")  # a macro in the reference header too
    return names


def test_library_exports_every_declared_symbol(xamg):
    out = subprocess.check_output(["nm", "-D", "--defined-only", xamg.LIB_PATH], text=True)
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    missing = declared_functions() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    assert set(xamg.C_API_SYMBOLS) <= exported
    assert set(xamg.EXT_SYMBOLS) <= exported


def test_reference_api_names_all_present(xamg):
    """Every function of api/c/xamg_c_api.h:43-117 is implemented."""
    assert len(xamg.C_API_SYMBOLS) == 55
    for name in xamg.C_API_SYMBOLS:
        assert hasattr(xamg.lib(), name)


def test_library_is_built_for_sm100a_only():
    """The build recipe compiles every CUDA source for sm_100a alone: one
    -gencode, machine code only, and no other arch flag anywhere."""
    mk = open(os.path.join(ROOT, "softx-d-21-00014_b200", "Makefile")).read()
    gencodes = re.findall(r"-gencode\s+arch=(\S+),code=(\S+)", mk)
    assert gencodes == [("compute_100a", "sm_100a")], gencodes
    assert not re.search(r"(-arch[= ]|--gpu-architecture|-code=)", mk.replace(
        "arch=compute_100a,code=sm_100a", ""))
    assert re.search(r"\$\(NVCC\)\s+\$\(NVFLAGS\)", mk) and "$(ARCH)" in mk.split("NVFLAGS :=")[1]


def test_generators_match_oracle(xamg, oracle):
    for dims in [(3, 3, 3), (5, 4, 3), (16, 16, 16)]:
        a = xamg.generate_cube(*dims)
        b = oracle.generate_cube(*dims)
        for u, v in zip(a, b):
            assert u.tobytes() == v.tobytes()


def test_diffusion_generators_are_symmetric(xamg):
    import scipy.sparse as sp
    for stencil, dims in [(7, (6, 5, 4)), (27, (5, 4, 6))]:
        row, col, val = xamg.generate_diffusion(stencil, *dims, 1.0, 4.0, 3)
        n = int(np.prod(dims))
        A = sp.csr_matrix((val.copy(), col.copy(), row.copy()), shape=(n, n))
        assert abs(A - A.T).max() < 1e-12 * abs(A).max()
        # diagonal first in every row, positive
        assert (col[row[:-1]] == np.arange(n)).all() and (val[row[:-1]] > 0).all()
        # Dirichlet: positive definite -> smallest eigenvalue > 0
        w = np.linalg.eigvalsh(A.toarray())
        assert w.min() > 0
    row, col, val = xamg.generate_diffusion(27, 10, 10, 10, 1.0, 1.0, 0)
    assert len(col) == (3 * 10 - 2) ** 3
    row, col, val = xamg.generate_diffusion(7, 10, 10, 10, 1.0, 1.0, 0)
    assert len(col) == 7 * 1000 - 6 * 100


def test_narrowing_entry_points_match_reference(xamg):
    R = ref_pins.load()
    if R is None:
        pytest.skip("reference narrowing headers not available")
    L = xamg.lib()
    for r in [0, 255, 256, 65535, 65536, 2**32 - 1, 2**32]:
        assert L.XAMG_b200_define_int_type(r) == R.ref_define_int_type(r)
    for args in [(223232, 32768, 32768, 32768), (7, 3, 3, 3), (10**6, 70000, 70000, 70000)]:
        assert L.XAMG_b200_encode_hash(*args, 0, 0) == R.ref_encode_hash(*args, 0)
        assert L.XAMG_b200_encode_hash(*args, 1, 0) == R.ref_encode_hash(*args, 1)


def test_params_roundtrip_on_host(xamg, capfd):
    """XAMG_param_* needs no GPU: add, change, override, defaults, print."""
    p = xamg.Params({"solver": {"method": "PBiCGStab", "rel_tolerance": 1e-6},
                     "preconditioner": {"method": "MultiGrid", "hypre_per_level_hierarchy": 1}},
                    overrides={"preconditioner": {"mg_coarsening_type": "8@lev0-1",
                                                  "mg_interpolation_type": "6@lev0-1"}})
    p.change("solver", "rel_tolerance", 1e-8)
    p.change("solver", "abs_tolerance", 1e-8)   # present after set_default
    with pytest.raises(xamg.XamgError) as e:
        p.change("solver", "no_such_key", 1)
    assert e.value.code == -2
    with pytest.raises(xamg.XamgError):
        p.change("coarse_grid_solver", "max_iters", 3)  # Direct has no max_iters
    p.change("coarse_grid_solver", "max_iters", 3, forced=True)
    p.print()
    out = capfd.readouterr().out
    # dictionary defaults (xamg_params_details.h:131-144): Jacobi smoothers, Direct coarse
    assert "[pre_smoother]" in out and "Jacobi" in out and "Direct" in out
    assert "mg_coarsening_type = 8 @lev0" in out and "@lev1" in out
    assert "relax_factor = 0.99" in out          # family default of the smoothers
    assert "mg_max_levels = 25" in out           # MultiGrid family default
    assert "rel_tolerance = 1e-08" in out


def test_bad_handles_return_codes(xamg):
    L = xamg.lib()
    assert L.XAMG_param_print(999) == -1
    assert L.XAMG_vector_set_val_d(1.0, 999) == -1
    assert L.XAMG_solver_solve1(1, 999) == -1
    assert "invalid" in xamg.last_error()


def test_no_cpu_fallback(xamg):
    """Without a CUDA device the library refuses instead of computing on the host."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    rc = xamg.lib().XAMG_init(0, None, b"")
    assert rc == -4  # XAMG_ERR_CUDA
    v = C.c_size_t()
    assert xamg.lib().XAMG_vector_create(C.byref(v), 2) == 0
    assert xamg.lib().XAMG_vector_alloc_d(10, 1, v.value) == -4


def test_param_ranges_and_allowed_sets(xamg):
    """Values outside the ranges and allowed sets of
    xamg_params_details.h:79-123 are refused with XAMG_ERR_INVALID_ARG by
    add, change, forced change and per-level overrides; boundary values are
    accepted."""
    L = xamg.lib()
    p = xamg.Params({"solver": {"method": "PBiCGStab"},
                     "preconditioner": {"method": "MultiGrid"},
                     "pre_smoother": {"method": "Chebyshev"}}, set_default=False)
    bad = [("pre_smoother", "polynomial_order", 0), ("pre_smoother", "polynomial_order", 5),
           ("pre_smoother", "spectrum_fraction", 1.5), ("preconditioner", "mg_cycle", 3),
           ("preconditioner", "mg_coarsening_type", 2), ("preconditioner", "mg_coarsening_type", 23),
           ("preconditioner", "mg_max_levels", 0), ("preconditioner", "mg_max_levels", 51),
           ("preconditioner", "mg_coarse_matrix_size", 2001),
           ("preconditioner", "mg_strength_threshold", -0.1),
           ("preconditioner", "mg_agg_interpolation_type", 0), ("solver", "rel_tolerance", -1e-8),
           ("solver", "convergence_check", 2), ("preconditioner", "gpu_index_compress", 4)]
    for role, key, value in bad:
        with pytest.raises(xamg.XamgError) as e:
            p.add(role, key, value)
        assert e.value.code == -2, (key, value)
        with pytest.raises(xamg.XamgError):
            p.change(role, key, value, forced=True)
    good = [("pre_smoother", "polynomial_order", 1), ("pre_smoother", "polynomial_order", 4),
            ("pre_smoother", "spectrum_fraction", 1.0), ("preconditioner", "mg_cycle", 2),
            ("preconditioner", "mg_coarsening_type", 22), ("preconditioner", "mg_max_levels", 50),
            ("preconditioner", "mg_coarse_matrix_size", 2000), ("solver", "max_iters", 65535),
            ("preconditioner", "gpu_index_compress", 3)]
    for role, key, value in good:
        p.add(role, key, value)
    p.change("preconditioner", "mg_cycle", 1)
    with pytest.raises(xamg.XamgError):
        p.change("preconditioner", "mg_cycle", 4)
    for spec in ("3@lev0", "1@lev2-4"):
        o = C.c_size_t()
        assert L.XAMG_param_override_create(C.byref(o)) == 0
        assert L.XAMG_param_override_add_value(b"mg_cycle", spec.encode(), o.value) == 0
        rc = L.XAMG_param_override_apply(b"preconditioner", p.h, o.value)
        assert rc == (-2 if spec.startswith("3") else 0), spec
        L.XAMG_param_override_destroy(o.value)
