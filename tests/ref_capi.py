"""ctypes driver of the reference itself: XAMG's own C API (api/c/xamg_c_api.cpp)
compiled unmodified from the reference sources, with the single-process
shims of oracle/ref_shim (MPI, argsparser's parameter dictionary, hypre), by
`make -C oracle ref` into oracle/_ref/libxamg_ref_nv<NV>.so (XAMG_NV is a
compile-time constant of the reference's C API).

Test infrastructure: the reference run here pins the CPU oracle (XAMG's
reduction order on one core, oracle mode 0 with ncores = 1) bit for bit. The
multigrid hierarchy that hypre would build is registered with the hypre
stand-in (xamg_ref_set_hierarchy) before the solver is created."""
import ctypes as C
import os
import subprocess
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
INT_KEYS = {"convergence_check", "convergence_info", "polynomial_order", "max_iters",
            "hypre_log", "hypre_per_level_hierarchy", "mg_reduced_precision", "mg_cycle",
            "mg_max_levels", "mg_coarse_matrix_size", "mg_num_paths", "mg_coarsening_type",
            "mg_interpolation_type", "mg_Pmax_elements", "mg_agg_num_levels",
            "mg_agg_interpolation_type", "mg_agg_Pmax_elements", "mg_agg_P12max_elements"}
# B200 extension keys that do not change the numbers the reference computes
# (index storage, graphs, launch tuning, the setup's seed, the GPU's
# Gauss-Seidel block size); any other extension key has no reference meaning
NEUTRAL_EXT_KEYS = {"gpu_index_compress", "gpu_graph", "gpu_spmv_tune", "gpu_seed",
                    "gpu_hsgs_rows", "gpu_persistent", "gpu_solve_graph"}
_libs = {}
sz = C.c_size_t


def lib_path(nv):
    return os.path.join(REF_DIR, f"libxamg_ref_nv{nv}.so")


def available(nv=1):
    if not os.path.exists(lib_path(nv)):
        subprocess.call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    return os.path.exists(lib_path(nv))


def lib(nv):
    if nv not in _libs:
        L = C.CDLL(lib_path(nv))
        L.XAMG_csr_matrix_alloc.argtypes = [C.c_uint64, C.c_uint64, sz]
        L.XAMG_csr_matrix_offset.argtypes = [C.c_int, C.c_int, sz]
        L.XAMG_param_add_value_s.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, sz]
        L.XAMG_param_add_value_i.argtypes = [C.c_char_p, C.c_char_p, C.c_uint16, sz]
        L.XAMG_param_add_value_d.argtypes = [C.c_char_p, C.c_char_p, C.c_float, sz]
        L.XAMG_param_override_add_value.argtypes = [C.c_char_p, C.c_char_p, sz]
        L.XAMG_param_override_apply.argtypes = [C.c_char_p, sz, sz]
        L.XAMG_vector_alloc_d.argtypes = [C.c_int, C.c_uint16, sz]
        L.XAMG_vector_upload_d.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint16, sz]
        L.XAMG_vector_download_d.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint16, sz]
        L.XAMG_vector_set_val_d.argtypes = [C.c_double, sz]
        L.XAMG_solver_solve1.argtypes = [C.c_uint16, sz]
        L.XAMG_solver_get_convergence_info.argtypes = [C.c_void_p, C.c_uint16, sz]
        L.xamg_ref_set_hierarchy.argtypes = [C.c_int] + [C.c_void_p] * 9
        assert L.XAMG_init(0, None, b"") == 0
        assert L.XAMG_get_nv() == nv
        _libs[nv] = L
    return _libs[nv]


def _call(L, name, *a):
    rc = getattr(L, name)(*a)
    assert rc == 0, (name, rc)


def register_hierarchy(L, hierarchy):
    """hierarchy: list of {A: (row, col, val), P: (row, col, val, ncols) or
    None, min_eig, max_eig}, as the library's export or the oracle-side setup
    gives it."""
    nl = len(hierarchy)
    keep = []

    def ptrs(arrs, dt):
        a = [np.ascontiguousarray(x, dt) for x in arrs]
        keep.extend(a)
        return (C.c_void_p * len(a))(*[x.ctypes.data for x in a])

    n = np.array([len(lv["A"][0]) - 1 for lv in hierarchy], np.int32)
    empty_u = np.zeros(1, np.uint32)
    empty_f = np.zeros(1, np.float64)
    P = [lv["P"] if lv["P"] is not None else (empty_u, empty_u, empty_f, 0) for lv in hierarchy]
    mn = np.array([lv["min_eig"] for lv in hierarchy], np.float64)
    mx = np.array([lv["max_eig"] for lv in hierarchy], np.float64)
    L.xamg_ref_set_hierarchy(nl, n.ctypes.data, ptrs([lv["A"][0] for lv in hierarchy], np.uint32),
                             ptrs([lv["A"][1] for lv in hierarchy], np.uint32),
                             ptrs([lv["A"][2] for lv in hierarchy], np.float64),
                             ptrs([p[0] for p in P], np.uint32), ptrs([p[1] for p in P], np.uint32),
                             ptrs([p[2] for p in P], np.float64), mn.ctypes.data, mx.ctypes.data)


class Solve:
    """One reference solver on a CSR matrix: XAMG_csr_matrix_*, part,
    matrix, parameters (with per-level overrides), vectors, solver."""

    def __init__(self, row, col, val, nv, params, overrides=None, hierarchy=None):
        L = self.L = lib(nv)
        self.nv, self.n = nv, len(row) - 1
        n = self.n
        if hierarchy is not None:
            register_hierarchy(L, hierarchy)
        self._r = np.ascontiguousarray(row, np.int32)
        self._c = np.ascontiguousarray(col, np.int32)
        self._v = np.ascontiguousarray(val, np.float64)
        m = sz()
        _call(L, "XAMG_csr_matrix_create", C.byref(m))
        _call(L, "XAMG_csr_matrix_alloc", n, len(col), m)
        _call(L, "XAMG_csr_matrix_fill", self._r.ctypes.data_as(C.c_void_p),
              self._c.ctypes.data_as(C.c_void_p), self._v.ctypes.data_as(C.c_void_p), m)
        _call(L, "XAMG_csr_matrix_offset", 0, 0, m)
        p, mid = sz(), sz()
        _call(L, "XAMG_part_create", C.byref(p))
        _call(L, "XAMG_part_construct", n, p)
        _call(L, "XAMG_matrix_create", C.byref(mid))
        _call(L, "XAMG_matrix_set_part", p, mid)
        _call(L, "XAMG_matrix_construct", m, mid)
        _call(L, "XAMG_csr_matrix_destroy", m)
        par = sz()
        _call(L, "XAMG_param_create", C.byref(par))
        for role, kv in params.items():
            for k, v in kv.items():
                if k.startswith("gpu_"):
                    if k not in NEUTRAL_EXT_KEYS:
                        raise ValueError(f"{k} has no counterpart in the reference")
                    continue
                r, kk = role.encode(), k.encode()
                if isinstance(v, str):
                    _call(L, "XAMG_param_add_value_s", r, kk, v.encode(), par)
                elif k in INT_KEYS:
                    _call(L, "XAMG_param_add_value_i", r, kk, int(v), par)
                else:
                    _call(L, "XAMG_param_add_value_d", r, kk, float(v), par)
        for role, ov in (overrides or {}).items():
            o = sz()
            _call(L, "XAMG_param_override_create", C.byref(o))
            for k, v in ov.items():
                _call(L, "XAMG_param_override_add_value", k.encode(), v.encode(), o)
            _call(L, "XAMG_param_override_apply", role.encode(), par, o)
            _call(L, "XAMG_param_override_destroy", o)
        L.XAMG_param_set_default(par)
        x, b = sz(), sz()
        for v in (x, b):
            _call(L, "XAMG_vector_create", C.byref(v), 2)
            _call(L, "XAMG_vector_set_part", p, v)
            _call(L, "XAMG_vector_alloc_d", n, nv, v)
        s = sz()
        _call(L, "XAMG_solver_create2", mid, par, x, b, C.byref(s))
        self.h = dict(m=mid, p=p, par=par, x=x, b=b, s=s)

    def solve(self, b, x0=None):
        """x (and the per-RHS convergence flags) of one XAMG_solver_solve1 from
        x0 (default zero)."""
        L, h, n, nv = self.L, self.h, self.n, self.nv
        b = np.ascontiguousarray(b, np.float64).ravel()
        _call(L, "XAMG_vector_upload_d", b.ctypes.data, n, 0, nv, h["b"])
        if x0 is None:
            _call(L, "XAMG_vector_set_val_d", 0.0, h["x"])
        else:
            x0 = np.ascontiguousarray(x0, np.float64).ravel()
            _call(L, "XAMG_vector_upload_d", x0.ctypes.data, n, 0, nv, h["x"])
        t0 = time.perf_counter()
        _call(L, "XAMG_solver_solve1", nv, h["s"])
        self.last_seconds = time.perf_counter() - t0
        x = np.zeros(n * nv)
        _call(L, "XAMG_vector_download_d", x.ctypes.data, n, 0, nv, h["x"])
        conv = np.zeros(nv, np.int32)
        _call(L, "XAMG_solver_get_convergence_info", conv.ctypes.data, nv, h["s"])
        return x, conv

    def close(self):
        L, h = self.L, self.h
        for k in ("x", "b"):
            L.XAMG_vector_destroy(h[k])
        L.XAMG_solver_destroy(h["s"])
        L.XAMG_matrix_destroy(h["m"])
        L.XAMG_param_destroy(h["par"])
