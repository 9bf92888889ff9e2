"""Python view of the XAMG C API as implemented by lib/libxamg_c_api.so.

The functions keep the reference C API's names and argument meaning
(api/c/xamg_c_api.h:43-117); they call straight into the shared library with
ctypes. A thin object layer (Matrix, Vector, Params, Solver) mirrors the
handle lifecycle of examples/c/example.c so that scripts read like the
reference's C example. Every call checks the status code and raises
XamgError with the library's message.

The library has no CPU fallback: on a machine without a CUDA device,
XAMG_init returns XAMG_ERR_CUDA and every call that needs the GPU fails.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libxamg_c_api.so")

ERRORS = {
    -1: "XAMG_ERR_INVALID_HANDLE", -2: "XAMG_ERR_INVALID_ARG", -3: "XAMG_ERR_NV_MISMATCH",
    -4: "XAMG_ERR_CUDA", -5: "XAMG_ERR_BREAKDOWN", -6: "XAMG_ERR_TIMEOUT",
    -7: "XAMG_ERR_NOT_INITIALIZED", -8: "XAMG_ERR_UNSUPPORTED", -9: "XAMG_ERR_ALLOC",
    -10: "XAMG_ERR_INTERNAL",
}

# Every symbol the headers in include/ declare (checked by the CPU tests).
C_API_SYMBOLS = [
    "XAMG_init", "XAMG_finalize", "XAMG_get_nv", "XAMG_id_get_proc", "XAMG_id_get_nprocs",
    "XAMG_id_get_comm_ptr", "XAMG_param_create", "XAMG_param_add_value_s",
    "XAMG_param_add_value_i", "XAMG_param_add_value_d", "XAMG_param_forced_change_value_s",
    "XAMG_param_forced_change_value_i", "XAMG_param_forced_change_value_d",
    "XAMG_param_change_value_s", "XAMG_param_change_value_i", "XAMG_param_change_value_d",
    "XAMG_param_override_create", "XAMG_param_override_add_value", "XAMG_param_override_apply",
    "XAMG_param_override_destroy", "XAMG_param_set_default", "XAMG_param_print",
    "XAMG_param_destroy", "XAMG_part_create", "XAMG_part_construct", "XAMG_part_get_numa_size",
    "XAMG_part_destroy", "XAMG_vector_create", "XAMG_vector_offset", "XAMG_vector_alloc_d",
    "XAMG_vector_set_part", "XAMG_vector_set_val_d", "XAMG_vector_download_d",
    "XAMG_vector_upload_v", "XAMG_vector_upload_d", "XAMG_vector_destroy",
    "XAMG_csr_matrix_create", "XAMG_csr_matrix_alloc", "XAMG_csr_matrix_fill",
    "XAMG_csr_matrix_offset", "XAMG_csr_matrix_get_nrows", "XAMG_csr_matrix_destroy",
    "XAMG_matrix_create", "XAMG_matrix_set_part", "XAMG_matrix_construct", "XAMG_matrix_destroy",
    "XAMG_solver_create1", "XAMG_solver_create2", "XAMG_solver_renew_params",
    "XAMG_solver_solve1", "XAMG_solver_solve2", "XAMG_solver_get_convergence_info",
    "XAMG_solver_destroy", "XAMG_timer", "XAMG_barrier",
]
EXT_SYMBOLS = [
    "XAMG_b200_last_error", "XAMG_b200_build_info", "XAMG_b200_spmv", "XAMG_b200_spmv_dot",
    "XAMG_b200_dot", "XAMG_b200_group1", "XAMG_b200_group2", "XAMG_b200_group4",
    "XAMG_b200_define_int_type", "XAMG_b200_encode_hash", "XAMG_b200_generate_cube",
    "XAMG_b200_generate_diffusion", "XAMG_b200_solver_stats", "XAMG_b200_solver_nlevels",
    "XAMG_b200_solver_level_info", "XAMG_b200_solver_level_download",
    "XAMG_b200_solver_hierarchy_export", "XAMG_b200_vector_device_ptr",
    "XAMG_b200_solver_level_csr", "XAMG_b200_kernel_launches", "XAMG_b200_stream",
    "XAMG_b200_set_device", "XAMG_b200_dot_noalloc", "XAMG_b200_wait_selftest",
    "XAMG_b200_kernel_arch", "XAMG_b200_grid_selftest",
    "XAMG_b200_solver_level_spmv", "XAMG_b200_read_system_size", "XAMG_b200_read_system",
    "XAMG_b200_write_system", "XAMG_b200_solver_hierarchy_save",
    "XAMG_b200_matrix_hierarchy_load", "XAMG_b200_gemm_bf16", "XAMG_b200_mlp_create",
    "XAMG_b200_mlp_destroy", "XAMG_b200_mlp_predict", "XAMG_b200_mlp_train_step",
    "XAMG_b200_mlp_gradients", "XAMG_b200_mlp_params", "XAMG_b200_solver_solve_batch",
    "XAMG_b200_solver_level_tuned", "XAMG_b200_stencil_layout", "XAMG_b200_solver_level_stencil",
    "XAMG_b200_solver_level_xstaged",
]


class XamgError(RuntimeError):
    def __init__(self, code, fn, msg):
        super().__init__(f"{fn} failed with {ERRORS.get(code, code)}: {msg}")
        self.code = code


class Csr(C.Structure):
    """XAMG_b200_csr: a CSR block in device memory."""
    _fields_ = [("nrows", C.c_uint64), ("ncols", C.c_uint64), ("nnz", C.c_uint64),
                ("row", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p),
                ("col_bytes", C.c_int), ("val_f32", C.c_int)]


_lib = None
sz = C.c_size_t
u16 = C.c_uint16
u64 = C.c_uint64
vp = C.c_void_p


def build():
    subprocess.check_call(["make", "-s", "-j8", "-C", HERE])


def lib():
    """Load the in-tree library (build it first if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = C.CDLL(LIB_PATH)
    sig = {
        "XAMG_init": (C.c_int, [C.c_int, vp, C.c_char_p]),
        "XAMG_finalize": (C.c_int, []),
        "XAMG_get_nv": (C.c_int, []),
        "XAMG_timer": (C.c_double, []),
        "XAMG_barrier": (C.c_int, []),
        "XAMG_param_create": (C.c_int, [C.POINTER(sz)]),
        "XAMG_param_add_value_s": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, sz]),
        "XAMG_param_add_value_i": (C.c_int, [C.c_char_p, C.c_char_p, u16, sz]),
        "XAMG_param_add_value_d": (C.c_int, [C.c_char_p, C.c_char_p, C.c_float, sz]),
        "XAMG_param_change_value_s": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, sz]),
        "XAMG_param_change_value_i": (C.c_int, [C.c_char_p, C.c_char_p, u16, sz]),
        "XAMG_param_change_value_d": (C.c_int, [C.c_char_p, C.c_char_p, C.c_float, sz]),
        "XAMG_param_forced_change_value_s": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, sz]),
        "XAMG_param_forced_change_value_i": (C.c_int, [C.c_char_p, C.c_char_p, u16, sz]),
        "XAMG_param_forced_change_value_d": (C.c_int, [C.c_char_p, C.c_char_p, C.c_float, sz]),
        "XAMG_param_override_create": (C.c_int, [C.POINTER(sz)]),
        "XAMG_param_override_add_value": (C.c_int, [C.c_char_p, C.c_char_p, sz]),
        "XAMG_param_override_apply": (C.c_int, [C.c_char_p, sz, sz]),
        "XAMG_param_override_destroy": (C.c_int, [sz]),
        "XAMG_param_set_default": (None, [sz]),
        "XAMG_param_print": (C.c_int, [sz]),
        "XAMG_param_destroy": (C.c_int, [sz]),
        "XAMG_part_create": (C.c_int, [C.POINTER(sz)]),
        "XAMG_part_construct": (C.c_int, [C.c_int, sz]),
        "XAMG_part_get_numa_size": (C.c_int, [sz]),
        "XAMG_part_destroy": (C.c_int, [sz]),
        "XAMG_vector_create": (C.c_int, [C.POINTER(sz), C.c_int]),
        "XAMG_vector_offset": (C.c_int, [u64, sz]),
        "XAMG_vector_alloc_d": (C.c_int, [C.c_int, u16, sz]),
        "XAMG_vector_set_part": (C.c_int, [sz, sz]),
        "XAMG_vector_set_val_d": (C.c_int, [C.c_double, sz]),
        "XAMG_vector_download_d": (C.c_int, [vp, u64, u64, u16, sz]),
        "XAMG_vector_upload_v": (C.c_int, [sz, sz]),
        "XAMG_vector_upload_d": (C.c_int, [vp, u64, u64, u16, sz]),
        "XAMG_vector_destroy": (C.c_int, [sz]),
        "XAMG_csr_matrix_create": (C.c_int, [C.POINTER(sz)]),
        "XAMG_csr_matrix_alloc": (C.c_int, [u64, u64, sz]),
        "XAMG_csr_matrix_fill": (C.c_int, [vp, vp, vp, sz]),
        "XAMG_csr_matrix_offset": (C.c_int, [C.c_int, C.c_int, sz]),
        "XAMG_csr_matrix_get_nrows": (C.c_uint32, [sz]),
        "XAMG_csr_matrix_destroy": (C.c_int, [sz]),
        "XAMG_matrix_create": (C.c_int, [C.POINTER(sz)]),
        "XAMG_matrix_set_part": (C.c_int, [sz, sz]),
        "XAMG_matrix_construct": (C.c_int, [sz, sz]),
        "XAMG_matrix_destroy": (C.c_int, [sz]),
        "XAMG_solver_create1": (C.c_int, [sz, sz, C.POINTER(sz)]),
        "XAMG_solver_create2": (C.c_int, [sz, sz, sz, sz, C.POINTER(sz)]),
        "XAMG_solver_renew_params": (C.c_int, [sz, sz]),
        "XAMG_solver_solve1": (C.c_int, [u16, sz]),
        "XAMG_solver_solve2": (C.c_int, [u16, sz, sz, sz]),
        "XAMG_solver_get_convergence_info": (C.c_int, [vp, u16, sz]),
        "XAMG_solver_destroy": (C.c_int, [sz]),
        "XAMG_b200_last_error": (C.c_int, [C.c_char_p, sz]),
        "XAMG_b200_build_info": (C.c_int, [C.c_char_p, sz]),
        "XAMG_b200_spmv": (C.c_int, [C.POINTER(Csr), vp, vp, C.c_int, C.c_int, vp]),
        "XAMG_b200_spmv_dot": (C.c_int, [C.POINTER(Csr), vp, vp, vp, vp, C.c_int, vp]),
        "XAMG_b200_dot": (C.c_int, [u64, C.c_int, vp, vp, vp, vp]),
        "XAMG_b200_dot_noalloc": (C.c_int, [u64, C.c_int, vp, vp, vp, vp]),
        "XAMG_b200_group1": (C.c_int, [u64, C.c_int, vp, vp, vp, vp, vp, vp]),
        "XAMG_b200_group2": (C.c_int, [u64, C.c_int, vp, vp, vp, vp, vp, vp]),
        "XAMG_b200_group4": (C.c_int, [u64, C.c_int, vp, vp, vp, vp, vp, vp, vp]),
        "XAMG_b200_define_int_type": (u16, [u64]),
        "XAMG_b200_encode_hash": (u16, [u64, u64, u64, u64, C.c_int, C.c_int]),
        "XAMG_b200_generate_cube": (C.c_int64, [u64, u64, u64, vp, vp, vp]),
        "XAMG_b200_generate_diffusion": (C.c_int64, [C.c_int, u64, u64, u64, C.c_double,
                                                     C.c_double, u64, vp, vp, vp]),
        "XAMG_b200_solver_stats": (C.c_int, [sz, vp, vp, vp, vp, C.c_int]),
        "XAMG_b200_solver_nlevels": (C.c_int, [sz]),
        "XAMG_b200_solver_level_info": (C.c_int, [sz, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp,
                                                  vp, vp]),
        "XAMG_b200_solver_level_download": (C.c_int, [sz, C.c_int, C.c_int, vp, vp, vp]),
        "XAMG_b200_solver_hierarchy_export": (C.c_int, [sz, C.c_int, C.c_int, vp, vp, vp]),
        "XAMG_b200_vector_device_ptr": (C.c_int, [sz, C.POINTER(vp)]),
        "XAMG_b200_solver_level_csr": (C.c_int, [sz, C.c_int, C.c_int, C.POINTER(Csr)]),
        "XAMG_b200_kernel_launches": (C.c_uint64, []),
        "XAMG_b200_stream": (vp, []),
        "XAMG_b200_set_device": (C.c_int, [C.c_int]),
        "XAMG_b200_wait_selftest": (C.c_int, [C.c_double, C.POINTER(C.c_int)]),
        "XAMG_b200_kernel_arch": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "XAMG_b200_grid_selftest": (C.c_int, [C.c_double, C.POINTER(C.c_int)]),
        "XAMG_b200_solver_level_spmv": (C.c_int, [C.c_size_t, C.c_int, C.c_int, vp, vp, C.c_int,
                                                  C.c_int, vp]),
        "XAMG_b200_read_system_size": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint32),
                                                 C.POINTER(C.c_uint32)]),
        "XAMG_b200_read_system": (C.c_int, [C.c_char_p, C.c_uint16, vp, vp, vp, vp, vp,
                                            C.POINTER(C.c_int)]),
        "XAMG_b200_write_system": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, vp, vp, vp,
                                             C.c_uint16, vp, vp]),
        "XAMG_b200_solver_hierarchy_save": (C.c_int, [C.c_size_t, C.c_char_p]),
        "XAMG_b200_gemm_bf16": (C.c_int, [u64, u64, u64, vp, vp, vp, u64, C.c_int, vp, vp, u64,
                                          vp]),
        "XAMG_b200_mlp_create": (C.c_int, [C.c_uint32, C.c_uint32, C.c_uint32, u64,
                                           C.POINTER(C.c_size_t)]),
        "XAMG_b200_mlp_destroy": (C.c_int, [C.c_size_t]),
        "XAMG_b200_mlp_predict": (C.c_int, [C.c_size_t, C.c_uint32, vp, vp]),
        "XAMG_b200_mlp_train_step": (C.c_int, [C.c_size_t, C.c_uint32, vp, vp, C.c_float,
                                               C.POINTER(C.c_double)]),
        "XAMG_b200_mlp_gradients": (C.c_int, [C.c_size_t, C.c_uint32, vp, vp, vp,
                                              C.POINTER(C.c_double)]),
        "XAMG_b200_mlp_params": (C.c_int, [C.c_size_t, vp, C.c_int, C.POINTER(u64)]),
        "XAMG_b200_matrix_hierarchy_load": (C.c_int, [C.c_size_t, C.c_char_p]),
        "XAMG_b200_solver_solve_batch": (C.c_int, [C.c_int, vp, vp, vp, vp]),
        "XAMG_b200_solver_level_tuned": (C.c_int, [C.c_size_t, C.c_int, C.c_int, vp]),
        "XAMG_b200_solver_level_xstaged": (C.c_int, [C.c_size_t, C.c_int, C.c_int,
                                                     C.POINTER(C.c_int)]),
        "XAMG_b200_stencil_layout": (C.c_int, [u64, vp, vp, C.POINTER(C.c_int),
                                               C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                               C.POINTER(C.c_int)]),
        "XAMG_b200_solver_level_stencil": (C.c_int, [C.c_size_t, C.c_int, C.c_int,
                                                     C.POINTER(C.c_int), C.POINTER(C.c_uint32),
                                                     C.POINTER(C.c_uint32), C.POINTER(C.c_int)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error():
    buf = C.create_string_buffer(1024)
    lib().XAMG_b200_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def kernel_launches():
    return lib().XAMG_b200_kernel_launches()


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if isinstance(rc, int) and rc < 0 and name not in ("XAMG_b200_define_int_type",
                                                       "XAMG_b200_encode_hash",
                                                       "XAMG_b200_kernel_launches"):
        raise XamgError(rc, name, last_error())
    return rc


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------- generators
def read_system(path, nv=1):
    """XAMG's binary system file: (row, col, val, b, x, found) with b, x as
    [n*nv] arrays (b = 1, x = 0 where the file holds none; found bit 0/1)."""
    n, nnz = C.c_uint32(), C.c_uint32()
    call("XAMG_b200_read_system_size", str(path).encode(), C.byref(n), C.byref(nnz))
    row = np.zeros(n.value + 1, np.uint32)
    col = np.zeros(nnz.value, np.uint32)
    val = np.zeros(nnz.value, np.float64)
    b = np.zeros(n.value * nv, np.float64)
    x = np.zeros(n.value * nv, np.float64)
    found = C.c_int()
    call("XAMG_b200_read_system", str(path).encode(), nv, _ptr(row), _ptr(col), _ptr(val),
         _ptr(b), _ptr(x), C.byref(found))
    return row, col, val, b, x, found.value


def write_system(path, row, col, val, nv=1, b=None, x=None):
    """Write XAMG's binary system file (x only together with b)."""
    row = np.ascontiguousarray(row, np.uint32)
    col = np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.float64)
    bb = None if b is None else np.ascontiguousarray(b, np.float64)
    xx = None if x is None else np.ascontiguousarray(x, np.float64)
    call("XAMG_b200_write_system", str(path).encode(), len(row) - 1, len(col), _ptr(row),
         _ptr(col), _ptr(val), nv, None if bb is None else _ptr(bb),
         None if xx is None else _ptr(xx))


def stencil_layout(row, col):
    """Grid-stencil detection on host CSR arrays (no GPU): (pattern, S, S2,
    diag_first), pattern -1 where the matrix does not qualify."""
    row = np.ascontiguousarray(row, np.uint32)
    col = np.ascontiguousarray(col, np.uint32)
    pat, S, S2, df = C.c_int(), C.c_uint32(), C.c_uint32(), C.c_int()
    call("XAMG_b200_stencil_layout", len(row) - 1, _ptr(row), _ptr(col), C.byref(pat),
         C.byref(S), C.byref(S2), C.byref(df))
    return pat.value, S.value, S2.value, df.value


def generate_cube(nx, ny, nz):
    """The reference's 7-point Laplacian (cube.inl) as numpy CSR arrays."""
    n = nx * ny * nz
    row = np.zeros(n + 1, np.uint32)
    col = np.zeros(7 * n, np.uint32)
    val = np.zeros(7 * n, np.float64)
    nnz = call("XAMG_b200_generate_cube", nx, ny, nz, _ptr(row), _ptr(col), _ptr(val))
    return row, col[:nnz].copy(), val[:nnz].copy()


def generate_diffusion(stencil, nx, ny, nz, sigma, aniso_z=1.0, seed=0):
    n = nx * ny * nz
    row = np.zeros(n + 1, np.uint32)
    col = np.zeros(stencil * n, np.uint32)
    val = np.zeros(stencil * n, np.float64)
    nnz = call("XAMG_b200_generate_diffusion", stencil, nx, ny, nz, sigma, aniso_z, seed,
               _ptr(row), _ptr(col), _ptr(val))
    return row, col[:nnz].copy(), val[:nnz].copy()


# ---------------------------------------------------------------- objects
def init(device=None):
    if device is not None:
        call("XAMG_b200_set_device", int(device))
    call("XAMG_init", 0, None, b"")


def stream():
    """The library's cudaStream_t as an integer."""
    return lib().XAMG_b200_stream()


def finalize():
    call("XAMG_finalize")


class Params:
    """XAMG_param_*: {role: {key: value}}; "value@levA-B" strings as overrides."""

    INT_KEYS = {"convergence_check", "convergence_info", "polynomial_order", "max_iters",
                "hypre_log", "hypre_per_level_hierarchy", "mg_reduced_precision", "mg_cycle",
                "mg_max_levels", "mg_coarse_matrix_size", "mg_num_paths", "mg_coarsening_type",
                "mg_interpolation_type", "mg_Pmax_elements", "mg_agg_num_levels",
                "mg_agg_interpolation_type", "mg_agg_Pmax_elements", "mg_agg_P12max_elements",
                "gpu_precond_f32", "gpu_coarse_f64", "gpu_index_compress", "gpu_hsgs_rows",
                "gpu_graph", "gpu_seed", "gpu_persistent", "gpu_spmv_tune", "gpu_level_bf16",
                "gpu_level_fp16", "gpu_solve_graph"}

    def __init__(self, spec=None, overrides=None, set_default=True):
        h = sz()
        call("XAMG_param_create", C.byref(h))
        self.h = h.value
        for role, kv in (spec or {}).items():
            for k, v in kv.items():
                self.add(role, k, v)
        for role, ov in (overrides or {}).items():
            o = sz()
            call("XAMG_param_override_create", C.byref(o))
            for k, v in ov.items():
                call("XAMG_param_override_add_value", k.encode(), v.encode(), o.value)
            call("XAMG_param_override_apply", role.encode(), self.h, o.value)
            call("XAMG_param_override_destroy", o.value)
        if set_default:
            lib().XAMG_param_set_default(self.h)

    def add(self, role, key, value):
        r, k = role.encode(), key.encode()
        if isinstance(value, str):
            call("XAMG_param_add_value_s", r, k, value.encode(), self.h)
        elif key in self.INT_KEYS:
            call("XAMG_param_add_value_i", r, k, int(value), self.h)
        else:
            call("XAMG_param_add_value_d", r, k, float(value), self.h)

    def change(self, role, key, value, forced=False):
        r, k = role.encode(), key.encode()
        pre = "XAMG_param_forced_change_value_" if forced else "XAMG_param_change_value_"
        if isinstance(value, str):
            call(pre + "s", r, k, value.encode(), self.h)
        elif key in self.INT_KEYS:
            call(pre + "i", r, k, int(value), self.h)
        else:
            call(pre + "d", r, k, float(value), self.h)

    def print(self):
        call("XAMG_param_print", self.h)


class Matrix:
    """XAMG_csr_matrix_* + XAMG_matrix_* for a square CSR held by one rank."""

    def __init__(self, row, col, val):
        n = len(row) - 1
        c = sz()
        call("XAMG_csr_matrix_create", C.byref(c))
        call("XAMG_csr_matrix_alloc", n, len(col), c.value)
        r32 = np.ascontiguousarray(row, np.int32)
        c32 = np.ascontiguousarray(col, np.int32)
        v64 = np.ascontiguousarray(val, np.float64)
        call("XAMG_csr_matrix_fill", _ptr(r32), _ptr(c32), _ptr(v64), c.value)
        call("XAMG_csr_matrix_offset", 0, 0, c.value)
        p = sz()
        call("XAMG_part_create", C.byref(p))
        call("XAMG_part_construct", n, p.value)
        m = sz()
        call("XAMG_matrix_create", C.byref(m))
        call("XAMG_matrix_set_part", p.value, m.value)
        call("XAMG_matrix_construct", c.value, m.value)
        call("XAMG_csr_matrix_destroy", c.value)
        self.h, self.part, self.n, self.nnz = m.value, p.value, n, len(col)

    def load_hierarchy(self, path):
        """Attach a hierarchy file written for this matrix (skips the setup of
        solvers created with the same multigrid parameters)."""
        call("XAMG_b200_matrix_hierarchy_load", self.h, str(path).encode())


class Mlp:
    """The learned-guess MLP (XAMG_b200_mlp_*): n_in -> h -> h -> n_out."""

    def __init__(self, n_in, n_hidden, n_out, seed=0):
        i = C.c_size_t()
        call("XAMG_b200_mlp_create", n_in, n_hidden, n_out, seed, C.byref(i))
        self.h, self.n_in, self.n_hidden, self.n_out = i.value, n_in, n_hidden, n_out

    def __del__(self):
        try:
            call("XAMG_b200_mlp_destroy", self.h)
        except Exception:
            pass

    def count(self):
        c = u64()
        call("XAMG_b200_mlp_params", self.h, None, 0, C.byref(c))
        return c.value

    def params(self):
        out = np.zeros(self.count(), np.float32)
        call("XAMG_b200_mlp_params", self.h, _ptr(out), 0, None)
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.count()
        call("XAMG_b200_mlp_params", self.h, _ptr(p), 1, None)

    def predict(self, X_ptr, Y_ptr, batch):
        call("XAMG_b200_mlp_predict", self.h, batch, X_ptr, Y_ptr)

    def train_step(self, X_ptr, T_ptr, batch, lr):
        loss = C.c_double()
        call("XAMG_b200_mlp_train_step", self.h, batch, X_ptr, T_ptr, lr, C.byref(loss))
        return loss.value

    def gradients(self, X_ptr, T_ptr, batch):
        g = np.zeros(self.count(), np.float32)
        loss = C.c_double()
        call("XAMG_b200_mlp_gradients", self.h, batch, X_ptr, T_ptr, _ptr(g), C.byref(loss))
        return g, loss.value


class Vector:
    """XAMG_vector_* of n rows and nv interleaved right-hand sides (device)."""

    def __init__(self, n, nv, part=None):
        v = sz()
        call("XAMG_vector_create", C.byref(v), 2)
        if part is not None:
            call("XAMG_vector_set_part", part, v.value)
        call("XAMG_vector_alloc_d", n, nv, v.value)
        self.h, self.n, self.nv = v.value, n, nv

    def set(self, value):
        call("XAMG_vector_set_val_d", float(value), self.h)

    def upload(self, a):
        a = np.ascontiguousarray(a, np.float64).reshape(-1)
        assert a.size == self.n * self.nv
        call("XAMG_vector_upload_d", _ptr(a), self.n, 0, self.nv, self.h)

    def download(self):
        out = np.empty(self.n * self.nv, np.float64)
        call("XAMG_vector_download_d", _ptr(out), self.n, 0, self.nv, self.h)
        return out

    def device_ptr(self):
        p = C.c_void_p()
        call("XAMG_b200_vector_device_ptr", self.h, C.byref(p))
        return p.value


def solve_batch(solvers, xs, bs):
    """XAMG_b200_solver_solve_batch: solver i solves x_i from b_i, all systems
    together (each on its own stream, the merged BiCGStab forms in lockstep)."""
    m = len(solvers)
    nv = np.array([x.nv for x in xs], np.uint16)
    xh = np.array([x.h for x in xs], np.uint64)
    bh = np.array([b.h for b in bs], np.uint64)
    sh = np.array([S.h for S in solvers], np.uint64)
    call("XAMG_b200_solver_solve_batch", m, _ptr(nv), _ptr(xh), _ptr(bh), _ptr(sh))


class Solver:
    """XAMG_solver_create2 + solve + statistics."""

    def __init__(self, matrix, params, x, b):
        s = sz()
        call("XAMG_solver_create2", matrix.h, params.h, x.h, b.h, C.byref(s))
        self.h, self.nv = s.value, x.nv

    def solve(self, x=None, b=None):
        if x is None:
            call("XAMG_solver_solve1", self.nv, self.h)
        else:
            call("XAMG_solver_solve2", self.nv, x.h, b.h, self.h)

    def renew(self, params):
        call("XAMG_solver_renew_params", params.h, self.h)

    def convergence_info(self):
        out = np.zeros(self.nv, np.int32)
        call("XAMG_solver_get_convergence_info", _ptr(out), self.nv, self.h)
        return out

    def stats(self):
        it = C.c_int()
        conv = np.zeros(self.nv, np.int32)
        a = np.zeros(self.nv)
        r = np.zeros(self.nv)
        call("XAMG_b200_solver_stats", self.h, C.byref(it), _ptr(conv), _ptr(a), _ptr(r),
             self.nv)
        return dict(iters=it.value, conv=conv, abs_res=a, rel_res=r)

    def nlevels(self):
        return call("XAMG_b200_solver_nlevels", self.h)

    def level_info(self, level, which):
        nr, nc, nz = u64(), u64(), u64()
        cb, f32 = C.c_int(), C.c_int()
        hsh = C.c_uint16()
        mn, mx = C.c_double(), C.c_double()
        call("XAMG_b200_solver_level_info", self.h, level, which, C.byref(nr), C.byref(nc),
             C.byref(nz), C.byref(cb), C.byref(f32), C.byref(hsh), C.byref(mn), C.byref(mx))
        return dict(nrows=nr.value, ncols=nc.value, nnz=nz.value, col_bytes=cb.value,
                    f32=bool(f32.value), bf16=f32.value == 2, fp16=f32.value == 3, hash=hsh.value, min_eig=mn.value,
                    max_eig=mx.value)

    def level_tuned(self, level, which):
        """The autotuner's launch-shape codes of a level matrix, as a
        [2][2][6] array (value float, x float, log2 nv)."""
        out = np.zeros(24, np.uint8)
        call("XAMG_b200_solver_level_tuned", self.h, level, which, _ptr(out))
        return out.reshape(2, 2, 6)

    def level_xstaged(self, level, which):
        """The nv the level matrix's x-staged copy was built for (0: none)."""
        v = C.c_int()
        call("XAMG_b200_solver_level_xstaged", self.h, level, which, C.byref(v))
        return v.value

    def level_stencil(self, level, which):
        """The level matrix's grid-stencil copy: (pattern, S, S2, diag_first),
        pattern -1 where it has none."""
        pat, S, S2, df = C.c_int(), C.c_uint32(), C.c_uint32(), C.c_int()
        call("XAMG_b200_solver_level_stencil", self.h, level, which, C.byref(pat), C.byref(S),
             C.byref(S2), C.byref(df))
        return pat.value, S.value, S2.value, df.value

    def level_download(self, level, which):
        info = self.level_info(level, which)
        row = np.zeros(info["nrows"] + 1, np.uint32)
        col = np.zeros(info["nnz"], {1: np.uint8, 2: np.uint16, 4: np.uint32,
                                     -2: np.int16}[info["col_bytes"]])
        if info["bf16"]:  # BF16 bits, widened to float32 below
            val = np.zeros(info["nnz"], np.uint16)
        else:  # FP16 values come back widened to float32, their scale applied
            val = np.zeros(info["nnz"], np.float32 if info["f32"] else np.float64)
        call("XAMG_b200_solver_level_download", self.h, level, which, _ptr(row), _ptr(col),
             _ptr(val))
        if info["bf16"]:
            val = (val.astype(np.uint32) << 16).view(np.float32)
        return row, col, val, info

    def save_hierarchy(self, path):
        """Write the multigrid hierarchy this solver was built from."""
        call("XAMG_b200_solver_hierarchy_save", self.h, str(path).encode())

    def level_spmv(self, level, which, x_ptr, y_ptr, nv, mode=0, stream=None):
        """y = A x on the solver's own level matrix (device pointers)."""
        call("XAMG_b200_solver_level_spmv", self.h, level, which, x_ptr, y_ptr, nv, mode,
             stream if stream is not None else globals()["stream"]())

    def level_csr(self, level, which):
        d = Csr()
        call("XAMG_b200_solver_level_csr", self.h, level, which, C.byref(d))
        return d

    def hierarchy(self):
        """The double-precision hierarchy the host setup built: list of
        dicts {A: (row, col, val), P: (row, col, val, ncols) or None, min_eig, max_eig}."""
        out = []
        nl = self.nlevels()
        for l in range(nl):
            ia = self.level_info(l, 0)
            row = np.zeros(ia["nrows"] + 1, np.uint32)
            col = np.zeros(ia["nnz"], np.uint32)
            val = np.zeros(ia["nnz"], np.float64)
            call("XAMG_b200_solver_hierarchy_export", self.h, l, 0, _ptr(row), _ptr(col),
                 _ptr(val))
            P = None
            if l + 1 < nl:
                ip = self.level_info(l, 2)
                pr = np.zeros(ip["nrows"] + 1, np.uint32)
                pc = np.zeros(ip["nnz"], np.uint32)
                pv = np.zeros(ip["nnz"], np.float64)
                call("XAMG_b200_solver_hierarchy_export", self.h, l, 2, _ptr(pr), _ptr(pc),
                     _ptr(pv))
                P = (pr, pc, pv, ip["ncols"])
            out.append(dict(A=(row, col, val), P=P, min_eig=ia["min_eig"],
                            max_eig=ia["max_eig"]))
        return out
