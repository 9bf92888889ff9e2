"""ctypes wrapper around the CPU oracle (oracle/liboracle.so).

Test infrastructure: the oracle is the checker, never the thing measured or
shipped. Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg
import this module.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def build():
    subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])


def threads():
    """Threads the oracle's SpMV loops run on (OMP_NUM_THREADS or all cores)."""
    return int(lib().or_threads())


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(ORACLE_DIR, "oracle.cpp")):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_define_int_type.restype = C.c_uint16
        L.or_define_int_type.argtypes = [C.c_uint64]
        L.or_encode_hash.restype = C.c_uint16
        L.or_encode_hash.argtypes = [C.c_uint64] * 4 + [C.c_int, C.c_int]
        L.or_set_reduction.argtypes = [C.c_int, C.c_int]
        L.or_core_range.argtypes = [C.c_uint64, C.c_int, C.c_int, C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_uint64)]
        for fn in (L.or_csr_ax_y, L.or_csr_axpy):
            fn.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64, u32p, u32p, C.c_void_p,
                           C.c_void_p, C.c_void_p, C.c_int]
        L.or_compress.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, u32p, u32p, u32p, u32p,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.or_transpose.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, u32p, u32p, f64p, u32p,
                                   u32p, f64p]
        L.or_inverse.argtypes = [C.c_int, C.c_uint64, C.c_void_p, C.c_void_p]
        L.or_inv_diag.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_uint64, u32p, u32p, f64p,
                                  C.c_void_p]
        L.or_cheby_coeffs.argtypes = [C.c_double, C.c_double, C.c_int, C.c_float, f64p]
        L.or_dot.argtypes = [C.c_uint64, C.c_int, f64p, f64p, f64p]
        L.or_group1.argtypes = [C.c_uint64, C.c_int, f64p, f64p, f64p, f64p, f64p]
        L.or_group2.argtypes = [C.c_uint64, C.c_int, f64p, f64p, f64p, f64p, f64p]
        L.or_group4.argtypes = [C.c_uint64, C.c_int, f64p, f64p, f64p, f64p, f64p, f64p]
        L.or_round_bf16.argtypes = [C.c_uint64, C.c_void_p, C.c_void_p]
        L.or_threads.restype = C.c_int
        L.or_generate_cube.restype = C.c_uint64
        L.or_generate_cube.argtypes = [C.c_uint64] * 3 + [u32p, u32p, f64p]
        L.or_sys_create.restype = C.c_void_p
        L.or_sys_create.argtypes = [C.c_int]
        L.or_sys_destroy.argtypes = [C.c_void_p]
        L.or_sys_set_param.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
        L.or_sys_set_hsgs_cores.argtypes = [C.c_void_p, C.c_int]
        L.or_sys_add_level.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, u32p, u32p, f64p,
                                       C.c_double, C.c_double]
        L.or_sys_add_interp.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, u32p,
                                        u32p, f64p]
        L.or_sys_setup.argtypes = [C.c_void_p]
        L.or_sys_solve.argtypes = [C.c_void_p, f64p, f64p, i32p, f64p, f64p]
        L.or_sys_level_matrix.restype = C.c_uint64
        L.or_sys_level_matrix.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.POINTER(C.c_int),
                                          C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        _lib = L
    return _lib


def set_reduction(mode, ncores=1):
    """mode 0: XAMG per-core sequential order; mode 1: the B200 kernels' fixed order."""
    lib().or_set_reduction(mode, ncores)


def define_int_type(r):
    return lib().or_define_int_type(r)


def encode_hash(nnz, ncols, bnrows, bncols, f32=False, reduced=False):
    return lib().or_encode_hash(nnz, ncols, bnrows, bncols, int(f32), int(reduced))


def core_range(n, ncores, core):
    off, sz = C.c_uint64(), C.c_uint64()
    lib().or_core_range(n, ncores, core, C.byref(off), C.byref(sz))
    return off.value, sz.value


def generate_cube(nx, ny, nz):
    n = nx * ny * nz
    row = np.zeros(n + 1, np.uint32)
    col = np.zeros(7 * n, np.uint32)
    val = np.zeros(7 * n, np.float64)
    nnz = lib().or_generate_cube(nx, ny, nz, row, col, val)
    return row, col[:nnz].copy(), val[:nnz].copy()


def csr_ax_y(row, col, val, x, nv, ncols=None, axpy_y=None):
    nrows = len(row) - 1
    ncols = ncols if ncols is not None else (x.size // nv)
    f32 = val.dtype == np.float32
    dt = np.float32 if f32 else np.float64
    val = np.ascontiguousarray(val, dt)
    x = np.ascontiguousarray(x, dt)
    if axpy_y is None:
        y = np.zeros(nrows * nv, dt)
        lib().or_csr_ax_y(int(f32), nrows, ncols, len(col), row, col, val.ctypes.data,
                          x.ctypes.data, y.ctypes.data, nv)
    else:
        y = np.ascontiguousarray(axpy_y, dt).copy()
        lib().or_csr_axpy(int(f32), nrows, ncols, len(col), row, col, val.ctypes.data,
                          x.ctypes.data, y.ctypes.data, nv)
    return y


def compress(row, col, block_ncols):
    row = row.astype(np.uint32).copy()
    col = col.astype(np.uint32).copy()
    nrows = len(row) - 1
    row_ind = np.zeros(nrows, np.uint32)
    col_ind = np.zeros(block_ncols, np.uint32)
    nr, nc = C.c_uint64(), C.c_uint64()
    lib().or_compress(nrows, block_ncols, len(col), row, col, row_ind, col_ind, C.byref(nr),
                      C.byref(nc))
    return row[:nr.value + 1], col, row_ind[:nr.value], col_ind[:nc.value]


def transpose(row, col, val, ncols):
    nrows = len(row) - 1
    trow = np.zeros(ncols + 1, np.uint32)
    tcol = np.zeros(len(col), np.uint32)
    tval = np.zeros(len(col), np.float64)
    lib().or_transpose(nrows, ncols, len(col), row.astype(np.uint32), col.astype(np.uint32),
                       val.astype(np.float64), trow, tcol, tval)
    return trow, tcol, tval


def inverse(a):
    a = np.ascontiguousarray(a)
    n = a.shape[0]
    out = np.zeros_like(a)
    lib().or_inverse(int(a.dtype == np.float32), n, a.ctypes.data, out.ctypes.data)
    return out


def inv_diag(row, col, val, f32=False, sqrt=False):
    n = len(row) - 1
    out = np.zeros(n, np.float32 if f32 else np.float64)
    lib().or_inv_diag(int(f32), int(sqrt), n, len(col), row, col, val, out.ctypes.data)
    return out


def cheby_coeffs(min_eig, max_eig, order, frac):
    out = np.zeros(order, np.float64)
    lib().or_cheby_coeffs(min_eig, max_eig, order, frac, out)
    return out


def round_bf16(a):
    """float32 array -> the same values rounded to BF16 (as float32)"""
    a = np.ascontiguousarray(a, np.float32)
    out = np.empty_like(a)
    lib().or_round_bf16(a.size, a.ctypes.data, out.ctypes.data)
    return out


def dot(x, y, nv):
    out = np.zeros(nv, np.float64)
    lib().or_dot(x.size // nv, nv, np.ascontiguousarray(x, np.float64),
                 np.ascontiguousarray(y, np.float64), out)
    return out


class System:
    """A whole XAMG solve on the oracle: levels, parameters, solve."""

    def __init__(self, nv):
        self.h = lib().or_sys_create(nv)
        self.nv = nv
        self.n = None

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_sys_destroy(self.h)
            self.h = None

    def set(self, role, key, value, level=-1):
        lib().or_sys_set_param(self.h, role.encode(), key.encode(), str(value).encode(), level)

    def set_params(self, params):
        """params: {role: {key: value}}; key 'k@lev' sets a per-level value."""
        for role, kv in params.items():
            for k, v in kv.items():
                if "@" in k:
                    key, lev = k.split("@")
                    self.set(role, key, v, int(lev))
                else:
                    self.set(role, k, v)

    def hsgs_cores(self, n):
        lib().or_sys_set_hsgs_cores(self.h, n)

    def add_level(self, row, col, val, min_eig=float("nan"), max_eig=float("nan")):
        n = len(row) - 1
        if self.n is None:
            self.n = n
        lib().or_sys_add_level(self.h, n, len(col), np.ascontiguousarray(row, np.uint32),
                               np.ascontiguousarray(col, np.uint32),
                               np.ascontiguousarray(val, np.float64), min_eig, max_eig)

    def add_interp(self, row, col, val, ncols):
        lib().or_sys_add_interp(self.h, len(row) - 1, ncols, len(col),
                                np.ascontiguousarray(row, np.uint32),
                                np.ascontiguousarray(col, np.uint32),
                                np.ascontiguousarray(val, np.float64))

    def setup(self):
        rc = lib().or_sys_setup(self.h)
        assert rc == 0

    def solve(self, b, x0=None):
        nv = self.nv
        b = np.ascontiguousarray(b, np.float64).ravel()
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, np.float64).ravel().copy()
        conv = np.zeros(nv, np.int32)
        a = np.zeros(nv)
        r = np.zeros(nv)
        it = lib().or_sys_solve(self.h, x, b, conv, a, r)
        return x, dict(iters=it, conv=conv, abs_res=a, rel_res=r)

    def level_matrix(self, level, which):
        """which: 0 A, 1 R, 2 P in the working precision the oracle derived."""
        L = lib()
        f32 = C.c_int()
        nr, nc = C.c_uint64(), C.c_uint64()
        nnz = L.or_sys_level_matrix(self.h, level, which, None, None, None, C.byref(f32),
                                    C.byref(nr), C.byref(nc))
        row = np.zeros(nr.value + 1, np.uint32)
        col = np.zeros(nnz, np.uint32)
        val = np.zeros(nnz, np.float32 if f32.value else np.float64)
        L.or_sys_level_matrix(self.h, level, which, row.ctypes.data, col.ctypes.data,
                              val.ctypes.data, C.byref(f32), C.byref(nr), C.byref(nc))
        return row, col, val, nc.value


# ---------------------------------------------------------------------------
# Inputs of the CPU arm (oracle/liboracle_setup.so): the seeded generators and
# the host multigrid setup compiled from the library's host-only sources, so
# that a process that must not load the CUDA library gets the same matrix and
# hierarchy bit for bit.
# ---------------------------------------------------------------------------
SETUP_LIB_PATH = os.path.join(ORACLE_DIR, "liboracle_setup.so")
_setup = None

# XAMG's MultiGrid family defaults (xamg_params_details.h:194-235) for the
# keys the host setup reads, plus the library's seed key.
MG_DEFAULTS = {"mg_strength_threshold": 0.5, "mg_max_row_sum": 0.9, "mg_max_levels": 25,
               "mg_coarse_matrix_size": 100, "mg_trunc_factor": 0.25, "mg_Pmax_elements": 4,
               "gpu_seed": 0}


def setup_lib():
    global _setup
    if _setup is None:
        if not os.path.exists(SETUP_LIB_PATH):
            build()
        L = C.CDLL(SETUP_LIB_PATH)
        L.XAMG_b200_generate_diffusion.restype = C.c_int64
        L.XAMG_b200_generate_diffusion.argtypes = [C.c_int] + [C.c_uint64] * 3 + [
            C.c_double, C.c_double, C.c_uint64, u32p, u32p, f64p]
        L.XAMG_b200_generate_cube.restype = C.c_int64
        L.XAMG_b200_generate_cube.argtypes = [C.c_uint64] * 3 + [u32p, u32p, f64p]
        L.os_hier_build.restype = C.c_void_p
        L.os_hier_build.argtypes = [C.c_uint64, C.c_uint64, u32p, u32p, f64p, C.c_float,
                                    C.c_float, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int]
        L.os_hier_free.argtypes = [C.c_void_p]
        L.os_hier_levels.restype = C.c_int
        L.os_hier_levels.argtypes = [C.c_void_p]
        L.os_hier_level.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.POINTER(C.c_uint64)] * 3 + [
            C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _setup = L
    return _setup


def setup_generate_diffusion(stencil, nx, ny, nz, sigma, az, seed):
    """The library's seeded diffusion generator (7- or 27-point)."""
    n = nx * ny * nz
    row = np.zeros(n + 1, np.uint32)
    col = np.zeros(stencil * n, np.uint32)
    val = np.zeros(stencil * n, np.float64)
    nnz = setup_lib().XAMG_b200_generate_diffusion(stencil, nx, ny, nz, sigma, az, seed, row, col,
                                                   val)
    assert nnz >= 0
    return row, col[:nnz].copy(), val[:nnz].copy()


def setup_hierarchy(row, col, val, mg_params):
    """The hierarchy the library's host setup builds for a MultiGrid list
    `mg_params` (XAMG defaults for missing keys): a list of dicts
    {A: (row, col, val), P: (row, col, val, ncols) or None, min_eig, max_eig},
    as the library's solver hierarchy export gives it."""
    L = setup_lib()
    p = dict(MG_DEFAULTS)
    p.update({k: v for k, v in mg_params.items() if k in MG_DEFAULTS})
    n = len(row) - 1
    h = L.os_hier_build(n, len(col), np.ascontiguousarray(row, np.uint32),
                        np.ascontiguousarray(col, np.uint32), np.ascontiguousarray(val, np.float64),
                        p["mg_strength_threshold"], p["mg_max_row_sum"], int(p["mg_max_levels"]),
                        int(p["mg_coarse_matrix_size"]), p["mg_trunc_factor"],
                        int(p["mg_Pmax_elements"]), int(p["gpu_seed"]))
    try:
        out = []
        nl = L.os_hier_levels(h)
        for lev in range(nl):
            mats = []
            for which in (0, 1):
                nr, nc, nz = C.c_uint64(), C.c_uint64(), C.c_uint64()
                mn, mx = C.c_double(), C.c_double()
                L.os_hier_level(h, lev, which, C.byref(nr), C.byref(nc), C.byref(nz), None, None,
                                None, C.byref(mn), C.byref(mx))
                if nr.value == 0:
                    mats.append(None)
                    continue
                r = np.zeros(nr.value + 1, np.uint32)
                c = np.zeros(nz.value, np.uint32)
                v = np.zeros(nz.value, np.float64)
                L.os_hier_level(h, lev, which, C.byref(nr), C.byref(nc), C.byref(nz),
                                r.ctypes.data, c.ctypes.data, v.ctypes.data, C.byref(mn),
                                C.byref(mx))
                mats.append((r, c, v, nc.value))
            out.append(dict(A=mats[0][:3], P=mats[1] if lev + 1 < nl else None,
                            min_eig=mn.value, max_eig=mx.value))
        return out
    finally:
        L.os_hier_free(h)
