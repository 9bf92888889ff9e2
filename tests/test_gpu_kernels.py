"""Kernel-level parity on the GPU, through the C ABI (XAMG_b200_* entry
points with device pointers): every SpMV element must equal the oracle's bit
for bit; reductions must equal the oracle's replay of the kernels' fixed
order bit for bit, and XAMG's sequential order to 1e-12 relative."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NVS = [1, 2, 4, 8, 16, 32]


def torch_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def random_csr(n, ncols, rng, max_row=30, empty_frac=0.1):
    row = [0]
    cols, vals = [], []
    for i in range(n):
        k = 0 if rng.random() < empty_frac else int(rng.integers(1, max_row + 1))
        k = min(k, ncols)
        c = rng.choice(ncols, size=k, replace=False)
        cols.extend(c.tolist())
        vals.extend((rng.standard_normal(k) * 10.0 ** rng.integers(-3, 4, k)).tolist())
        row.append(len(cols))
    return (np.array(row, np.uint32), np.array(cols, np.uint32), np.array(vals, np.float64))


def dev_csr(xamg, row, col, val, ncols, col_bytes, f32):
    ctype = {1: np.uint8, 2: np.uint16, 4: np.uint32}[col_bytes]
    keep = [torch_dev(row), torch_dev(col.astype(ctype)),
            torch_dev(val.astype(np.float32 if f32 else np.float64))]
    d = xamg.Csr(len(row) - 1, ncols, len(col), keep[0].data_ptr(), keep[1].data_ptr(),
                 keep[2].data_ptr(), col_bytes, int(f32))
    return d, keep


@pytest.mark.parametrize("nv", NVS)
@pytest.mark.parametrize("col_bytes,ncols", [(1, 200), (2, 5000), (4, 70000)])
@pytest.mark.parametrize("f32", [False, True])
def test_spmv_bit_exact(gpu, oracle, nv, col_bytes, ncols, f32):
    rng = np.random.default_rng(nv * 100 + col_bytes * 7 + int(f32))
    n = 3000
    row, col, val = random_csr(n, ncols, rng)
    dt = np.float32 if f32 else np.float64
    x = rng.standard_normal(ncols * nv).astype(dt)
    y0 = rng.standard_normal(n * nv).astype(dt)
    A, keep = dev_csr(gpu, row, col, val, ncols, col_bytes, f32)
    xd = torch_dev(x)
    for mode in (0, 1):
        yd = torch_dev(y0.copy())
        gpu.call("XAMG_b200_spmv", C.byref(A), xd.data_ptr(), yd.data_ptr(), nv, mode, None)
        import torch
        torch.cuda.synchronize()
        got = yd.cpu().numpy()
        want = oracle.csr_ax_y(row, col, val.astype(dt), x, nv, ncols=ncols,
                               axpy_y=(y0 if mode == 1 else None))
        assert got.tobytes() == want.tobytes(), f"mode {mode}: {np.abs(got - want).max()}"


def test_spmv_edge_cases(gpu, oracle):
    import torch
    rng = np.random.default_rng(11)
    # a single row, a matrix with no entries, a long dense row
    for n, ncols, max_row, empty in [(1, 5, 5, 0.0), (50, 50, 0, 1.0), (4, 3000, 3000, 0.0)]:
        row, col, val = random_csr(n, ncols, rng, max_row=max(max_row, 1), empty_frac=empty)
        for nv in (1, 8):
            x = rng.standard_normal(ncols * nv)
            A, keep = dev_csr(gpu, row, col, val, ncols, 4, False)
            yd = torch_dev(np.full(n * nv, 7.0))
            xd = torch_dev(x)
            gpu.call("XAMG_b200_spmv", C.byref(A), xd.data_ptr(), yd.data_ptr(), nv, 0, None)
            torch.cuda.synchronize()
            want = oracle.csr_ax_y(row, col, val, x, nv, ncols=ncols)
            assert yd.cpu().numpy().tobytes() == want.tobytes()


def test_spmv_cube_rounding_kats(gpu):
    """The order and no-FMA known answers of the oracle tests, on the GPU."""
    import torch
    e = 2.0**-30
    row = np.array([0, 3, 5], np.uint32)
    col = np.array([0, 1, 2, 3, 4], np.uint32)
    val = np.array([1e16, 1.0, -1e16, -1.0, 1 + e])
    x = np.array([1.0, 1.0, 1.0, 1.0, 1 - e])
    A, keep = dev_csr(gpu, row, col, val, 5, 4, False)
    xd, yd = torch_dev(x), torch_dev(np.zeros(2))
    gpu.call("XAMG_b200_spmv", C.byref(A), xd.data_ptr(), yd.data_ptr(), 1, 0, None)
    torch.cuda.synchronize()
    assert yd.cpu().numpy().tolist() == [0.0, 0.0]


@pytest.mark.parametrize("nv", NVS)
@pytest.mark.parametrize("n", [1, 97, 4096, 300001])
def test_reductions_canonical(gpu, oracle, nv, n):
    import torch
    rng = np.random.default_rng(n + nv)
    x = rng.standard_normal(n * nv)
    y = rng.standard_normal(n * nv)
    xd, yd = torch_dev(x), torch_dev(y)
    out = np.zeros(nv)
    gpu.call("XAMG_b200_dot", n, nv, xd.data_ptr(), yd.data_ptr(),
             out.ctypes.data_as(C.c_void_p), None)
    oracle.set_reduction(1)
    try:
        want = oracle.dot(x, y, nv)
    finally:
        oracle.set_reduction(0)
    assert out.tobytes() == want.tobytes()
    seq = oracle.dot(x, y, nv)
    np.testing.assert_allclose(out, seq, rtol=1e-11, atol=1e-11 * np.abs(x * y).sum())


@pytest.mark.parametrize("nv", [1, 8, 32])
def test_merged_groups_canonical(gpu, oracle, nv):
    import torch
    n = 20000
    rng = np.random.default_rng(nv)
    r0 = rng.standard_normal(n * nv)
    b = rng.standard_normal(n * nv)
    s = rng.standard_normal(n * nv)
    t = rng.standard_normal(n * nv)
    om = rng.standard_normal(nv)
    oracle.set_reduction(1)
    try:
        # group1
        r0d, bd = torch_dev(r0), torch_dev(b)
        pd, rd = torch_dev(np.zeros(n * nv)), torch_dev(np.zeros(n * nv))
        rho = np.zeros(nv)
        gpu.call("XAMG_b200_group1", n, nv, r0d.data_ptr(), bd.data_ptr(), pd.data_ptr(),
                 rd.data_ptr(), rho.ctypes.data_as(C.c_void_p), None)
        o_r0, o_b = r0.copy(), b.copy()
        o_p, o_r, o_rho = np.zeros(n * nv), np.zeros(n * nv), np.zeros(nv)
        oracle.lib().or_group1(n, nv, o_r0, o_b, o_p, o_r, o_rho)
        assert r0d.cpu().numpy().tobytes() == o_r0.tobytes()
        assert pd.cpu().numpy().tobytes() == o_p.tobytes()
        assert rho.tobytes() == o_rho.tobytes()
        # group2
        phi, psi, th = np.zeros(nv), np.zeros(nv), np.zeros(nv)
        td, sd, r0dd = torch_dev(t), torch_dev(s), torch_dev(r0)  # kept alive across the calls
        gpu.call("XAMG_b200_group2", n, nv, td.data_ptr(), sd.data_ptr(),
                 phi.ctypes.data_as(C.c_void_p), psi.ctypes.data_as(C.c_void_p),
                 th.ctypes.data_as(C.c_void_p), None)
        o = [np.zeros(nv) for _ in range(3)]
        oracle.lib().or_group2(n, nv, t, s, *o)
        assert phi.tobytes() == o[0].tobytes() and psi.tobytes() == o[1].tobytes()
        assert th.tobytes() == o[2].tobytes()
        # group4
        rd = torch_dev(np.zeros(n * nv))
        rho4 = np.zeros(nv)
        gpu.call("XAMG_b200_group4", n, nv, sd.data_ptr(), td.data_ptr(),
                 r0dd.data_ptr(), rd.data_ptr(), om.ctypes.data_as(C.c_void_p),
                 rho4.ctypes.data_as(C.c_void_p), None)
        o_r, o_rho = np.zeros(n * nv), np.zeros(nv)
        oracle.lib().or_group4(n, nv, s, t, r0, o_r, om, o_rho)
        assert rd.cpu().numpy().tobytes() == o_r.tobytes()
        assert rho4.tobytes() == o_rho.tobytes()
    finally:
        oracle.set_reduction(0)
    torch.cuda.synchronize()


@pytest.mark.parametrize("nv", [1, 8])
def test_spmv_dot_fused(gpu, oracle, nv):
    import torch
    row, col, val = gpu.generate_cube(20, 20, 20)
    n = len(row) - 1
    rng = np.random.default_rng(3)
    x, z = rng.standard_normal(n * nv), rng.standard_normal(n * nv)
    A, keep = dev_csr(gpu, row, col, val, n, 2, False)
    vd = torch_dev(np.zeros(n * nv))
    dot = np.zeros(nv)
    xd, zd = torch_dev(x), torch_dev(z)  # kept alive until the kernel has run
    gpu.call("XAMG_b200_spmv_dot", C.byref(A), xd.data_ptr(), vd.data_ptr(),
             zd.data_ptr(), dot.ctypes.data_as(C.c_void_p), nv, None)
    v = oracle.csr_ax_y(row, col, val, x, nv, ncols=n)
    assert vd.cpu().numpy().tobytes() == v.tobytes()
    oracle.set_reduction(1)
    try:
        assert dot.tobytes() == oracle.dot(v, z, nv).tobytes()
    finally:
        oracle.set_reduction(0)


def test_kernels_are_sm100_machine_code(gpu):
    """The CUDA runtime reports the library's kernels as sm_100 machine code."""
    import ctypes as C
    b, p = C.c_int(), C.c_int()
    gpu.call("XAMG_b200_kernel_arch", C.byref(b), C.byref(p))
    assert b.value == 100, (b.value, p.value)
