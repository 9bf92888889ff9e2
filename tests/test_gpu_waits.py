"""Bounded waits. The SpMV kernels wait on an mbarrier for the bulk copies of
their staged matrix entries; every such wait gives up after a time limit,
raises a flag that the solve call turns into XAMG_ERR_TIMEOUT, and leaves no
copy in flight. Here a kernel waits on a barrier that nothing completes: the
wait must end by itself within its limit, report the timeout, and leave the
GPU context usable for the next call."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_reports(gpu):
    out = C.c_int(-1)
    t0 = time.perf_counter()
    gpu.call("XAMG_b200_wait_selftest", 0.02, C.byref(out))
    dt = time.perf_counter() - t0
    assert out.value == 1
    assert dt < 1.0
    # the flag was cleared and the context still works
    row, col, val = gpu.generate_cube(8, 8, 8)
    n = len(row) - 1
    import torch
    rd = torch.from_numpy(row).cuda()
    cd = torch.from_numpy(col).cuda()
    vd = torch.from_numpy(val).cuda()
    A = gpu.Csr(n, n, len(col), rd.data_ptr(), cd.data_ptr(), vd.data_ptr(), 4, 0)
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    gpu.call("XAMG_b200_spmv", C.byref(A), x.data_ptr(), y.data_ptr(), 1, 0,
             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    want = np.add.reduceat(val, row[:-1]) if n else np.zeros(0)
    np.testing.assert_allclose(y.cpu().numpy(), want, rtol=1e-12, atol=1e-12)


def test_wait_selftest_rejects_long_limits(gpu):
    out = C.c_int(-1)
    rc = gpu.lib().XAMG_b200_wait_selftest(5.0, C.byref(out))
    assert rc == -2
