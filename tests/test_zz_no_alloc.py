"""XAMG_b200_dot_noalloc, the dot product for callers that cannot allocate
device memory (an application whose device memory belongs to its own pool
allocator, or a loop where a synchronising cudaMalloc is not allowed): called
through the C ABI twice in a row on the same inputs, it must give what
XAMG_b200_dot gives, bit for bit. Collected last so that a run that stops at
the first failure has run every other test first; it also passes alone in a
fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nv,n", [(1, 1000), (8, 300001), (32, 77777)])
def test_dot_noalloc_matches_dot(gpu, nv, n):
    import torch
    rng = np.random.default_rng(nv + n)
    x = torch.from_numpy(rng.standard_normal(n * nv)).cuda()
    y = torch.from_numpy(rng.standard_normal(n * nv)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    want = np.zeros(nv)
    gpu.call("XAMG_b200_dot", n, nv, x.data_ptr(), y.data_ptr(),
             want.ctypes.data_as(C.c_void_p), stream)
    for _ in range(2):
        out = torch.full((nv,), np.nan, dtype=torch.float64, device="cuda")
        gpu.call("XAMG_b200_dot_noalloc", n, nv, x.data_ptr(), y.data_ptr(), out.data_ptr(),
                 stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got.tobytes() == want.tobytes()
    ref = (x.cpu().numpy().reshape(n, nv) * y.cpu().numpy().reshape(n, nv)).sum(axis=0)
    np.testing.assert_allclose(want, ref, rtol=1e-10, atol=1e-9)


def test_dot_noalloc_rejects_unsupported_nv(gpu):
    import torch
    x = torch.zeros(30, dtype=torch.float64, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = gpu.lib().XAMG_b200_dot_noalloc(10, 3, x.data_ptr(), x.data_ptr(), out.data_ptr(), None)
    assert rc == -2


def test_dot_noalloc_allocates_nothing(gpu):
    """XAMG_init resolved the array and loaded the entry point's kernels, so
    calls on the library's device (every supported nv, repeated) leave the
    device's free memory exactly as it was."""
    import torch
    n = 50000
    x = torch.ones(n * 32, dtype=torch.float64, device="cuda")
    out = torch.zeros(32, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        for nv in (1, 2, 4, 8, 16, 32):
            gpu.call("XAMG_b200_dot_noalloc", n, nv, x.data_ptr(), x.data_ptr(),
                     out.data_ptr(), stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert out.cpu().numpy().tolist() == [float(n)] * 32
