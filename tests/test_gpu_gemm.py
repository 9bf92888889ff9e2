"""The tcgen05 BF16 GEMM (XAMG_b200_gemm_bf16) against a float64 product of the
same BF16-rounded operands. FP32 accumulation differs from the exact sum by at
most K * 2^-24 * (|A| |B|^T) per element (plus one BF16 rounding of the
output for the BF16 modes); the tests allow twice that."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(gpu, M, N, K, mode, seed, bias=True):
    import torch
    g = torch.Generator().manual_seed(seed)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    bv = torch.randn(N, generator=g) if bias else None
    aux = torch.randn(M, N, generator=g).to(torch.bfloat16)
    out_dt = torch.float32 if mode == 0 else torch.bfloat16
    Ad, Bd = A.cuda(), B.cuda()
    Cd = torch.full((M, N), float("nan"), dtype=out_dt, device="cuda")
    bd = bv.cuda() if bias else None
    auxd = aux.cuda()
    gpu.call("XAMG_b200_gemm_bf16", M, N, K, Ad.data_ptr(), Bd.data_ptr(), Cd.data_ptr(), N, mode,
             bd.data_ptr() if bias else None, auxd.data_ptr(), N,
             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    a = A.double().numpy()
    b = B.double().numpy()
    ref = a @ b.T
    bound = 2.0 * K * 2.0 ** -24 * (np.abs(a) @ np.abs(b).T) + 1e-30
    if bias and mode != 3:
        ref = ref + bv.double().numpy()[None, :]
        bound = bound + 2.0 ** -23 * np.abs(ref)
    if mode == 2:
        ref = np.maximum(ref, 0.0)
    if mode == 3:
        ref = np.where(aux.double().numpy() > 0, ref, 0.0)
    got = Cd.double().cpu().numpy()
    if mode != 0:
        bound = bound + 2.0 ** -8 * np.abs(ref)
    return got, ref, bound


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 640), (384, 256, 1024),
                                   (1024, 1024, 4096)])
def test_gemm_f32_bias(gpu, M, N, K):
    got, ref, bound = run(gpu, M, N, K, 0, seed=M + N + K)
    assert np.all(np.abs(got - ref) <= bound), np.abs(got - ref).max()


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_gemm_bf16_modes(gpu, mode):
    got, ref, bound = run(gpu, 256, 256, 512, mode, seed=mode)
    assert np.all(np.abs(got - ref) <= bound), np.abs(got - ref).max()


def test_gemm_rejects_bad_shapes(gpu):
    import torch
    A = torch.zeros(128, 64, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(128, 128, dtype=torch.float32, device="cuda")
    rc = gpu.lib().XAMG_b200_gemm_bf16(100, 128, 64, A.data_ptr(), A.data_ptr(), C.data_ptr(),
                                       128, 0, None, None, 0, None)
    assert rc == -2
