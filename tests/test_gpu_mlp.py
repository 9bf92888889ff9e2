"""The learned-guess MLP on the GPU (forward and backward on the tcgen05 GEMM)
against its CPU restatement (oracle/mlp_oracle.py): the same BF16 rounding
points, FP32 instead of float64 accumulation. Gradients must agree to 1 % of
each block's largest entry; a few steps of Adam must reduce the loss of a
learnable map tenfold."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import mlp_oracle as MO  # noqa: E402

pytestmark = pytest.mark.gpu


def blocks(g, n_in, h, n_out):
    sizes = [h * n_in, h, h * h, h, n_out * h, n_out]
    out, off = [], 0
    for s in sizes:
        out.append(g[off:off + s])
        off += s
    return out


@pytest.mark.parametrize("n_in,h,n_out,B", [(256, 128, 128, 128), (128, 256, 384, 256)])
def test_gradients_against_oracle(gpu, n_in, h, n_out, B):
    import torch
    m = gpu.Mlp(n_in, h, n_out, seed=3)
    p = m.params()
    rng = np.random.default_rng(4)
    X = rng.standard_normal((B, n_in)).astype(np.float32)
    T = rng.standard_normal((B, n_out)).astype(np.float32)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    Yd = torch.empty(B, n_out, dtype=torch.float32, device="cuda")
    m.predict(Xd.data_ptr(), Yd.data_ptr(), B)
    g, loss = m.gradients(Xd.data_ptr(), Td.data_ptr(), B)
    _, _, _, Yr = MO.forward(p.astype(np.float64), X.astype(np.float64), n_in, h, n_out)
    gr, lr_ = MO.gradients(p.astype(np.float64), X.astype(np.float64), T.astype(np.float64),
                           n_in, h, n_out)
    Y = Yd.cpu().numpy()
    assert np.abs(Y - Yr).max() <= 1e-2 * np.abs(Yr).max()
    assert abs(loss - lr_) <= 1e-3 * lr_
    for gb, rb in zip(blocks(g, n_in, h, n_out), blocks(gr, n_in, h, n_out)):
        assert np.abs(gb - rb).max() <= 1e-2 * np.abs(rb).max() + 1e-12


def test_training_reduces_the_loss(gpu):
    import torch
    n_in, h, n_out, B = 128, 256, 128, 512
    rng = np.random.default_rng(5)
    M = rng.standard_normal((n_in, n_out)) / np.sqrt(n_in)
    X = rng.standard_normal((B, n_in)).astype(np.float32)
    T = (X @ M).astype(np.float32)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    m = gpu.Mlp(n_in, h, n_out, seed=6)
    first = m.train_step(Xd.data_ptr(), Td.data_ptr(), B, 1e-3)
    for _ in range(300):
        last = m.train_step(Xd.data_ptr(), Td.data_ptr(), B, 1e-3)
    assert last < first / 10, (first, last)
