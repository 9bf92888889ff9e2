"""CPU restatement of the learned-guess MLP (test infrastructure only: the
checker of softx-d-21-00014_b200/csrc/mlp.cu; nothing in the library uses
it). float64 arithmetic with BF16 rounding at the points where the GPU stores
BF16: the input, the weights, both hidden activations and every backward
activation gradient; the GPU accumulates in FP32, so results agree to FP32
accumulation error plus an occasional BF16 rounding flip."""
import numpy as np


def bf16(a, on=True):
    """Round float64/float32 values to the nearest BF16 (ties to even);
    identity when on is False."""
    if not on:
        return np.asarray(a, np.float64)
    a32 = np.asarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split(params, n_in, h, n_out):
    out, off = [], 0
    for i, o in ((n_in, h), (h, h), (h, n_out)):
        W = params[off:off + o * i].reshape(o, i).astype(np.float64)
        off += o * i
        b = params[off:off + o].astype(np.float64)
        off += o
        out.append((W, b))
    return out


def forward(params, X, n_in, h, n_out, rnd=True):
    (W1, b1), (W2, b2), (W3, b3) = split(params, n_in, h, n_out)
    x = bf16(X, rnd)
    H1 = bf16(np.maximum(x @ bf16(W1, rnd).T + b1, 0.0), rnd)
    H2 = bf16(np.maximum(H1 @ bf16(W2, rnd).T + b2, 0.0), rnd)
    Y = H2 @ bf16(W3, rnd).T + b3
    return x, H1, H2, Y


def gradients(params, X, T, n_in, h, n_out, rnd=True):
    """(flat gradient in the library's parameter order, loss)."""
    (W1, b1), (W2, b2), (W3, b3) = split(params, n_in, h, n_out)
    x, H1, H2, Y = forward(params, X, n_in, h, n_out, rnd)
    B = X.shape[0]
    d = Y - T
    loss = float((d * d).mean())
    dY = bf16(2.0 / (B * n_out) * d, rnd)
    gW3, gb3 = dY.T @ H2, dY.sum(axis=0)
    dH2 = bf16(np.where(H2 > 0, dY @ bf16(W3, rnd), 0.0), rnd)
    gW2, gb2 = dH2.T @ H1, dH2.sum(axis=0)
    dH1 = bf16(np.where(H1 > 0, dH2 @ bf16(W2, rnd), 0.0), rnd)
    gW1, gb1 = dH1.T @ x, dH1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return g, loss
