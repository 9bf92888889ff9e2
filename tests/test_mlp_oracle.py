"""The CPU restatement of the learned-guess MLP (oracle/mlp_oracle.py): its
back-propagated gradients must match central finite differences of its own
loss (with BF16 rounding switched off), and its BF16 rounding must agree with
torch's."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                "oracle"))
import mlp_oracle as MO  # noqa: E402


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n_in, h, n_out, B = 6, 5, 4, 7
    n = h * n_in + h + h * h + h + n_out * h + n_out
    p = rng.standard_normal(n) * 0.5
    X = rng.standard_normal((B, n_in))
    T = rng.standard_normal((B, n_out))
    g, _ = MO.gradients(p, X, T, n_in, h, n_out, rnd=False)
    eps = 1e-6
    for i in rng.choice(n, 40, replace=False):
        q = p.copy()
        q[i] += eps
        lp = MO.gradients(q, X, T, n_in, h, n_out, rnd=False)[1]
        q[i] -= 2 * eps
        lm = MO.gradients(q, X, T, n_in, h, n_out, rnd=False)[1]
        assert abs((lp - lm) / (2 * eps) - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(1).standard_normal(10000) * 10.0 ** np.random.default_rng(2).integers(-5, 5, 10000)
    want = torch.from_numpy(x.astype(np.float32)).to(torch.bfloat16).double().numpy()
    assert np.array_equal(MO.bf16(x), want)
