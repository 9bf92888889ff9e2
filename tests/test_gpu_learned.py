"""The learned coarse initial guess end to end on a small matrix (the
benchmark description's configuration 4 at 32^3): training pairs from the
solver, the MLP trained on the GPU (its loss must fall at least tenfold), and
held-out solves from the zero guess and from the learned guess, which is kept
per right-hand side only when its initial residual is below the zero guess's.
Both must converge; the guess must be kept for most right-hand sides, at
least halve the initial residual, and not add iterations."""
import os
import sys

import pytest

pytestmark = pytest.mark.gpu


def test_learned_guess_pipeline(gpu):
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "softx-d-21-00014_b200"))
    import learned
    out = learned.run(n_edge=32, n_train=512, n_eval=64, nv=32, steps=200, level=2, hidden=256,
                      log=lambda *a: None)
    assert out["final_loss"] < out["first_loss"] / 10
    assert out["learned_iters"] <= out["zero_iters"]
    # the smoothed guess of the trained network passes the acceptance test
    # for most held-out right-hand sides and at least halves their initial
    # residual (measured: all kept, 0.20 of the zero guess's residual)
    assert out["guesses_kept"] >= 0.5
    assert out["initial_residual_ratio"] <= 0.5
