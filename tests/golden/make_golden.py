"""Regenerates tests/golden/oracle_solves.json: the oracle's own results on
fixed seeded inputs, committed so that later changes to the oracle show up.
Run from the repository root: python tests/golden/make_golden.py"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_py as O  # noqa: E402


def config1(nv, seed=0):
    row, col, val = O.generate_cube(32, 32, 32)
    params = {"solver": {"method": "MergedPBiCGStab", "max_iters": 1000,
                         "rel_tolerance": 1e-8, "abs_tolerance": 0},
              "preconditioner": {"method": "Jacobi"}}
    S = O.System(nv)
    S.set_params(params)
    S.add_level(row, col, val)
    S.setup()
    b = np.random.default_rng(seed).uniform(-1, 1, (len(row) - 1) * nv)
    x, st = S.solve(b)
    return dict(params=params, seed=seed, iters=st["iters"], conv=st["conv"].tolist(),
                rel_res=st["rel_res"].tolist(), abs_res=st["abs_res"].tolist())


if __name__ == "__main__":
    out = {"config1_nv1": config1(1)}
    json.dump(out, open(os.path.join(HERE, "oracle_solves.json"), "w"), indent=1)
    print(json.dumps(out, indent=1))
