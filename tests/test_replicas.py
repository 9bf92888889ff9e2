"""Several-GPU layer on the CPU: two gloo ranks (world size 2, spawned
processes, rendezvous on 127.0.0.1) run the replica host logic that bench.py
uses under torchrun: the block partition, max/sum over ranks, barriers, and
independent per-rank solves (here on the oracle) whose gathered results equal
one process solving every block."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


PARAMS = {"solver": {"method": "MergedPBiCGStab", "rel_tolerance": 1e-8, "max_iters": 200},
          "preconditioner": {"method": "Jacobi"}}


def _solve_block(blk, nv, n_edge):
    import oracle_py as O
    row, col, val = O.generate_cube(n_edge, n_edge, n_edge)
    n = len(row) - 1
    b = np.random.default_rng(500 + blk).uniform(-1, 1, n * nv)
    s = O.System(nv)
    s.set_params(PARAMS)
    s.add_level(row, col, val)
    s.setup()
    x, st = s.solve(b)
    return x, st["iters"]


def _rank_main(rank, world, port, total_blocks, nv, n_edge, out_dir):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import torch.distributed as dist
    import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    ws, r, local = replicas.dist_env()
    assert (ws, r, local) == (world, rank, rank)
    mine = replicas.rhs_blocks(total_blocks, ws, r)
    replicas.barrier()
    res = {blk: _solve_block(blk, nv, n_edge) for blk in mine}
    iters = sum(it for _, it in res.values())
    tot_iters = replicas.sum_over_ranks(iters)
    worst = replicas.max_over_ranks(float(rank + 1))
    # every rank reports what it solved
    objs = [None] * ws
    dist.all_gather_object(objs, {blk: x.tolist() for blk, (x, _) in res.items()})
    replicas.barrier()
    dist.destroy_process_group()
    if rank == 0:
        merged = {}
        for o in objs:
            merged.update(o)
        np.save(os.path.join(out_dir, "merged.npy"),
                np.array([merged[k] for k in sorted(merged)], dtype=np.float64))
        with open(os.path.join(out_dir, "meta.txt"), "w") as f:
            f.write(f"{sorted(merged)} {tot_iters} {worst}\n")


def test_rhs_blocks_partition():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))
    import replicas
    for total in range(0, 13):
        for world in range(1, 9):
            got = [b for r in range(world) for b in replicas.rhs_blocks(total, world, r)]
            assert got == list(range(total))
            sizes = [len(replicas.rhs_blocks(total, world, r)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.rhs_blocks(4, 2, 2)


def test_assign_systems_balanced():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))
    import numpy as np
    import replicas
    rng = np.random.default_rng(3)
    edges = rng.choice(np.arange(16, 97, 8), 64)
    nvs = rng.choice([1, 4, 16], 64)
    work = (edges.astype(float) ** 3 * nvs).tolist()
    assert replicas.assign_systems(work, 1) == [0] * 64
    for world in (2, 4, 8):
        owner = replicas.assign_systems(work, world)
        assert owner == replicas.assign_systems(work, world)  # deterministic
        assert sorted(set(owner)) == list(range(world))
        load = [sum(w for w, o in zip(work, owner) if o == r) for r in range(world)]
        # greedy largest-first: no rank exceeds the mean by more than the largest system
        assert max(load) <= sum(work) / world + max(work)
    with pytest.raises(ValueError):
        replicas.assign_systems(work, 0)


def test_two_gloo_ranks_solve_their_own_blocks(tmp_path):
    import torch.multiprocessing as mp
    world, total_blocks, nv, n_edge = 2, 3, 2, 8
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, total_blocks, nv, n_edge, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    blocks, tot_iters, worst = open(tmp_path / "meta.txt").read().rsplit(" ", 2)
    assert blocks == "[0, 1, 2]"
    assert float(worst) == 2.0
    merged = np.load(tmp_path / "merged.npy")
    ref_iters = 0
    for blk in range(total_blocks):
        x, it = _solve_block(blk, nv, n_edge)
        ref_iters += it
        assert merged[blk].tobytes() == np.asarray(x, np.float64).tobytes()
    assert float(tot_iters) == ref_iters
