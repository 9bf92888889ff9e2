"""Benchmark of the B200 solve phase: ms per right-hand side to a 1e-8
relative residual, the chosen (FP32-preconditioner) form against plain FP64
on the same matrix, and the fine-level SpMV as a fraction of HBM bandwidth.

Workload (default): 27-point variable-coefficient diffusion (trilinear finite
elements, per-cell kappa = exp(N(0,1)), seed 0) on a 128^3 node grid
(2,097,152 rows, 55,742,968 nonzeros), nv = 8 right-hand sides uniform in
[-1,1]; PBiCGStab (merged form) preconditioned by an AMG V(1,1) cycle with
Chebyshev degree-2 smoothers (PMIS, strength 0.25, extended+i); relative
tolerance 1e-8. Synthetic inputs stand in for the benchmark matrices.

A step is one solve of the nv-block from x = 0. `value` times K steps with
the right-hand side resident in device memory (CUDA events on the library's
stream); `e2e` times the same solves through the C API with host buffers:
upload b, solve, download x. Under torchrun every rank solves its own
right-hand-side block on its own GPU (weak scaling, no data-path
collective); times are the maximum over ranks.

--impl reference times the reference's own solve phase (XAMG's C API built
from the reference sources into oracle/_ref with single-process stand-ins for
MPI, argsparser and hypre: one rank, one core) on the same workload, alone in
its process: inputs and hierarchy from oracle/liboracle_setup.so, then whole
solves to the tolerance, one per step. The reference's MPI+shm parallel build
cannot run here (no MPI); cpu_baseline of the GPU arm times the oracle port
on all host threads beside it.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "softx-d-21-00014_b200"))

WORKLOADS = {
    "amg27": dict(desc="27-pt var-kappa Q1 FE 128^3, nv=8, PBiCGStab + AMG V(1,1) Chebyshev-2",
                  stencil=27, grid=128, sigma=1.0, aniso=1.0, nv=8, smoother="Chebyshev",
                  order=2, bf16_levels=2),
    "poisson32": dict(desc="7-pt Poisson 32^3 (cube.inl), nv=1, MergedPBiCGStab + Jacobi",
                      stencil=0, grid=32, sigma=0.0, aniso=1.0, nv=1, smoother=None, order=0),
    "aniso192": dict(desc="27-pt var-kappa Q1 FE 192^3, kappa=exp(N(0,4)), 4:1 z-anisotropy, nv=32, "
                          "PBiCGStab + AMG V(2,2) Chebyshev-3",
                     stencil=27, grid=192, sigma=2.0, aniso=4.0, nv=32, smoother="Chebyshev",
                     order=3, sweeps=2),
    "batch64": dict(desc="64 uneven 7-pt var-kappa systems, edge in {16,24,...,96}, "
                         "kappa=exp(N(0,1.5^2)), nv in {1,4,16}, PBiCGStab + AMG V(1,1) HSGS "
                         "FP32, batch solve vs one solve per call",
                    stencil=7, grid=96, sigma=1.5, aniso=1.0, nv=0, smoother="HSGS", order=0,
                    systems=64),
    "learned96": dict(desc="7-pt var-kappa 96^3, nv=32, learned coarse guess vs zero guess "
                           "(4096 training, 1024 held-out Gaussian-source RHS)",
                      stencil=7, grid=96, sigma=1.0, aniso=1.0, nv=32, smoother="Chebyshev",
                      order=2),
}


def params_for(w, reduced):
    if w["smoother"] is None:
        return {"solver": {"method": "MergedPBiCGStab", "max_iters": 1000,
                           "rel_tolerance": 1e-8, "abs_tolerance": 0},
                "preconditioner": {"method": "Jacobi"}}
    sm = {"method": w["smoother"], "polynomial_order": w["order"]}
    if w.get("sweeps", 1) != 1:
        sm["max_iters"] = w["sweeps"]
    # plain: XAMG's FP64 method with XAMG's index narrowing. chosen: the whole
    # multigrid preconditioner (finest level included) in FP32 with 2-byte
    # column offsets where they fit, and on the workloads where it measured
    # faster the finest levels' matrix values stored in BF16 (bf16_levels);
    # the outer iteration stays FP64. (The grid-stencil copy,
    # gpu_index_compress = 3, measured slower in these solves.)
    prec = {"method": "MultiGrid", "max_iters": 1, "mg_agg_num_levels": 0,
            "mg_strength_threshold": 0.25, "mg_coarsening_type": 8,
            "mg_interpolation_type": 6, "mg_coarse_matrix_size": 500,
            "mg_reduced_precision": 0, "gpu_index_compress": 1}
    solver = {"method": "MergedPBiCGStab", "max_iters": 500, "rel_tolerance": 1e-8,
              "abs_tolerance": 0, "gpu_index_compress": 1}
    if reduced:
        prec.update(gpu_precond_f32=1, gpu_index_compress=2,
                    gpu_level_bf16=w.get("bf16_levels", 0))
        solver.update(gpu_index_compress=2)
    return {"solver": solver, "preconditioner": prec,
            "pre_smoother": sm, "post_smoother": dict(sm),
            "coarse_grid_solver": {"method": "Direct"}}


def make_matrix(X, w):
    g = w["grid"]
    if w["stencil"] == 0:
        return X.generate_cube(g, g, g)
    return X.generate_diffusion(w["stencil"], g, g, g, w["sigma"], w["aniso"], 0)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap,utilization.gpu")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        util = [float(r[7]) for r in self.rows if len(r) > 7 and r[7].isdigit()]
        loaded = [s for s, u in zip(sm, util) if u > 0] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(loaded)) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


from replicas import dist_env, rhs_blocks  # noqa: E402
import replicas  # noqa: E402


def max_over_ranks(v, ws):
    return replicas.max_over_ranks(v) if ws > 1 else v


def barrier(ws):
    if ws > 1:
        replicas.barrier()


def run_ours(args, w):
    import torch
    import xamg_b200 as X
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    X.init(device=local)
    stream = torch.cuda.ExternalStream(X.stream())
    nv = w["nv"]
    t0 = time.time()
    row, col, val = make_matrix(X, w)
    n = len(row) - 1
    M = X.Matrix(row, col, val)
    # weak scaling: one right-hand-side block per rank, seeded by its index
    rng = np.random.default_rng(1000 + rhs_blocks(ws, ws, rank)[0])
    b = rng.uniform(-1, 1, n * nv)
    bv, xv = X.Vector(n, nv), X.Vector(n, nv)
    bv.upload(b)
    xv.set(0.0)
    solvers = {}
    for name, reduced in (("fp64", False), ("chosen", True)):
        if w["smoother"] is None and reduced:
            continue
        if args.solves_only and args.solves_only != name:
            continue
        solvers[name] = X.Solver(M, X.Params(params_for(w, reduced)), xv, bv)
    setup_s = time.time() - t0
    chosen = "chosen" if "chosen" in solvers else "fp64"

    # pinned host buffers for the end-to-end arm
    bh = torch.from_numpy(b).pin_memory()
    xh_pin = torch.empty(n * nv, dtype=torch.float64).pin_memory()

    def timed(S, K, e2e=False):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        barrier(ws)
        torch.cuda.synchronize()
        k0 = X.kernel_launches()
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(K):
                if e2e:
                    X.call("XAMG_vector_upload_d", bh.data_ptr(), n, 0, nv, bv.h)
                xv.set(0.0)
                S.solve()
                if e2e:
                    X.call("XAMG_vector_download_d", xh_pin.data_ptr(), n, 0, nv, xv.h)
            ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
        barrier(ws)
        ms = ev0.elapsed_time(ev1)
        return max_over_ranks(ms, ws), X.kernel_launches() - k0, xh_pin.numpy().copy()

    if args.solves_only:
        # profiling aid: W + K solves of one arm and nothing else
        S = solvers[args.solves_only]
        for _ in range(args.warmup):
            xv.set(0.0)
            S.solve()
        ms, launches, _ = timed(S, args.steps)
        return {"arm": args.solves_only, "ms_per_rhs": ms / (args.steps * nv),
                "iters": S.stats()["iters"], "launches_per_solve": launches / args.steps}

    if args.roofline_only:
        return roofline(X, torch, stream, solvers[chosen], n, nv, args,
                        which=3 if w["smoother"] else 0, reps=args.steps)

    res = {}
    for name, S in solvers.items():
        for _ in range(args.warmup):
            xv.set(0.0)
            S.solve()
        st = S.stats()
        with ClockSampler(local) as cs:
            ms, launches, _ = timed(S, args.steps)
        res[name] = dict(ms=ms, launches=launches, iters=st["iters"], conv=st["conv"].tolist(),
                         rel_res=st["rel_res"].tolist(), clocks=cs.summary(), x=xv.download())
    S = solvers[chosen]
    ms_e2e, _, xh = timed(S, args.steps, e2e=True)
    # true residual of the chosen solve
    import scipy.sparse as sp
    A = sp.csr_matrix((val.copy(), col.copy(), row.copy()), shape=(n, n))
    Xs, Bs = xh.reshape(n, nv), b.reshape(n, nv)
    true_rel = (np.linalg.norm(Bs - A @ Xs, axis=0) / np.linalg.norm(Bs, axis=0)).max()

    # which=3: the multigrid cycle's level-0 operator; a solver without a
    # multigrid hierarchy (Jacobi-preconditioned configuration 1) has only A
    rf = roofline(X, torch, stream, S, n, nv, args, which=3 if w["smoother"] else 0)
    rf64 = roofline(X, torch, stream, S, n, nv, args, which=0)
    # the plain FP64 method's level-0 SpMV (XAMG's narrowing, FP64 values)
    rf_plain = roofline(X, torch, stream, solvers["fp64"], n, nv, args,
                        which=3 if w["smoother"] else 0)

    total_rhs = args.steps * nv * ws
    out = {
        "metric": "ms/RHS to 1e-8 residual: chosen vs plain FP64 on 1 B200; SpMV % of HBM BW",
        "value": res[chosen]["ms"] / total_rhs * ws,
        "unit": "ms/RHS",
        "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res[chosen]["ms"] / args.steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": ("f64 outer / f32 preconditioner" +
                  (f" (bf16 values on the {w['bf16_levels']} finest levels)"
                   if w.get("bf16_levels") else "")) if chosen == "chosen" else "f64",
        "data": "synthetic",
        "config": config_of(w, n, len(col)),
        "iters": {k: v["iters"] for k, v in res.items()},
        "plain_fp64_ms_per_rhs": res["fp64"]["ms"] / total_rhs * ws,
        "chosen_vs_fp64_speedup": res["fp64"]["ms"] / res[chosen]["ms"],
        "true_rel_residual": float(true_rel),
        "e2e": {"value": ms_e2e / total_rhs * ws, "unit": "ms/RHS",
                "h2d_bytes_per_step": n * nv * 8, "d2h_bytes_per_step": n * nv * 8},
        "gpu_launches": int(res[chosen]["launches"]),
        "roofline": rf,
        "roofline_krylov_spmv": rf64,
        "roofline_plain_spmv": rf_plain,
        "clocks": res[chosen]["clocks"],
        "setup_s": setup_s,
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb, errs, oit = cpu_baseline(solvers["fp64"], w, row, col, val, b,
                                     {k: v["x"] for k, v in res.items()})
        out["cpu_baseline"] = cb
        out["rel_err_vs_oracle"] = errs
        out["iters"]["oracle_fp64"] = oit
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out if rank == 0 else None


def roofline(X, torch, stream, S, n, nv, args, which=3, reps=50):
    """The finest level's SpMV y = A x through XAMG_b200_solver_level_spmv on
    the solver's own uploaded matrix, as its solves run it: which=3 the operator the multigrid cycle applies (the
    FP32 copy in the chosen form: the smoother and residual SpMVs, the largest
    share of the solve), which=0 the Krylov level's FP64 matrix. Algorithmic
    bytes per launch: values and narrowed columns once, row pointers, x read
    and y written once (x's reuse across rows is served by the caches)."""
    A0 = S.level_csr(0, which)
    esz = 4 if A0.val_f32 else 8                    # x and y elements
    vsz = {0: 8, 1: 4, 2: 2, 3: 2}[A0.val_f32]       # stored values (2: BF16, 3: FP16)
    vname = {2: ", BF16 values", 3: ", FP16 values"}.get(A0.val_f32, "")
    # a grid-stencil copy (gpu_index_compress = 3) is what the SpMV reads:
    # one value per slot and row, a 4-byte entry mask per row, no columns
    st_pat = S.level_stencil(0, which)[0]
    dt = torch.float32 if A0.val_f32 else torch.float64
    xd = torch.empty(n * nv, dtype=dt, device="cuda").uniform_(-1, 1)
    yd = torch.empty(n * nv, dtype=dt, device="cuda")
    torch.cuda.synchronize()
    for _ in range(3):
        S.level_spmv(0, which, xd.data_ptr(), yd.data_ptr(), nv)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(reps):
            S.level_spmv(0, which, xd.data_ptr(), yd.data_ptr(), nv)
        e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    fname = "float" if esz == 4 else "double"
    if st_pat >= 0:
        slots = 27 if st_pat == 0 else 7
        alg = slots * n * vsz + n * 4 + 2 * n * nv * esz
        kname = f"k_spmv_stencil<{fname}> level 0, EStore, nv={nv}, " \
                f"{slots}-slot grid stencil" + vname
        tkey = f"{args.workload}_n{n}_which{which}_nv{nv}_v{vsz}_st{slots}"
    else:
        alg = A0.nnz * (vsz + abs(A0.col_bytes)) + (n + 1) * 4 + 2 * n * nv * esz
        kname = f"k_spmv<{fname}> level 0, EStore, nv={nv}, " \
                f"col_bytes={A0.col_bytes}" + vname
        tkey = f"{args.workload}_n{n}_which{which}_nv{nv}_v{vsz}"
    achieved = alg / (ms * 1e-3) / 1e9
    peak, peak_kind = peaks()
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "spmv_traffic.json")
    if os.path.exists(tfile):
        t = json.load(open(tfile)).get(tkey)
        if t:
            traffic = t["dram_bytes_per_launch"]
    return {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
            "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": traffic, "algorithmic_bytes": int(alg), "ms_per_launch": ms,
            "launches_timed": reps}


def config_of(w, n, nnz):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": w["desc"], "rows": n, "nnz": int(nnz), "nv": w["nv"],
            "rhs_per_gpu_per_step": w["nv"], "tolerance": 1e-8,
            "l2": "inputs larger than L2 (matrix > 126 MB)" if nnz * 12 > 126e6
            else "L2-resident inputs (no flush)"}


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_py
    return oracle_py


class OracleSolve:
    """The oracle (the restatement of XAMG's FP64 CPU solve phase) set up for
    the plain-FP64 method of workload w on a given hierarchy: full solves from
    x = 0 to the relative tolerance, dot products in XAMG's order over one
    core range per host thread (as XAMG's ranks sum them), every loop on the
    host threads."""

    def __init__(self, w, row, col, val, hierarchy):
        O = oracle_module()
        self.O = O
        self.nv = w["nv"]
        self.sysm = O.System(self.nv)
        self.sysm.set_params(params_for(w, False))
        if hierarchy is None:
            self.sysm.add_level(row, col, val)
        else:
            for lv in hierarchy:
                self.sysm.add_level(*lv["A"], lv["min_eig"], lv["max_eig"])
                if lv["P"] is not None:
                    self.sysm.add_interp(*lv["P"])
        self.sysm.setup()
        self.cores = O.threads()

    def solve(self, b):
        """(x, stats, seconds) of one whole solve."""
        self.O.set_reduction(0, self.cores)
        try:
            t0 = time.perf_counter()
            x, st = self.sysm.solve(b)
            return x, st, time.perf_counter() - t0
        finally:
            self.O.set_reduction(0)


def oracle_inputs(w):
    """Matrix, right-hand side and hierarchy of workload w without the CUDA
    library: the seeded generators and the host multigrid setup compiled into
    oracle/liboracle_setup.so from the library's host-only sources."""
    O = oracle_module()
    g = w["grid"]
    if w["stencil"] == 0:
        row, col, val = O.generate_cube(g, g, g)
    else:
        row, col, val = O.setup_generate_diffusion(w["stencil"], g, g, g, w["sigma"], w["aniso"], 0)
    n = len(row) - 1
    b = np.random.default_rng(1000).uniform(-1, 1, n * w["nv"])
    H = None
    if w["smoother"] is not None:
        H = O.setup_hierarchy(row, col, val, params_for(w, False)["preconditioner"])
    return row, col, val, b, H


def rel_err(x, ref, nv):
    """max over right-hand sides of ||x - ref|| / ||ref||"""
    X, R = x.reshape(-1, nv), ref.reshape(-1, nv)
    return float((np.linalg.norm(X - R, axis=0) / np.linalg.norm(R, axis=0)).max())


def cpu_baseline(S, w, row, col, val, b, xs):
    """One whole plain-FP64 solve of the same system on the oracle (the
    hierarchy the GPU solver built), timed on the host threads; its solution
    gives each GPU result's relative error against the FP64 CPU oracle."""
    arm = OracleSolve(w, row, col, val, S.hierarchy() if w["smoother"] else None)
    x, st, dt = arm.solve(b)
    cb = {"value": dt * 1e3 / w["nv"], "unit": "ms/RHS", "cores": arm.cores, "kind": "port",
          "sample": f"one whole plain-FP64 solve of the same {w['nv']} right-hand sides to 1e-8 "
                    f"({st['iters']} iterations, {dt:.1f} s), XAMG's reduction order over "
                    f"{arm.cores} core ranges"}
    errs = {k: rel_err(v, x, w["nv"]) for k, v in xs.items()}
    return cb, errs, int(st["iters"])


class quiet_stdout:
    """Sends what native code prints to stdout (the reference's log lines)
    to stderr, so that stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def run_reference(args, w):
    """CPU arm, alone in this process (no CUDA library, no GPU): the
    reference's own solve phase, XAMG's C API compiled unmodified from its
    sources into oracle/_ref with single-process stand-ins for MPI,
    argsparser's parameter dictionary and hypre (one rank: one core), on the
    same matrix, right-hand sides and hierarchy (oracle/liboracle_setup.so;
    the hierarchy is registered with the hypre stand-in). Each step is one
    whole plain-FP64 solve of the nv right-hand sides from x = 0 to the
    tolerance; whole solves take tens of seconds at full size, so after
    min(W, 1) warm-up solves it times at most K solves within a time budget
    and reports the number it timed. Without oracle/_ref (no reference
    sources where it was built) the oracle port on all host threads stands
    in (kind "port"). Under torchrun only rank 0 runs it."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ref_capi
    t0 = time.time()
    row, col, val, b, H = oracle_inputs(w)
    n, nv = len(row) - 1, w["nv"]
    use_ref = ref_capi.available(nv)
    with quiet_stdout():
        if use_ref:
            S = ref_capi.Solve(row, col, val, nv, params_for(w, False), hierarchy=H)
            def one():
                x, conv = S.solve(b)
                return x, int(conv.sum()), S.last_seconds
            cores, kind = 1, "reference"
        else:
            arm = OracleSolve(w, row, col, val, H)
            def one():
                x, st, dt = arm.solve(b)
                return x, int(st["conv"].sum()), dt
            cores, kind = arm.cores, "port"
        setup_s = time.time() - t0
        warm = min(args.warmup, 1)
        for _ in range(warm):
            one()
        total, steps, budget = 0.0, 0, 90.0
        while steps < args.steps and (steps == 0 or total < budget):
            x, nconv, dt = one()
            total += dt
            steps += 1
    v = total * 1e3 / (steps * nv)
    import scipy.sparse as sp
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    Xs, Bs = x.reshape(n, nv), b.reshape(n, nv)
    true_rel = (np.linalg.norm(Bs - A @ Xs, axis=0) / np.linalg.norm(Bs, axis=0)).max()
    what = ("XAMG's own solve phase built from the reference sources, one rank"
            if use_ref else "the oracle port, XAMG's reduction order over the host threads")
    cb = {"value": v, "unit": "ms/RHS", "cores": cores, "kind": kind,
          "sample": f"each step one whole plain-FP64 solve of the {nv} right-hand sides to 1e-8 "
                    f"({what}); {steps} steps timed after {warm} warm-up, "
                    f"{nconv}/{nv} right-hand sides converged"}
    return {"impl": "reference",
            "metric": "ms/RHS to 1e-8 residual: chosen vs plain FP64 on 1 B200; SpMV % of HBM BW",
            "value": v, "unit": "ms/RHS", "n_gpus": ws, "steps": steps, "steps_requested": args.steps,
            "warmup": warm, "ms_per_step": total * 1e3 / steps,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(w, n, len(col)),
            "true_rel_residual": float(true_rel), "setup_s": setup_s, "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "ms/RHS", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def batch_params(reduced):
    """Configuration 3's method: merged PBiCGStab with an AMG V(1,1)
    hybrid-Gauss-Seidel preconditioner, FP32 with 2-byte relative columns
    (chosen) or XAMG's FP64 method (plain)."""
    sm = {"method": "HSGS", "max_iters": 1}
    prec = {"method": "MultiGrid", "max_iters": 1, "mg_agg_num_levels": 0,
            "mg_strength_threshold": 0.25, "mg_coarsening_type": 8,
            "mg_interpolation_type": 6, "mg_coarse_matrix_size": 500,
            "mg_reduced_precision": 0, "gpu_index_compress": 1}
    solver = {"method": "MergedPBiCGStab", "max_iters": 500, "rel_tolerance": 1e-8,
              "abs_tolerance": 0, "gpu_index_compress": 1}
    if reduced:
        prec.update(gpu_precond_f32=1, gpu_index_compress=2)
        solver.update(gpu_index_compress=2)
    return {"solver": solver, "preconditioner": prec, "pre_smoother": sm,
            "post_smoother": dict(sm), "coarse_grid_solver": {"method": "Direct"}}


def run_batch(args, w):
    """Configuration 3: the systems solved by one XAMG_b200_solver_solve_batch
    call per step (chosen: FP32 preconditioner, every system on its own
    stream, lockstep iterations) against one XAMG_solver_solve2 call per
    system (the same solvers, and XAMG's plain FP64 method). Synthetic
    systems: edges and nv drawn from a seeded generator. Under torchrun the
    systems are shared out among the ranks (largest first, to the least
    loaded rank; replicas.assign_systems) with no data-path collective: the
    total work is fixed, so the scaling is strong, and every time is the
    maximum over ranks."""
    import torch
    import xamg_b200 as X
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    X.init(device=local)
    stream = torch.cuda.ExternalStream(X.stream())
    rng = np.random.default_rng(3)
    m = w["systems"]
    edges = rng.choice(np.arange(16, 97, 8), m)
    nvs = rng.choice([1, 4, 16], m)
    owner = replicas.assign_systems((edges.astype(float) ** 3 * nvs).tolist(), ws)
    t0 = time.time()
    sysm = []
    for i in range(m):
        e, nv = int(edges[i]), int(nvs[i])
        n = e ** 3
        b = rng.uniform(-1, 1, n * nv)  # drawn on every rank: the same b whatever the split
        if owner[i] != rank:
            continue
        row, col, val = X.generate_diffusion(7, e, e, e, w["sigma"], 1.0, 100 + i)
        M = X.Matrix(row, col, val)
        bv, xv = X.Vector(n, nv), X.Vector(n, nv)
        bv.upload(b)
        xv.set(0.0)
        S = X.Solver(M, X.Params(batch_params(True)), xv, bv)
        P = X.Solver(M, X.Params(batch_params(False)), xv, bv)
        sysm.append(dict(M=M, b=b, bv=bv, xv=xv, S=S, P=P, n=n, nv=nv, edge=e,
                         bh=torch.from_numpy(b).pin_memory(),
                         xh=torch.empty(n * nv, dtype=torch.float64).pin_memory(),
                         row=row, col=col, val=val))
    setup_s = max_over_ranks(time.time() - t0, ws)
    total_rhs = int(nvs.sum())
    Ss = [d["S"] for d in sysm]
    xs = [d["xv"] for d in sysm]
    bs = [d["bv"] for d in sysm]

    def step(kind, e2e=False):
        if e2e:
            for d in sysm:
                X.call("XAMG_vector_upload_d", d["bh"].data_ptr(), d["n"], 0, d["nv"], d["bv"].h)
        for d in sysm:
            d["xv"].set(0.0)
        if kind == "batch":
            X.solve_batch(Ss, xs, bs)
        else:
            for d in sysm:
                (d["S"] if kind == "single" else d["P"]).solve(d["xv"], d["bv"])
        if e2e:
            for d in sysm:
                X.call("XAMG_vector_download_d", d["xh"].data_ptr(), d["n"], 0, d["nv"],
                       d["xv"].h)

    def timed(kind, K, e2e=False):
        for _ in range(args.warmup):
            step(kind)
        barrier(ws)
        torch.cuda.synchronize()
        k0 = X.kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(K):
                step(kind, e2e)
            e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(ws)
        ms = max_over_ranks(e0.elapsed_time(e1) / K, ws)
        launches = replicas.sum_over_ranks((X.kernel_launches() - k0) // K) if ws > 1 \
            else (X.kernel_launches() - k0) // K
        return ms, int(launches)

    with ClockSampler(local) as cs:
        ms_batch, launches = timed("batch", args.steps)
    ms_single, _ = timed("single", args.steps)
    ms_plain, _ = timed("plain", max(1, args.steps // 2))
    ms_e2e, _ = timed("batch", args.steps, e2e=True)
    iters = [int(np.max(d["S"].stats()["iters"])) for d in sysm]
    # true residuals of the batch solve (from the last e2e step's downloads)
    import scipy.sparse as sp
    worst = 0.0
    for d in sysm:
        A = sp.csr_matrix((d["val"].copy(), d["col"].copy(), d["row"].copy()),
                          shape=(d["n"], d["n"]))
        Xs, Bs = d["xh"].numpy().reshape(d["n"], d["nv"]), d["b"].reshape(d["n"], d["nv"])
        worst = max(worst, float((np.linalg.norm(Bs - A @ Xs, axis=0) /
                                  np.linalg.norm(Bs, axis=0)).max()))
    worst = max_over_ranks(worst, ws)
    it_min = -max_over_ranks(-min(iters), ws)
    it_max = max_over_ranks(max(iters), ws)
    big = int(np.argmax([d["n"] * d["nv"] for d in sysm]))
    rf = roofline(X, torch, stream, sysm[big]["S"], sysm[big]["n"], sysm[big]["nv"], args)
    rf["kernel"] += f" (largest system: {sysm[big]['edge']}^3, nv={sysm[big]['nv']})"
    clocks = cs.summary()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return None
    vec_bytes = int(sum(int(e) ** 3 * int(v) * 8 for e, v in zip(edges, nvs)))
    return {
        "metric": "ms/RHS to 1e-8 residual: batch solve vs one solve per call",
        "value": ms_batch / total_rhs, "unit": "ms/RHS", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_batch, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64 outer / f32 preconditioner",
        "data": "synthetic",
        "config": {"workload": w["desc"], "systems": m,
                   "rows": int(sum(int(e) ** 3 for e in edges)),
                   "rhs_per_step": total_rhs, "edges": edges.tolist(), "nv": nvs.tolist(),
                   "systems_per_rank": [owner.count(r) for r in range(ws)],
                   "tolerance": 1e-8, "l2": "inputs larger than L2 (all systems' matrices)"},
        "iters": {"min": int(it_min), "max": int(it_max)},
        "one_call_per_system_ms_per_rhs": ms_single / total_rhs,
        "plain_fp64_ms_per_rhs": ms_plain / total_rhs,
        "batch_vs_one_call_speedup": ms_single / ms_batch,
        "chosen_vs_fp64_speedup": ms_plain / ms_batch,
        "true_rel_residual": worst,
        "e2e": {"value": ms_e2e / total_rhs, "unit": "ms/RHS",
                "h2d_bytes_per_step": vec_bytes, "d2h_bytes_per_step": vec_bytes},
        "gpu_launches": launches, "roofline": rf, "clocks": clocks,
        "setup_s": setup_s,
    }


def run_learned(args, w):
    """The learned coarse initial guess (configuration 4): not the headline
    metric; one JSON line with both guesses' iterations and ms/RHS."""
    import xamg_b200 as X
    import learned
    X.init()
    r = learned.run(n_edge=w["grid"], n_train=4096, n_eval=1024, nv=w["nv"], steps=400,
                    level=3, hidden=1024, log=lambda *a: print(*a, file=sys.stderr))
    return {"metric": "ms/RHS to 1e-8, learned coarse initial guess vs zero guess",
            "value": r["learned_ms_per_rhs"], "unit": "ms/RHS", "n_gpus": 1,
            "higher_is_better": False, "data": "synthetic",
            "config": {"workload": w["desc"]}, "learned": r}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="amg27", choices=sorted(WORKLOADS))
    ap.add_argument("--grid", type=int, default=None, help="override the grid edge")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--solves-only", choices=["fp64", "chosen"], default=None,
                    help="set up one arm, then only its warm-up and timed solves: the command "
                         "to profile that arm's launches")
    ap.add_argument("--roofline-only", action="store_true",
                    help="set up, then time only the level-0 SpMV (--steps launches): "
                         "the command to profile that kernel")
    args = ap.parse_args()
    w = dict(WORKLOADS[args.workload])
    if args.grid:
        w["grid"] = args.grid
        w["desc"] = w["desc"].replace("128^3", f"{args.grid}^3").replace("32^3", f"{args.grid}^3")
    if args.workload == "learned96" and args.impl != "reference":
        out = run_learned(args, w)
    elif args.workload == "batch64" and args.impl != "reference":
        out = run_batch(args, w)
    else:
        out = run_reference(args, w) if args.impl == "reference" else run_ours(args, w)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
