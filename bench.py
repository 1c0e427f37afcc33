"""Benchmark of the PDLP hot path on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Workload: the synthetic LP with known optimum at scale -- m = 2,000,000
equality rows, n = 5,000,000 columns, 8 nonzeros per column (40M nonzeros,
FP64 values, int32 indices), Ruiz scaling with 10 passes -- solved to 1e-8
relative KKT (the reference's definition).

* One step = one restart chunk of the FP64 solve: restart_every = 40 PDHG
  iterations and the KKT check that ends them (the reference checks once per
  restart_every iterations, pdlp.cpp:229).  The solve is driven chunk by chunk
  through the stepwise C ABI (mc_pdlp_ctx_begin / _iterate / _finish); setup
  (upload, transpose, Ruiz) happens before the warm-up chunks.
* ``value``: PDHG iterations/s over the K timed chunks (CUDA events on the
  engine's stream), model resident in HBM, whole job (sum over ranks / max
  time over ranks).
* ``forms``: each full solve once -- FP64 and FP32 + FP64 refinement, to 1e-8
  and to 1e-4 -- with time to tolerance, iterations and the objective error
  against the generator's analytic optimum.
* ``e2e``: one full FP64 solve to 1e-8 through the public API from pinned HOST
  buffers; the host->device copy of the model and the device->host copy of
  the solution are inside the timed region; value = iterations / wall time.
* ``roofline``: the dominant kernel's algorithmic bytes per launch over its
  mean CUDA-event duration (a profiled 400-iteration solve, events on the
  engine's stream), against the measured HBM copy bandwidth; ``traffic`` from
  the committed ncu summary of the same kernel on the same LP.
* ``cpu_baseline``: the reference's own CPU solve_pdlp (oracle/_ref, built
  from the reference sources) on the same LP, rank 0, one core: setup-only
  and 40-iteration samples, steady iterations/s.
* ``--impl reference``: the reference CPU PDLP alone, same metric, config and
  step (40 iterations, setup excluded).
* ``--workload config2|batch1|batch2``: the precision-stress LP, the 256
  uneven LPs and the 512 node variants (batched; FP32 + refinement with FP64
  beside it); ``--ncu-case``: a short profiled solve for ncu captures.
* ``--workload presolve``: the device presolve of a 5.6M-nonzero canonical
  model (step = one full presolve), against the C restatement and, at the
  reference's 4096-row cap, the reference's own presolve.
* ``--budget-s``: legs that would start after this wall time are skipped, so
  the JSON line is always printed.

N > 1 (torchrun): a single LP does not shard (replicas only), so every rank
solves its own replica; no collective touches the data path.  The batch
workloads shard by LP (nonzero-balanced, weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "markov-zip1_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

METRIC = "time-to-1e-8 KKT & SpMV HBM GB/s: plain FP64 vs FP32+refine+warm-start PDLP"
UNIT = "PDHG iterations/s (solve to 1e-8 relative KKT)"
WORKLOADS = {
    # synthetic LP with known optimum, FP64 values, int32 indices
    "config1": dict(m=2_000_000, n=5_000_000, k=8, seed=1, family="standard",
                    label="synthetic LP m=2M n=5M 8 nnz/col (40M nnz), FP64, Ruiz 10 passes, tolerance 1e-8"),
    # precision stress: |a| log-uniform over six decades, 20% boxed columns
    "config2": dict(m=1_000_000, n=3_000_000, k=10, seed=1, family="precision",
                    label="precision-stress LP m=1M n=3M 10 nnz/col (30M nnz), |a| in [1e-3,1e3], tolerance 1e-8"),
}
WORKLOAD = dict(WORKLOADS["config1"])
TOL = 1e-8


def peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_bytes(kind: str, m: int, n: int, nnz: int, fp: int = 8) -> float:
    """Algorithmic bytes of one launch of a fused kernel (each array touched once).

    primal: col pointers 4(n+1), row indices 4nnz, values fp*nnz, the y gather
            fp*m, reads c, col_norm, lo, hi, x, x_avg (6 fp n), writes x,
            x_bar, x_avg (3 fp n)
    dual:   row pointers 4(m+1), column indices 4nnz, values fp*nnz, the x_bar
            gather fp*n, reads y, y_avg, b_lo, b_hi, row_norm (5 fp m),
            writes y, y_avg (2 fp m)
    """
    if kind == "primal":
        return 4 * (n + 1) + (4 + fp) * nnz + fp * m + 9 * fp * n
    if kind == "dual":
        return 4 * (m + 1) + (4 + fp) * nnz + fp * n + 7 * fp * m
    raise ValueError(kind)


def ncu_traffic(kernel: str):
    """dram bytes per launch from the committed ncu summary, if any."""
    f = ROOT / "profiles" / "traffic_config1.txt"
    if WORKLOAD["label"] != WORKLOADS["config1"]["label"] or not f.exists():
        return None
    for line in f.read_text().splitlines():
        parts = line.split()
        if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
            return float(parts[2])
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"mc_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def init_dist(world: int, backend: str):
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return dist


def max_over_ranks(dist, value: float, device) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value: float, device) -> float:
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def make_model(seed: int):
    from mcpdlp import generators
    w = WORKLOAD
    return generators.random_lp(seed, w["m"], w["n"], w["k"], w["family"])


def cpu_reference_sample(model, warmup_runs: int = 1, timed_runs: int = 1, iters: int = 40) -> dict:
    """The reference CPU solve_pdlp on the same LP: setup-only runs and
    `iters`-iteration runs; steady iterations/s = iters / (T_iters - T_setup)."""
    from oracle import ReferencePdlp, OraclePort
    from mcpdlp import _abi
    if ReferencePdlp.available():
        solver, kind = ReferencePdlp(), "reference"
    else:
        solver, kind = OraclePort(), "port"
    o = _abi.default_options_struct()
    o.primal_tolerance = o.dual_tolerance = o.gap_tolerance = TOL
    # the reference PDLP is single-threaded: pin it to one core for the sample
    saved = os.sched_getaffinity(0) if hasattr(os, "sched_getaffinity") else None
    if saved:
        os.sched_setaffinity(0, {max(saved)})
    try:
        t_setup, t_run, r = _time_cpu_solves(solver, model, o, warmup_runs, timed_runs, iters)
    finally:
        if saved:
            os.sched_setaffinity(0, saved)
    setup = float(np.median(t_setup))
    per_iter = max(1e-9, (float(np.median(t_run)) - setup) / iters)
    return dict(value=1.0 / per_iter, unit=UNIT, cores=1, kind=kind,
                sample=(f"reference solve_pdlp on the same LP ({WORKLOAD['label']}): "
                        f"{len(t_setup)} setup-only solves (max_iterations=0, {setup:.2f} s) and "
                        f"{len(t_run)} solves of {iters} iterations; steady rate = {iters} / "
                        f"(T_{iters} - T_0); one pinned core of {host_cpu()}"),
                setup_s=setup, ms_per_iteration=per_iter * 1e3, last_primal=r.primal_infeasibility)


def host_cpu() -> str:
    model = "unknown CPU"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{model} ({os.cpu_count()} logical cores on the host)"


def _time_cpu_solves(solver, model, o, warmup_runs: int, timed_runs: int, iters: int):
    t_setup = []
    for _ in range(max(1, warmup_runs)):
        o.max_iterations = 0
        t0 = time.perf_counter()
        solver.solve(model, o)
        t_setup.append(time.perf_counter() - t0)
    t_run = []
    for _ in range(max(1, timed_runs)):
        o.max_iterations = iters
        t0 = time.perf_counter()
        r = solver.solve(model, o)
        t_run.append(time.perf_counter() - t0)
    return t_setup, t_run, r


def run_reference_arm(args) -> None:
    world, rank, local = dist_env()
    if rank != 0:
        return
    model = make_model(WORKLOAD["seed"])
    t0 = time.perf_counter()
    sample = cpu_reference_sample(model, warmup_runs=max(1, args.warmup), timed_runs=max(1, args.steps))
    wall = time.perf_counter() - t0
    line = {
        "metric": METRIC, "value": sample["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sample["ms_per_iteration"] * 40,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, known optimum)", "impl": "reference",
        "config": dict(workload=WORKLOAD["label"], m=WORKLOAD["m"], n=WORKLOAD["n"],
                       nnz=WORKLOAD["n"] * WORKLOAD["k"], seed=WORKLOAD["seed"],
                       step="40 PDHG iterations of the reference CPU PDLP (setup excluded)"),
        "cpu_baseline": {k: sample[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": sample["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)


def run_ncu_case(args) -> None:
    """A short profiled solve of the workload (for ncu captures of the hot
    kernels): setup plus `--ncu-iterations` PDHG iterations."""
    import torch
    import mcpdlp
    from mcpdlp import PdlpOptions, Precision
    model = make_model(WORKLOAD["seed"])
    ctx = mcpdlp.Context(0)
    dm = mcpdlp.DeviceModel(model)
    x = torch.empty(model.num_cols, dtype=torch.float64, device="cuda")
    y = torch.empty(model.num_rows, dtype=torch.float64, device="cuda")
    o = PdlpOptions(max_iterations=args.ncu_iterations, profile_kernels=True,
                    precision=Precision.fp32_refine if args.precision == "fp32_refine" else Precision.fp64)
    o.set_tolerance(TOL)
    r = ctx.solve_device(dm, o, x, y)
    print(json.dumps({"ncu_case": args.precision, "iterations": r.iterations,
                      "launches": r.extra["launches_by_kind"]}), flush=True)
    ctx.close()


def batch_models(workload: str, world: int = 1, rank: int = 0):
    """The batch workload's LPs of this rank (weak scaling: N ranks share a
    batch N times the single-GPU batch, sharded by nonzeros; a rank generates
    only the LPs of its shard)."""
    from mcpdlp import generators
    from mcpdlp.parallel import shard_by_nnz
    if workload == "batch1":
        shapes = generators.batch_part1_shapes(1, 256 * world)
        mine = shard_by_nnz([n * k for (_, n, k) in shapes], world)[rank]
        return (generators.batch_part1(1, 256 * world, only=mine),
                "256 uneven LPs per GPU (m~U[100,20000], n~U[2m,4m], k~U{4..12}), batched, tolerance 1e-6", None)
    mine = shard_by_nnz([1] * (512 * world), world)[rank]
    base, models, _ = generators.batch_part2(1, 512 * world, only=mine)
    return (models, "512 node variants per GPU of one LP (m=5000, n=15000, 8 nnz/col), batched, tolerance 1e-6",
            base)


def run_batch_ncu_case(args) -> None:
    """A short batched solve of the batch workload (for ncu captures)."""
    import mcpdlp
    from mcpdlp import PdlpOptions, Precision
    models, _, base = batch_models(args.workload)
    ctx = mcpdlp.Context(0)
    o = PdlpOptions(max_iterations=args.ncu_iterations, profile_kernels=True,
                    precision=Precision.fp32_refine if args.precision == "fp32_refine" else Precision.fp64)
    o.set_tolerance(1e-6)
    if args.shared_matrix and base is not None:
        res = ctx.solve_variants(base, [m_.var_lower for m_ in models], [m_.var_upper for m_ in models], o)
    else:
        res = ctx.solve_batch(models, o)
    print(json.dumps({"ncu_case": args.workload, "precision": args.precision, "shared_matrix": args.shared_matrix,
                      "iterations": max(r.iterations for r in res),
                      "launches": res[0].extra["launches_by_kind"],
                      "kernel_ms": res[0].extra["kernel_ms_by_kind"]}), flush=True)
    ctx.close()


def run_batch_arm(args) -> None:
    """Batched solves (one launch set for many LPs): part1 = 256 uneven LPs
    (m ~ U[100,20000], n ~ U[2m,4m], 4-12 nnz/col), part2 = 512 node variants
    of one LP (m=5000, n=15000, 8 nnz/col) with 1-10 bounds tightened; to 1e-6."""
    import torch
    import mcpdlp
    from mcpdlp import PdlpOptions, generators
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    models, label, base = batch_models(args.workload, world, rank)
    ctx = mcpdlp.Context(local)
    from mcpdlp import Precision

    def timed(precision, solve=None):
        o = PdlpOptions(device=local, precision=precision)
        o.set_tolerance(1e-6)
        solve = solve or (lambda: ctx.solve_batch(models, o))
        for _ in range(args.warmup):
            solve()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = None
        for _ in range(args.steps):
            res = solve()
        return max_over_ranks(dist, time.perf_counter() - t0, dev), res

    # the FP32 + FP64-refinement form is the workload's; plain FP64 beside it
    el, res = timed(Precision.fp32_refine)
    el64, res64 = timed(Precision.fp64)
    lps = sum_over_ranks(dist, float(len(models) * args.steps), dev)
    shared = {}
    if base is not None:
        # the node variants with the matrix read once per iteration for all of them
        lows, ups = [m_.var_lower for m_ in models], [m_.var_upper for m_ in models]
        for form, prec in (("fp64", Precision.fp64), ("fp32_refine", Precision.fp32_refine)):
            ov = PdlpOptions(device=local, precision=prec)
            ov.set_tolerance(1e-6)
            shared[form] = timed(prec, lambda ov=ov: ctx.solve_variants(base, lows, ups, ov))

    def summary(rs):
        st = [r.status.name for r in rs]
        errs = [abs(r.objective - m.info["optimum"]) / abs(m.info["optimum"]) for r, m in zip(rs, models)
                if r.status.name == "optimal" and "optimum" in m.info and args.workload == "batch1"]
        certs = [r.extra["certificate"] for r in rs if r.status.name == "infeasible_or_unbounded"]
        return {"statuses": {k: st.count(k) for k in sorted(set(st))},
                "certificates": {k: certs.count(k) for k in sorted(set(certs))},
                "max_iterations_in_batch": max(r.iterations for r in rs),
                "max_objective_rel_err_vs_analytic": max(errs) if errs else None}

    line = {"metric": "batched PDLP solves to 1e-6 relative KKT", "value": lps / el, "unit": "LPs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded generators)",
            "config": dict(workload=label, lps=len(models), nnz=sum(m.nnz for m in models),
                           form="FP32 PDHG + FP64 residuals/restarts/refinement, packed CSR, CUDA graph"),
            **summary(res),
            "forms": {"fp32_refine": {"LPs_per_s": lps / el, "ms_per_step": el * 1e3 / args.steps},
                      "fp64": {"LPs_per_s": lps / el64, "ms_per_step": el64 * 1e3 / args.steps,
                               **summary(res64)}},
            "gpu_launches": res[0].extra["kernel_launches"] * args.steps}
    for form, (elv, resv) in shared.items():
        packed_el, packed_res = (el64, res64) if form == "fp64" else (el, res)
        agree = sum(1 for a, b in zip(resv, packed_res) if a.status == b.status)
        line["forms"][f"shared_matrix_{form}"] = {
            "LPs_per_s": lps / elv, "ms_per_step": elv * 1e3 / args.steps,
            "speedup_vs_packed_same_form": packed_el / elv, "status_agrees_with_packed": f"{agree}/{len(models)}",
            "engine": "mc_pdlp_ctx_solve_variants: one matrix, variant-minor iterates", **summary(resv)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


PRESOLVE = dict(m=1_000_000, n=1_500_000, k=4, seed=1, chains=64, chain_len=32,
                label="canonical model m=1M n=1.5M ~4 nnz/col (5.6M nnz): 5% singleton rows, 64 staircases "
                      "of 32 rows, 1% empty rows and columns, 0.1% entries below the pivot tolerance")


def run_presolve_arm(args) -> None:
    """Device presolve of a large canonical model (src/presolve/presolve.cpp:20).
    One step = one full presolve (all passes) of the model resident in HBM;
    value = nonzeros presolved per second.  e2e = presolve() from host arrays
    with the reduced model and record stack read back.  A single model does
    not shard: under torchrun every rank presolves its own copy (replicas)."""
    import ctypes as C
    import torch
    import mcpdlp
    from mcpdlp import _abi, _lib, _raise, generators
    from mcpdlp.presolve import CanonicalModel, PresolveOptions, postsolve, presolve
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    w = PRESOLVE
    c = generators.presolve_workload(w["seed"], w["m"], w["n"], k=w["k"], chains=w["chains"],
                                     chain_len=w["chain_len"])
    ctx = mcpdlp.Context(local)
    lib = _lib.engine()
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=dev)
    keep = [torch.from_numpy(a).to(dev) for a in (c.col_start, c.row_index, c.value, c.rhs, c.objective)]
    s = _abi.McCanonicalLp()
    s.num_rows, s.num_cols, s.nnz = c.num_rows, c.num_cols, c.nnz
    s.col_start, s.row_index, s.value, s.rhs, s.objective = (t.data_ptr() for t in keep)
    s.objective_offset = c.objective_offset
    o = PresolveOptions().to_struct()
    torch.cuda.synchronize()

    def device_presolve():
        ptr = C.c_void_p()
        _raise(lib.mc_presolve_run(ctx.handle, C.byref(s), C.byref(o), C.byref(ptr)))
        info = _abi.McPresolveInfo()
        lib.mc_presolve_get_info(ptr, C.byref(info))
        lib.mc_presolve_free(ptr)
        return info

    for _ in range(max(args.warmup, 1)):
        info = device_presolve()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            info = device_presolve()
        e1.record(stream)
        torch.cuda.synchronize()
    clock = clocks.summary()
    el = max_over_ranks(dist, e0.elapsed_time(e1) / 1e3, dev)
    per = el / args.steps
    total_nnz = sum_over_ranks(dist, float(c.nnz * args.steps), dev)
    # e2e: from pinned host arrays, the reduced model and the stack read back
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hc = CanonicalModel(c.num_rows, c.num_cols, pin(c.col_start), pin(c.row_index), pin(c.value), pin(c.rhs),
                        pin(c.objective), c.objective_offset)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = presolve(hc, ctx=ctx)
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0, dev)
    red = g.model
    st = g.stack
    # postsolve of a seeded reduced solution (host arrays in and out)
    rng = np.random.default_rng(7)
    sol = type("ReducedSolution", (), {})()
    sol.primal, sol.dual = rng.uniform(0.0, 2.0, red.num_cols), rng.normal(size=red.num_rows)
    postsolve(st, sol, c, ctx=ctx)
    t0 = time.perf_counter()
    postsolve(st, sol, c, ctx=ctx)
    post_s = time.perf_counter() - t0
    h2d = c.col_start.nbytes + c.row_index.nbytes + c.value.nbytes + c.rhs.nbytes + c.objective.nbytes
    d2h = sum(a.nbytes for a in (red.col_start, red.row_index, red.value, red.rhs, red.objective, st.kind, st.index,
                                 st.variable, st.value, st.value2, st.incident_start, st.incident_row,
                                 st.incident_coefficient, st.presolved_to_original_rows,
                                 st.presolved_to_original_cols))
    # matrix sweeps of the run: every pass reads the CSR (empty rows) and the
    # CSC (empty columns); every singleton round reads the CSR rows >= P
    passes = int(info.passes_executed) + (1 if info.passes_executed < PresolveOptions().max_passes else 0)
    sweep = 4 * (c.num_rows + 1) + 13 * c.nnz
    csc_sweep = 4 * (c.num_cols + 1) + 13 * c.nnz
    algo_bytes = passes * (sweep + csc_sweep) + int(info.scan_rounds) * sweep
    hbm, src = peaks()
    line = {"metric": "canonical-model presolve throughput (reference presolve semantics, bit-exact)",
            "value": total_nnz / el, "unit": "nonzeros/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": dict(workload=w["label"], m=c.num_rows, n=c.num_cols, nnz=c.nnz, seed=w["seed"],
                           l2="model (>126 MB with its CSR copy) larger than L2"),
            "presolve": dict(passes_executed=int(info.passes_executed), rounds=int(info.scan_rounds),
                             records=int(info.records), presolved_rows=int(info.presolved_rows),
                             presolved_cols=int(info.presolved_cols), status=int(info.status)),
            "postsolve_e2e_ms": post_s * 1e3,
            "e2e": {"value": c.nnz / e2e_s, "unit": "nonzeros/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "s_per_step": e2e_s},
            "roofline": {"bound": "hbm", "achieved": algo_bytes / per / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": algo_bytes / per / 1e9 / hbm, "traffic": None, "peak_source": src,
                         "note": "all matrix sweeps of one presolve (passes x (CSR + CSC) + rounds x CSR, "
                                 "13 B per nonzero each) over its event time"},
            "clocks": clock}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import OraclePort, presolve_mismatch
        port = OraclePort()
        t0 = time.perf_counter()
        a = port.presolve(c)
        cpu_s = time.perf_counter() - t0
        bad = presolve_mismatch(g, a)
        line["parity_vs_oracle"] = "bit-identical model, stack, maps, statistics" if bad is None else f"MISMATCH: {bad}"
        line["cpu_baseline"] = {"value": c.nnz / cpu_s, "unit": "nonzeros/s", "cores": 1, "kind": "port",
                                "sample": "one full presolve of the same model by the C restatement (the "
                                          "reference caps canonical models at 4096 rows/columns)"}
        # like for like with the reference itself at its size cap
        small = generators.presolve_workload(1, 4096, 4096, k=3, chains=8, chain_len=16)
        from oracle import ReferencePdlp
        if ReferencePdlp.available():
            ref = ReferencePdlp()
            ref.presolve(small)
            t0 = time.perf_counter()
            for _ in range(20):
                ref.presolve(small)
            ref_s = (time.perf_counter() - t0) / 20
            presolve(small, ctx=ctx)
            walls, inside = [], []
            for _ in range(20):
                t0 = time.perf_counter()
                r = presolve(small, ctx=ctx)
                walls.append(time.perf_counter() - t0)
                inside.append(r.extra["presolve_ms"])
                del r
            line["at_reference_cap"] = {"model": "4096 x 4096, 3 nnz/col", "nnz": small.nnz,
                                        "reference_cpu_ms": ref_s * 1e3,
                                        "device_e2e_ms_median": float(np.median(walls)) * 1e3,
                                        "device_e2e_ms_min": float(np.min(walls)) * 1e3,
                                        "device_presolve_call_ms_median": float(np.median(inside)),
                                        "note": "e2e: presolve() from host arrays with the result read back; "
                                                "presolve_call: mc_presolve_run alone"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del keep
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _event_timer(torch, stream):
    """Start/stop CUDA events on the engine's own stream."""
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    return e0, e1


def timed_solve(ctx, torch, stream, dist, dev, fn):
    """One full solve `fn()` bracketed by a barrier and synchronisation; the
    time is the CUDA-event interval on the engine stream (max over ranks)."""
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = _event_timer(torch, stream)
    e0.record(stream)
    t0 = time.perf_counter()
    r = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    el = max(e0.elapsed_time(e1) / 1e3, 0.0)
    return r, max_over_ranks(dist, el, dev), max_over_ranks(dist, wall, dev)


def run_engine_arm(args) -> None:
    import torch
    import mcpdlp
    from mcpdlp import PdlpOptions, Precision

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    t_start = time.perf_counter()

    def over_budget() -> bool:
        # every rank takes the same decision (max over ranks of the elapsed time)
        return max_over_ranks(dist, time.perf_counter() - t_start, dev) > args.budget_s

    model = make_model(WORKLOAD["seed"])
    m, n, nnz = model.num_rows, model.num_cols, model.nnz
    optimum = model.info["optimum"]
    ctx = mcpdlp.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=dev)
    dmodel = mcpdlp.DeviceModel(model, f"cuda:{local}")
    x = torch.empty(n, dtype=torch.float64, device=dev)
    y = torch.empty(m, dtype=torch.float64, device=dev)
    R = 40

    def options(precision=Precision.fp64, tol=TOL, **kw):
        o = PdlpOptions(device=local, precision=precision, **kw)
        o.set_tolerance(tol)
        return o

    # ---- value: steady PDHG iterations/s, one step = one restart chunk
    # (restart_every = 40 iterations and its KKT check) of the FP64 solve to
    # 1e-8, model resident in HBM; setup (transpose, Ruiz) before the timed region
    # clocks are sampled from the warm-up chunks through the first full solve
    # (the timed chunks alone last well under a second)
    clocks = ClockSampler(local).__enter__()
    sess = ctx.begin(dmodel, options())
    for _ in range(args.warmup):
        sess.iterate(1)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = _event_timer(torch, stream)
    e0.record(stream)
    for _ in range(args.steps):
        sess.iterate(1)
    e1.record(stream)
    torch.cuda.synchronize()
    step_s = max(e0.elapsed_time(e1) / 1e3, 1e-9)
    chunks_run = args.warmup + args.steps
    stepped = sess.finish(x, y)
    loop_launches = sum(v for k, v in stepped.extra["launches_by_kind"].items() if k != "setup") - 1
    launches = (loop_launches // max(1, chunks_run)) * args.steps if not sess.finished else None
    t_max = max_over_ranks(dist, step_s, dev)
    value = sum_over_ranks(dist, float(R * args.steps), dev) / t_max

    forms = {}
    clock = None
    # ---- each full solve once: FP64 and FP32 + FP64 refinement, to 1e-8 and 1e-4
    for name, prec, tol in (("fp64", Precision.fp64, TOL), ("fp32_refine", Precision.fp32_refine, TOL),
                            ("fp64_1e-4", Precision.fp64, 1e-4), ("fp32_refine_1e-4", Precision.fp32_refine, 1e-4)):
        if over_budget():
            forms[name] = {"skipped": f"wall budget of {args.budget_s:.0f} s reached"}
            continue
        r, el, wall = timed_solve(ctx, torch, stream, dist, dev, lambda: ctx.solve_device(dmodel, options(prec, tol), x, y))
        forms[name] = {"time_to_tol_s": el, "iterations": r.iterations, "status": r.status.name,
                       "iterations_per_s": r.iterations / el,
                       "objective": r.objective,
                       "objective_rel_err_vs_analytic": abs(r.objective - optimum) / abs(optimum),
                       "kkt": {"primal": r.primal_infeasibility, "dual": r.dual_infeasibility,
                               "gap": r.duality_gap},
                       "setup_and_transfer_ms": r.h2d_ms}
        if name == "fp64":
            clocks.__exit__(None, None, None)
            clock = clocks.summary()
            clock["window"] = "warm-up and timed chunks, then the full FP64 solve to 1e-8"
    if clock is None:
        clocks.__exit__(None, None, None)
        clock = clocks.summary()
    if "time_to_tol_s" in forms.get("fp64", {}) and "time_to_tol_s" in forms.get("fp32_refine", {}):
        forms["speedup_time_to_1e-8_fp32_refine_vs_fp64"] = (forms["fp64"]["time_to_tol_s"]
                                                            / forms["fp32_refine"]["time_to_tol_s"])

    # ---- the learned warm start (FP32 + refinement + GNN start, combined): a network
    # trained on GPU-solved LPs of the same generator at this LP's shape and
    # small sizes (m in [200, 600], n = 2.5m, 8 per column, 1024 seeds), fed
    # to the engine as (a) its predicted initial primal weight with the
    # reference's cold point, and (b) that weight with its predicted dual, the
    # guard on (the engine keeps the cold point if the prediction scores
    # worse); time to 1e-8 includes the prediction
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    hmodel = mcpdlp.Model(m, n, pin(model.col_start), pin(model.row_index), pin(model.value),
                          pin(model.objective), pin(model.var_lower), pin(model.var_upper),
                          pin(model.row_lower), pin(model.row_upper))
    if not args.no_learned and not over_budget():
        from mcpdlp import generators
        from mcpdlp.learn import WarmStartNet, solve_targets
        t0 = time.perf_counter()
        sizes = [generators.uniform_int(sd, 0, 200, 600) for sd in range(1024)]
        fam = [generators.random_lp(sd, mm, (5 * mm) // 2, WORKLOAD["k"]) for sd, mm in enumerate(sizes)]
        to = PdlpOptions(device=local, max_iterations=20000)
        to.set_tolerance(1e-8)
        net = WarmStartNet(local, 3, 0)
        net.fit(solve_targets(ctx, fam, to, margin=0.0), epochs=6, lr=2e-3)
        train_s = time.perf_counter() - t0
        for name, with_dual in (("fp32_refine_learned_weight", False), ("fp32_refine_learned_weight_dual", True)):
            if over_budget():
                forms[name] = {"skipped": f"wall budget of {args.budget_s:.0f} s reached"}
                continue

            # prediction from the host model (wall time, synchronised), then the
            # solve on the device-resident model timed like the plain forms
            torch.cuda.synchronize()
            tp = time.perf_counter()
            _, py, lw = net.predict(hmodel)
            w0 = float(min(max(math.exp(lw), 1e-6), 1e6))
            py_dev = torch.from_numpy(np.ascontiguousarray(py)).to(dev) if with_dual else None
            torch.cuda.synchronize()
            pred_s = max_over_ranks(dist, time.perf_counter() - tp, dev)
            o = options(Precision.fp32_refine, warm_start_guard=with_dual)
            o.initial_primal_weight = w0
            o.initial_dual = py_dev
            r, el, wall = timed_solve(ctx, torch, stream, dist, dev, lambda o=o: ctx.solve_device(dmodel, o, x, y))
            forms[name] = {"time_to_tol_s": pred_s + el, "prediction_s": pred_s, "solve_s": el,
                           "iterations": r.iterations, "status": r.status.name,
                           "objective_rel_err_vs_analytic": abs(r.objective - optimum) / abs(optimum),
                           "warm_start_used": r.extra["warm_start_used"],
                           "initial_primal_weight": w0,
                           "start": ("predicted dual and primal weight, primal from the reference's cold start"
                                     if with_dual else "predicted primal weight, the reference's cold point"),
                           "includes": "prediction (host model, wall) + the solve (events, model resident)",
                           "training_s": train_s, "training": "1024 GPU-solved LPs of the generator at "
                                                               "m in [200,600], n = 2.5m, 8 per column, 6 epochs"}
            if with_dual:
                forms[name]["start_score"] = {"prediction": r.extra["warm_start_score"],
                                              "cold": r.extra["cold_start_score"]}
            if "time_to_tol_s" in forms.get("fp64", {}):
                forms[name]["speedup_time_to_1e-8_vs_fp64"] = (forms["fp64"]["time_to_tol_s"]
                                                               / forms[name]["time_to_tol_s"])

    # ---- e2e: one full FP64 solve to 1e-8 through the public API from pinned
    # host buffers; H2D of the model and D2H of the solution in the timed region
    h2d_bytes = 4 * (n + 1) + 12 * nnz + 8 * 3 * n + 8 * 2 * m
    d2h_bytes = 8 * (n + m)
    e2e = None
    if not over_budget():
        r, el, wall = timed_solve(ctx, torch, stream, dist, dev, lambda: ctx.solve(hmodel, options()))
        e2e = {"value": sum_over_ranks(dist, float(r.iterations), dev) / wall, "unit": UNIT,
               "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
               "s_per_solve": wall, "iterations": r.iterations, "status": r.status.name,
               "objective_rel_err_vs_analytic": abs(r.objective - optimum) / abs(optimum),
               "h2d_ms": r.h2d_ms, "d2h_ms": r.d2h_ms,
               "step": "one full solve to 1e-8 (upload, setup, iterations, download)"}
        last_e2e = r
        # the post-solve check on the device (verify_primal, as the CLI runs it)
        t0 = time.perf_counter()
        vrep = ctx.verify_primal(hmodel, last_e2e.primal, last_e2e.objective, TOL, TOL)
        verify = {"s": time.perf_counter() - t0, "passed": vrep["passed"],
                  "maximum_row_violation": vrep["maximum_row_violation"],
                  "objective_difference": vrep["objective_difference"]}
    else:
        verify = None

    # ---- roofline of the dominant kernel: a profiled 400-iteration solve
    # (CUDA events around every launch, on the engine stream)
    prof = ctx.solve_device(dmodel, options(profile_kernels=True, max_iterations=400), x, y)
    kms = prof.extra["kernel_ms_by_kind"]
    kl = prof.extra["launches_by_kind"]
    per_launch = {k: kms[k] / kl[k] for k in ("primal", "dual") if kl.get(k)}
    dominant = max(("primal", "dual"), key=lambda k: kms.get(k, 0.0))
    algo = kernel_bytes(dominant, m, n, nnz)
    achieved = algo / (per_launch[dominant] / 1e3) / 1e9
    peak, peak_kind = peaks()
    traffic = ncu_traffic(dominant)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": f"k_{dominant}",
                "peak_source": f"hbm_gbs ({peak_kind})", "algorithmic_bytes_per_launch": algo,
                "ms_per_launch": per_launch[dominant],
                "other_kernel": {k: {"ms_per_launch": v, "algorithmic_bytes_per_launch": kernel_bytes(k, m, n, nnz),
                                     "achieved_gbs": kernel_bytes(k, m, n, nnz) / (v / 1e3) / 1e9,
                                     "frac": kernel_bytes(k, m, n, nnz) / (v / 1e3) / 1e9 / peak}
                                 for k, v in per_launch.items() if k != dominant},
                "time_share": {k: kms[k] / max(1e-9, sum(kms.values())) for k in kms if kms[k] > 0}}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, known optimum)",
        "config": dict(workload=WORKLOAD["label"], m=m, n=n, nnz=nnz, seed=WORKLOAD["seed"],
                       step=f"one restart chunk ({R} PDHG iterations and the KKT check) of the FP64 solve "
                            "to 1e-8, model resident in HBM, setup before the timed region",
                       l2="inputs larger than L2 (960 MB of matrix read per iteration)",
                       parallelism=f"replicas x{world}"),
        "clocks": clock,
        "gpu_launches": launches,
        "forms": forms,
        "e2e": e2e,
        "roofline": roofline,
        "verify_primal_device": verify,
        "wall_s": time.perf_counter() - t_start,
    }
    if "time_to_tol_s" in forms.get("fp64", {}):
        f = forms["fp64"]
        line.update(time_to_tol_s=f["time_to_tol_s"], iterations_to_tol=f["iterations"], status=f["status"],
                    objective=f["objective"], objective_rel_err_vs_analytic=f["objective_rel_err_vs_analytic"],
                    kkt=f["kkt"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_reference_sample(model)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line["wall_s"] = time.perf_counter() - t_start
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned warm-start forms")
    ap.add_argument("--budget-s", type=float, default=900.0,
                    help="wall-time budget: legs after it are skipped (the JSON line is still printed)")
    ap.add_argument("--ncu-case", action="store_true",
                    help="run one short profiled solve of the workload (for ncu) and exit")
    ap.add_argument("--ncu-iterations", type=int, default=12)
    ap.add_argument("--shared-matrix", action="store_true",
                    help="with --ncu-case --workload batch2: the variant solve (one matrix) instead of the packed batch")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32_refine"])
    ap.add_argument("--workload", default="config1", choices=["config1", "config2", "batch1", "batch2", "presolve"])
    args = ap.parse_args()
    if args.workload in WORKLOADS:
        WORKLOAD.clear()
        WORKLOAD.update(WORKLOADS[args.workload])
    if args.workload == "presolve":
        run_presolve_arm(args)
    elif args.workload in ("batch1", "batch2"):
        if args.ncu_case:
            run_batch_ncu_case(args)
        else:
            run_batch_arm(args)
    elif args.ncu_case:
        run_ncu_case(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_engine_arm(args)


if __name__ == "__main__":
    main()
