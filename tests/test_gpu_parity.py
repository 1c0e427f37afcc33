"""GPU PDLP vs the oracle and the reference's golden vectors (needs a B200).

Parity bar (floating point): same termination status as the reference CPU
PDLP, and at 1e-8 relative KKT the objective within 1e-6 relative of the
reference's; the GPU's own reported residuals meet the tolerance.  At 1e-4
the objective is compared at the tolerance's scale (1e-3 relative).
Iteration counts are recorded but need not match: the SpMV summation order
differs from the reference's sequential CSC loop.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

import mcpdlp
from conftest import options, rel
from mcpdlp import PdlpOptions, PdlpStatus, generators
from test_oracle import GOLDEN, load_model, synthetic

pytestmark = pytest.mark.gpu

OBJ_TOL = {"0.0001": 1e-3, "1e-08": 1e-6}


def gpu_opts(tol: float, **kw) -> PdlpOptions:
    o = PdlpOptions(**kw)
    o.set_tolerance(tol)
    return o


def check_against(res, gold: dict, tol_key: str) -> None:
    tol = float(tol_key)
    assert res.status == gold["status"]
    if res.status == PdlpStatus.optimal:
        assert res.primal_infeasibility <= tol
        assert res.dual_infeasibility <= tol
        assert res.duality_gap <= tol
    assert rel(res.objective, gold["objective"]) <= OBJ_TOL[tol_key], (res.objective, gold["objective"])
    assert res.backend_actually_used == "cuda"


@pytest.mark.parametrize("name", list(GOLDEN["models"]))
@pytest.mark.parametrize("tol", ["0.0001", "1e-08"])
def test_golden_models(gpu_ctx, name, tol):
    m = load_model(name)
    res = gpu_ctx.solve(m, gpu_opts(float(tol)))
    gold = GOLDEN["models"][name]["results"][tol]
    check_against(res, gold, tol)


@pytest.mark.parametrize("name", list(GOLDEN["synthetic"]))
@pytest.mark.parametrize("tol", ["0.0001", "1e-08"])
def test_golden_synthetic(gpu_ctx, name, tol):
    m = synthetic(name)
    res = gpu_ctx.solve(m, gpu_opts(float(tol)))
    check_against(res, GOLDEN["synthetic"][name]["results"][tol], tol)
    if tol == "1e-08":
        # error against the analytic FP64 optimum c.x* = b.y*
        assert rel(res.objective, m.info["optimum"]) < 1e-6


@pytest.mark.parametrize("seed", range(4, 10))
def test_config0_seeds_vs_oracle(gpu_ctx, oracle, seed):
    m = generators.random_lp(seed, 1000, 3000, 6)
    for tol in (1e-4, 1e-8):
        cpu = oracle.solve(m, options(tol))
        res = gpu_ctx.solve(m, gpu_opts(tol))
        assert res.status == cpu.status
        assert rel(res.objective, cpu.objective) <= (1e-6 if tol == 1e-8 else 1e-3)


def test_first_check_tracks_oracle_closely(gpu_ctx, oracle):
    """Over one restart chunk the trajectories agree to rounding level."""
    m = synthetic("config0_s1")
    cpu = oracle.solve(m, options(1e-12, max_iterations=40), trace_capacity=4)
    res = gpu_ctx.solve(m, gpu_opts(1e-12, max_iterations=40), trace_capacity=4)
    assert res.iterations == cpu.iterations == 40
    assert res.trace["iteration"].tolist() == cpu.trace["iteration"].tolist()
    np.testing.assert_allclose(res.trace["primal_infeasibility"], cpu.trace["primal_infeasibility"], rtol=1e-9)
    np.testing.assert_allclose(res.trace["dual_infeasibility"], cpu.trace["dual_infeasibility"], rtol=1e-9)
    np.testing.assert_allclose(res.trace["step_size"], cpu.trace["step_size"], rtol=1e-12)
    np.testing.assert_allclose(res.primal, cpu.primal, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(res.dual, cpu.dual, rtol=1e-9, atol=1e-12)


OPTION_SETS = [
    dict(restart_strategy=mcpdlp.RestartStrategy.none),
    dict(restart_strategy=mcpdlp.RestartStrategy.fixed),
    dict(adaptive_step_size=False),
    dict(adaptive_primal_weight=False),
    dict(ruiz_scaling=False),
    dict(restart_every=7),
    dict(initial_primal_weight=3.0, step_size_reduction=0.5),
]


@pytest.mark.parametrize("kw", OPTION_SETS, ids=lambda d: ",".join(f"{k}={int(v) if isinstance(v, bool) else v}" for k, v in d.items()))
def test_option_variants_vs_oracle(gpu_ctx, oracle, kw):
    from test_oracle import random_small_lp
    for seed in range(4):
        m = random_small_lp(seed)
        okw = {k: int(v) for k, v in kw.items()}
        cpu = oracle.solve(m, options(1e-8, max_iterations=20000, **okw))
        res = gpu_ctx.solve(m, gpu_opts(1e-8, max_iterations=20000, **kw))
        assert res.status == cpu.status, (seed, kw)
        if cpu.status == 0:
            assert rel(res.objective, cpu.objective) <= 1e-6, (seed, kw)


@pytest.mark.parametrize("max_iterations", [0, 1, 39, 40, 55, 81])
def test_iteration_limit_edges(gpu_ctx, oracle, max_iterations):
    """Partial final chunk and the zero-iteration evaluation (pdlp.cpp:263-275)."""
    m = synthetic("small_s7")
    cpu = oracle.solve(m, options(1e-12, max_iterations=max_iterations))
    res = gpu_ctx.solve(m, gpu_opts(1e-12, max_iterations=max_iterations))
    assert res.status == cpu.status == PdlpStatus.iteration_limit
    assert res.iterations == cpu.iterations == max_iterations
    assert rel(res.objective, cpu.objective) <= 1e-9
    np.testing.assert_allclose(res.primal_infeasibility, cpu.primal_infeasibility, rtol=1e-7, atol=1e-15)


def test_trivial_models(gpu_ctx):
    """pdlp.cpp:144-149: m == 0 or n == 0 is optimal with empty vectors."""
    empty = mcpdlp.Model(0, 3, np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0),
                         np.ones(3), np.zeros(3), np.ones(3), np.zeros(0), np.zeros(0))
    r = gpu_ctx.solve(empty)
    assert r.status == PdlpStatus.optimal and r.message == "trivial" and r.iterations == 0


def test_empty_rows_and_columns(gpu_ctx, oracle):
    m = mcpdlp.from_triplets(4, 5, [0, 0, 2], [0, 1, 1], [1.0, 2.0, -1.0],
                             objective=[1.0, 1.0, 0.0, -1.0, 0.0],
                             var_lower=[0, 0, 0, 0, -np.inf], var_upper=[4, 4, 1, 2, np.inf],
                             row_lower=[1.0, -np.inf, -3.0, -np.inf], row_upper=[np.inf, 5, 3, np.inf])
    cpu = oracle.solve(m, options(1e-8))
    res = gpu_ctx.solve(m, gpu_opts(1e-8))
    assert res.status == cpu.status
    assert rel(res.objective, cpu.objective) <= 1e-6


def test_maximize_with_offset(gpu_ctx, oracle):
    """Maximise + offset.  The reference's duality gap adds the raw (maximise)
    objective to a minimisation-sign dual objective (pdlp.cpp:113-131), so a
    maximise LP with a nonzero optimum never meets the gap test and ends at
    the iteration limit; the engine reproduces that status and the iterate."""
    m = synthetic("small_s7")
    m.objective = -m.objective
    m.objective_sense = mcpdlp.ObjectiveSense.maximize
    m.objective_offset = 12.5
    cpu = oracle.solve(m, options(1e-8, max_iterations=4000))
    res = gpu_ctx.solve(m, gpu_opts(1e-8, max_iterations=4000))
    assert res.status == cpu.status == PdlpStatus.iteration_limit
    assert res.iterations == cpu.iterations == 4000
    assert rel(res.objective, cpu.objective) <= 1e-6
    assert rel(res.duality_gap, cpu.duality_gap) <= 1e-6


def test_deterministic(gpu_ctx):
    m = synthetic("config0_s2")
    a = gpu_ctx.solve(m, gpu_opts(1e-8))
    b = gpu_ctx.solve(m, gpu_opts(1e-8))
    assert a.iterations == b.iterations and a.objective == b.objective
    assert np.array_equal(a.primal, b.primal) and np.array_equal(a.dual, b.dual)


def test_warm_start_from_solution(gpu_ctx, oracle):
    m = synthetic("config0_s1")
    cpu = oracle.solve(m, options(1e-8))
    o = gpu_opts(1e-8)
    o.initial_primal, o.initial_dual = cpu.primal, cpu.dual
    res = gpu_ctx.solve(m, o)
    assert res.status == PdlpStatus.optimal
    assert res.iterations == 40
    assert rel(res.objective, cpu.objective) <= 1e-8


def test_device_resident_input_matches_host(gpu_ctx):
    import torch
    m = synthetic("config0_s3")
    host = gpu_ctx.solve(m, gpu_opts(1e-8))
    dm = mcpdlp.DeviceModel(m)
    x = torch.zeros(m.num_cols, dtype=torch.float64, device="cuda")
    y = torch.zeros(m.num_rows, dtype=torch.float64, device="cuda")
    dev = gpu_ctx.solve_device(dm, gpu_opts(1e-8), x, y)
    assert dev.iterations == host.iterations and dev.objective == host.objective
    assert np.array_equal(x.cpu().numpy(), host.primal)
    assert np.array_equal(y.cpu().numpy(), host.dual)


def test_device_resident_warm_start_matches_host(gpu_ctx):
    """A device model takes device starting points; the result equals the
    host solve from the same points (and host arrays are refused)."""
    import dataclasses
    import torch
    m = synthetic("config0_s3")
    cold = gpu_ctx.solve(m, gpu_opts(1e-8))
    x0, y0 = 0.9 * cold.primal, 0.9 * cold.dual
    ho = gpu_opts(1e-8)
    ho.initial_primal, ho.initial_dual = x0, y0
    host = gpu_ctx.solve(m, ho)
    dm = mcpdlp.DeviceModel(m)
    do = dataclasses.replace(ho, initial_primal=torch.from_numpy(x0).cuda(), initial_dual=torch.from_numpy(y0).cuda())
    x = torch.zeros(m.num_cols, dtype=torch.float64, device="cuda")
    y = torch.zeros(m.num_rows, dtype=torch.float64, device="cuda")
    dev = gpu_ctx.solve_device(dm, do, x, y)
    assert dev.iterations == host.iterations and dev.objective == host.objective
    assert np.array_equal(y.cpu().numpy(), host.dual)
    with pytest.raises(ValueError):
        gpu_ctx.solve_device(dm, ho)


def test_nonfinite_objective_is_numerical_failure(gpu_ctx):
    """NaN data ends as numerical_failure (the reference would run on to its
    iteration limit on NaNs; the engine stops at the next check)."""
    m = synthetic("small_s7")
    m.objective[3] = np.nan
    res = gpu_ctx.solve(m, gpu_opts(1e-8, max_iterations=400))
    assert res.status == PdlpStatus.numerical_failure
    assert res.iterations == 40


def test_invalid_matrix_is_rejected_before_use(gpu_ctx):
    import torch
    m = synthetic("small_s7")
    dm = mcpdlp.DeviceModel(m)
    dm.row_index[5] = m.num_rows + 7      # out of range: caught by device validation
    with pytest.raises(ValueError, match="row index out of range"):
        gpu_ctx.solve_device(dm, gpu_opts(1e-6))
    # the context stays usable
    assert gpu_ctx.solve(m, gpu_opts(1e-4)).status == PdlpStatus.optimal
    del torch


def test_allocation_failure_is_reported(gpu_ctx):
    from mcpdlp import _lib
    lib = _lib.engine()
    with mcpdlp.Context(0) as fresh:
        lib.mc_test_inject_alloc_failures(1)
        with pytest.raises(mcpdlp.EngineError, match="out_of_memory"):
            fresh.solve(synthetic("small_s7"), gpu_opts(1e-4))
        lib.mc_test_inject_alloc_failures(0)
        assert fresh.solve(synthetic("small_s7"), gpu_opts(1e-4)).status == PdlpStatus.optimal


def test_profiled_solve_matches_graph_solve(gpu_ctx):
    m = synthetic("config0_s1")
    a = gpu_ctx.solve(m, gpu_opts(1e-8))
    b = gpu_ctx.solve(m, gpu_opts(1e-8, profile_kernels=True))
    assert a.iterations == b.iterations and a.objective == b.objective
    assert b.extra["kernel_ms_by_kind"]["primal"] > 0
    assert a.extra["kernel_launches"] == b.extra["kernel_launches"]


@pytest.mark.parametrize("name", list(GOLDEN["simplex"]))
def test_transport_against_simplex_optimum(gpu_ctx, name):
    """Transportation LPs (no analytic optimum): the reference primal simplex's
    FP64 optimum is the yardstick.  Where the reference PDLP converges at 1e-8,
    the GPU PDLP must too, within 1e-6 of the simplex objective; where the
    reference stalls at its iteration limit, the GPU result is still within
    1e-4 of the optimum and is never claimed optimal away from it."""
    from test_oracle import transport_case
    g = GOLDEN["simplex"][name]
    res = gpu_ctx.solve(transport_case(name), gpu_opts(1e-8))
    if g["pdlp_1e8"]["status"] == 0:
        assert res.status == PdlpStatus.optimal
        assert rel(res.objective, g["objective"]) <= 1e-6
    else:
        assert rel(res.objective, g["objective"]) <= 1e-4
        if res.status == PdlpStatus.optimal:
            assert rel(res.objective, g["objective"]) <= 1e-6


NETLIB_CASES = [(n, "fp64") for n in sorted(GOLDEN["netlib_optimal"])] + [
    (n, "fp32_refine") for n in ("netlib_afiro", "netlib_sc50a", "netlib_sc50b")]


@pytest.mark.parametrize("name,precision", NETLIB_CASES)
def test_netlib_published_optima(gpu_ctx, name, precision):
    """Known answers: the published Netlib optima (the reference's
    scripts/run_netlib.py:19-93) at 1e-8 relative KKT (the mixed form on the
    models its own tests cover)."""
    from mcpdlp import Precision
    res = gpu_ctx.solve(load_model(name), gpu_opts(1e-8, precision=Precision[precision]))
    best = GOLDEN["netlib_optimal"][name]
    assert res.status == PdlpStatus.optimal
    assert abs(res.objective - best) <= 1e-6 * max(1.0, abs(best)), (res.objective, best)
