"""Mixed-precision form (FP32 iterations, FP64 checks and re-centring) vs the
reference (needs a B200).

The form has no counterpart in the reference; its oracle is the reference's
FP64 CPU PDLP on the same LP.  Bar: same termination status, objective within
1e-6 relative at 1e-8 relative KKT (the reference's KKT, evaluated in FP64),
and the error against the analytic optimum of the synthetic LPs.
"""
from __future__ import annotations

import numpy as np
import pytest

import mcpdlp
from conftest import options, rel
from mcpdlp import PdlpOptions, PdlpStatus, Precision, generators
from test_oracle import GOLDEN, load_model, synthetic

pytestmark = pytest.mark.gpu


def mixed(tol: float, **kw) -> PdlpOptions:
    o = PdlpOptions(precision=Precision.fp32_refine, **kw)
    o.set_tolerance(tol)
    return o


@pytest.mark.parametrize("name", list(GOLDEN["synthetic"]))
def test_synthetic_to_1e8(gpu_ctx, name):
    m = synthetic(name)
    gold = GOLDEN["synthetic"][name]["results"]["1e-08"]
    res = gpu_ctx.solve(m, mixed(1e-8))
    assert res.status == gold["status"] == PdlpStatus.optimal
    assert max(res.primal_infeasibility, res.dual_infeasibility, res.duality_gap) <= 1e-8
    assert rel(res.objective, gold["objective"]) <= 1e-6
    assert rel(res.objective, m.info["optimum"]) <= 1e-6


@pytest.mark.parametrize("name", ["blend_pdlp", "equality_pdlp", "tiny_simplex", "netlib_afiro",
                                  "netlib_sc50a", "netlib_sc50b", "netlib_blend", "netlib_scsd1"])
def test_golden_models_to_1e8(gpu_ctx, name):
    m = load_model(name)
    gold = GOLDEN["models"][name]["results"]["1e-08"]
    res = gpu_ctx.solve(m, mixed(1e-8))
    assert res.status == gold["status"]
    assert rel(res.objective, gold["objective"]) <= 1e-6


@pytest.mark.parametrize("seed", range(4, 8))
def test_config0_seeds(gpu_ctx, oracle, seed):
    m = generators.random_lp(seed, 1000, 3000, 6)
    cpu = oracle.solve(m, options(1e-8))
    res = gpu_ctx.solve(m, mixed(1e-8))
    assert res.status == cpu.status == PdlpStatus.optimal
    assert rel(res.objective, cpu.objective) <= 1e-6
    # same algorithm: the iteration count stays close to the FP64 reference's
    assert res.iterations <= 2 * cpu.iterations + 200


def test_precision_family(gpu_ctx, oracle):
    """|a| over six decades (the precision-stress family, small)."""
    m = synthetic("precision_s1")
    cpu = oracle.solve(m, options(1e-8))
    res = gpu_ctx.solve(m, mixed(1e-8))
    assert res.status == cpu.status
    assert rel(res.objective, cpu.objective) <= 1e-6


def test_deterministic_and_device_input(gpu_ctx):
    import torch
    m = synthetic("config0_s2")
    a = gpu_ctx.solve(m, mixed(1e-8))
    b = gpu_ctx.solve(m, mixed(1e-8))
    assert a.iterations == b.iterations and a.objective == b.objective
    assert np.array_equal(a.primal, b.primal)
    dm = mcpdlp.DeviceModel(m)
    x = torch.zeros(m.num_cols, dtype=torch.float64, device="cuda")
    y = torch.zeros(m.num_rows, dtype=torch.float64, device="cuda")
    d = gpu_ctx.solve_device(dm, mixed(1e-8), x, y)
    assert d.iterations == a.iterations and d.objective == a.objective
    assert np.array_equal(x.cpu().numpy(), a.primal)


@pytest.mark.parametrize("max_iterations", [0, 40, 55])
def test_iteration_limit_edges(gpu_ctx, max_iterations):
    m = synthetic("small_s7")
    res = gpu_ctx.solve(m, mixed(1e-12, max_iterations=max_iterations))
    assert res.status == PdlpStatus.iteration_limit
    assert res.iterations == max_iterations


def test_invalid_lanes_rejected(gpu_ctx):
    with pytest.raises(ValueError, match="power of two"):
        gpu_ctx.solve(synthetic("small_s7"), mixed(1e-6, lanes_per_row=-1))
    with pytest.raises(ValueError, match="power of two"):
        gpu_ctx.solve(synthetic("small_s7"), mixed(1e-6, lanes_per_column=3))
