"""Stepwise solves (mc_pdlp_ctx_begin / _iterate / _finish) on the GPU.

The reference runs the PDHG loop of solve_pdlp in one call
(src/lp/first_order/pdlp.cpp:194-275); the stepwise form drives the same loop
a few restart chunks at a time.  Driven to the end it must give the one-shot
solve's result bit for bit; stopped early it must give what a one-shot solve
with max_iterations at the same point gives.
"""
from __future__ import annotations

import numpy as np
import pytest

import mcpdlp
from mcpdlp import PdlpOptions, PdlpStatus, Precision, generators

pytestmark = pytest.mark.gpu


def opts(tol=1e-8, **kw) -> PdlpOptions:
    o = PdlpOptions(**kw)
    o.set_tolerance(tol)
    return o


def same(a, b) -> None:
    assert a.status == b.status
    assert a.iterations == b.iterations
    assert a.objective == b.objective
    assert a.primal_infeasibility == b.primal_infeasibility
    assert a.dual_infeasibility == b.dual_infeasibility
    assert a.duality_gap == b.duality_gap
    assert np.array_equal(np.asarray(a.primal), np.asarray(b.primal))
    assert np.array_equal(np.asarray(a.dual), np.asarray(b.dual))


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
@pytest.mark.parametrize("chunks", [1, 3, 1 << 30])
def test_stepwise_equals_one_shot(gpu_ctx, precision, chunks):
    m = generators.random_lp(1, 1000, 3000, 6)
    o = opts(precision=precision)
    ref = gpu_ctx.solve(m, o)
    assert ref.status == PdlpStatus.optimal
    s = gpu_ctx.begin(m, o)
    steps = 0
    while not s.finished:
        s.iterate(chunks)
        steps += 1
        assert steps < 10000
    assert s.iterations == ref.iterations
    same(s.finish(), ref)


def test_stepwise_stopped_early_equals_iteration_limit(gpu_ctx):
    m = generators.random_lp(2, 1000, 3000, 6)
    s = gpu_ctx.begin(m, opts())
    it, fin = s.iterate(5)
    assert (it, fin) == (200, False)
    early = s.finish()
    ref = gpu_ctx.solve(m, opts(max_iterations=200))
    assert early.status == PdlpStatus.iteration_limit
    same(early, ref)


def test_stepwise_partial_last_chunk(gpu_ctx):
    # max_iterations not a multiple of restart_every: the last whole chunk ends
    # the loop and finish runs the remaining 17 iterations and the final check
    m = generators.random_lp(3, 500, 1500, 6)
    o = opts(max_iterations=137)
    s = gpu_ctx.begin(m, o)
    while not s.finished:
        s.iterate(1)
    assert s.iterations == 120
    same(s.finish(), gpu_ctx.solve(m, o))


def test_stepwise_with_trace_and_warm_start(gpu_ctx):
    m = generators.random_lp(4, 800, 2400, 6)
    cold = gpu_ctx.solve(m, opts())
    o = opts(warm_start_guard=True)
    o.initial_primal = cold.primal * 0.9
    o.initial_dual = cold.dual * 0.9
    ref = gpu_ctx.solve(m, o, trace_capacity=64)
    s = gpu_ctx.begin(m, o, trace_capacity=64)
    while not s.finished:
        s.iterate(2)
    got = s.finish()
    same(got, ref)
    for k in ref.trace:
        assert np.array_equal(got.trace[k], ref.trace[k])
    assert got.extra["warm_start_used"] == ref.extra["warm_start_used"]


def test_stepwise_device_model(gpu_ctx):
    import torch
    m = generators.random_lp(5, 1000, 3000, 6)
    dm = mcpdlp.DeviceModel(m)
    x0 = torch.empty(m.num_cols, dtype=torch.float64, device="cuda")
    y0 = torch.empty(m.num_rows, dtype=torch.float64, device="cuda")
    ref = gpu_ctx.solve_device(dm, opts(), x0, y0)
    x1 = torch.empty_like(x0)
    y1 = torch.empty_like(y0)
    s = gpu_ctx.begin(dm, opts())
    while not s.finished:
        s.iterate(4)
    got = s.finish(x1, y1)
    assert got.iterations == ref.iterations and got.objective == ref.objective
    assert torch.equal(x0, x1) and torch.equal(y0, y1)


def test_other_call_ends_the_session(gpu_ctx):
    m = generators.random_lp(6, 300, 900, 6)
    s = gpu_ctx.begin(m, opts())
    s.iterate(1)
    gpu_ctx.solve(m, opts(1e-4))            # reuses the context's buffers
    with pytest.raises(ValueError, match="no solve in progress"):
        s.iterate(1)
    with pytest.raises(ValueError, match="no solve in progress"):
        s.finish()


def test_trivial_model_stepwise(gpu_ctx):
    m = mcpdlp.from_triplets(0, 2, [], [], [], objective=[1.0, 2.0], var_lower=[0.0, 0.0],
                             var_upper=[1.0, 1.0], row_lower=[], row_upper=[])
    s = gpu_ctx.begin(m, opts())
    assert s.iterate(3) == (0, True)
    r = s.finish()
    assert r.status == PdlpStatus.optimal and r.message == "trivial"
