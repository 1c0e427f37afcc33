"""Batched solves (mc_pdlp_ctx_solve_batch) vs the oracle (needs a B200).

Every LP of a batch runs the reference algorithm on its own, so each result
must match the oracle's solve of that LP alone: same status and objective
within 1e-6 relative at 1e-8 KKT.  Node variants with a crossed bound are
infeasible; the reference runs them to its iteration limit, the batch
certifies them at setup (status infeasible_or_unbounded).
"""
from __future__ import annotations

import numpy as np
import pytest

import mcpdlp
from conftest import options, rel
from mcpdlp import PdlpOptions, PdlpStatus, generators
from test_oracle import synthetic

pytestmark = pytest.mark.gpu


def opts(tol: float, **kw) -> PdlpOptions:
    o = PdlpOptions(**kw)
    o.set_tolerance(tol)
    return o


def test_uneven_batch_matches_solo_solves(gpu_ctx, oracle):
    models = generators.batch_part1(5, count=10, m_range=(100, 600))
    res = gpu_ctx.solve_batch(models, opts(1e-8))
    assert len(res) == len(models)
    for m, r in zip(models, res):
        cpu = oracle.solve(m, options(1e-8))
        assert r.status == cpu.status == PdlpStatus.optimal, m.name
        assert rel(r.objective, cpu.objective) <= 1e-6, m.name
        assert rel(r.objective, m.info["optimum"]) <= 1e-6, m.name
        assert max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap) <= 1e-8
        assert len(r.primal) == m.num_cols and len(r.dual) == m.num_rows


def test_node_variants_status_and_objective(gpu_ctx, oracle):
    base, variants, _ = generators.batch_part2(2, variants=20, m=400, n=1200, k=8)
    res = gpu_ctx.solve_batch(variants, opts(1e-6))
    for v, r in zip(variants, res):
        crossed = bool(np.any(v.var_lower > v.var_upper))
        if crossed:
            assert r.status == PdlpStatus.infeasible_or_unbounded, v.name
            continue
        cpu = oracle.solve(v, options(1e-6, max_iterations=20000))
        assert r.status == cpu.status, v.name
        if cpu.status == PdlpStatus.optimal:
            assert rel(r.objective, cpu.objective) <= 1e-4, v.name


def test_row_activity_certificate(gpu_ctx):
    """x1 + x2 = 5 with 0 <= x <= 2: the row's activity interval [0, 4] misses 5."""
    bad = mcpdlp.from_triplets(1, 2, [0, 0], [0, 1], [1.0, 1.0], objective=[1.0, 1.0],
                               var_lower=[0.0, 0.0], var_upper=[2.0, 2.0], row_lower=[5.0],
                               row_upper=[5.0])
    good = synthetic("small_s7")
    res = gpu_ctx.solve_batch([bad, good], opts(1e-6))
    assert res[0].status == PdlpStatus.infeasible_or_unbounded
    assert res[1].status == PdlpStatus.optimal


def test_batch_of_one_agrees_with_single_solve(gpu_ctx):
    m = synthetic("config0_s1")
    single = gpu_ctx.solve(m, opts(1e-8))
    (b,) = gpu_ctx.solve_batch([m], opts(1e-8))
    assert b.status == single.status == PdlpStatus.optimal
    assert rel(b.objective, single.objective) <= 1e-7


def test_batch_deterministic(gpu_ctx):
    models = generators.batch_part1(6, count=6, m_range=(100, 400))
    a = gpu_ctx.solve_batch(models, opts(1e-8))
    b = gpu_ctx.solve_batch(models, opts(1e-8))
    for x, y in zip(a, b):
        assert x.iterations == y.iterations and x.objective == y.objective
        assert np.array_equal(x.primal, y.primal)


def test_batch_iteration_limit_and_trivial_members(gpu_ctx):
    empty = mcpdlp.Model(0, 2, np.zeros(3, np.int32), np.zeros(0, np.int32), np.zeros(0),
                         np.ones(2), np.zeros(2), np.ones(2), np.zeros(0), np.zeros(0))
    m = synthetic("small_s7")
    res = gpu_ctx.solve_batch([m, empty, m], opts(1e-12, max_iterations=55))
    assert res[0].status == res[2].status == PdlpStatus.iteration_limit
    assert res[0].iterations == res[2].iterations == 55
    assert res[0].objective == res[2].objective
    assert res[1].status == PdlpStatus.optimal and res[1].message == "trivial"


def test_mixed_batch_matches_solo_solves(gpu_ctx, oracle):
    """FP32 + FP64-refinement batch: every LP still reaches 1e-8 relative KKT
    (residuals evaluated in FP64) and agrees with the oracle's solo solve and
    the analytic optimum within 1e-6."""
    from mcpdlp import Precision
    models = generators.batch_part1(7, count=8, m_range=(100, 600))
    res = gpu_ctx.solve_batch(models, opts(1e-8, precision=Precision.fp32_refine))
    for m, r in zip(models, res):
        cpu = oracle.solve(m, options(1e-8))
        assert r.status == cpu.status == PdlpStatus.optimal, m.name
        assert max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap) <= 1e-8
        assert rel(r.objective, cpu.objective) <= 1e-6, m.name
        assert rel(r.objective, m.info["optimum"]) <= 1e-6, m.name
        assert r.extra["refinement_rounds"] == r.extra["restarts"] > 0


def test_mixed_batch_node_variants(gpu_ctx, oracle):
    from mcpdlp import Precision
    base, variants, _ = generators.batch_part2(3, variants=16, m=400, n=1200, k=8)
    res = gpu_ctx.solve_batch(variants, opts(1e-6, precision=Precision.fp32_refine))
    for v, r in zip(variants, res):
        if np.any(v.var_lower > v.var_upper):
            assert r.status == PdlpStatus.infeasible_or_unbounded, v.name
            continue
        cpu = oracle.solve(v, options(1e-6, max_iterations=20000))
        if cpu.status == PdlpStatus.optimal:
            assert r.status == PdlpStatus.optimal, v.name
            assert rel(r.objective, cpu.objective) <= 1e-4, v.name


@pytest.mark.parametrize("lanes", [(1, 1), (2, 8), (32, 32)])
def test_batch_lanes_given_or_tuned_agree(gpu_ctx, lanes):
    """Explicit lanes bypass the autotuner; every lane count runs the same
    algorithm, so statuses agree and objectives within 1e-7."""
    models = generators.batch_part1(8, count=5, m_range=(100, 500))
    tuned = gpu_ctx.solve_batch(models, opts(1e-8))
    fixed = gpu_ctx.solve_batch(models, opts(1e-8, lanes_per_column=lanes[0], lanes_per_row=lanes[1]))
    for a, b in zip(tuned, fixed):
        assert a.status == b.status == PdlpStatus.optimal
        assert rel(a.objective, b.objective) <= 1e-7


def test_work_queue_with_early_finishers(gpu_ctx, oracle):
    """LPs that converge at very different iteration counts, and members
    certified infeasible at setup, leave the work queue while the rest run on;
    the survivors' results are those of their solo solves."""
    bad = mcpdlp.from_triplets(1, 2, [0, 0], [0, 1], [1.0, 1.0], objective=[1.0, 1.0],
                               var_lower=[0.0, 0.0], var_upper=[2.0, 2.0], row_lower=[5.0],
                               row_upper=[5.0])
    slow = generators.transport(4, 30, 40)
    fast = synthetic("small_s7")
    models = [fast, bad, slow, fast]
    res = gpu_ctx.solve_batch(models, opts(1e-8))
    assert res[1].status == PdlpStatus.infeasible_or_unbounded
    for i in (0, 2, 3):
        cpu = oracle.solve(models[i], options(1e-8))
        assert res[i].status == cpu.status
        assert rel(res[i].objective, cpu.objective) <= 1e-6
    assert res[2].iterations > 10 * res[0].iterations
    assert res[0].iterations == res[3].iterations and res[0].objective == res[3].objective


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_batch_warm_start_from_solutions(gpu_ctx, precision):
    """mc_pdlp_ctx_solve_batch_warm: every LP started at its own solution stops
    at the first check (40 iterations) with the same objective; LPs given no
    start (None) run from the cold start as in a plain batch."""
    from mcpdlp import Precision
    models = generators.batch_part1(9, count=6, m_range=(100, 500))
    o = opts(1e-8, precision=Precision[precision])
    cold = gpu_ctx.solve_batch(models, o)
    xs = [r.primal if b % 3 else None for b, r in enumerate(cold)]
    ys = [r.dual if b % 3 else None for b, r in enumerate(cold)]
    warm = gpu_ctx.solve_batch(models, o, initial_primal=xs, initial_dual=ys)
    for b, (c, w) in enumerate(zip(cold, warm)):
        assert c.status == w.status == PdlpStatus.optimal
        if b % 3:
            assert w.iterations == 40, (b, w.iterations)
            assert rel(w.objective, c.objective) <= 1e-7
        else:
            assert w.iterations == c.iterations and w.objective == c.objective


def test_batch_maximize_and_offset_members(gpu_ctx, oracle):
    """Per-LP objective sense and offset in one batch: each member follows its
    own solve (a maximisation LP stops at the iteration limit, as the reference
    does: its gap mixes the maximisation objective with a minimisation-sign
    dual objective, src/lp/first_order/pdlp.cpp:113-131)."""
    mx = generators.random_lp(31, 120, 360, 5)
    mx.objective_sense, mx.objective_offset = 1, 7.5
    mn = generators.random_lp(32, 150, 450, 5)
    mn.objective_offset = -2.25
    o = opts(1e-8, max_iterations=2000)
    res = gpu_ctx.solve_batch([mx, mn], o)
    for model, r in zip((mx, mn), res):
        single = gpu_ctx.solve(model, o)
        cpu = oracle.solve(model, options(1e-8, max_iterations=2000))
        assert r.status == single.status == cpu.status
        assert rel(r.objective, cpu.objective) <= 1e-6
    assert res[0].status == PdlpStatus.iteration_limit
    assert res[1].status == PdlpStatus.optimal
    assert rel(res[1].objective, mn.info["optimum"] + mn.objective_offset) <= 1e-6
