"""Variants of one LP solved together (mc_pdlp_ctx_solve_variants; needs a B200).

The variants differ only in their variable bounds -- the node LPs of one
branching round (bounds tightened as src/milp/milp_solver.cpp:401-447 does).
Every variant runs the reference algorithm (src/lp/first_order/pdlp.cpp:
139-276) on its own LP, so each result must match the oracle's solve of that
LP alone (same status; objective within 1e-6 relative at 1e-8 KKT) and the
packed batch's result; infeasible variants carry certificates that the CPU
checker (oracle/certificates.py) accepts.
"""
from __future__ import annotations

import numpy as np
import pytest

from certificates import check_certificate
from conftest import options, rel
from mcpdlp import PdlpOptions, PdlpStatus, Precision, generators

pytestmark = pytest.mark.gpu


def opts(tol: float, **kw) -> PdlpOptions:
    o = PdlpOptions(**kw)
    o.set_tolerance(tol)
    return o


def node_round(seed: int, count: int, m=300, n=900):
    base, variants, _ = generators.batch_part2(seed, variants=count, m=m, n=n, k=8)
    return base, variants


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
def test_variants_match_solo_solves_and_the_batch(gpu_ctx, oracle, precision):
    base, variants = node_round(3, 37)   # not a multiple of 32: a partly filled warp
    res = gpu_ctx.solve_variants(base, [v.var_lower for v in variants], [v.var_upper for v in variants],
                                 opts(1e-8, precision=precision))
    batch = gpu_ctx.solve_batch(variants, opts(1e-8, precision=precision))
    assert len(res) == len(variants)
    optimal = 0
    for v, r, b in zip(variants, res, batch):
        assert r.status == b.status, v.name
        if r.status == PdlpStatus.infeasible_or_unbounded:
            assert check_certificate(v, r.extra["certificate"], r.extra["certificate_index"], r.dual)
            continue
        cpu = oracle.solve(v, options(1e-8))
        assert r.status == cpu.status, (v.name, r.status, cpu.status)
        if cpu.status == PdlpStatus.optimal:
            optimal += 1
            assert max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap) <= 1e-8
            assert rel(r.objective, cpu.objective) <= 1e-6, v.name
            assert rel(r.objective, b.objective) <= 1e-6, v.name
            assert len(r.primal) == v.num_cols and len(r.dual) == v.num_rows
            assert np.all(r.primal >= v.var_lower - 1e-9) and np.all(r.primal <= v.var_upper + 1e-9)
    assert optimal > 0


def test_base_bounds_variant_is_the_base_lp(gpu_ctx, oracle):
    base, variants = node_round(4, 5)
    lows = [None] + [v.var_lower for v in variants]
    ups = [None] + [v.var_upper for v in variants]
    res = gpu_ctx.solve_variants(base, lows, ups, opts(1e-8))
    single = gpu_ctx.solve(base, opts(1e-8))
    cpu = oracle.solve(base, options(1e-8))
    assert res[0].status == single.status == cpu.status == PdlpStatus.optimal
    assert rel(res[0].objective, cpu.objective) <= 1e-6
    assert rel(res[0].objective, base.info["optimum"]) <= 1e-6


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
def test_variants_deterministic_and_warm_started(gpu_ctx, precision):
    base, variants = node_round(5, 12)
    lows, ups = [v.var_lower for v in variants], [v.var_upper for v in variants]
    a = gpu_ctx.solve_variants(base, lows, ups, opts(1e-8, precision=precision))
    b = gpu_ctx.solve_variants(base, lows, ups, opts(1e-8, precision=precision))
    for x, y in zip(a, b):
        assert x.status == y.status and x.iterations == y.iterations and x.objective == y.objective
        assert np.array_equal(x.primal, y.primal) and np.array_equal(x.dual, y.dual)
    starts_x = [r.primal if r.status == PdlpStatus.optimal else None for r in a]
    starts_y = [r.dual if r.status == PdlpStatus.optimal else None for r in a]
    w = gpu_ctx.solve_variants(base, lows, ups, opts(1e-8, precision=precision), initial_primal=starts_x,
                               initial_dual=starts_y)
    for cold, warm in zip(a, w):
        assert warm.status == cold.status
        if cold.status == PdlpStatus.optimal:
            assert warm.iterations == 40, warm.iterations
            assert rel(warm.objective, cold.objective) <= 1e-7


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
def test_infeasible_variants_are_certified(gpu_ctx, precision):
    base, variants = node_round(6, 40)
    # and the base with one crossed pair of bounds (column 3 only)
    crossed = base.copy()
    crossed.var_lower = crossed.var_lower.copy()
    crossed.var_lower[3] = crossed.var_upper[3] + 0.5
    vs = variants + [crossed]
    res = gpu_ctx.solve_variants(base, [v.var_lower for v in vs], [v.var_upper for v in vs],
                                 opts(1e-6, precision=precision))
    kinds = set()
    for v, r in zip(vs, res):
        if r.status == PdlpStatus.infeasible_or_unbounded:
            kinds.add(r.extra["certificate"])
            assert check_certificate(v, r.extra["certificate"], r.extra["certificate_index"], r.dual), v.name
        else:
            assert r.extra["certificate"] == "none"
    assert res[-1].extra["certificate"] == "crossed_bounds" and res[-1].extra["certificate_index"] == 3


def test_variants_bad_arrays_rejected(gpu_ctx):
    base, variants = node_round(7, 2)
    with pytest.raises(ValueError):
        gpu_ctx.solve_variants(base, [variants[0].var_lower[:-1]], [variants[0].var_upper], opts(1e-6))
