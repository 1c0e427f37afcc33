"""Device presolve / postsolve against the oracle (needs a B200).

presolve (src/presolve/presolve.cpp:20-217) must give bit-identical reduced
models, record stacks, maps, statistics, statuses and messages to the
oracle's restatement (itself pinned bit-for-bit to the reference by
tests/test_presolve_oracle.py); postsolve (presolve.cpp:219-317) identical
primal values and duals / objective within 1e-12 relative (double-double on
the device where the reference sums in long double).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from mcpdlp import generators
from mcpdlp.presolve import CanonicalModel, PresolveOptions, SolveStatus, postsolve, presolve
from test_presolve_oracle import GOLDEN, canonical_digest, check_against_golden, load_case, reduced_solution, same

pytestmark = pytest.mark.gpu


def post_close(gpu, cpu) -> None:
    assert np.array_equal(gpu.primal, cpu.primal)
    scale = 1.0 + float(np.max(np.abs(cpu.dual), initial=0.0))
    assert np.allclose(gpu.dual, cpu.dual, rtol=1e-12, atol=1e-12 * scale), float(np.max(np.abs(gpu.dual - cpu.dual)))
    assert abs(gpu.objective - cpu.objective) <= 1e-12 * (1.0 + abs(cpu.objective))


class _Sol:
    """A reduced solution (primal, dual), as lp::reference::Result carries it."""

    def __init__(self, x, y):
        self.primal, self.dual = x, y


def run_both(gpu_ctx, oracle, c, opts=None):
    g = presolve(c, opts, ctx=gpu_ctx)
    o = oracle.presolve(c, opts)
    same(g, o)
    if g.status == SolveStatus.optimal:
        rx, ry = reduced_solution(g, 3)
        post_close(postsolve(g.stack, _Sol(rx, ry), c, ctx=gpu_ctx), oracle.postsolve(o, c, rx, ry))
    return g


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_golden_cases(gpu_ctx, oracle, name):
    c = load_case(name)
    g = presolve(c, ctx=gpu_ctx)
    post = None
    if g.status == SolveStatus.optimal:
        rx, ry = reduced_solution(g, GOLDEN[name]["result"]["post"]["seed"])
        post = postsolve(g.stack, _Sol(rx, ry), c, ctx=gpu_ctx)
        post_close(post, oracle.postsolve(oracle.presolve(c), c, rx, ry))
        post = None  # postsolve sums differ from long double in the last bits: compared above
    check_against_golden(g, post, GOLDEN[name]["result"])


def test_reference_unit_answers(gpu_ctx):
    """tests/presolve_test.cpp:30-96 through the device."""
    assert presolve(load_case("canon_empty_row"), ctx=gpu_ctx).status == SolveStatus.infeasible
    assert presolve(load_case("canon_empty_column"), ctx=gpu_ctx).status == SolveStatus.unbounded
    c = load_case("canon_row_singleton")
    res = presolve(c, ctx=gpu_ctx)
    assert res.status == SolveStatus.optimal and res.statistics.row_singletons_removed >= 1
    post = postsolve(res.stack, _Sol(np.zeros(res.model.num_cols), np.zeros(res.model.num_rows)), c, ctx=gpu_ctx)
    assert abs(post.primal[0] - 3.0) < 1e-9 and abs(post.primal[1] - 4.0) < 1e-9
    assert abs(post.objective - 50.0) < 1e-9


@pytest.mark.parametrize("seed", range(16))
@pytest.mark.parametrize("kind", ["feasible", "infeasible_row", "infeasible_singleton", "unbounded"])
def test_generated_models_match_oracle(gpu_ctx, oracle, seed, kind):
    c = generators.presolve_lp(300 + seed, 80 + 17 * seed, 100 + 23 * seed, k=2 + seed % 3,
                               singletons=0.04 + 0.02 * (seed % 5), chains=1 + seed % 4, chain_len=3 + seed % 7,
                               tiny=0.02, kind=kind)
    run_both(gpu_ctx, oracle, c)


@pytest.mark.parametrize("opts", [PresolveOptions(max_passes=0), PresolveOptions(max_passes=1),
                                  PresolveOptions(max_passes=12), PresolveOptions(pivot_tolerance=0.5),
                                  PresolveOptions(feasibility_tolerance=10.0), PresolveOptions(dual_tolerance=2.0)])
def test_options_match_oracle(gpu_ctx, oracle, opts):
    for seed, kind in ((1, "feasible"), (2, "infeasible_singleton"), (3, "unbounded"), (4, "infeasible_row")):
        run_both(gpu_ctx, oracle, generators.presolve_lp(seed, 150, 200, kind=kind), opts)


def test_long_cascades_take_rounds(gpu_ctx, oracle):
    """Staircases of 40 rows: each singleton makes the next row one in the
    same pass (forward) or the next pass (backward); the device walks them in
    rounds and must still match the sequential walk exactly."""
    c = generators.presolve_lp(77, 600, 700, k=2, singletons=0.01, chains=3, chain_len=40, tiny=0.0)
    g = run_both(gpu_ctx, oracle, c, PresolveOptions(max_passes=60))
    assert g.extra["scan_rounds"] > g.statistics.passes_executed + 1
    assert g.statistics.row_singletons_removed >= 3 * 40


def test_large_model_beyond_reference_cap(gpu_ctx, oracle):
    """The reference caps canonical models at 4096 rows and columns
    (src/linalg/sparse_basis.cpp:27-28); the device presolve does not."""
    c = generators.presolve_lp(5, 12000, 16000, k=3, singletons=0.05, chains=4, chain_len=8)
    g = run_both(gpu_ctx, oracle, c)
    assert g.statistics.original_rows > 4096 and g.statistics.presolved_rows < c.num_rows


def test_invalid_models_rejected(gpu_ctx):
    good = generators.presolve_lp(9, 30, 40)
    c = dataclasses.replace(good, value=good.value.copy())
    c.value[0] = 0.0
    with pytest.raises(ValueError):
        presolve(c, ctx=gpu_ctx)
    c = dataclasses.replace(good, rhs=good.rhs.copy())
    c.rhs[3] = np.inf
    with pytest.raises(ValueError):
        presolve(c, ctx=gpu_ctx)
    c = dataclasses.replace(good, row_index=good.row_index.copy())
    j = int(np.argmax(np.diff(good.col_start) >= 2))
    p = good.col_start[j]
    c.row_index[p], c.row_index[p + 1] = c.row_index[p + 1], c.row_index[p]
    with pytest.raises(ValueError):
        presolve(c, ctx=gpu_ctx)
    with pytest.raises(ValueError):
        presolve(dataclasses.replace(good, objective_offset=np.nan), ctx=gpu_ctx)
    # postsolve against a model of another shape
    res = presolve(good, ctx=gpu_ctx)
    with pytest.raises(ValueError):
        postsolve(res.stack, _Sol(np.zeros(1), np.zeros(1)), generators.presolve_lp(9, 31, 40), ctx=gpu_ctx)


def test_empty_models(gpu_ctx, oracle):
    for c in (CanonicalModel(0, 0, [0], [], [], [], []),
              CanonicalModel(3, 0, [0], [], [], [0.0, 0.0, 0.0], []),
              CanonicalModel(0, 2, [0, 0, 0], [], [], [], [1.0, 2.0])):
        run_both(gpu_ctx, oracle, c)


def test_repeatable_and_results_independent(gpu_ctx):
    c = generators.presolve_lp(11, 300, 400)
    a, b = presolve(c, ctx=gpu_ctx), presolve(c, ctx=gpu_ctx)
    same(a, b)
    assert canonical_digest(a.model) == canonical_digest(b.model)
    del b  # freeing one result leaves the other usable
    rx, ry = reduced_solution(a, 1)
    p1 = postsolve(a.stack, _Sol(rx, ry), c, ctx=gpu_ctx)
    p2 = postsolve(a.stack, _Sol(rx, ry), c, ctx=gpu_ctx)
    assert np.array_equal(p1.primal, p2.primal) and np.array_equal(p1.dual, p2.dual)
    assert p1.objective == p2.objective
