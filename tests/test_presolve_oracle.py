"""The presolve oracle is pinned to the reference (CPU-only tests).

* against the committed golden vectors made by the reference's own presolve
  and postsolve (tests/golden/make_golden.py, ``presolve`` section):
  bit-for-bit equal reduced models, record stacks, maps, statistics, and
  postsolve outputs;
* against the reference library, live, where oracle/_ref is built: seeded
  generated models of every outcome and option setting;
* the reference's own known answers (tests/presolve_test.cpp:30-96).
"""
from __future__ import annotations

import dataclasses
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from mcpdlp import generators
from mcpdlp.presolve import CanonicalModel, PresolveOptions, SolveStatus

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"
GOLDEN = json.loads((GOLDEN_DIR / "golden.json").read_text())["presolve"]


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def canonical_digest(c) -> str:
    return sha(np.array([c.num_rows, c.num_cols]), c.col_start, c.row_index, c.value, c.rhs, c.objective,
               np.array([c.objective_offset]))


def load_case(name: str) -> CanonicalModel:
    g = GOLDEN[name]
    if "file" in g:
        z = np.load(GOLDEN_DIR / g["file"])
        c = CanonicalModel(int(z["num_rows"]), int(z["num_cols"]), z["col_start"], z["row_index"], z["value"],
                           z["rhs"], z["objective"], float(z["objective_offset"]))
    else:
        c = generators.presolve_lp(g["seed"], g["m"], g["n"], kind=g["kind"])
    assert canonical_digest(c) == g["digest"], f"{name}: fixture or generator changed"
    return c


def check_against_golden(res, post, gold: dict) -> None:
    assert int(res.status) == gold["status"]
    assert res.message == gold["message"]
    assert dataclasses.asdict(res.statistics) == gold["statistics"]
    assert res.model.objective_offset == gold["objective_offset"]
    assert canonical_digest(res.model) == gold["model_sha256"]
    st = res.stack
    assert sha(st.kind, st.index, st.variable, st.value, st.value2, st.incident_start, st.incident_row,
               st.incident_coefficient) == gold["stack_sha256"]
    assert sha(st.presolved_to_original_rows, st.presolved_to_original_cols) == gold["maps_sha256"]
    if post is not None:
        assert sha(post.primal) == gold["post"]["primal_sha256"]
        assert sha(post.dual) == gold["post"]["dual_sha256"]
        assert post.objective == gold["post"]["objective"]


def reduced_solution(res, seed: int = 7):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 2.0, res.model.num_cols), rng.normal(size=res.model.num_rows)


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_matches_reference_golden(oracle, name):
    c = load_case(name)
    res = oracle.presolve(c)
    post = None
    if res.status == SolveStatus.optimal:
        rx, ry = reduced_solution(res, GOLDEN[name]["result"]["post"]["seed"])
        post = oracle.postsolve(res, c, rx, ry)
    check_against_golden(res, post, GOLDEN[name]["result"])


def test_reference_unit_answers(oracle):
    """tests/presolve_test.cpp:30-96 through the oracle."""
    assert oracle.presolve(load_case("canon_empty_row")).status == SolveStatus.infeasible
    assert oracle.presolve(load_case("canon_empty_column")).status == SolveStatus.unbounded
    c = load_case("canon_row_singleton")
    res = oracle.presolve(c)
    assert res.status == SolveStatus.optimal and res.statistics.row_singletons_removed >= 1
    post = oracle.postsolve(res, c, np.zeros(res.model.num_cols), np.zeros(res.model.num_rows))
    assert abs(post.primal[0] - 3.0) < 1e-9 and abs(post.primal[1] - 4.0) < 1e-9
    assert abs(post.objective - 50.0) < 1e-9


CASES = [(seed, kind) for seed in range(12) for kind in ("feasible", "infeasible_row", "infeasible_singleton",
                                                          "unbounded")]


def same(a, b) -> None:
    from oracle import presolve_mismatch
    bad = presolve_mismatch(a, b)
    assert bad is None, bad


@pytest.mark.parametrize("seed,kind", CASES)
def test_oracle_matches_reference_live(oracle, reference, seed, kind):
    c = generators.presolve_lp(100 + seed, 60 + 11 * seed, 80 + 13 * seed, k=2 + seed % 3,
                               singletons=0.05 + 0.02 * (seed % 4), chains=1 + seed % 3, chain_len=3 + seed % 5,
                               tiny=0.02, kind=kind)
    a, b = oracle.presolve(c), reference.presolve(c)
    same(a, b)
    if a.status == SolveStatus.optimal:
        rx, ry = reduced_solution(a, seed)
        pa, pb = oracle.postsolve(a, c, rx, ry), reference.postsolve(c, rx, ry)
        assert np.array_equal(pa.primal, pb.primal) and np.array_equal(pa.dual, pb.dual)
        assert pa.objective == pb.objective
        # a shorter reduced solution leaves the missing entries 0 (presolve.cpp:261-272)
        pa, pb = oracle.postsolve(a, c, rx[:-1], ry[:-1]), reference.postsolve(c, rx[:-1], ry[:-1])
        assert np.array_equal(pa.primal, pb.primal) and np.array_equal(pa.dual, pb.dual)


@pytest.mark.parametrize("opts", [PresolveOptions(max_passes=0), PresolveOptions(max_passes=1),
                                  PresolveOptions(pivot_tolerance=0.5), PresolveOptions(feasibility_tolerance=10.0),
                                  PresolveOptions(dual_tolerance=2.0)])
def test_oracle_options_match_reference(oracle, reference, opts):
    for seed, kind in ((1, "feasible"), (2, "infeasible_singleton"), (3, "unbounded"), (4, "infeasible_row")):
        c = generators.presolve_lp(seed, 150, 200, kind=kind)
        same(oracle.presolve(c, opts), reference.presolve(c, opts))


def test_invalid_models_rejected_like_the_reference(oracle, reference):
    good = generators.presolve_lp(9, 30, 40)
    bad = []
    c = dataclasses.replace(good, value=good.value.copy())
    c.value[0] = 0.0  # explicit zero
    bad.append(c)
    c = dataclasses.replace(good, rhs=good.rhs.copy())
    c.rhs[3] = np.inf
    bad.append(c)
    c = dataclasses.replace(good, objective=good.objective.copy())
    c.objective[2] = np.nan
    bad.append(c)
    c = dataclasses.replace(good, row_index=good.row_index.copy())
    j = int(np.argmax(np.diff(good.col_start) >= 2))
    p = good.col_start[j]
    c.row_index[p], c.row_index[p + 1] = c.row_index[p + 1], c.row_index[p]  # unsorted column
    bad.append(c)
    bad.append(dataclasses.replace(good, objective_offset=np.inf))
    for c in bad:
        with pytest.raises(ValueError):
            reference.presolve(c)
        with pytest.raises(ValueError):
            oracle.presolve(c)


def test_empty_models(oracle, reference):
    for c in (CanonicalModel(0, 0, [0], [], [], [], []),
              CanonicalModel(3, 0, [0], [], [], [0.0, 0.0, 0.0], []),
              CanonicalModel(0, 2, [0, 0, 0], [], [], [], [1.0, 2.0])):
        same(oracle.presolve(c), reference.presolve(c))


def test_presolve_workload_is_seeded_and_valid(oracle):
    """The timing workload's generator (bench.py --workload presolve, at a
    small size): the same arrays for the same seed, a model the reference's
    validate() accepts, and every reduction kind present."""
    a = generators.presolve_workload(3, 20000, 30000, k=3, chains=8, chain_len=10)
    b = generators.presolve_workload(3, 20000, 30000, k=3, chains=8, chain_len=10)
    assert canonical_digest(a) == canonical_digest(b)
    res = oracle.presolve(a)
    assert res.status == SolveStatus.optimal
    st = res.statistics
    assert st.empty_rows_removed > 0 and st.empty_cols_removed > 0 and st.row_singletons_removed > 0
    assert st.passes_executed >= 2
