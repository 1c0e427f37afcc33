"""The CPU oracle is pinned to the reference (CPU-only tests).

* against the committed golden vectors made by the reference itself
  (tests/golden/make_golden.py): bit-for-bit equal results;
* against the reference library, live, where oracle/_ref is built: random
  small LPs across option settings, bit-for-bit;
* the reference's own known answers (tests/pdlp_test.cpp, ADR-P3-05).
"""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

from conftest import options
from mcpdlp import generators
from mcpdlp.model import Model, from_triplets

GOLDEN_DIR = Path(__file__).resolve().parent / "golden"
GOLDEN = json.loads((GOLDEN_DIR / "golden.json").read_text())


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def load_model(name: str) -> Model:
    z = np.load(GOLDEN_DIR / GOLDEN["models"][name]["file"])
    return Model(int(z["num_rows"]), int(z["num_cols"]), z["col_start"], z["row_index"],
                 z["value"], z["objective"], z["var_lower"], z["var_upper"], z["row_lower"],
                 z["row_upper"], float(z["objective_offset"]), int(z["objective_sense"]), name=name)


def synthetic(name: str) -> Model:
    g = GOLDEN["synthetic"][name]
    return generators.random_lp(g["seed"], g["m"], g["n"], g["k"], g["family"])


def check_exact(res, gold: dict) -> None:
    assert res.status == gold["status"]
    assert res.iterations == gold["iterations"]
    assert res.objective == gold["objective"]
    assert res.primal_infeasibility == gold["primal_infeasibility"]
    assert res.dual_infeasibility == gold["dual_infeasibility"]
    assert res.duality_gap == gold["duality_gap"]
    assert sha(res.primal) == gold["primal_sha256"]
    assert sha(res.dual) == gold["dual_sha256"]


FAST_MODELS = [n for n in GOLDEN["models"] if n not in ("netlib_sc105", "netlib_recipe", "netlib_scsd6")]


@pytest.mark.parametrize("name", FAST_MODELS)
@pytest.mark.parametrize("tol", ["0.0001", "1e-08"])
def test_oracle_bit_exact_on_golden_models(oracle, name, tol):
    m = load_model(name)
    res = oracle.solve(m, options(float(tol)))
    check_exact(res, GOLDEN["models"][name]["results"][tol])


@pytest.mark.slow
@pytest.mark.parametrize("name", ["netlib_sc105", "netlib_scsd6"])
def test_oracle_bit_exact_on_long_netlib(oracle, name):
    m = load_model(name)
    res = oracle.solve(m, options(1e-8))
    check_exact(res, GOLDEN["models"][name]["results"]["1e-08"])


@pytest.mark.parametrize("name", list(GOLDEN["synthetic"]))
def test_generator_is_pinned(name):
    m = synthetic(name)
    digest = sha(m.col_start, m.row_index, m.value, m.objective, m.var_lower, m.var_upper,
                 m.row_lower, m.row_upper)
    assert digest == GOLDEN["synthetic"][name]["digest"]
    assert m.info["optimum"] == pytest.approx(GOLDEN["synthetic"][name]["optimum"], rel=0, abs=0)


@pytest.mark.parametrize("name", list(GOLDEN["synthetic"]))
@pytest.mark.parametrize("tol", ["0.0001", "1e-08"])
def test_oracle_bit_exact_on_golden_synthetic(oracle, name, tol):
    m = synthetic(name)
    res = oracle.solve(m, options(float(tol)))
    check_exact(res, GOLDEN["synthetic"][name]["results"][tol])


@pytest.mark.parametrize("name", list(GOLDEN["ruiz"]))
def test_oracle_ruiz_bit_exact(oracle, name):
    e = oracle.equilibrate(synthetic(name), 10)
    g = GOLDEN["ruiz"][name]
    assert e["iterations"] == g["iterations"]
    assert e["converged"] == g["converged"]
    assert sha(e["value"]) == g["value_sha256"]
    assert sha(e["row_scale"], e["col_scale"]) == g["scales_sha256"]
    assert sha(e["objective"], e["var_lower"], e["var_upper"], e["row_lower"], e["row_upper"]) == g["bounds_sha256"]


def test_reference_known_answers(oracle):
    """tests/pdlp_test.cpp:62 (-7), :119 (5); ADR-P3-05 (-9 at 1e-6)."""
    assert abs(oracle.solve(load_model("blend_pdlp"), options(1e-4)).objective + 7.0) < 0.1
    assert abs(oracle.solve(load_model("equality_pdlp"), options(1e-4)).objective - 5.0) < 0.1
    r = oracle.solve(load_model("tiny_simplex"), options(1e-6))
    assert r.status == 0 and abs(r.objective + 9.0) < 1e-4


def test_synthetic_optimum_is_analytic(oracle):
    m = synthetic("config0_s1")
    r = oracle.solve(m, options(1e-8))
    assert abs(r.objective - m.info["optimum"]) / abs(m.info["optimum"]) < 1e-8
    assert abs(m.info["optimum"] - m.info["dual_optimum"]) / abs(m.info["optimum"]) < 1e-12


# ---------------------------------------------------------------- live pin
def random_small_lp(seed: int) -> Model:
    """Mixed bound kinds, ranged/one-sided rows, maximise, offset."""
    rng = np.random.default_rng(seed)
    m, n = int(rng.integers(3, 30)), int(rng.integers(3, 40))
    rows, cols, vals = [], [], []
    for j in range(n):
        k = int(rng.integers(1, min(m, 4) + 1))
        for r in rng.choice(m, size=k, replace=False):
            rows.append(int(r)); cols.append(j); vals.append(float(rng.normal()))
    x0 = rng.uniform(0, 2, n)
    A = np.zeros((m, n))
    for r, c, v in zip(rows, cols, vals):
        A[r, c] += v
    act = A @ x0
    kind = rng.integers(0, 4, m)
    rl = np.where(kind == 0, act, np.where(kind == 1, -np.inf, act - rng.uniform(0, 1, m)))
    ru = np.where(kind == 0, act, np.where(kind == 2, np.inf, act + rng.uniform(0, 1, m)))
    vk = rng.integers(0, 4, n)
    vl = np.where(vk == 0, -np.inf, 0.0)
    vu = np.where(vk == 1, np.inf, 5.0)
    return from_triplets(m, n, rows, cols, vals, objective=rng.normal(size=n), var_lower=vl,
                         var_upper=vu, row_lower=rl, row_upper=ru,
                         objective_offset=float(rng.normal()), objective_sense=int(rng.integers(0, 2)))


OPTION_SETS = [
    dict(),
    dict(restart_strategy=0),
    dict(restart_strategy=2),
    dict(adaptive_step_size=0),
    dict(adaptive_primal_weight=0),
    dict(ruiz_scaling=0),
    dict(restart_every=7, max_iterations=300),
    dict(max_iterations=0),
    dict(max_iterations=55),
    dict(initial_primal_weight=3.0, step_size_reduction=0.5),
]


@pytest.mark.parametrize("seed", range(12))
def test_oracle_matches_reference_live(oracle, reference, seed):
    m = random_small_lp(seed)
    for kw in OPTION_SETS:
        kw = dict(kw)
        o = options(1e-6, max_iterations=kw.pop("max_iterations", 4000), **kw)
        a = oracle.solve(m, o)
        b = reference.solve(m, o)
        assert (a.status, a.iterations, a.objective) == (b.status, b.iterations, b.objective), kw
        assert (a.primal_infeasibility, a.dual_infeasibility, a.duality_gap) == (
            b.primal_infeasibility, b.dual_infeasibility, b.duality_gap)
        assert np.array_equal(a.primal, b.primal) and np.array_equal(a.dual, b.dual)


def test_oracle_ruiz_matches_reference_live(oracle, reference):
    for seed in range(6):
        m = random_small_lp(100 + seed)
        a, b = oracle.equilibrate(m, 10), reference.equilibrate(m, 10)
        for k in ("value", "objective", "var_lower", "var_upper", "row_lower", "row_upper",
                  "row_scale", "col_scale"):
            assert np.array_equal(a[k], b[k]), k
        assert a["iterations"] == b["iterations"]


def test_reference_verifier_accepts_oracle_solution(oracle, reference):
    """The CLI's post-solve check (apps/markov_cero_solve.cpp:164-178)."""
    m = load_model("blend_pdlp")
    r = oracle.solve(m, options(1e-4))
    rep = reference.verify_primal(m, r.primal, r.objective, 1e-4)
    assert rep["passed"]


# ------------------------------------------------- primal simplex optimum
SIMPLEX = GOLDEN["simplex"]


def transport_case(name: str) -> Model:
    g = SIMPLEX[name]
    return generators.transport(g["seed"], g["suppliers"], g["customers"])


@pytest.mark.parametrize("name", list(SIMPLEX))
def test_transport_generator_is_pinned(name):
    m = transport_case(name)
    assert sha(m.col_start, m.row_index, m.value, m.objective, m.var_lower, m.var_upper,
               m.row_lower, m.row_upper) == SIMPLEX[name]["digest"]


@pytest.mark.parametrize("name", ["transport_2_20x30", "transport_4_30x40"])
def test_reference_simplex_reproduces_golden(reference, name):
    r = reference.simplex(transport_case(name))
    assert r["status"] == SIMPLEX[name]["status"] == "optimal"
    assert r["objective"] == SIMPLEX[name]["objective"]


@pytest.mark.parametrize("name", list(SIMPLEX))
def test_oracle_pdlp_against_simplex_optimum(oracle, name):
    """The reference PDLP at 1e-8 (restated) against the simplex's FP64
    optimum: where it converges, within 1e-6 relative (src/lp/reference/
    revised_simplex.cpp is the FP64 optimum of the transportation family)."""
    g = SIMPLEX[name]
    r = oracle.solve(transport_case(name), options(1e-8))
    assert (r.status, r.iterations, r.objective) == (g["pdlp_1e8"]["status"], g["pdlp_1e8"]["iterations"],
                                                     g["pdlp_1e8"]["objective"])
    if r.status == 0:
        assert abs(r.objective - g["objective"]) <= 1e-6 * abs(g["objective"])


@pytest.mark.parametrize("name", ["netlib_afiro", "netlib_sc50a", "netlib_sc50b"])
def test_oracle_reaches_published_netlib_optima(oracle, name):
    """Known answers: the published Netlib optima (the reference's
    scripts/run_netlib.py:19-93), reached by the PDLP at 1e-8 within 1e-6."""
    r = oracle.solve(load_model(name), options(1e-8))
    best = GOLDEN["netlib_optimal"][name]
    assert r.status == 0
    assert abs(r.objective - best) <= 1e-6 * max(1.0, abs(best))
