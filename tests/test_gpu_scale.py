"""Parity at scale: the GPU engine against the reference CPU PDLP on seeded
LPs far above the unit-test sizes (needs a B200).

The reference results are committed fixtures (tests/golden/golden.json,
section "scale", made by tests/golden/make_golden.py --only scale, which runs
the reference's own solve_pdlp, src/lp/first_order/pdlp.cpp:139-276):

* standard_4m: the 40M-nonzero LP's generator at m = 200,000, n = 500,000,
  8 nonzeros per column (4M nonzeros).  The reference reaches 1e-4 and 1e-8.
  Bar: same status, objective within 1e-6 relative of the reference's at
  1e-8 (1e-3 at 1e-4), and the error against the analytic optimum b.y*.
* precision_600k: the precision-stress generator (|a| log-uniform over six
  decades, 20% boxed columns) at m = 20,000, n = 60,000, 10 nonzeros per
  column.  The reference stalls there: iteration limit (100,000) at both
  tolerances, relative KKT about 4e-4.  Bar: the GPU stalls too (same
  status), and its objective at the limit is as close to the analytic
  optimum as the reference's (within 10x of its error).
"""
from __future__ import annotations

import pytest

from conftest import rel
from mcpdlp import PdlpOptions, PdlpStatus, Precision, generators
from test_oracle import GOLDEN, sha

pytestmark = pytest.mark.gpu

SCALE = GOLDEN["scale"]
OBJ_TOL = {"0.0001": 1e-3, "1e-08": 1e-6}


def scale_model(name: str):
    g = SCALE[name]
    m = generators.random_lp(g["seed"], g["m"], g["n"], g["k"], g["family"])
    assert sha(m.col_start, m.row_index, m.value, m.objective, m.var_lower, m.var_upper,
               m.row_lower, m.row_upper) == g["digest"]
    return m


@pytest.fixture(scope="module")
def models():
    return {name: scale_model(name) for name in SCALE}


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
@pytest.mark.parametrize("tol", ["0.0001", "1e-08"])
def test_standard_4m_against_reference(gpu_ctx, models, precision, tol):
    m = models["standard_4m"]
    gold = SCALE["standard_4m"]["results"][tol]
    o = PdlpOptions(precision=precision)
    o.set_tolerance(float(tol))
    r = gpu_ctx.solve(m, o)
    assert gold["status"] == PdlpStatus.optimal
    assert r.status == gold["status"]
    assert max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap) <= float(tol)
    assert rel(r.objective, gold["objective"]) <= OBJ_TOL[tol], (r.objective, gold["objective"])
    opt = SCALE["standard_4m"]["optimum"]
    err = abs(r.objective - opt) / abs(opt)
    # the reference's own error against b.y* at this tolerance bounds ours (with slack)
    assert err <= max(10 * gold["objective_rel_err_vs_analytic"], 1e-11 if tol == "1e-08" else 1e-6), err
    print(f"standard_4m {precision.name} tol {tol}: gpu {r.iterations} it, obj {r.objective!r} "
          f"(err vs b.y* {err:.2e}); reference {gold['iterations']} it, obj {gold['objective']!r} "
          f"(err {gold['objective_rel_err_vs_analytic']:.2e})")


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
def test_precision_600k_stalls_like_reference(gpu_ctx, models, precision):
    m = models["precision_600k"]
    gold = SCALE["precision_600k"]["results"]["1e-08"]
    assert gold["status"] == PdlpStatus.iteration_limit
    o = PdlpOptions(precision=precision)
    o.set_tolerance(1e-8)
    r = gpu_ctx.solve(m, o)
    assert r.status == gold["status"]
    assert r.iterations == gold["iterations"] == 100000
    opt = SCALE["precision_600k"]["optimum"]
    err = abs(r.objective - opt) / abs(opt)
    assert err <= 10 * gold["objective_rel_err_vs_analytic"], (err, gold["objective_rel_err_vs_analytic"])
    print(f"precision_600k {precision.name}: gpu obj err {err:.2e} kkt "
          f"{max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap):.2e}; reference err "
          f"{gold['objective_rel_err_vs_analytic']:.2e} kkt "
          f"{max(gold['primal_infeasibility'], gold['dual_infeasibility'], gold['duality_gap']):.2e}")
