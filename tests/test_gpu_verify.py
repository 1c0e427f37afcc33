"""Device verify_primal (mc_verify_primal) against the reference's own
verify_primal (src/verify/primal_verifier.cpp:44-103, oracle/_ref) on the same
candidates (needs a B200).

The reference sums row activities and the objective in long double; the device
in double-double.  Pass/fail, the violation counts and the lowest violating
index of every kind must agree exactly; the maxima and the recomputed
objective within 1e-12 relative.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import mcpdlp
from conftest import rel
from mcpdlp import PdlpOptions, _abi, _lib, generators
from test_oracle import load_model, synthetic

pytestmark = pytest.mark.gpu


def solved(gpu_ctx, m, tol=1e-8):
    o = PdlpOptions()
    o.set_tolerance(tol)
    r = gpu_ctx.solve(m, o)
    return r.primal, r.objective


def check_same(dev: dict, ref: dict) -> None:
    assert dev["passed"] == ref["passed"]
    assert dev["violations"] == ref["violations"]
    assert dev["first_index"] == ref["first_index"]
    for k in ("maximum_row_violation", "maximum_variable_violation"):
        assert abs(dev[k] - ref[k]) <= 1e-12 * max(1.0, abs(ref[k])), k
    assert rel(dev["recomputed_objective"], ref["recomputed_objective"]) <= 1e-14
    assert abs(dev["objective_difference"] - ref["objective_difference"]) <= 1e-12 * max(
        1.0, abs(ref["recomputed_objective"]))


MODELS = ["netlib_afiro", "netlib_sc50a", "blend_pdlp", "tiny_simplex", "config0_s1", "precision_s1", "transport"]


def model_named(name):
    if name.startswith("config0") or name.startswith("precision"):
        return synthetic(name)
    if name == "transport":
        return generators.transport(4, 30, 40)
    return load_model(name)


@pytest.mark.parametrize("name", MODELS)
def test_solution_passes_like_the_reference(gpu_ctx, reference, name):
    """The CLI's post-solve check: candidate = the PDLP solution, tolerance =
    the solve tolerance (apps/markov_cero_solve.cpp:164-168)."""
    m = model_named(name)
    for tol in (1e-4, 1e-8):
        x, obj = solved(gpu_ctx, m, tol)
        dev = gpu_ctx.verify_primal(m, x, obj, tol, tol)
        check_same(dev, reference.verify_report(m, x, obj, tol, tol))


@pytest.mark.parametrize("name", MODELS)
def test_perturbed_candidates(gpu_ctx, reference, name):
    """Violations of every kind: shifted entries past their bounds, a wrong
    claimed objective, a tolerance tighter than the solve's."""
    m = model_named(name)
    x, obj = solved(gpu_ctx, m, 1e-4)
    rng = np.random.default_rng(11)
    y = x.copy()
    pick = rng.choice(m.num_cols, size=min(7, m.num_cols), replace=False)
    y[pick] += rng.choice([-1.0, 1.0], size=len(pick)) * (1.0 + 10 * rng.random(len(pick)))
    for cand, claimed, tol in ((y, obj, 1e-7), (x, obj * (1 + 1e-3) + 1e-3, 1e-6), (x, obj, 1e-9)):
        dev = gpu_ctx.verify_primal(m, cand, claimed, tol, tol)
        check_same(dev, reference.verify_report(m, cand, claimed, tol, tol))
    assert not gpu_ctx.verify_primal(m, y, obj, 1e-7, 1e-7)["passed"]


def test_device_resident_input(gpu_ctx, reference):
    import torch
    m = synthetic("config0_s1")
    x, obj = solved(gpu_ctx, m, 1e-6)
    dm = mcpdlp.DeviceModel(m)
    dx = torch.from_numpy(x).cuda()
    lp = dm.to_struct()
    rep = _abi.McVerifyReport()
    _lib.check(_lib.engine().mc_verify_primal(gpu_ctx.handle, C.addressof(lp), dx.data_ptr(), obj, 1e-6, 1e-6,
                                              1e-6, 1e-6, C.addressof(rep)))
    host = gpu_ctx.verify_primal(m, x, obj, 1e-6, 1e-6)
    assert bool(rep.passed) == host["passed"]
    assert rep.recomputed_objective == host["recomputed_objective"]
    assert rep.maximum_row_violation == host["maximum_row_violation"]


def test_invalid_inputs_are_errors(gpu_ctx):
    m = synthetic("small_s7")
    x = np.zeros(m.num_cols)
    x[4] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        gpu_ctx.verify_primal(m, x, 0.0)
    with pytest.raises(ValueError, match="tolerances"):
        gpu_ctx.verify_primal(m, np.zeros(m.num_cols), 0.0, feasibility_tolerance=1e-3)
    with pytest.raises(ValueError, match="claimed objective"):
        gpu_ctx.verify_primal(m, np.zeros(m.num_cols), float("inf"))
    # the context stays usable
    assert gpu_ctx.verify_primal(m, np.zeros(m.num_cols), 0.0, 1e-4, 1e-4)["violations"]["row_lower"] >= 0


def test_empty_rows_and_empty_models(gpu_ctx, reference):
    """Rows without entries have activity 0 and are still checked against
    their bounds; a model without rows or without nonzeros verifies its
    variable bounds and objective only -- as the reference does."""
    inf = np.inf
    # row 1 has no entries and bounds [1, 2]: activity 0 violates its lower bound
    m = mcpdlp.from_triplets(3, 2, [0, 2], [0, 1], [1.0, 2.0], objective=[1.0, -1.0],
                             var_lower=[0.0, 0.0], var_upper=[4.0, inf], row_lower=[0.0, 1.0, -inf],
                             row_upper=[3.0, 2.0, 5.0])
    for x, claimed in (([1.0, 1.0], 0.0), ([5.0, 3.0], 2.0), ([0.5, 0.25], 0.25)):
        x = np.array(x)
        check_same(gpu_ctx.verify_primal(m, x, claimed, 1e-7, 1e-7),
                   reference.verify_report(m, x, claimed, 1e-7, 1e-7))
    no_rows = mcpdlp.Model(0, 2, np.zeros(3, np.int32), np.zeros(0, np.int32), np.zeros(0),
                           np.array([1.0, 2.0]), np.zeros(2), np.ones(2), np.zeros(0), np.zeros(0))
    no_nnz = mcpdlp.Model(2, 2, np.zeros(3, np.int32), np.zeros(0, np.int32), np.zeros(0),
                          np.array([1.0, 2.0]), np.zeros(2), np.ones(2), np.array([-1.0, 0.5]),
                          np.array([1.0, 1.0]))
    for mm in (no_rows, no_nnz):
        for x in (np.array([0.5, 0.5]), np.array([2.0, -1.0])):
            check_same(gpu_ctx.verify_primal(mm, x, 1.5, 1e-7, 1e-7),
                       reference.verify_report(mm, x, 1.5, 1e-7, 1e-7))
