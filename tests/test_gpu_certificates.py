"""Infeasibility certificates of batched solves (needs a B200).

The reference PDLP never reports infeasibility (pdlp.hpp:43 declares the
status; pdlp.cpp runs infeasible LPs to its iteration limit), so every
certificate the batched engine returns is checked on its own by the CPU
checker oracle/certificates.py in exact rational arithmetic:

* node variants of one LP (bounds tightened as the reference's branching
  does, src/milp/milp_solver.cpp:401-447): every infeasible result carries a
  crossed-bounds, row-activity or dual-ray certificate that the checker
  accepts, and every feasible variant's result is not infeasible;
* LPs whose infeasibility no single row or bound shows (a row that is the
  sum of two others with a shifted right-hand side): found during the
  iterations as a dual ray (the dual average diverges along it), in both
  precision forms, while feasible LPs of the same batch converge.
"""
from __future__ import annotations

import numpy as np
import pytest

import mcpdlp
from certificates import check_certificate, dual_ray_margin
from conftest import options
from mcpdlp import PdlpOptions, PdlpStatus, Precision, generators

pytestmark = pytest.mark.gpu


def opts(tol: float, **kw) -> PdlpOptions:
    o = PdlpOptions(**kw)
    o.set_tolerance(tol)
    return o


def hidden_infeasible(seed: int, m: int = 150, n: int = 450, shift: float = 1.0):
    """A feasible random LP plus the equality row (row a + row b) whose
    right-hand side is b_a + b_b + shift: no single row's activity interval
    over the box [0, 10] excludes its bounds, but the system is infeasible."""
    base = generators.random_lp(seed, m, n, 6)
    rows, cols, vals = [], [], []
    for j in range(n):
        for p in range(base.col_start[j], base.col_start[j + 1]):
            rows.append(int(base.row_index[p]))
            cols.append(j)
            vals.append(float(base.value[p]))
    a, b = 0, 1
    extra = [(r, c, v) for r, c, v in zip(rows, cols, vals) if r in (a, b)]
    rows += [m] * len(extra)
    cols += [c for _, c, _ in extra]
    vals += [v for _, _, v in extra]
    rhs = float(base.row_lower[a] + base.row_lower[b] + shift)
    return mcpdlp.from_triplets(m + 1, n, rows, cols, vals, objective=base.objective,
                                var_lower=base.var_lower, var_upper=base.var_upper,
                                row_lower=np.append(base.row_lower, rhs),
                                row_upper=np.append(base.row_upper, rhs), name=f"hidden-{seed}")


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
def test_node_variant_certificates_check_out(gpu_ctx, oracle, precision):
    base, variants, _ = generators.batch_part2(4, variants=48, m=400, n=1200, k=8)
    res = gpu_ctx.solve_batch(variants, opts(1e-6, precision=precision))
    infeasible = 0
    for v, r in zip(variants, res):
        if r.status == PdlpStatus.infeasible_or_unbounded:
            infeasible += 1
            kind, idx = r.extra["certificate"], r.extra["certificate_index"]
            assert kind != "none", v.name
            assert check_certificate(v, kind, idx, r.dual), (v.name, kind, idx)
        else:
            assert r.extra["certificate"] == "none"
            assert r.status == PdlpStatus.optimal, (v.name, r.status)
    assert infeasible > 0


@pytest.mark.parametrize("precision", [Precision.fp64, Precision.fp32_refine])
def test_hidden_infeasibility_found_as_dual_ray(gpu_ctx, oracle, precision):
    hidden = [hidden_infeasible(s) for s in (11, 12, 13)]
    feasible = [generators.random_lp(s, 150, 450, 6) for s in (21, 22)]
    models = [hidden[0], feasible[0], hidden[1], feasible[1], hidden[2]]
    res = gpu_ctx.solve_batch(models, opts(1e-8, precision=precision))
    for model, r in zip(models, res):
        if model.name.startswith("hidden"):
            assert r.status == PdlpStatus.infeasible_or_unbounded, (model.name, r.status, r.iterations)
            assert r.extra["certificate"] == "dual_ray"
            assert r.extra["certificate_index"] == -1
            margin = dual_ray_margin(model, r.dual)
            assert margin is not None and margin > 0
            assert r.iterations < 100000
            # the reference runs these to its iteration limit
            cpu = oracle.solve(model, options(1e-8, max_iterations=2000))
            assert cpu.status == PdlpStatus.iteration_limit
        else:
            assert r.status == PdlpStatus.optimal and r.extra["certificate"] == "none"


def test_single_solve_keeps_the_reference_status(gpu_ctx):
    # one LP through mc_pdlp_ctx_solve: no certificates, the reference's
    # behaviour (iteration limit on an infeasible LP)
    m = hidden_infeasible(14)
    r = gpu_ctx.solve(m, opts(1e-8, max_iterations=4000))
    assert r.status == PdlpStatus.iteration_limit
    assert r.extra["certificate"] == "none" and r.extra["certificate_index"] == -1
