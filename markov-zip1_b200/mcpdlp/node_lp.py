"""Node-LP relaxations of branch and bound, solved as one GPU batch.

The reference solves each open node's LP relaxation on its own with the dense
simplex (``solve_node_relaxation``, src/milp/node_lp.cpp:9-82, capped at 1024
canonical rows).  Here all the nodes of one branching round go to the engine's
batched PDLP (``mc_pdlp_ctx_solve_batch``) together: every node is the parent
model with tightened variable bounds (src/milp/milp_solver.cpp:401-447), so a
round is exactly the batch of node variants the batched engine is built for.

    results = solve_node_relaxations(ctx, [down, up, ...], max_iterations=100000)

Statuses are the reference's ``lp::reference::SolveStatus`` names.  A node
whose bounds cross, or whose row activity interval misses a row's bounds, is
certified ``infeasible`` at setup (the engine's certificates); PDLP does not
otherwise detect infeasibility, so such a node ends at ``iteration_limit``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import Context, PdlpOptions, PdlpStatus, Precision
from .model import Model

# lp::reference::SolveStatus (include/markov_cero/lp/reference/revised_simplex.hpp)
SOLVE_STATUS = ("optimal", "infeasible", "unbounded", "iteration_limit", "invalid_model",
                "invalid_options", "resource_limit", "numerical_failure")

_FROM_PDLP = {
    PdlpStatus.optimal: "optimal",
    PdlpStatus.infeasible_or_unbounded: "infeasible",   # certified at setup
    PdlpStatus.iteration_limit: "iteration_limit",
    PdlpStatus.numerical_failure: "numerical_failure",
}


@dataclass
class NodeLpResult:
    """NodeLpResult (include/markov_cero/milp/node_lp.hpp:13-19) without the
    simplex basis, which PDLP does not produce."""
    status: str = "infeasible"
    primal: np.ndarray = field(default_factory=lambda: np.zeros(0))
    objective: float = 0.0
    iterations: int = 0


def solve_node_relaxations(ctx: Context, nodes: list, max_iterations: int = 500000,
                           feasibility_tolerance: float = 1e-7,
                           precision: Precision = Precision.fp64,
                           options: Optional[PdlpOptions] = None,
                           warm_primal: Optional[list] = None, warm_dual: Optional[list] = None) -> list:
    """LP relaxations of `nodes` (Models) in one batched solve.  The defaults
    are milp::Options' max_iterations and feasibility_tolerance
    (include/markov_cero/milp/milp_solver.hpp:15-32); the tolerance is the
    PDLP relative KKT tolerance.  warm_primal / warm_dual (a point or None per
    node) start each node where its parent ended, as the reference's node
    solve starts the dual simplex from the parent's basis
    (src/milp/node_lp.cpp:44-60)."""
    o = options or PdlpOptions()
    o.max_iterations = max_iterations
    o.set_tolerance(feasibility_tolerance)
    o.precision = precision
    out = []
    for r in ctx.solve_batch(list(nodes), o, initial_primal=warm_primal, initial_dual=warm_dual):
        res = NodeLpResult(status=_FROM_PDLP[r.status], iterations=r.iterations)
        if res.status == "optimal":
            res.primal = r.primal
            res.objective = r.objective
        out.append(res)
    return out


def branch_children(node: Model, primal: np.ndarray, branch_var: int):
    """The two children of a node branched on `branch_var` at its LP value
    (src/milp/milp_solver.cpp:401-447): down x_k <= floor(v), up x_k >= ceil(v);
    a child whose new bound crosses the node's other bound by more than 1e-9 is
    not created (None)."""
    v = float(primal[branch_var])
    lo, hi = node.var_lower[branch_var], node.var_upper[branch_var]
    f, c = math.floor(v), math.ceil(v)
    down = up = None
    if not (math.isfinite(lo) and f < lo - 1e-9):
        down = node.copy()
        down.var_upper = node.var_upper.copy()
        down.var_upper[branch_var] = f
        down.name = f"{node.name}-x{branch_var}<={f}"
    if not (math.isfinite(hi) and c > hi + 1e-9):
        up = node.copy()
        up.var_lower = node.var_lower.copy()
        up.var_lower[branch_var] = c
        up.name = f"{node.name}-x{branch_var}>={c}"
    return down, up
