"""Node-LP relaxations of branch and bound, solved together on the GPU.

The reference solves each open node's LP relaxation on its own with the dense
simplex (``solve_node_relaxation``, src/milp/node_lp.cpp:9-82, capped at 1024
canonical rows).  Here all the nodes of one branching round go to the engine
together.  Every node is the parent model with tightened variable bounds
(src/milp/milp_solver.cpp:401-447), so when the nodes share the matrix, the
objective and the row bounds -- the normal case -- they run in the variant
engine (``mc_pdlp_ctx_solve_variants``: the matrix stored and read once per
iteration for all of them); nodes of different models run in the packed batch
(``mc_pdlp_ctx_solve_batch``).

    results = solve_node_relaxations(ctx, [down, up, ...], max_iterations=100000)

Statuses are the reference's ``lp::reference::SolveStatus`` names.  A node is
``infeasible`` when the engine certifies it: crossed bounds or a row activity
interval that misses a row's bounds (at setup), or a dual ray found during the
iterations (Farkas certificate); an infeasible node that yields no certificate
ends at ``iteration_limit``.
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
    PdlpStatus.infeasible_or_unbounded: "infeasible",   # certified (setup or dual ray)
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


def share_matrix(nodes: list) -> bool:
    """True when every node has the first node's matrix, objective, offset,
    sense and row bounds (they differ at most in their variable bounds)."""
    a = nodes[0]
    same = lambda x, y: x is y or (x.shape == y.shape and np.array_equal(x, y))  # noqa: E731
    for b in nodes[1:]:
        if (b.num_rows, b.num_cols, b.nnz, b.objective_offset, int(b.objective_sense)) != \
                (a.num_rows, a.num_cols, a.nnz, a.objective_offset, int(a.objective_sense)):
            return False
        if not all(same(getattr(a, f), getattr(b, f)) for f in ("col_start", "row_index", "value", "objective",
                                                                 "row_lower", "row_upper")):
            return False
    return True


def solve_node_relaxations(ctx: Context, nodes: list, max_iterations: int = 500000,
                           feasibility_tolerance: float = 1e-7,
                           precision: Precision = Precision.fp64,
                           options: Optional[PdlpOptions] = None,
                           warm_primal: Optional[list] = None, warm_dual: Optional[list] = None,
                           shared_matrix: Optional[bool] = None) -> list:
    """LP relaxations of `nodes` (Models) solved together.  The defaults are
    milp::Options' max_iterations and feasibility_tolerance
    (include/markov_cero/milp/milp_solver.hpp:15-32); the tolerance is the
    PDLP relative KKT tolerance.  warm_primal / warm_dual (a point or None per
    node) start each node where its parent ended, as the reference's node
    solve starts the dual simplex from the parent's basis
    (src/milp/node_lp.cpp:44-60).  shared_matrix: None = the variant engine
    when the nodes share the matrix (share_matrix), True / False to force
    the variant engine / the packed batch."""
    o = options or PdlpOptions()
    o.max_iterations = max_iterations
    o.set_tolerance(feasibility_tolerance)
    o.precision = precision
    nodes = list(nodes)
    if shared_matrix is None:
        shared_matrix = len(nodes) > 1 and share_matrix(nodes)
    if shared_matrix:
        if not share_matrix(nodes):
            raise ValueError("shared_matrix=True needs nodes that differ only in their variable bounds")
        res = ctx.solve_variants(nodes[0], [n_.var_lower for n_ in nodes], [n_.var_upper for n_ in nodes], o,
                                 initial_primal=warm_primal, initial_dual=warm_dual)
    else:
        res = ctx.solve_batch(nodes, o, initial_primal=warm_primal, initial_dual=warm_dual)
    out = []
    for r in res:
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
