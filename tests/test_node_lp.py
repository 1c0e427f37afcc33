"""Node-LP relaxations of branch and bound as one batched solve
(mcpdlp.node_lp).  CPU: the branching rule; GPU: node statuses and objectives
against the reference's primal simplex on every node."""
from __future__ import annotations

import math

import numpy as np
import pytest

import mcpdlp
from conftest import rel
from mcpdlp import generators
from mcpdlp.node_lp import SOLVE_STATUS, branch_children, solve_node_relaxations


def test_branch_children_follow_the_reference_rule():
    """src/milp/milp_solver.cpp:401-447: down x_k <= floor(v), up x_k >= ceil(v),
    a child is dropped when its bound crosses the other by more than 1e-9."""
    m = generators.random_lp(3, 20, 60, 4)
    x = np.full(m.num_cols, 2.5)
    down, up = branch_children(m, x, 7)
    assert down.var_upper[7] == 2.0 and down.var_lower[7] == m.var_lower[7]
    assert up.var_lower[7] == 3.0 and up.var_upper[7] == m.var_upper[7]
    assert np.array_equal(np.delete(down.var_upper, 7), np.delete(m.var_upper, 7))
    assert m.var_upper[7] == 10.0 and m.var_lower[7] == 0.0       # parent untouched
    node = m.copy()
    node.var_lower = m.var_lower.copy()
    node.var_lower[7] = 3.0
    d, u = branch_children(node, x, 7)          # floor 2 < lower 3: no down child
    assert d is None and u is not None
    node.var_upper = m.var_upper.copy()
    node.var_upper[7] = 2.0
    node.var_lower[7] = 0.0
    d, u = branch_children(node, x, 7)          # ceil 3 > upper 2: no up child
    assert u is None and d is not None
    assert SOLVE_STATUS[0] == "optimal" and SOLVE_STATUS[3] == "iteration_limit"


@pytest.mark.gpu
def test_node_round_against_simplex(gpu_ctx, reference):
    base = generators.transport(2, 20, 30)
    root = reference.simplex(base)
    assert root["status"] == "optimal"
    x = root["primal"]
    base.info["x_star"] = x
    # one branching round: both children of the six most fractional
    # variables, grandchildren of the first two, and two node variants with
    # crossed bounds (the config-3 generator's tightening)
    order = np.argsort(-np.abs(x - np.round(x)))[:6]
    nodes = []
    for j in order:
        nodes += [c for c in branch_children(base, x, int(j)) if c is not None]
    for c in list(nodes[:2]):
        nodes += [g for g in branch_children(c, x, int(order[2])) if g is not None]
    nodes += [generators.tighten_bounds(base, 100 + s)[0] for s in range(2)]
    res = solve_node_relaxations(gpu_ctx, nodes, max_iterations=100000, feasibility_tolerance=1e-7)
    optimal = 0
    for node, r in zip(nodes, res):
        if np.any(node.var_lower > node.var_upper):
            # the reference rejects crossed bounds before its simplex runs
            # (canonicalize: "inconsistent variable bounds"); the batch
            # certifies such a node infeasible at setup
            assert r.status == "infeasible", node.name
            continue
        s = reference.simplex(node)
        if r.status == "infeasible":
            assert s["status"] == "infeasible", node.name        # the certificate is sound
        if s["status"] == "infeasible":
            assert r.status in ("infeasible", "iteration_limit"), node.name
        if r.status == "optimal":
            assert s["status"] == "optimal", node.name
            assert rel(r.objective, s["objective"]) <= 1e-5, node.name
            assert np.all(r.primal >= node.var_lower - 1e-6) and np.all(r.primal <= node.var_upper + 1e-6)
            optimal += 1
    assert optimal >= len(nodes) // 2


@pytest.mark.gpu
def test_children_warm_started_from_the_parent(gpu_ctx):
    """Children started from the parent's PDLP solution reach the same
    objectives (within the tolerance) as from a cold start, in far fewer
    iterations."""
    base = generators.random_lp(21, 300, 900, 6)
    parent = solve_node_relaxations(gpu_ctx, [base], max_iterations=100000, feasibility_tolerance=1e-7)[0]
    assert parent.status == "optimal"
    x = parent.primal
    par = gpu_ctx.solve(base, mcpdlp.PdlpOptions(primal_tolerance=1e-7, dual_tolerance=1e-7, gap_tolerance=1e-7))
    order = np.argsort(-np.abs(x - np.round(x)))[:8]
    nodes = []
    for j in order:
        nodes += [c for c in branch_children(base, x, int(j)) if c is not None]
    cold = solve_node_relaxations(gpu_ctx, nodes, max_iterations=100000, feasibility_tolerance=1e-7)
    warm = solve_node_relaxations(gpu_ctx, nodes, max_iterations=100000, feasibility_tolerance=1e-7,
                                  warm_primal=[par.primal] * len(nodes), warm_dual=[par.dual] * len(nodes))
    both = [(c, w) for c, w in zip(cold, warm) if c.status == w.status == "optimal"]
    assert len(both) >= len(nodes) // 2
    for c, w in both:
        assert rel(c.objective, w.objective) <= 1e-5
    assert sum(w.iterations for _, w in both) < 0.8 * sum(c.iterations for c, _ in both)


@pytest.mark.gpu
def test_shared_matrix_round_matches_the_packed_batch(gpu_ctx):
    """A round whose nodes share the matrix runs in the variant engine by
    default; it must give the packed batch's statuses and objectives."""
    base = generators.random_lp(23, 300, 900, 6)
    parent = solve_node_relaxations(gpu_ctx, [base], max_iterations=100000, feasibility_tolerance=1e-7)[0]
    x = parent.primal
    order = np.argsort(-np.abs(x - np.round(x)))[:10]
    nodes = []
    for j in order:
        nodes += [c for c in branch_children(base, x, int(j)) if c is not None]
    nodes += [generators.tighten_bounds(base, 200 + s)[0] for s in range(4)]
    from mcpdlp.node_lp import share_matrix
    assert share_matrix(nodes)
    shared = solve_node_relaxations(gpu_ctx, nodes, max_iterations=100000, feasibility_tolerance=1e-7)
    packed = solve_node_relaxations(gpu_ctx, nodes, max_iterations=100000, feasibility_tolerance=1e-7,
                                    shared_matrix=False)
    for node, a, b in zip(nodes, shared, packed):
        assert a.status == b.status, node.name
        if a.status == "optimal":
            assert rel(a.objective, b.objective) <= 1e-6, node.name


def test_share_matrix_detects_other_models():
    a = generators.random_lp(5, 30, 90, 4)
    b = a.copy()
    b.var_upper = b.var_upper.copy()
    b.var_upper[3] = 1.0
    from mcpdlp.node_lp import share_matrix
    assert share_matrix([a, b])
    c = a.copy()
    c.objective = c.objective.copy()
    c.objective[0] += 1.0
    assert not share_matrix([a, c])
    assert not share_matrix([a, generators.random_lp(6, 30, 90, 4)])
