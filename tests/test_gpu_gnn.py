"""The learned warm start on the GPU (needs a B200).

* loss, gradient and prediction of the FP32 CUDA kernels against the FP64
  CPU oracle (oracle/gnn_oracle.py), on the same parameters;
* training steps reduce the loss; the network learns across instances;
* the engine's guard: a bad prediction falls back to the cold start, a good
  one is used (PDHG always runs to the same tolerance).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import gnn_oracle as G
import mcpdlp
from conftest import options, rel
from mcpdlp import PdlpOptions, PdlpStatus, generators
from mcpdlp.learn import Target, WarmStartNet, solve_targets, solve_warm

pytestmark = pytest.mark.gpu


def small_target(seed: int, S: int = 6, D: int = 7) -> Target:
    m = generators.transport(seed, S, D)
    rng = np.random.default_rng(seed)
    return Target(m, rng.uniform(0, 30, m.num_cols), rng.normal(0, 0.2, m.num_rows), 0.3)


@pytest.mark.parametrize("seed", [1, 2])
def test_loss_and_gradient_match_oracle(seed):
    net = WarmStartNet(0, 3, seed)
    t = small_target(seed)
    loss, grad = net.loss_and_grad(t)
    theta = net.params.astype(np.float64)
    loss_c, grad_c, _ = G.loss_and_grad(theta, t.model, t.x, t.y, t.log_omega)
    assert abs(loss - loss_c) <= 1e-4 * abs(loss_c) + 1e-7
    err = np.linalg.norm(grad - grad_c) / np.linalg.norm(grad_c)
    assert err <= 1e-4, err
    big = np.abs(grad_c) > 1e-3 * np.abs(grad_c).max()
    np.testing.assert_allclose(grad[big], grad_c[big], rtol=2e-3)
    net.close()


def test_gradient_on_a_random_lp():
    """Mixed-sign coefficients, boxed and free bounds, ranged rows."""
    from test_oracle import random_small_lp
    m = random_small_lp(3)
    rng = np.random.default_rng(0)
    t = Target(m, rng.normal(size=m.num_cols), rng.normal(size=m.num_rows), -0.2)
    net = WarmStartNet(0, 3, 7)
    loss, grad = net.loss_and_grad(t)
    loss_c, grad_c, _ = G.loss_and_grad(net.params.astype(np.float64), m, t.x, t.y, t.log_omega)
    assert abs(loss - loss_c) <= 1e-4 * abs(loss_c) + 1e-7
    assert np.linalg.norm(grad - grad_c) / np.linalg.norm(grad_c) <= 1e-4


def test_prediction_matches_oracle():
    net = WarmStartNet(0, 3, 3)
    m = generators.transport(4, 9, 8)
    x, y, lw = net.predict(m)
    xc, yc, lwc = G.predict(net.params.astype(np.float64), m)
    np.testing.assert_allclose(x, xc, rtol=1e-4, atol=1e-4 * (np.abs(xc).max() + 1e-30))
    np.testing.assert_allclose(y, yc, rtol=1e-4, atol=1e-4 * (np.abs(yc).max() + 1e-30))
    assert abs(lw - lwc) <= 1e-4 * (1 + abs(lwc))


def test_training_reduces_loss_and_generalises(gpu_ctx):
    train = [generators.transport(s, 5 + s % 4, 6 + s % 3) for s in range(40)]
    held = [generators.transport(1000 + s, 5 + s % 4, 6 + s % 3) for s in range(8)]
    o = PdlpOptions(max_iterations=20000)
    o.set_tolerance(1e-8)
    data = solve_targets(gpu_ctx, train, o)
    test = solve_targets(gpu_ctx, held, o)
    net = WarmStartNet(0, 3, 0)
    before = np.mean([net.loss_and_grad(t)[0] for t in test])
    hist = net.fit(data, epochs=4, lr=3e-3)
    after = np.mean([net.loss_and_grad(t)[0] for t in test])
    assert hist[-1] < hist[0]
    assert after < 0.5 * before, (before, after)


def test_guard_falls_back_from_a_bad_prediction(gpu_ctx, oracle):
    m = generators.transport(5, 12, 10)
    o = PdlpOptions(max_iterations=100000, warm_start_guard=True)
    o.set_tolerance(1e-6)
    o.initial_primal = np.full(m.num_cols, 1e4)
    o.initial_dual = np.full(m.num_rows, -1e3)
    o.initial_primal_weight = 1e5
    r = gpu_ctx.solve(m, o)
    cold = gpu_ctx.solve(m, PdlpOptions(max_iterations=100000, primal_tolerance=1e-6, dual_tolerance=1e-6,
                                        gap_tolerance=1e-6))
    assert not r.extra["warm_start_used"]
    assert r.extra["warm_start_score"] > r.extra["cold_start_score"]
    assert r.iterations == cold.iterations and r.objective == cold.objective


def test_guard_uses_a_good_prediction(gpu_ctx, oracle):
    m = generators.transport(6, 10, 12)
    cpu = oracle.solve(m, options(1e-8, max_iterations=200000))
    o = PdlpOptions(max_iterations=100000, warm_start_guard=True)
    o.set_tolerance(1e-6)
    o.initial_primal, o.initial_dual = cpu.primal, cpu.dual
    r = gpu_ctx.solve(m, o)
    assert r.extra["warm_start_used"]
    assert r.extra["warm_start_score"] <= r.extra["cold_start_score"]
    assert r.status == PdlpStatus.optimal and r.iterations == 40


def test_solve_warm_runs_to_the_same_tolerance(gpu_ctx):
    net = WarmStartNet(0, 3, 0)
    m = generators.transport(7, 8, 9)
    o = PdlpOptions(max_iterations=100000)
    o.set_tolerance(1e-6)
    r = solve_warm(gpu_ctx, net, m, o)
    assert r.status in (PdlpStatus.optimal, PdlpStatus.iteration_limit)
    if r.status == PdlpStatus.optimal:
        assert max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap) <= 1e-6
    assert math.isfinite(r.extra["warm_start_score"]) or not r.extra["warm_start_used"]


def test_device_built_instance_matches_host_build(gpu_ctx, monkeypatch):
    """Large LPs are built on the device (the engine's transpose, norms and
    features in kernels); the result must be the host build's, bit for bit."""
    m = generators.random_lp(8, 3000, 9000, 6)
    net = WarmStartNet(0, 3, 0)
    monkeypatch.setenv("MC_GNN_DEVICE_BUILD_MIN_NNZ", str(1 << 40))
    xh, yh, wh = net.predict(m)
    monkeypatch.setenv("MC_GNN_DEVICE_BUILD_MIN_NNZ", "0")
    xd, yd, wd = net.predict(m)
    assert np.array_equal(xh, xd) and np.array_equal(yh, yd) and wh == wd
    t = solve_targets(gpu_ctx, [m], PdlpOptions(max_iterations=2000), margin=0.0)[0]
    monkeypatch.setenv("MC_GNN_DEVICE_BUILD_MIN_NNZ", str(1 << 40))
    lh, gh = net.loss_and_grad(t)
    monkeypatch.setenv("MC_GNN_DEVICE_BUILD_MIN_NNZ", "0")
    ld, gd = net.loss_and_grad(t)
    assert lh == ld and np.array_equal(gh, gd)


def test_predicted_weight_form_runs_to_the_same_tolerance(gpu_ctx, oracle):
    """halves="weight": the reference's cold point with the predicted initial
    primal weight (initial_primal_weight, pdlp.hpp:31) -- same optimum."""
    net = WarmStartNet(0, 3, 0)
    m = generators.random_lp(5, 200, 600, 6)
    o = PdlpOptions(max_iterations=100000)
    o.set_tolerance(1e-8)
    r = solve_warm(gpu_ctx, net, m, o, halves="weight")
    assert r.status == PdlpStatus.optimal
    assert max(r.primal_infeasibility, r.dual_infeasibility, r.duality_gap) <= 1e-8
    assert abs(r.objective - m.info["optimum"]) <= 1e-6 * abs(m.info["optimum"])
    assert not r.extra["warm_start_used"]


def test_trained_network_gains_over_untrained_and_cold(gpu_ctx):
    """What training buys, on held-out instances: the trained network's
    prediction starts closer to optimality (the reference's KKT score, as the
    engine's guard measures it) than both the cold start and the same network
    untrained.  (Measured on B200 with this setup: 15 of 16 held-out LPs, start
    scores 1-4% below the cold start's.)  On this family the reference
    algorithm's iteration count is erratic in the start point, so the test
    asserts the start-point gain only."""
    def family(seed):
        S = generators.uniform_int(seed, 0, 15, 30)
        D = generators.uniform_int(seed, 1, 15, 30)
        return generators.transport(seed, S, D)
    train = [family(s) for s in range(512)]
    held = [family(9000 + s) for s in range(16)]
    o = PdlpOptions(max_iterations=20000)
    o.set_tolerance(1e-8)
    data = solve_targets(gpu_ctx, train, o)
    untrained = WarmStartNet(0, 3, 0)
    trained = WarmStartNet(0, 3, 0)
    trained.fit(data, epochs=4, lr=2e-3)
    e = PdlpOptions(max_iterations=2000)
    e.set_tolerance(1e-4)
    better_than_cold = better_than_untrained = 0
    for m in held:
        rt = solve_warm(gpu_ctx, trained, m, e)     # the guard scores both starts
        ru = solve_warm(gpu_ctx, untrained, m, e)
        better_than_cold += rt.extra["warm_start_score"] < rt.extra["cold_start_score"]
        better_than_untrained += rt.extra["warm_start_score"] < ru.extra["warm_start_score"]
    assert better_than_cold >= 13, better_than_cold
    assert better_than_untrained >= 13, better_than_untrained


def test_trained_network_saves_iterations_on_random_lps(gpu_ctx):
    """The iteration gain on the config-0 random-LP family (m in [200, 600],
    n = 3m, 6 nonzeros per column), where PDHG converges smoothly: trained on
    1024 GPU-solved instances, the guarded warm start (predicted point, the
    reference's derived primal weight) reaches 1e-8 in fewer iterations in
    total than the cold start on held-out instances.  (Measured on B200 with
    this setup: 676 against 736 iterations on average, 8% fewer.)"""
    def family(seed):
        m = generators.uniform_int(seed, 0, 200, 600)
        return generators.random_lp(seed, m, 3 * m, 6)
    train = [family(s) for s in range(1024)]
    o = PdlpOptions(max_iterations=20000)
    o.set_tolerance(1e-8)
    data = solve_targets(gpu_ctx, train, o, margin=0.0)
    net = WarmStartNet(0, 3, 0)
    net.fit(data, epochs=6, lr=2e-3)
    cold_total = warm_total = 0
    for seed in range(10_000_000, 10_000_000 + 24):
        m = family(seed)
        cold = gpu_ctx.solve(m, o)
        warm = solve_warm(gpu_ctx, net, m, o)
        assert cold.status == warm.status == PdlpStatus.optimal
        assert rel(cold.objective, warm.objective) <= 1e-6
        cold_total += cold.iterations
        warm_total += warm.iterations
    assert warm_total < cold_total, (warm_total, cold_total)
