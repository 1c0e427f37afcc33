"""Learned warm start for PDLP (the engine's GNN, include/mc_pdlp.h).

    net = WarmStartNet(device=0, rounds=3, seed=0)
    data = solve_targets(ctx, models, options)       # GPU PDLP solutions as targets
    net.fit(data, epochs=3, lr=1e-3)
    res = solve_warm(ctx, net, model, options)        # guarded warm start

``solve_warm`` feeds the network's prediction to the engine with
``warm_start_guard`` on: the engine evaluates the reference's KKT score of the
prediction and of the cold start and runs from the better-scoring point, and
PDHG runs to the same tolerance either way.

CLI (training and evaluation on the transportation family, or on the config-0
random-LP family with --family random):

    python -m mcpdlp.learn --train 4096 --test 256 --out gnn.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import time
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import Context, PdlpOptions, PdlpResult, _abi, _lib
from .model import Model


@dataclass
class Target:
    model: Model
    x: np.ndarray
    y: np.ndarray
    log_omega: float
    result: Optional[PdlpResult] = None


class WarmStartNet:
    """The device-resident network (mc_gnn)."""

    def __init__(self, device: int = 0, rounds: int = 3, seed: int = 0):
        self._lib = _lib.engine()
        self._h = C.c_void_p()
        _lib.check(self._lib.mc_gnn_create(device, rounds, seed, C.byref(self._h)))
        n = C.c_int64(0)
        _lib.check(self._lib.mc_gnn_num_params(self._h, C.byref(n)))
        self.num_params = n.value
        self.rounds = rounds

    def close(self) -> None:
        if self._h:
            self._lib.mc_gnn_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        _lib.check(self._lib.mc_gnn_get_params(self._h, out.ctypes.data))
        return out

    @params.setter
    def params(self, value: np.ndarray) -> None:
        v = np.ascontiguousarray(value, np.float32)
        if v.size != self.num_params:
            raise ValueError("parameter count mismatch")
        _lib.check(self._lib.mc_gnn_set_params(self._h, v.ctypes.data))

    def predict(self, model: Model):
        lp = model.to_struct()
        x = np.zeros(model.num_cols)
        y = np.zeros(model.num_rows)
        lw = C.c_double(0)
        _lib.check(self._lib.mc_gnn_predict(self._h, C.addressof(lp), x.ctypes.data, y.ctypes.data,
                                            C.byref(lw)))
        return x, y, lw.value

    def loss_and_grad(self, t: Target):
        lp = t.model.to_struct()
        loss = C.c_double(0)
        g = np.zeros(self.num_params, np.float32)
        _lib.check(self._lib.mc_gnn_loss_and_grad(self._h, C.addressof(lp), t.x.ctypes.data,
                                                  t.y.ctypes.data, t.log_omega, C.byref(loss),
                                                  g.ctypes.data))
        return loss.value, g

    def train_step(self, t: Target, lr: float) -> float:
        lp = t.model.to_struct()
        loss = C.c_double(0)
        _lib.check(self._lib.mc_gnn_train_step(self._h, C.addressof(lp), t.x.ctypes.data,
                                               t.y.ctypes.data, t.log_omega, lr, C.byref(loss)))
        return loss.value

    def fit(self, data: list, epochs: int = 3, lr: float = 1e-3, seed: int = 0, log=None) -> list:
        rng = np.random.default_rng(seed)
        history = []
        for ep in range(epochs):
            order = rng.permutation(len(data))
            losses = [self.train_step(data[i], lr * (0.5 ** ep)) for i in order]
            history.append(float(np.mean(losses)))
            if log:
                log(f"epoch {ep}: mean loss {history[-1]:.5f}")
        return history

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, rounds=self.rounds)

    def load(self, path: str) -> None:
        z = np.load(path)
        self.params = z["params"]


def b_scale(model: Model) -> float:
    """max(1, |finite row bounds|_inf): the network's primal unit."""
    s = 1.0
    for a in (model.row_lower, model.row_upper):
        f = a[np.isfinite(a)]
        if len(f):
            s = max(s, float(np.abs(f).max()))
    return s


def shaped_primal(model: Model, x: np.ndarray, margin: float = 0.05) -> np.ndarray:
    """Training target for the primal: entries at a finite bound are pushed
    `margin` (in units of |b|_inf) beyond it, so that the prediction lands
    outside the box there and the engine's projection makes it exact.  The
    reference's dual residual sums |x_j - proj(x_j - g_j)|^2 over all columns,
    so exact bound values matter for a warm start to score well."""
    t = x.copy()
    tol = 1e-6 * b_scale(model)
    m = margin * b_scale(model)
    lo, hi = model.var_lower, model.var_upper
    at_lo = np.isfinite(lo) & (x <= lo + tol)
    at_hi = np.isfinite(hi) & (x >= hi - tol)
    t[at_lo] = lo[at_lo] - m
    t[at_hi] = hi[at_hi] + m
    return t


def solve_targets(ctx: Context, models: list, options: PdlpOptions, batch: int = 128,
                  margin: float = 0.05) -> list:
    """GPU PDLP solutions of `models` (batched) as training targets."""
    out = []
    for s in range(0, len(models), batch):
        chunk = models[s:s + batch]
        for m, r in zip(chunk, ctx.solve_batch(chunk, options)):
            out.append(Target(m, shaped_primal(m, r.primal, margin) if margin > 0 else r.primal, r.dual,
                              math.log(max(r.extra["final_primal_weight"], 1e-12)), r))
    return out


def solve_warm(ctx: Context, net: WarmStartNet, model: Model, options: PdlpOptions,
               guard: bool = True, use_weight: bool = False) -> PdlpResult:
    """Solve from the network's prediction, guarded by the engine (guard=False
    forces the prediction, for measuring what it does on its own).

    The predicted point is used with the reference's own initial primal weight
    (derived from the scaled norms of c and b): on B200 the predicted weight,
    trained on each solve's final weight, costs iterations (on held-out
    config-0 family LPs at 1e-8: 844 iterations from the predicted weight
    alone, 869 from the solve's own final weight, 736 cold), while the
    predicted point with the derived weight takes 676.  use_weight=True passes
    the predicted weight too."""
    x, y, lw = net.predict(model)
    o = PdlpOptions(**{k: getattr(options, k) for k in options.__dataclass_fields__})
    o.initial_primal, o.initial_dual = x, y
    o.initial_primal_weight = float(min(max(math.exp(lw), 1e-6), 1e6)) if use_weight else 0.0
    o.warm_start_guard = guard
    return ctx.solve(model, o)


def main() -> None:
    from . import generators
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--test", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--target-iterations", type=int, default=20000)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--max-iterations", type=int, default=100000)
    ap.add_argument("--margin", type=float, default=0.05)
    ap.add_argument("--size", type=int, nargs=2, default=[50, 500],
                    help="suppliers and customers uniform in [lo, hi] (the workload: 50 500)")
    ap.add_argument("--family", default="transport", choices=["transport", "random"],
                    help="transport: S, D in --size; random: the config-0 generator with m in --size, "
                         "n = 3m, 6 nonzeros per column")
    ap.add_argument("--out", default="")
    args = ap.parse_args()
    ctx = Context(0)
    t0 = time.time()
    def family(seed):
        if args.family == "random":
            m = generators.uniform_int(seed, 0, *args.size)
            return generators.random_lp(seed, m, 3 * m, 6)
        S = generators.uniform_int(seed, 0, *args.size)
        D = generators.uniform_int(seed, 1, *args.size)
        return generators.transport(seed, S, D)
    train_models = [family(seed) for seed in range(args.train)]
    topt = PdlpOptions(max_iterations=args.target_iterations)
    topt.set_tolerance(1e-8)
    data = solve_targets(ctx, train_models, topt, margin=args.margin)
    t_data = time.time() - t0
    net = WarmStartNet(0, 3, 0)
    t0 = time.time()
    hist = net.fit(data, epochs=args.epochs, lr=args.lr, log=print)
    t_train = time.time() - t0
    if args.out:
        net.save(args.out)
    eopt = PdlpOptions(max_iterations=args.max_iterations)
    eopt.set_tolerance(args.tol)
    rows = []
    for seed in range(10_000_000, 10_000_000 + args.test):
        m = family(seed)
        cold = ctx.solve(m, eopt)
        warm = solve_warm(ctx, net, m, eopt)
        forced = solve_warm(ctx, net, m, eopt, guard=False)
        rows.append(dict(m=m.num_rows, n=m.num_cols, cold_it=cold.iterations, warm_it=warm.iterations,
                         cold_ms=cold.total_ms, warm_ms=warm.total_ms, cold_status=cold.status.name,
                         warm_status=warm.status.name, used=warm.extra["warm_start_used"],
                         forced_it=forced.iterations, forced_status=forced.status.name,
                         warm_score=warm.extra["warm_start_score"], cold_score=warm.extra["cold_start_score"],
                         cold_kkt=max(cold.primal_infeasibility, cold.dual_infeasibility, cold.duality_gap),
                         warm_kkt=max(warm.primal_infeasibility, warm.dual_infeasibility, warm.duality_gap)))
    summary = dict(train=args.train, test=args.test, epochs=args.epochs, loss=hist, data_s=t_data,
                   train_s=t_train, tol=args.tol,
                   cold_optimal=sum(r["cold_status"] == "optimal" for r in rows),
                   warm_optimal=sum(r["warm_status"] == "optimal" for r in rows),
                   warm_used=sum(r["used"] for r in rows),
                   mean_cold_it=float(np.mean([r["cold_it"] for r in rows])),
                   mean_warm_it=float(np.mean([r["warm_it"] for r in rows])),
                   mean_forced_it=float(np.mean([r["forced_it"] for r in rows])),
                   forced_optimal=sum(r["forced_status"] == "optimal" for r in rows),
                   size=args.size,
                   mean_cold_ms=float(np.mean([r["cold_ms"] for r in rows])),
                   mean_warm_ms=float(np.mean([r["warm_ms"] for r in rows])),
                   median_start_score_ratio=float(np.median([r["warm_score"] / max(r["cold_score"], 1e-300)
                                                             for r in rows])))
    print(json.dumps(summary))
    if args.out:
        with open(args.out + ".json", "w") as f:
            json.dump(dict(summary=summary, rows=rows), f)


if __name__ == "__main__":
    main()
