"""Generate the golden fixtures of the PDLP path from the reference itself.

Run in a checkout where the reference sources exist (oracle/Makefile builds
oracle/_ref/libref_pdlp.so from them):

    python tests/golden/make_golden.py

Writes, next to this script:
  * <name>.npz   -- small LPs in CSC form (the reference's PDLP unit-test
                   models, tests/pdlp_test.cpp:12-129; the ADR-P3-05 model
                   examples/phase3/tiny_simplex.mps; Netlib models from
                   data/netlib that the reference PDLP solves), parsed by the
                   reference's own MPS reader;
  * golden.json  -- the reference solve_pdlp result on each (status,
                   iterations, objective, residuals, SHA-256 of the primal and
                   dual bytes) at 1e-4 and 1e-8, the same for seeded synthetic
                   LPs (regenerated from their seed, pinned by a SHA-256 of the
                   generated arrays), equilibrate_model digests, and the
                   reference primal simplex's optimum of small seeded
                   transportation LPs (the FP64 optimum of that family, which
                   has no analytic one), and the published optimal objectives of
                   the Netlib fixtures (the reference's scripts/run_netlib.py).

    python tests/golden/make_golden.py --only simplex   # refresh that section
    python tests/golden/make_golden.py --only netlib    # the published Netlib optima
    python tests/golden/make_golden.py --only scale     # larger seeded LPs (minutes)
    python tests/golden/make_golden.py --only presolve  # presolve / postsolve of canonical models

The ``presolve`` section holds the reference's presolve and postsolve
(src/presolve/presolve.cpp) on canonical models: the models of the
reference's presolve unit tests (tests/presolve_test.cpp:30-96, written out
as canon_*.npz), the canonical form (sparse_canonicalize) of the Netlib
fixtures, and seeded generated models (mcpdlp.generators.presolve_lp, pinned
by a SHA-256 of the generated arrays) in all four outcomes; per model the
status, message, statistics, objective offset and SHA-256 digests of the
reduced model, the record stack and the maps, and of postsolve's primal and
dual for a seeded reduced solution.

The ``scale`` section holds the reference solve_pdlp on seeded LPs far above
the unit-test sizes: the 40M-nonzero LP's generator at m = 200,000,
n = 500,000, 8 nonzeros per column (4M nonzeros), and the precision-stress
generator at m = 20,000, n = 60,000, 10 nonzeros per column (600k nonzeros),
each at 1e-4 and 1e-8 (one process per solve; about five minutes of CPU).
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "markov-zip1_b200"))
sys.path.insert(0, str(ROOT / "oracle"))

from mcpdlp import _abi, generators  # noqa: E402
from mcpdlp.model import Model, from_triplets  # noqa: E402
import oracle as orc  # noqa: E402

REF = orc.REFERENCE_SOURCES   # MC_REFERENCE_DIR, else /root/reference
NETLIB = ["afiro", "sc50a", "sc50b", "sc105", "blend", "recipe", "scsd1", "scsd6"]
SYNTHETIC = [  # (name, seed, m, n, k, family)
    ("config0_s1", 1, 1000, 3000, 6, "standard"),
    ("config0_s2", 2, 1000, 3000, 6, "standard"),
    ("config0_s3", 3, 1000, 3000, 6, "standard"),
    ("small_s7", 7, 200, 600, 6, "standard"),
    ("precision_s1", 1, 300, 900, 10, "precision"),
]
TOLS = [1e-4, 1e-8]
SCALE = [  # (name, seed, m, n, k, family)
    ("standard_4m", 1, 200_000, 500_000, 8, "standard"),
    ("precision_600k", 1, 20_000, 60_000, 10, "precision"),
]
TRANSPORT = [  # (seed, suppliers, customers): within the simplex's dense limits
    (1, 20, 30), (2, 20, 30), (3, 25, 35), (4, 30, 40), (5, 40, 50), (6, 40, 60),
]


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def model_digest(m: Model) -> str:
    return sha(m.col_start, m.row_index, m.value, m.objective, m.var_lower, m.var_upper,
               m.row_lower, m.row_upper)


def blend_lp() -> Model:
    # tests/pdlp_test.cpp:12-48: min -x1 - 2 x2, x1 + x2 <= 4, x1 <= 3, x2 <= 3, 0 <= x <= 10
    inf = np.inf
    return from_triplets(3, 2, [0, 0, 1, 2], [0, 1, 0, 1], [1.0, 1.0, 1.0, 1.0],
                         objective=[-1.0, -2.0], var_lower=[0.0, 0.0], var_upper=[10.0, 10.0],
                         row_lower=[-inf, -inf, -inf], row_upper=[4.0, 3.0, 3.0], name="blend_pdlp")


def equality_lp() -> Model:
    # tests/pdlp_test.cpp:82-109: min x1 + x2, x1 + x2 = 5, 0 <= x <= 5
    return from_triplets(1, 2, [0, 0], [0, 1], [1.0, 1.0], objective=[1.0, 1.0],
                         var_lower=[0.0, 0.0], var_upper=[5.0, 5.0], row_lower=[5.0],
                         row_upper=[5.0], name="equality_pdlp")


def save_model(m: Model, name: str) -> None:
    np.savez_compressed(HERE / f"{name}.npz", num_rows=m.num_rows, num_cols=m.num_cols,
                        col_start=m.col_start, row_index=m.row_index, value=m.value,
                        objective=m.objective, var_lower=m.var_lower, var_upper=m.var_upper,
                        row_lower=m.row_lower, row_upper=m.row_upper,
                        objective_offset=m.objective_offset, objective_sense=int(m.objective_sense))


def opts(tol: float, max_iter: int = 100000):
    o = _abi.default_options_struct()
    o.primal_tolerance = o.dual_tolerance = o.gap_tolerance = tol
    o.max_iterations = max_iter
    return o


def record(ref, m: Model) -> dict:
    out = {}
    for tol in TOLS:
        r = ref.solve(m, opts(tol))
        out[f"{tol:g}"] = dict(status=r.status, iterations=r.iterations, objective=r.objective,
                               primal_infeasibility=r.primal_infeasibility,
                               dual_infeasibility=r.dual_infeasibility, duality_gap=r.duality_gap,
                               primal_sha256=sha(r.primal), dual_sha256=sha(r.dual),
                               message=r.message)
    return out


def netlib_optima() -> dict:
    """The published Netlib optimal objectives the reference's benchmark
    script carries (scripts/run_netlib.py:19-93), for the fixtures here."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("run_netlib", REF / "scripts" / "run_netlib.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return {f"netlib_{k}": float(v["optimal"]) for k, v in mod.NETLIB_BENCHMARKS.items()
            if k in NETLIB and "optimal" in v}


def simplex_section(ref) -> dict:
    out = {}
    for seed, S, D in TRANSPORT:
        m = generators.transport(seed, S, D)
        r = ref.simplex(m)
        p = ref.solve(m, opts(1e-8))
        out[f"transport_{seed}_{S}x{D}"] = dict(seed=seed, suppliers=S, customers=D,
                                                digest=model_digest(m), status=r["status"],
                                                objective=r["objective"],
                                                iterations=r["iterations"],
                                                pdlp_1e8=dict(status=p.status, iterations=p.iterations,
                                                              objective=p.objective))
        print("simplex", seed, S, D, r["status"], r["objective"], "pdlp", p.status, p.iterations)
    return out


def _scale_job(job) -> dict:
    """One reference solve of a SCALE model at one tolerance (own process)."""
    import time
    name, seed, m_, n_, k_, fam, tol = job
    ref = orc.ReferencePdlp()
    m = generators.random_lp(seed, m_, n_, k_, fam)
    t0 = time.perf_counter()
    r = ref.solve(m, opts(tol))
    wall = time.perf_counter() - t0
    opt = m.info["optimum"]
    out = dict(status=r.status, iterations=r.iterations, objective=r.objective,
               primal_infeasibility=r.primal_infeasibility, dual_infeasibility=r.dual_infeasibility,
               duality_gap=r.duality_gap, restarts=r.restarts, wall_s=wall,
               objective_rel_err_vs_analytic=abs(r.objective - opt) / abs(opt))
    print(name, f"{tol:g}", out, flush=True)
    return dict(name=name, tol=f"{tol:g}", digest=model_digest(m), optimum=opt, result=out)


def scale_section() -> dict:
    import multiprocessing as mp
    jobs = [(*case, tol) for case in SCALE for tol in TOLS]
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        done = pool.map(_scale_job, jobs)
    out = {}
    for name, seed, m_, n_, k_, fam in SCALE:
        mine = [d for d in done if d["name"] == name]
        out[name] = dict(seed=seed, m=m_, n=n_, k=k_, family=fam, digest=mine[0]["digest"],
                         optimum=mine[0]["optimum"], results={d["tol"]: d["result"] for d in mine})
    return out


PRESOLVE_GENERATED = [  # (name, seed, m, n, kind)
    ("gen_feasible_s1", 1, 200, 300, "feasible"),
    ("gen_feasible_s2", 2, 400, 500, "feasible"),
    ("gen_feasible_s3", 3, 120, 150, "feasible"),
    ("gen_infeasible_row_s4", 4, 200, 300, "infeasible_row"),
    ("gen_infeasible_singleton_s5", 5, 200, 300, "infeasible_singleton"),
    ("gen_unbounded_s6", 6, 200, 300, "unbounded"),
]


def presolve_unit_models() -> list:
    """The canonical models of the reference's presolve tests
    (tests/presolve_test.cpp:30-96); the blend LP there goes through
    sparse_canonicalize as in the test."""
    from mcpdlp.presolve import CanonicalModel
    out = [
        ("canon_empty_row", CanonicalModel(1, 1, [0, 0], [], [], [10.0], [1.0])),
        ("canon_empty_column", CanonicalModel(1, 1, [0, 0], [], [], [0.0], [-5.0])),
        ("canon_row_singleton", CanonicalModel(2, 2, [0, 2, 3], [0, 1, 1], [2.0, 1.0, 1.0], [6.0, 7.0],
                                               [10.0, 5.0])),
    ]
    return out


def presolve_blend_lp() -> Model:
    # tests/presolve_test.cpp:12-28: min 40 A + 30 B, A + B = 100, 0.01 A + 0.03 B <= 2, A, B >= 0
    inf = np.inf
    return from_triplets(2, 2, [0, 0, 1, 1], [0, 1, 0, 1], [1.0, 1.0, 0.01, 0.03], objective=[40.0, 30.0],
                         var_lower=[0.0, 0.0], var_upper=[inf, inf], row_lower=[100.0, -inf],
                         row_upper=[100.0, 2.0], name="presolve_blend")


def save_canonical(c, name: str) -> None:
    np.savez_compressed(HERE / f"{name}.npz", num_rows=c.num_rows, num_cols=c.num_cols, col_start=c.col_start,
                        row_index=c.row_index, value=c.value, rhs=c.rhs, objective=c.objective,
                        objective_offset=c.objective_offset)


def canonical_digest(c) -> str:
    return sha(np.array([c.num_rows, c.num_cols]), c.col_start, c.row_index, c.value, c.rhs, c.objective,
               np.array([c.objective_offset]))


def presolve_record(ref, c) -> dict:
    import dataclasses
    try:
        r = ref.presolve(c)
    except ValueError as e:
        return dict(error=str(e))
    st = r.stack
    out = dict(status=int(r.status), message=r.message, statistics=dataclasses.asdict(r.statistics),
               objective_offset=r.model.objective_offset, model_sha256=canonical_digest(r.model),
               stack_sha256=sha(st.kind, st.index, st.variable, st.value, st.value2, st.incident_start,
                                st.incident_row, st.incident_coefficient),
               maps_sha256=sha(st.presolved_to_original_rows, st.presolved_to_original_cols))
    if r.status == 0:
        rng = np.random.default_rng(7)
        rx = rng.uniform(0.0, 2.0, r.model.num_cols)
        ry = rng.normal(size=r.model.num_rows)
        p = ref.postsolve(c, rx, ry)
        out["post"] = dict(seed=7, primal_sha256=sha(p.primal), dual_sha256=sha(p.dual), objective=p.objective)
    return out


def presolve_section(ref) -> dict:
    out = {}
    cases = presolve_unit_models()
    cases.append(("canon_presolve_blend", ref.canonical_model(presolve_blend_lp())))
    for name in NETLIB:
        cases.append((f"canon_netlib_{name}", ref.canonical_model(ref.parse_mps(REF / "data/netlib" / f"{name}.mps"))))
    for name, c in cases:
        save_canonical(c, name)
        out[name] = dict(file=f"{name}.npz", digest=canonical_digest(c), m=c.num_rows, n=c.num_cols, nnz=c.nnz,
                         result=presolve_record(ref, c))
        print(name, out[name]["result"].get("status"), out[name]["result"].get("statistics"))
    for name, seed, m_, n_, kind in PRESOLVE_GENERATED:
        c = generators.presolve_lp(seed, m_, n_, kind=kind)
        out[name] = dict(seed=seed, m=m_, n=n_, kind=kind, digest=canonical_digest(c), result=presolve_record(ref, c))
        print(name, out[name]["result"].get("status"), out[name]["result"].get("message"))
    return out


def main() -> None:
    orc.build(reference=True)
    ref = orc.ReferencePdlp()
    if "--only" in sys.argv:
        golden = json.loads((HERE / "golden.json").read_text())
        what = sys.argv[sys.argv.index("--only") + 1]
        if what == "simplex":
            golden["simplex"] = simplex_section(ref)
        elif what == "netlib":
            golden["netlib_optimal"] = netlib_optima()
        elif what == "scale":
            golden["scale"] = scale_section()
        elif what == "presolve":
            golden["presolve"] = presolve_section(ref)
        (HERE / "golden.json").write_text(json.dumps(golden, indent=1, sort_keys=True))
        return
    golden = {"models": {}, "synthetic": {}, "ruiz": {}}
    fixtures = [blend_lp(), equality_lp(), ref.parse_mps(REF / "examples/phase3/tiny_simplex.mps")]
    fixtures[2].name = "tiny_simplex"
    for name in NETLIB:
        mm = ref.parse_mps(REF / "data/netlib" / f"{name}.mps")
        mm.name = f"netlib_{name}"
        fixtures.append(mm)
    for m in fixtures:
        save_model(m, m.name)
        golden["models"][m.name] = dict(file=f"{m.name}.npz", m=m.num_rows, n=m.num_cols,
                                        nnz=m.nnz, digest=model_digest(m), results=record(ref, m))
        print(m.name, {k: (v["status"], v["iterations"], v["objective"])
                       for k, v in golden["models"][m.name]["results"].items()})
    for name, seed, mm, nn, kk, fam in SYNTHETIC:
        m = generators.random_lp(seed, mm, nn, kk, fam)
        golden["synthetic"][name] = dict(seed=seed, m=mm, n=nn, k=kk, family=fam,
                                         digest=model_digest(m), optimum=m.info["optimum"],
                                         results=record(ref, m))
        print(name, {k: (v["status"], v["iterations"], v["objective"])
                     for k, v in golden["synthetic"][name]["results"].items()})
        e = ref.equilibrate(m, 10)
        golden["ruiz"][name] = dict(iterations=e["iterations"], converged=e["converged"],
                                    value_sha256=sha(e["value"]),
                                    scales_sha256=sha(e["row_scale"], e["col_scale"]),
                                    bounds_sha256=sha(e["objective"], e["var_lower"], e["var_upper"],
                                                      e["row_lower"], e["row_upper"]))
    golden["simplex"] = simplex_section(ref)
    golden["netlib_optimal"] = netlib_optima()
    golden["scale"] = scale_section()
    golden["presolve"] = presolve_section(ref)
    (HERE / "golden.json").write_text(json.dumps(golden, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
