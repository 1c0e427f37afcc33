"""The boundary compiled into the reference solver.

markov-zip1_b200/binding/Makefile links the reference's own sources (its
solve_pdlp compiled as solve_pdlp_cpu, its CLI main renamed) with the GPU
module markov-zip1_b200/binding/*.cpp and lib/libmcpdlp.so into
markov-zip1_b200/binding/_build/:

* pdlp_test -- the reference's tests/pdlp_test.cpp (asserts on).  With
  MARKOV_CERO_PDLP_BACKEND=gpu every solve_pdlp of the process goes to the
  GPU engine; with no visible GPU that must fail loudly (no CPU fallback).
* ruiz_scaling_test -- the reference's tests/ruiz_scaling_test.cpp with its
  equilibrate() calls routed to the device (binding/ruiz_gpu.cpp).
* presolve_test -- the reference's tests/presolve_test.cpp with its
  presolve()/postsolve() calls routed to the device presolve
  (binding/presolve_gpu.cpp); with no visible GPU it must fail loudly.
* markov-cero-solve -- the reference CLI with `--engine pdlp-gpu`
  (apps/markov_cero_solve.cpp:136-189), checked on the ADR-P3-05 model
  (docs/decisions/ADR-P3-05-pdhg-pdlp.md:11-23: objective -9.0000013 at
  tolerance 1e-6, optimal, verified) and on Netlib fixtures against their
  published optima.

The MPS files are written here from the committed fixtures (parsed by the
reference's own reader when they were made), so a machine that runs these
tests needs no reference checkout; the binaries are built where the
reference sources are.
"""
from __future__ import annotations

import json
import math
import os
import subprocess
from pathlib import Path

import pytest

from test_oracle import GOLDEN, load_model

BUILD = Path(__file__).resolve().parent.parent / "markov-zip1_b200" / "binding" / "_build"
PDLP_TEST = BUILD / "pdlp_test"
CLI = BUILD / "markov-cero-solve"
PRESOLVE_TEST = BUILD / "presolve_test"
RUIZ_TEST = BUILD / "ruiz_scaling_test"

needs_build = pytest.mark.skipif(not (PDLP_TEST.exists() and CLI.exists()),
                                 reason="integration build absent (needs the reference sources)")


def write_mps(model, path: Path) -> None:
    """Free-format MPS of a fixture model (rows E/L/G with RANGES for boxed
    rows; explicit bounds per column)."""
    m, n = model.num_rows, model.num_cols
    assert model.objective_offset == 0.0
    num = lambda v: repr(float(v))  # noqa: E731  shortest round-trip form
    kinds, rhs, ranges = [], {}, {}
    for i in range(m):
        lo, hi = model.row_lower[i], model.row_upper[i]
        if lo == hi:
            kinds.append("E")
            rhs[i] = lo
        elif math.isinf(lo) and math.isinf(hi):
            kinds.append("N")
        elif math.isinf(lo):
            kinds.append("L")
            rhs[i] = hi
        elif math.isinf(hi):
            kinds.append("G")
            rhs[i] = lo
        else:
            kinds.append("G")
            rhs[i] = lo
            ranges[i] = hi - lo
    out = ["NAME FIXTURE", "ROWS", " N COST"]
    out += [f" {k} R{i}" for i, k in enumerate(kinds)]
    out.append("COLUMNS")
    for j in range(n):
        if model.objective[j] != 0.0:
            out.append(f" C{j} COST {num(model.objective[j])}")
        for p in range(model.col_start[j], model.col_start[j + 1]):
            out.append(f" C{j} R{model.row_index[p]} {num(model.value[p])}")
    out.append("RHS")
    out += [f" RHS R{i} {num(v)}" for i, v in rhs.items() if v != 0.0]
    if ranges:
        out.append("RANGES")
        out += [f" RNG R{i} {num(v)}" for i, v in ranges.items()]
    out.append("BOUNDS")
    for j in range(n):
        lo, hi = model.var_lower[j], model.var_upper[j]
        if lo == hi:
            out.append(f" FX BND C{j} {num(lo)}")
            continue
        if math.isinf(lo) and math.isinf(hi):
            out.append(f" FR BND C{j}")
            continue
        out.append(f" MI BND C{j}" if math.isinf(lo) else f" LO BND C{j} {num(lo)}")
        if not math.isinf(hi):
            out.append(f" UP BND C{j} {num(hi)}")
    out.append("ENDATA")
    path.write_text("\n".join(out) + "\n")


def run(cmd, env_extra=None, timeout=300):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([str(c) for c in cmd], capture_output=True, text=True, env=env, timeout=timeout)


# ------------------------------------------------------------- CPU (here)
@needs_build
def test_reference_pdlp_test_cpu_backend_through_dispatch():
    r = run([PDLP_TEST])
    assert r.returncode == 0, r.stderr
    assert "All PDLP unit tests PASSED" in r.stdout


@pytest.mark.skipif(not PRESOLVE_TEST.exists(), reason="integration build absent (needs the reference sources)")
def test_reference_presolve_test_without_device_fails_loudly():
    r = run([PRESOLVE_TEST], {"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode != 0
    assert "no CPU fallback" in (r.stdout + r.stderr)


@pytest.mark.skipif(not RUIZ_TEST.exists(), reason="integration build absent (needs the reference sources)")
def test_reference_ruiz_test_without_device_fails_loudly():
    r = run([RUIZ_TEST], {"CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode != 0
    assert "no CPU fallback" in (r.stdout + r.stderr)


@needs_build
def test_gpu_request_without_device_fails_loudly():
    # a GPU request never falls back to the CPU solver
    r = run([PDLP_TEST], {"MARKOV_CERO_PDLP_BACKEND": "gpu", "CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode != 0
    assert "no CPU fallback" in (r.stdout + r.stderr)


@needs_build
def test_cli_engine_pdlp_gpu_without_device_is_a_numerical_failure(tmp_path):
    mps = tmp_path / "tiny_simplex.mps"
    write_mps(load_model("tiny_simplex"), mps)
    r = run([CLI, mps, "--engine", "pdlp-gpu", "--tolerance", "1e-6"], {"CUDA_VISIBLE_DEVICES": ""})
    out = json.loads(r.stdout.strip().splitlines()[0])
    assert out["status"] == "NumericalFailure" and out["backend"] == "gpu"
    assert "no CPU fallback" in out["error"]
    assert r.returncode != 0


@needs_build
def test_cli_cpu_pdlp_on_written_fixture_matches_adr(tmp_path):
    # the MPS writer round-trips the ADR model through the reference's reader
    mps = tmp_path / "tiny_simplex.mps"
    write_mps(load_model("tiny_simplex"), mps)
    r = run([CLI, mps, "--engine", "pdlp", "--tolerance", "1e-6"])
    out = json.loads(r.stdout.strip().splitlines()[0])
    assert r.returncode == 0 and out["status"] == "Optimal" and out["verified"]
    assert abs(out["objective"] - (-9.0000013)) < 1e-6


@needs_build
def test_cli_cpu_pdlp_on_written_netlib_matches_golden(tmp_path):
    # written fixture -> reference reader -> reference CPU PDLP: the golden result
    mps = tmp_path / "afiro.mps"
    write_mps(load_model("netlib_afiro"), mps)
    r = run([CLI, mps, "--engine", "pdlp", "--tolerance", "1e-8"])
    out = json.loads(r.stdout.strip().splitlines()[0])
    gold = GOLDEN["models"]["netlib_afiro"]["results"]["1e-08"]
    assert out["status"] == "Optimal" and out["lp_iterations"] == gold["iterations"]
    assert out["objective"] == gold["objective"]


# ------------------------------------------------------------------- GPU
@pytest.mark.skipif(not PRESOLVE_TEST.exists(), reason="integration build absent (needs the reference sources)")
@pytest.mark.gpu
def test_reference_presolve_test_on_gpu():
    """tests/presolve_test.cpp (asserts on): infeasible empty row, unbounded
    empty column, the row-singleton reduction and its postsolve (x = (3, 4),
    objective 50), and the blend model with presolve against the simplex
    without it -- every presolve/postsolve on the device."""
    r = run([PRESOLVE_TEST])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "presolve tests passed" in r.stdout


@pytest.mark.skipif(not RUIZ_TEST.exists(), reason="integration build absent (needs the reference sources)")
@pytest.mark.gpu
def test_reference_ruiz_test_on_gpu():
    """tests/ruiz_scaling_test.cpp (asserts on): the equilibrated norms, and
    the blend model scaled on the device, solved by the reference simplex and
    unscaled, against the unscaled solve."""
    r = run([RUIZ_TEST])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ruiz scaling tests passed" in r.stdout


@needs_build
@pytest.mark.gpu
def test_reference_pdlp_test_on_gpu():
    r = run([PDLP_TEST], {"MARKOV_CERO_PDLP_BACKEND": "gpu"})
    assert r.returncode == 0, r.stdout + r.stderr
    assert "All PDLP unit tests PASSED" in r.stdout


@needs_build
@pytest.mark.gpu
def test_cli_engine_pdlp_gpu_on_adr_model(tmp_path):
    mps = tmp_path / "tiny_simplex.mps"
    write_mps(load_model("tiny_simplex"), mps)
    r = run([CLI, mps, "--engine", "pdlp-gpu", "--tolerance", "1e-6"])
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[0])
    assert out["status"] == "Optimal" and out["verified"] and out["original_verified"]
    assert out["backend"] == "gpu" and out["kernel_ms"] > 0.0
    assert abs(out["objective"] - (-9.0)) < 1e-5
    assert "[gpu H2D=" in r.stderr and "VERIFIED" in r.stderr


@needs_build
@pytest.mark.gpu
@pytest.mark.parametrize("name", ["netlib_afiro", "netlib_sc50a", "netlib_sc50b", "netlib_sc105"])
def test_cli_engine_pdlp_gpu_on_netlib(tmp_path, name):
    mps = tmp_path / f"{name}.mps"
    model = load_model(name)
    write_mps(model, mps)
    r = run([CLI, mps, "--engine", "pdlp-gpu", "--tolerance", "1e-8"])
    assert r.returncode == 0, r.stdout + r.stderr
    out = json.loads(r.stdout.strip().splitlines()[0])
    assert out["status"] == "Optimal" and out["verified"]
    gold = GOLDEN["models"][name]["results"]["1e-08"]
    assert abs(out["objective"] - gold["objective"]) <= 1e-6 * max(1.0, abs(gold["objective"]))
    published = GOLDEN["netlib_optimal"][name]
    assert abs(out["objective"] - published) <= 1e-5 * max(1.0, abs(published))
