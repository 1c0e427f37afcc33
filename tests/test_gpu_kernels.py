"""Kernel-level parity through the C ABI (needs a B200).

* device CSC -> CSR transpose: bit-exact against a CPU transpose (rows in
  ascending column order), including long rows (block sort paths);
* Ruiz equilibration: bit-exact against the oracle (values of both copies,
  scales, bounds, objective, pass count);
* SpMV: within 1e-13 of the oracle relative to sum |a_ij x_j|.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import mcpdlp
from mcpdlp import _lib, generators
from mcpdlp.model import Model
from test_oracle import synthetic

pytestmark = pytest.mark.gpu


def cpu_transpose(m: Model):
    """CSR(A) with ascending columns per row (numpy, stable)."""
    cols = np.repeat(np.arange(m.num_cols, dtype=np.int32), np.diff(m.col_start))
    order = np.lexsort((cols, m.row_index))
    row_start = np.zeros(m.num_rows + 1, np.int64)
    np.add.at(row_start, m.row_index.astype(np.int64) + 1, 1)
    return np.cumsum(row_start).astype(np.int32), cols[order], m.value[order]


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_transpose(ctx, m: Model):
    import torch
    rs = torch.zeros(m.num_rows + 1, dtype=torch.int32, device="cuda")
    ci = torch.zeros(max(m.nnz, 1), dtype=torch.int32, device="cuda")
    cv = torch.zeros(max(m.nnz, 1), dtype=torch.float64, device="cuda")
    cs, ri, v = dev(m.col_start), dev(m.row_index), dev(m.value)
    _lib.check(_lib.engine().mc_csc_to_csr(ctx.handle, m.num_rows, m.num_cols, m.nnz, cs.data_ptr(),
                                           ri.data_ptr(), v.data_ptr(), rs.data_ptr(), ci.data_ptr(),
                                           cv.data_ptr()))
    return rs.cpu().numpy(), ci.cpu().numpy()[: m.nnz], cv.cpu().numpy()[: m.nnz]


def long_row_model(seed: int, row_lengths) -> Model:
    """Rows of chosen lengths (to reach the shared-memory and rank sorts)."""
    rng = np.random.default_rng(seed)
    m = len(row_lengths)
    n = max(row_lengths) + 5
    rows, cols = [], []
    for i, L in enumerate(row_lengths):
        for j in rng.choice(n, size=L, replace=False):
            rows.append(i); cols.append(int(j))
    vals = rng.normal(size=len(rows))
    vals[vals == 0] = 1.0
    return mcpdlp.from_triplets(m, n, rows, cols, vals, objective=np.ones(n), var_lower=np.zeros(n),
                                var_upper=np.ones(n), row_lower=np.zeros(m), row_upper=np.ones(m))


@pytest.mark.parametrize("case", ["config0", "precision", "transport", "long_rows", "single"])
def test_transpose_bit_exact(gpu_ctx, case):
    if case == "config0":
        m = synthetic("config0_s1")
    elif case == "precision":
        m = synthetic("precision_s1")
    elif case == "transport":
        m = generators.transport(3, 60, 80)
    elif case == "long_rows":
        m = long_row_model(0, [3, 40, 33, 700, 4096, 4097, 9000, 1, 0, 32])
    else:
        m = mcpdlp.from_triplets(1, 1, [0], [0], [2.0], objective=[1.0], var_lower=[0.0],
                                 var_upper=[1.0], row_lower=[0.0], row_upper=[1.0])
    rs, ci, cv = gpu_transpose(gpu_ctx, m)
    ers, eci, ecv = cpu_transpose(m)
    assert np.array_equal(rs, ers)
    assert np.array_equal(ci, eci)
    assert np.array_equal(cv, ecv)


@pytest.mark.parametrize("name", ["config0_s1", "precision_s1", "small_s7"])
def test_ruiz_bit_exact(gpu_ctx, oracle, name):
    import torch
    m = synthetic(name)
    exp = oracle.equilibrate(m, 10)
    rs, ci, cv = gpu_transpose(gpu_ctx, m)
    d_rs, d_ci, d_cv = dev(rs), dev(ci), dev(cv)
    cs, ri, v = dev(m.col_start), dev(m.row_index), dev(m.value)
    obj, vl, vu = dev(m.objective), dev(m.var_lower), dev(m.var_upper)
    rl, ru = dev(m.row_lower), dev(m.row_upper)
    row_scale = torch.zeros(m.num_rows, dtype=torch.float64, device="cuda")
    col_scale = torch.zeros(m.num_cols, dtype=torch.float64, device="cuda")
    it = C.c_int64(0)
    _lib.check(_lib.engine().mc_ruiz_equilibrate(
        gpu_ctx.handle, m.num_rows, m.num_cols, m.nnz, cs.data_ptr(), ri.data_ptr(), v.data_ptr(),
        d_rs.data_ptr(), d_ci.data_ptr(), d_cv.data_ptr(), obj.data_ptr(), vl.data_ptr(),
        vu.data_ptr(), rl.data_ptr(), ru.data_ptr(), 10, row_scale.data_ptr(), col_scale.data_ptr(),
        C.addressof(it)))
    assert it.value == exp["iterations"]
    assert np.array_equal(v.cpu().numpy(), exp["value"])
    assert np.array_equal(row_scale.cpu().numpy(), exp["row_scale"])
    assert np.array_equal(col_scale.cpu().numpy(), exp["col_scale"])
    for t, k in ((obj, "objective"), (vl, "var_lower"), (vu, "var_upper"), (rl, "row_lower"),
                 (ru, "row_upper")):
        assert np.array_equal(t.cpu().numpy(), exp[k]), k
    # the CSR copy is the same scaled matrix, permuted
    ers, eci, ecv = cpu_transpose(Model(m.num_rows, m.num_cols, m.col_start, m.row_index,
                                        exp["value"], m.objective, m.var_lower, m.var_upper,
                                        m.row_lower, m.row_upper))
    assert np.array_equal(d_cv.cpu().numpy(), ecv)


@pytest.mark.parametrize("name", ["config0_s1", "precision_s1"])
def test_spmv_matches_oracle(gpu_ctx, oracle, name):
    import torch
    m = synthetic(name)
    rng = np.random.default_rng(5)
    x = rng.normal(size=m.num_cols)
    x[rng.random(m.num_cols) < 0.2] = 0.0
    expect = oracle.spmv(m, x)
    rs, ci, cv = cpu_transpose(m)
    y = torch.zeros(m.num_rows, dtype=torch.float64, device="cuda")
    xs = dev(x)
    d_rs, d_ci, d_cv = dev(rs), dev(ci), dev(cv)
    _lib.check(_lib.engine().mc_spmv_csr(gpu_ctx.handle, m.num_rows, m.num_cols, d_rs.data_ptr(),
                                         d_ci.data_ptr(), d_cv.data_ptr(), xs.data_ptr(),
                                         y.data_ptr()))
    got = y.cpu().numpy()
    absum = np.zeros(m.num_rows)
    for j in range(m.num_cols):
        for p in range(m.col_start[j], m.col_start[j + 1]):
            absum[m.row_index[p]] += abs(m.value[p] * x[j])
    assert np.all(np.abs(got - expect) <= 1e-13 * np.maximum(absum, 1e-300))


CANONICAL_OPTIONS = [dict(), dict(min_scale=0.5, max_scale=2.0), dict(tolerance=0.5), dict(max_iterations=3)]


@pytest.mark.parametrize("name", ["netlib_afiro", "small_s7", "precision_s1", "transport"])
@pytest.mark.parametrize("opt", range(len(CANONICAL_OPTIONS)))
def test_canonical_ruiz_bit_exact(gpu_ctx, reference, name, opt):
    """mc_ruiz_equilibrate_canonical against the reference's equilibrate
    (src/scale/ruiz_scaling.cpp:20-125) on the CLI's canonical model of the LP:
    values, rhs, objective, clamped scales, inverses, pass count, converged.
    (The reference's sparse canonical form caps the model size, so the LPs are
    the small golden ones.)"""
    import torch
    from test_oracle import load_model
    m = (generators.transport(2, 20, 30) if name == "transport" else
         load_model(name) if name.startswith("netlib") else synthetic(name))
    kw = dict(max_iterations=10, tolerance=1e-3, min_scale=1e-4, max_scale=1e4)
    kw.update(CANONICAL_OPTIONS[opt])
    ref = reference.canonical_equilibrate(m, **kw)
    cm, cn, nnz = ref["m"], ref["n"], ref["nnz"]
    cs, ri, v = dev(ref["col_start"]), dev(ref["row_index"]), dev(ref["value_in"])
    rhs, obj = dev(ref["rhs_in"]), dev(ref["objective_in"])
    scales = [torch.zeros(k, dtype=torch.float64, device="cuda") for k in (cm, cn, cm, cn)]
    it, conv = C.c_int64(-1), C.c_int32(-1)
    _lib.check(_lib.engine().mc_ruiz_equilibrate_canonical(
        gpu_ctx.handle, cm, cn, nnz, cs.data_ptr(), ri.data_ptr(), v.data_ptr(), rhs.data_ptr(), obj.data_ptr(),
        kw["max_iterations"], kw["tolerance"], kw["min_scale"], kw["max_scale"], *[t.data_ptr() for t in scales],
        C.addressof(it), C.addressof(conv)))
    assert it.value == ref["iterations"] and bool(conv.value) == ref["converged"]
    for t, k in ((v, "value"), (rhs, "rhs"), (obj, "objective"), (scales[0], "row_scale"),
                 (scales[1], "col_scale"), (scales[2], "inv_row_scale"), (scales[3], "inv_col_scale")):
        assert np.array_equal(t.cpu().numpy(), ref[k]), k
