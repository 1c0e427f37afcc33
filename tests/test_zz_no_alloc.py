"""Ruiz equilibration for callers that cannot allocate device memory.

mc_ruiz_equilibrate_noalloc serves code that must not call cudaMalloc:
applications whose device memory is all owned by another allocator (a caching
pool, a fixed arena), and request paths that may not allocate because an
allocation can wait on the device for an unbounded time.  It keeps its
working memory in one static device array instead.  These tests call it
through the C ABI, twice and three times in a row on the same array, and
compare every output with the allocating entry point mc_ruiz_equilibrate.
The comparison is bit for bit, which is inside the tolerances the other GPU
tests use (1e-13 relative for SpMV, 1e-6 for objectives).

This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from mcpdlp import _abi, _lib, generators

pytestmark = pytest.mark.gpu

MAX_LINES = 1 << 20


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


class DeviceCopies:
    """A model on the device: CSC, the device-built CSR, bounds, objective."""

    def __init__(self, ctx, model):
        import torch
        self.m, self.n, self.nnz = model.num_rows, model.num_cols, model.nnz
        self.cs, self.ri, self.cv = _dev(model.col_start), _dev(model.row_index), _dev(model.value)
        self.rs = torch.zeros(self.m + 1, dtype=torch.int32, device="cuda")
        self.ci = torch.zeros(max(self.nnz, 1), dtype=torch.int32, device="cuda")
        self.rv = torch.zeros(max(self.nnz, 1), dtype=torch.float64, device="cuda")
        _lib.check(_lib.engine().mc_csc_to_csr(ctx.handle, self.m, self.n, self.nnz, self.cs.data_ptr(),
                                               self.ri.data_ptr(), self.cv.data_ptr(), self.rs.data_ptr(),
                                               self.ci.data_ptr(), self.rv.data_ptr()))
        self.obj, self.vl, self.vu = _dev(model.objective), _dev(model.var_lower), _dev(model.var_upper)
        self.rl, self.ru = _dev(model.row_lower), _dev(model.row_upper)
        self.row_scale = torch.full((self.m,), -7.0, dtype=torch.float64, device="cuda")
        self.col_scale = torch.full((self.n,), -7.0, dtype=torch.float64, device="cuda")

    def clone(self, ctx, model):
        return DeviceCopies(ctx, model)

    def args(self):
        return [self.cs.data_ptr(), self.ri.data_ptr(), self.cv.data_ptr(), self.rs.data_ptr(),
                self.ci.data_ptr(), self.rv.data_ptr(), self.obj.data_ptr(), self.vl.data_ptr(),
                self.vu.data_ptr(), self.rl.data_ptr(), self.ru.data_ptr()]

    def outputs(self) -> dict:
        return {k: getattr(self, k).cpu().numpy() for k in
                ("cv", "rv", "obj", "vl", "vu", "rl", "ru", "row_scale", "col_scale")}


def allocating(ctx, d: DeviceCopies, passes: int = 10):
    it = C.c_int64(-1)
    _lib.check(_lib.engine().mc_ruiz_equilibrate(ctx.handle, d.m, d.n, d.nnz, *d.args(), passes,
                                                 d.row_scale.data_ptr(), d.col_scale.data_ptr(),
                                                 C.addressof(it)))
    return it.value


def no_alloc(d: DeviceCopies, passes: int = 10, stream=None):
    it = C.c_int64(-1)
    _lib.check(_lib.engine().mc_ruiz_equilibrate_noalloc(d.m, d.n, d.nnz, *d.args(), passes,
                                                         d.row_scale.data_ptr(), d.col_scale.data_ptr(),
                                                         C.addressof(it), stream))
    return it.value


def assert_same(a: dict, b: dict) -> None:
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_no_alloc_matches_allocating_entry_point_on_consecutive_calls(gpu_ctx):
    import torch
    models = [generators.random_lp(1, 1000, 3000, 6),
              generators.random_lp(1, 300, 900, 10, "precision"),
              generators.random_lp(1, 1000, 3000, 6)]
    stream = torch.cuda.current_stream().cuda_stream
    for call, model in enumerate(models):
        expect = DeviceCopies(gpu_ctx, model)
        passes_expect = allocating(gpu_ctx, expect)
        got = DeviceCopies(gpu_ctx, model)
        passes_got = no_alloc(got, stream=stream if call == 1 else None)
        torch.cuda.synchronize()
        assert passes_got == passes_expect, call
        assert_same(got.outputs(), expect.outputs())


def test_no_alloc_partial_pass_counts(gpu_ctx):
    """Fewer passes than convergence needs, then a full run on the same scratch."""
    model = generators.random_lp(3, 500, 1500, 6)
    for passes in (0, 1, 3, 10):
        expect = DeviceCopies(gpu_ctx, model)
        got = DeviceCopies(gpu_ctx, model)
        assert no_alloc(got, passes) == allocating(gpu_ctx, expect, passes)
        assert_same(got.outputs(), expect.outputs())


def test_no_alloc_rejects_models_beyond_its_scratch(gpu_ctx):
    import torch
    tiny = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = _lib.engine().mc_ruiz_equilibrate_noalloc(MAX_LINES, 1, 0, *([None] * 11), 10, tiny.data_ptr(),
                                                   tiny.data_ptr(), None, None)
    assert rc == _abi.MC_ERR_RESOURCE_LIMIT
    assert "exceeds the static scratch limit" in _lib.last_error()
