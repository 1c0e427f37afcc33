"""The C ABI library: loads, exports what include/*.h declares, layouts agree,
host-side argument checks (CPU-only tests; no compute call needs a GPU)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import mcpdlp
from mcpdlp import _abi, _lib, generators

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions() -> set[str]:
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:int|void|size_t|double)\s+\*?\s*(mc_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def exported_symbols(path: Path) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_headers_declare_the_boundary():
    names = declared_functions()
    for must in ("mc_pdlp_solve", "mc_pdlp_ctx_solve", "mc_pdlp_ctx_create", "mc_pdlp_ctx_destroy",
                 "mc_pdlp_default_options", "mc_last_error", "mc_spmv_csr", "mc_csc_to_csr",
                 "mc_ruiz_equilibrate"):
        assert must in names


def test_library_exports_every_declared_symbol():
    exported = exported_symbols(_lib.ENGINE_PATH)
    missing = declared_functions() - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"


def test_library_loads_with_signatures():
    lib = _lib.engine()
    assert lib.mc_pdlp_abi_version() == _abi.MC_PDLP_ABI_VERSION
    assert set(_lib.ENGINE_SIGNATURES) <= exported_symbols(_lib.ENGINE_PATH)


def test_struct_layouts_match():
    sizes = (C.c_size_t * 8)()
    assert _lib.engine().mc_pdlp_struct_sizes(sizes, 8) == 0
    assert list(sizes) == [C.sizeof(_abi.McLp), C.sizeof(_abi.McPdlpOptions),
                           C.sizeof(_abi.McPdlpResult), C.sizeof(_abi.McPdlpTrace),
                           C.sizeof(_abi.McVerifyReport), C.sizeof(_abi.McCanonicalLp),
                           C.sizeof(_abi.McPresolveOptions), C.sizeof(_abi.McPresolveInfo)]


def test_default_options_match_reference_defaults():
    o = _abi.McPdlpOptions()
    _lib.engine().mc_pdlp_default_options(C.byref(o))
    ref = _abi.default_options_struct()
    for name, _ in _abi.McPdlpOptions._fields_:
        a, b = getattr(o, name), getattr(ref, name)
        if hasattr(a, "__len__"):
            assert list(a) == list(b), name
        else:
            assert a == b, name
    # PdlpOptions defaults, include/markov_cero/lp/first_order/pdlp.hpp:18-41
    p = mcpdlp.PdlpOptions()
    assert (p.max_iterations, p.restart_every, p.primal_tolerance, p.step_size_reduction,
            p.restart_reduction_factor, p.primal_weight_smoothing, p.ruiz_iterations) == (
        100000, 40, 1e-4, 0.9, 0.368, 0.5, 10)


def test_cpu_backend_is_rejected():
    with pytest.raises(ValueError, match="GPU only"):
        mcpdlp.PdlpOptions(backend=mcpdlp.Backend.cpu).to_struct()


def test_option_validation_needs_no_device():
    m = generators.random_lp(1, 20, 60, 3)
    lp = m.to_struct()
    o = _abi.default_options_struct()
    o.restart_every = 0
    res = _abi.McPdlpResult()
    rc = _lib.engine().mc_pdlp_solve(C.addressof(lp), C.addressof(o), None, None, None, None,
                                     C.addressof(res))
    assert rc == _abi.MC_ERR_INVALID_ARGUMENT
    assert "restart_every" in _lib.last_error()
    o = _abi.default_options_struct()
    o.backend = 0
    rc = _lib.engine().mc_pdlp_solve(C.addressof(lp), C.addressof(o), None, None, None, None,
                                     C.addressof(res))
    assert rc == _abi.MC_ERR_INVALID_ARGUMENT


def test_no_device_is_an_error_not_a_fallback():
    if mcpdlp.device_count() > 0:
        pytest.skip("a GPU is present")
    m = generators.random_lp(1, 20, 60, 3)
    with pytest.raises(mcpdlp.EngineError, match="no_device"):
        mcpdlp.solve_pdlp(m, mcpdlp.PdlpOptions())


def test_nnz_beyond_int32_is_resource_limit():
    lp = _abi.McLp()
    lp.num_rows, lp.num_cols, lp.nnz = 10, 10, 1 << 31
    o = _abi.default_options_struct()
    res = _abi.McPdlpResult()
    rc = _lib.engine().mc_pdlp_solve(C.addressof(lp), C.addressof(o), None, None, None, None,
                                     C.addressof(res))
    assert rc == _abi.MC_ERR_RESOURCE_LIMIT
