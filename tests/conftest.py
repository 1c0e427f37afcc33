"""Shared fixtures.  Tests marked ``gpu`` need a B200; the rest run on CPU.

The native libraries are built in-tree on first use (make is incremental).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "markov-zip1_b200"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")
    config.addinivalue_line("markers", "slow: larger instances")


def _ensure_built() -> None:
    lib = PKG / "lib"
    if not (lib / "libmcpdlp.so").exists() or not (lib / "liblpgen.so").exists():
        subprocess.run(["make", "-C", str(PKG), "-j8"], check=True, capture_output=True)
    if not (ROOT / "oracle" / "build" / "liboracle_pdlp.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), "oracle"], check=True,
                       capture_output=True)
    from oracle import REFERENCE_SOURCES
    ref_src = REFERENCE_SOURCES / "src" / "lp" / "first_order" / "pdlp.cpp"
    if ref_src.exists() and not (ROOT / "oracle" / "_ref" / "libref_pdlp.so").exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle"), f"REF={REFERENCE_SOURCES}", "ref"],
                       check=True, capture_output=True)
    if ref_src.exists() and not (PKG / "binding" / "_build" / "markov-cero-solve").exists():
        subprocess.run(["make", "-C", str(PKG / "binding"), f"REF={REFERENCE_SOURCES}", "-j8"],
                       check=True, capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def oracle():
    from oracle import OraclePort
    return OraclePort()


@pytest.fixture(scope="session")
def reference():
    from oracle import ReferencePdlp
    if not ReferencePdlp.available():
        pytest.skip("reference library oracle/_ref/libref_pdlp.so not built")
    return ReferencePdlp()


@pytest.fixture(scope="session")
def gpu_ctx():
    import mcpdlp
    if mcpdlp.device_count() == 0:
        pytest.fail("no sm_100 device visible: gpu tests must run on a B200")
    ctx = mcpdlp.Context(0)
    yield ctx
    ctx.close()


def options(tol: float = 1e-4, **kw):
    """Default options at a tolerance (ctypes struct, for the oracles)."""
    from mcpdlp import _abi
    o = _abi.default_options_struct()
    o.primal_tolerance = o.dual_tolerance = o.gap_tolerance = tol
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def rel(a: float, b: float) -> float:
    return abs(a - b) / max(1.0, abs(b))
