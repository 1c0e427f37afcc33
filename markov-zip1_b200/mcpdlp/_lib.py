"""Loading of the in-tree native libraries.

``libmcpdlp.so`` is the CUDA engine (the product); ``liblpgen.so`` holds the
seeded workload generators.  Both are built in-tree by the package Makefile
(``make -C markov-zip1_b200``).  There is no fallback: if the engine library
is missing, every solve raises ``EngineUnavailable``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

from . import _abi

PKG_ROOT = Path(__file__).resolve().parent.parent          # markov-zip1_b200/
LIB_DIR = PKG_ROOT / "lib"
ENGINE_PATH = LIB_DIR / "libmcpdlp.so"
LPGEN_PATH = LIB_DIR / "liblpgen.so"

_lock = threading.Lock()
_engine = None
_lpgen = None


class EngineUnavailable(RuntimeError):
    """The CUDA engine library is missing or cannot be loaded."""


class EngineError(RuntimeError):
    """A C-ABI call returned an error code."""

    def __init__(self, code: int, message: str):
        self.code = code
        name = _abi.ERROR_NAMES.get(code, str(code))
        super().__init__(f"{name}: {message}")


_VP = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64

ENGINE_SIGNATURES = {
    "mc_pdlp_abi_version": ([], C.c_int),
    "mc_pdlp_default_options": ([_VP], None),
    "mc_pdlp_struct_sizes": ([_VP, C.c_int], C.c_int),
    "mc_test_inject_alloc_failures": ([C.c_int], C.c_int),
    "mc_last_error": ([C.c_char_p, C.c_size_t], C.c_int),
    "mc_device_count": ([_VP], C.c_int),
    "mc_pdlp_ctx_create": ([C.c_int, _VP], C.c_int),
    "mc_pdlp_ctx_destroy": ([_VP], C.c_int),
    "mc_pdlp_ctx_solve": ([_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_pdlp_solve": ([_VP, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_pdlp_ctx_stream": ([_VP, _VP], C.c_int),
    "mc_pdlp_ctx_begin": ([_VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_pdlp_ctx_iterate": ([_VP, _I64, _VP, _VP], C.c_int),
    "mc_pdlp_ctx_finish": ([_VP, _VP, _VP, _VP], C.c_int),
    "mc_pdlp_ctx_solve_batch": ([_VP, _VP, C.c_int32, _VP, _VP, _VP, _VP], C.c_int),
    "mc_pdlp_ctx_solve_variants": ([_VP, _VP, C.c_int32, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_pdlp_ctx_solve_batch_warm": ([_VP, _VP, C.c_int32, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_gnn_create": ([C.c_int, C.c_int, C.c_uint64, _VP], C.c_int),
    "mc_gnn_destroy": ([_VP], C.c_int),
    "mc_gnn_num_params": ([_VP, _VP], C.c_int),
    "mc_gnn_get_params": ([_VP, _VP], C.c_int),
    "mc_gnn_set_params": ([_VP, _VP], C.c_int),
    "mc_gnn_predict": ([_VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_gnn_loss_and_grad": ([_VP, _VP, _VP, _VP, C.c_double, _VP, _VP], C.c_int),
    "mc_gnn_train_step": ([_VP, _VP, _VP, _VP, C.c_double, C.c_float, _VP], C.c_int),
    "mc_spmv_csr": ([_VP, _I32, _I32, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_csc_to_csr": ([_VP, _I32, _I32, _I64, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_ruiz_equilibrate": ([_VP, _I32, _I32, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                             _VP, _VP, _VP, _I64, _VP, _VP, _VP], C.c_int),
    "mc_lp_file_write": ([C.c_char_p, _VP], C.c_int),
    "mc_lp_file_info": ([C.c_char_p, _VP, _VP, _VP], C.c_int),
    "mc_lp_file_read": ([C.c_char_p, _VP], C.c_int),
    "mc_ruiz_equilibrate_canonical": ([_VP, _I32, _I32, _I64, _VP, _VP, _VP, _VP, _VP, _I64, C.c_double,
                                       C.c_double, C.c_double, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_verify_primal": ([_VP, _VP, _VP, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _VP],
                         C.c_int),
    "mc_ruiz_equilibrate_noalloc": ([_I32, _I32, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP,
                                     _VP, _VP, _VP, _I64, _VP, _VP, _VP, _VP], C.c_int),
    "mc_presolve_default_options": ([_VP], None),
    "mc_presolve_run": ([_VP, _VP, _VP, _VP], C.c_int),
    "mc_presolve_get_info": ([_VP, _VP], C.c_int),
    "mc_presolve_get_model": ([_VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_presolve_get_maps": ([_VP, _VP, _VP], C.c_int),
    "mc_presolve_get_records": ([_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP], C.c_int),
    "mc_postsolve": ([_VP, _VP, _VP, _I64, _VP, _I64, _VP, _VP, _VP], C.c_int),
    "mc_presolve_free": ([_VP], None),
    "mc_presolve_load": ([_VP, _VP, _I64, _VP, _VP, _VP, _VP, _VP, _I64, _VP, _I64, _VP, _VP], C.c_int),
}


def engine() -> C.CDLL:
    """The engine library with argtypes set; raises EngineUnavailable."""
    global _engine
    with _lock:
        if _engine is None:
            if not ENGINE_PATH.exists():
                raise EngineUnavailable(
                    f"{ENGINE_PATH} is not built; run `make -C {PKG_ROOT}` "
                    "(there is no CPU fallback)")
            try:
                lib = C.CDLL(str(ENGINE_PATH))
            except OSError as e:
                raise EngineUnavailable(f"cannot load {ENGINE_PATH}: {e}") from e
            for name, (args, res) in ENGINE_SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = args
                fn.restype = res
            _engine = lib
        return _engine


def last_error() -> str:
    buf = C.create_string_buffer(512)
    engine().mc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    if code != _abi.MC_OK:
        raise EngineError(code, last_error())


def lpgen() -> C.CDLL:
    global _lpgen
    with _lock:
        if _lpgen is None:
            if not LPGEN_PATH.exists():
                raise EngineUnavailable(f"{LPGEN_PATH} is not built; run `make -C {PKG_ROOT}`")
            lib = C.CDLL(str(LPGEN_PATH))
            lib.lpgen_random_lp.argtypes = [C.c_uint64, _I32, _I32, _I32, _I32] + [_VP] * 11
            lib.lpgen_random_lp.restype = C.c_int
            lib.lpgen_transport.argtypes = [C.c_uint64, _I32, _I32] + [_VP] * 10
            lib.lpgen_transport.restype = C.c_int
            lib.lpgen_uniform_int.argtypes = [C.c_uint64, C.c_uint64, _I64, _I64]
            lib.lpgen_uniform_int.restype = _I64
            lib.lpgen_uniform01.argtypes = [C.c_uint64, C.c_uint64]
            lib.lpgen_uniform01.restype = C.c_double
            lib.lpgen_tighten_bounds.argtypes = [C.c_uint64, _I32, _VP, _VP, _VP, _VP]
            lib.lpgen_tighten_bounds.restype = C.c_int
            _lpgen = lib
        return _lpgen


def engine_built() -> bool:
    return ENGINE_PATH.exists()


def build(verbose: bool = False) -> None:
    """Compile the native libraries in-tree (nvcc for sm_100a, gcc)."""
    import subprocess
    cmd = ["make", "-C", str(PKG_ROOT), f"-j{min(8, os.cpu_count() or 1)}"]
    out = subprocess.run(cmd, capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"native build failed:\n{out.stdout}\n{out.stderr}")
