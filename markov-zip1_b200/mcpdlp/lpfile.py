"""Binary CSC model files (mc_lp_file_*, format "MCLPCSC1").

    lpfile.write(model, "config1.mclp")
    m = lpfile.read("config1.mclp")              # Model in host memory
    dm = lpfile.read_device("config1.mclp")      # DeviceModel, streamed to the GPU

They carry models past the reference MPS reader's limits
(include/markov_cero/io/mps.hpp:13-20).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi, _lib
from .model import Model


def _path(path) -> bytes:
    return os.fsencode(os.fspath(path))


def _raise(code: int) -> None:
    if code == _abi.MC_ERR_INVALID_ARGUMENT:
        raise ValueError(_lib.last_error())
    _lib.check(code)


def write(model: Model, path) -> None:
    lp = model.to_struct()
    _raise(_lib.engine().mc_lp_file_write(_path(path), C.addressof(lp)))


def info(path) -> tuple[int, int, int]:
    m, n, z = C.c_int32(), C.c_int32(), C.c_int64()
    _raise(_lib.engine().mc_lp_file_info(_path(path), C.byref(m), C.byref(n), C.byref(z)))
    return m.value, n.value, z.value


def read(path) -> Model:
    m, n, z = info(path)
    arrays = dict(col_start=np.zeros(n + 1, np.int32), row_index=np.zeros(z, np.int32),
                  value=np.zeros(z), objective=np.zeros(n), var_lower=np.zeros(n), var_upper=np.zeros(n),
                  row_lower=np.zeros(m), row_upper=np.zeros(m))
    lp = _abi.McLp()
    lp.num_rows, lp.num_cols, lp.nnz = m, n, z
    for k, a in arrays.items():
        setattr(lp, k, a.ctypes.data if a.size else None)
    lp.memory = _abi.MC_MEMORY_HOST
    _raise(_lib.engine().mc_lp_file_read(_path(path), C.addressof(lp)))
    return Model(m, n, arrays["col_start"], arrays["row_index"], arrays["value"], arrays["objective"],
                 arrays["var_lower"], arrays["var_upper"], arrays["row_lower"], arrays["row_upper"],
                 lp.objective_offset, lp.objective_sense, name=os.path.basename(os.fspath(path)))


def read_device(path, device: str = "cuda:0"):
    """The model straight into device memory (torch tensors of a DeviceModel)."""
    import torch
    from . import DeviceModel
    m, n, z = info(path)
    dev = torch.device(device)
    dm = DeviceModel.__new__(DeviceModel)
    dm.num_rows, dm.num_cols, dm.nnz = m, n, z
    i32 = dict(dtype=torch.int32, device=dev)
    f64 = dict(dtype=torch.float64, device=dev)
    dm.col_start = torch.empty(n + 1, **i32)
    dm.row_index = torch.empty(max(z, 1), **i32)
    dm.value = torch.empty(max(z, 1), **f64)
    dm.objective, dm.var_lower, dm.var_upper = (torch.empty(max(n, 1), **f64) for _ in range(3))
    dm.row_lower, dm.row_upper = (torch.empty(max(m, 1), **f64) for _ in range(2))
    lp = _abi.McLp()
    lp.num_rows, lp.num_cols, lp.nnz = m, n, z
    for k in ("col_start", "row_index", "value", "objective", "var_lower", "var_upper", "row_lower",
              "row_upper"):
        setattr(lp, k, getattr(dm, k).data_ptr())
    lp.memory = _abi.MC_MEMORY_DEVICE
    with torch.cuda.device(dev):
        _raise(_lib.engine().mc_lp_file_read(_path(path), C.addressof(lp)))
    dm.objective_offset = lp.objective_offset
    dm.objective_sense = lp.objective_sense
    return dm
