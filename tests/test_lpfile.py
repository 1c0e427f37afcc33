"""Binary CSC model files (mc_lp_file_*): host round trips and header checks on
CPU; streaming into device memory and solving on the GPU."""
from __future__ import annotations

import numpy as np
import pytest

import mcpdlp
from conftest import rel
from mcpdlp import PdlpOptions, generators, lpfile
from test_oracle import load_model


def same(a, b) -> None:
    assert (a.num_rows, a.num_cols, a.nnz) == (b.num_rows, b.num_cols, b.nnz)
    for k in ("col_start", "row_index", "value", "objective", "var_lower", "var_upper", "row_lower",
              "row_upper"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    assert a.objective_offset == b.objective_offset and int(a.objective_sense) == int(b.objective_sense)


@pytest.mark.parametrize("which", ["netlib_afiro", "tiny_simplex", "random", "maximise", "empty_rows", "no_rows"])
def test_host_round_trip(tmp_path, which):
    if which == "random":
        m = generators.random_lp(3, 300, 900, 6, "precision")   # infinite upper bounds
    elif which == "maximise":
        m = generators.random_lp(4, 50, 150, 4)
        m.objective_sense, m.objective_offset = 1, -2.5
    elif which == "empty_rows":
        m = mcpdlp.Model(3, 2, np.array([0, 1, 1], np.int32), np.array([2], np.int32), np.array([1.5]),
                         np.ones(2), np.zeros(2), np.full(2, np.inf), np.full(3, -np.inf), np.ones(3))
    elif which == "no_rows":
        m = mcpdlp.Model(0, 2, np.zeros(3, np.int32), np.zeros(0, np.int32), np.zeros(0), np.ones(2),
                         np.zeros(2), np.ones(2), np.zeros(0), np.zeros(0))
    else:
        m = load_model(which)
    path = tmp_path / f"{which}.mclp"
    lpfile.write(m, path)
    assert lpfile.info(path) == (m.num_rows, m.num_cols, m.nnz)
    assert path.stat().st_size == 64 + 4 * (m.num_cols + 1) + 12 * m.nnz + 24 * m.num_cols + 16 * m.num_rows
    same(lpfile.read(path), m)


def test_bad_files_are_rejected(tmp_path):
    m = generators.random_lp(5, 40, 120, 4)
    good = tmp_path / "good.mclp"
    lpfile.write(m, good)
    raw = good.read_bytes()
    (tmp_path / "short.mclp").write_bytes(raw[:-8])
    with pytest.raises(ValueError, match="bytes, header says"):
        lpfile.read(tmp_path / "short.mclp")
    (tmp_path / "magic.mclp").write_bytes(b"XXXX" + raw[4:])
    with pytest.raises(ValueError, match="not an MCLPCSC1"):
        lpfile.info(tmp_path / "magic.mclp")
    bad = bytearray(raw)
    bad[8:12] = (-5).to_bytes(4, "little", signed=True)
    (tmp_path / "neg.mclp").write_bytes(bytes(bad))
    with pytest.raises(ValueError, match="bad header"):
        lpfile.info(tmp_path / "neg.mclp")
    with pytest.raises(ValueError, match="cannot open"):
        lpfile.info(tmp_path / "missing.mclp")


@pytest.mark.gpu
def test_device_stream_and_solve(gpu_ctx, tmp_path):
    """A model larger than one staging buffer (8 MiB) streamed into device
    memory solves exactly as the same model from host memory."""
    import torch
    m = generators.random_lp(2, 100_000, 250_000, 8)      # 2M nonzeros, 33 MB file
    path = tmp_path / "m.mclp"
    lpfile.write(m, path)
    dm = lpfile.read_device(path)
    assert torch.equal(dm.value.cpu(), torch.from_numpy(m.value))
    assert torch.equal(dm.row_upper.cpu(), torch.from_numpy(m.row_upper))
    o = PdlpOptions()
    o.set_tolerance(1e-6)
    a = gpu_ctx.solve(m, o)
    b = gpu_ctx.solve_device(dm, o)
    assert a.status == b.status and a.iterations == b.iterations and a.objective == b.objective
    assert rel(a.objective, m.info["optimum"]) < 1e-4
