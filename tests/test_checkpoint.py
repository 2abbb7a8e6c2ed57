"""Checkpoint files (reference naming <case>_<block>_T<step>, raw float64 in
the reference's node layout, JSON manifest): round trip and validation on
the host; on the GPU, a restarted solver continues bit for bit."""
import numpy as np
import pytest

from mplb_b200 import checkpoint, config


def test_round_trip_and_naming(tmp_path):
    case = config.lchannel_app(8, inflow=0.01)
    rng = np.random.default_rng(0)
    fields = {}
    for b in case.block_ids:
        nx, ny, nz = case.size3(b)
        fields[b] = rng.standard_normal((nz, ny, nx, case.q))
    man = checkpoint.write(str(tmp_path), case, 1234, fields)
    assert man.endswith(f"{case.case_name}_T1234.json")
    for b in case.block_ids:
        assert (tmp_path / f"{case.case_name}_{b}_T1234.f64").exists()
    back = checkpoint.read(str(tmp_path), case, 1234)
    for b in case.block_ids:
        assert np.array_equal(back[b], fields[b])


def test_rejects_mismatched_case(tmp_path):
    case = config.cavity(2, 16, 0.05, re=100)
    nx, ny, nz = case.size3(0)
    checkpoint.write(str(tmp_path), case, 7, {0: np.zeros((nz, ny, nx, 9))})
    other = config.cavity(2, 24, 0.05, re=100)
    with pytest.raises(ValueError):
        checkpoint.read(str(tmp_path), other, 7)
    with pytest.raises(ValueError):
        checkpoint.write(str(tmp_path), case, 8, {0: np.zeros((3, 3, 9))})


@pytest.mark.gpu
def test_restart_continues_bitwise(gpu_lib, tmp_path):
    from mplb_b200 import Solver
    case = config.cavity(3, 20, 0.05, re=100)
    a = Solver(case)
    a.init_uniform()
    a.stream_collision(25)
    checkpoint.save(a, str(tmp_path), 25)
    a.stream_collision(15)
    b = checkpoint.restart(case, str(tmp_path), 25)
    b.stream_collision(15)
    assert np.array_equal(a.f(0), b.f(0))
    a.update_macro_vars()
    b.update_macro_vars()
    for x, y in zip(a.macro(0), b.macro(0)):
        assert np.array_equal(x, y)
    a.close()
    b.close()
