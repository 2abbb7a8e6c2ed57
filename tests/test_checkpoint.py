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


def test_rejects_other_precision(tmp_path):
    case = config.cavity(2, 16, 0.05, re=100)
    nx, ny, nz = case.size3(0)
    checkpoint.write(str(tmp_path), case, 9, {0: np.zeros((nz, ny, nx, 9))})
    fp16 = config.cavity(2, 16, 0.05, re=100, precision="fp16")
    with pytest.raises(ValueError, match="precision|fp64"):
        checkpoint.read(str(tmp_path), fp16, 9)


@pytest.mark.gpu
def test_restart_keeps_check_periods(gpu_lib, tmp_path):
    """A run restarted at step 25 with check period 10 checks at 30, 40, 50
    (the absolute steps, as the reference's Iterate(start) counts), with the
    residuals of the uninterrupted run."""
    from mplb_b200 import Solver
    case = config.cavity(3, 16, 0.05, re=100)
    case.check_period = 10
    a = Solver(case)
    a.init_uniform()
    a.stream_collision(25)
    checkpoint.save(a, str(tmp_path), 25)
    b = checkpoint.restart(case, str(tmp_path), 25)
    assert b.steps_done == 25
    # both take their q_old from the moments of the step-25 state
    a.update_macro_vars()
    a.calc_residual_error(10)
    b.update_macro_vars()
    b.calc_residual_error(10)
    ha = a.iterate(criterion=0.0, max_steps=50)
    hb = b.iterate(criterion=0.0, max_steps=50)
    assert [h[0] for h in hb] == [30, 40, 50]
    assert [h[0] for h in ha] == [30, 40, 50]
    np.testing.assert_array_equal([h[1] for h in ha], [h[1] for h in hb])
    a.close()
    b.close()


@pytest.mark.gpu
def test_fp16_rounding_follows_the_step(gpu_lib):
    """The FP16 form draws its stochastic rounding from the step count: the
    same state stepped from the same step count gives the same bits, from
    another step count other bits (a restart sets the count, so it takes
    the uninterrupted run's draws)."""
    from mplb_b200 import Solver
    case = config.cavity(3, 16, 0.05, re=100, precision="fp16")
    s = Solver(case)
    s.init_uniform()
    s.stream_collision(5)
    f = s.f(0)
    out = {}
    for start in (25, 0, 25):
        t = Solver(case)
        t.upload_f(0, f)
        t.set_step(start)
        t.stream_collision(10)
        out.setdefault(start, []).append(t.f(0))
        t.close()
    s.close()
    assert np.array_equal(out[25][0], out[25][1])
    assert not np.array_equal(out[25][0], out[0][0])
