"""Parity of the CUDA path (through the C ABI) with the reference.

FP64 results are compared bit for bit with the golden fixtures made by the
reference itself and with the oracle (the C restatement) on the same
inputs; residuals, whose reductions sum in a different order, within a
relative 1e-12."""
import dataclasses

import numpy as np
import pytest

import golden_cases
from mplb_b200 import Solver, abi, config
from mplb_b200.solver import MplbGpuError

pytestmark = pytest.mark.gpu


def run_gpu(case, steps):
    s = Solver(case)
    s.init_uniform()
    cp = case.check_period
    hist = []
    for _ in range(steps // cp):
        s.stream_collision(cp)
        s.update_macro_vars()
        hist.append(s.calc_residual_error(cp))
    s.stream_collision(steps % cp)
    s.update_macro_vars()
    return s, hist


@pytest.mark.parametrize("name", golden_cases.names(include_long=True))
def test_gpu_matches_reference_golden(gpu_lib, name):
    g = golden_cases.load(name)
    s, hist = run_gpu(g["case"], g["steps"])
    for b in g["case"].block_ids:
        for got, want in zip(s.macro(b), g["macro"][b]):
            assert np.array_equal(got, want), name
        assert np.array_equal(s.f(b), g["f"][b]), name
    np.testing.assert_allclose([h[0] for h in hist], g["residual_max"],
                               rtol=1e-12, atol=0)
    np.testing.assert_allclose(np.array([h[1] for h in hist]),
                               g["residual_per_var"], rtol=1e-12, atol=1e-300)
    s.close()


ORACLE_CASES = {
    "cavity3d_bb": (lambda: config.cavity(3, 11, 0.05, re=100,
                                          wall="HalfwayBounceBack"), 40, 20),
    "cavity2d_bb": (lambda: config.cavity(2, 21, 0.05, re=100,
                                          wall="HalfwayBounceBack"), 100, 50),
    "poiseuille2d_bb": (lambda: config.poiseuille(
        2, 8, 10, g_lattice=1e-4, wall="HalfwayBounceBack"), 100, 50),
    "lchannel_bb": (lambda: config.lchannel(leg=9, side=6, depth=4,
                                            wall="HalfwayBounceBack"), 40, 20),
    "lchannel_eqm": (lambda: config.lchannel(leg=14, side=9, depth=7), 50, 25),
    # blocks of two nodes along an axis (no interior region)
    "tiny3d_3x2x4": (lambda: dataclasses.replace(
        config.cavity(3, 4, 0.05, re=50), block_sizes=[(3, 2, 4)]), 12, 4),
    "tiny3d_2x2x2": (lambda: dataclasses.replace(
        config.cavity(3, 2, 0.05, re=50), block_sizes=[(2, 2, 2)]), 12, 4),
    "tiny2d_2x5": (lambda: dataclasses.replace(
        config.cavity(2, 5, 0.05, re=50), block_sizes=[(2, 5)]), 12, 4),
    "odd3d_37x5x3": (lambda: dataclasses.replace(
        config.cavity(3, 37, 0.05, re=200), block_sizes=[(37, 5, 3)]), 20, 10),
    "cavity3d_edges": (lambda: config.cavity(
        3, 9, 0.05, re=100,
        order=("Front", "Left", "Right", "Top", "Bottom", "Back")), 30, 10),
}


@pytest.mark.parametrize("name", sorted(ORACLE_CASES))
def test_gpu_matches_oracle(gpu_lib, oracle_mod, name):
    build, steps, cp = ORACLE_CASES[name]
    case = build()
    case.check_period = cp
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    s = Solver(case)
    s.init_uniform()
    for b in case.block_ids:
        assert np.array_equal(s.f(b), o.f(b)), "initial f"
    for _ in range(steps // cp):
        o.step(cp)
        s.stream_collision(cp)
        o.update_macro()
        s.update_macro_vars()
        ro = o.residual(cp)
        rs = s.calc_residual_error(cp)
        np.testing.assert_allclose(rs[0], ro[0], rtol=1e-12)
        for b in case.block_ids:
            assert np.array_equal(s.f(b), o.f(b)), name
            for got, want in zip(s.macro(b), o.macro(b)):
                assert np.array_equal(got, want), name
    s.close()


def test_restart_from_uploaded_f(gpu_lib):
    case = config.lchannel_app(8, inflow=0.01)
    a = Solver(case)
    a.init_uniform()
    a.stream_collision(17)
    saved = {b: a.f(b) for b in case.block_ids}
    a.stream_collision(13)
    b_ = Solver(case)
    for b in case.block_ids:
        b_.upload_f(b, saved[b])
    b_.stream_collision(13)
    for b in case.block_ids:
        assert np.array_equal(a.f(b), b_.f(b))


def test_mass_conserved_in_closed_cavity(gpu_lib):
    case = config.cavity(3, 24, 0.05, re=100, wall="HalfwayBounceBack")
    s = Solver(case)
    s.init_uniform()
    m0 = s.mass()
    s.stream_collision(200)
    assert abs(s.mass() - m0) < 1e-10 * m0
    assert s.check_health() == abi.OK


def test_errors_are_reported(gpu_lib):
    case = config.cavity(3, 8, 0.05, re=10,
                         scheme="Scheme_StreamCollision_Swap")
    case.boundaries[0].scheme = "FDPeriodic"
    with pytest.raises(MplbGpuError) as e:
        Solver(case)
    assert e.value.status == abi.ERR_UNSUPPORTED
    s = Solver(config.cavity(2, 8, 0.05, re=10))
    with pytest.raises(MplbGpuError) as e:
        s.stream_collision(1)
    assert e.value.status == abi.ERR_STATE
    with pytest.raises(MplbGpuError) as e:
        s.init_macro(5)
    assert e.value.status == abi.ERR_INVALID


def test_divergence_is_detected(gpu_lib):
    case = config.cavity(2, 12, 0.05, re=10)
    s = Solver(case)
    s.init_uniform()
    f = s.f(0)
    f[0, 5, 5, :] = np.nan
    s.upload_f(0, f)
    s.stream_collision(2)
    assert s.check_health() == abi.ERR_DIVERGED


@pytest.mark.parametrize("name", sorted(golden_cases.apps()))
def test_gpu_matches_reference_app_files(gpu_lib, name):
    """The reference's own case files (Apps/*/*.json) through the JSON front
    end on the GPU: bit for bit the reference's run of the file."""
    case, steps, want = golden_cases.apps()[name]
    s = Solver(case)
    s.init_uniform()
    s.stream_collision(steps)
    s.update_macro_vars()
    assert golden_cases.fingerprint(case, s.f, s.macro) == want
    s.close()


@pytest.mark.parametrize("name", sorted(golden_cases.bench_cases()))
def test_gpu_matches_reference_bench_cases(gpu_lib, name):
    """The benchmark cavity (D3Q19, Re 400, lid 0.05) at 64^3 for 300 steps
    and the 3-block L-channel at 96/32/32 for 200 steps: f and moments bit
    for bit the reference's run (SHA-256 digests), residual history within
    summation order."""
    case, steps, residual, want = golden_cases.bench_cases()[name]
    s, hist = run_gpu(case, steps)
    assert golden_cases.fingerprint(case, s.f, s.macro) == want
    np.testing.assert_allclose([h[0] for h in hist],
                               [r[1] for r in residual], rtol=1e-12, atol=0)
    s.close()
