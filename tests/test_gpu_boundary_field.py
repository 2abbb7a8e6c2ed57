"""Per-node wall velocity on the B200 (mplbgpu_set_boundary_velocity, an
extension of the reference's uniform GivenVars): the L-channel with its
seeded +-1 % inlet perturbation and a cavity with a per-node halfway
bounce-back lid, bit for bit against the oracle restatement given the same
field; a field of equal values bit for bit the uniform run; clearing the
field; the FP32 form against FP64; the rejections."""
import numpy as np
import pytest

from mplb_b200 import Solver, abi, config
from mplb_b200.solver import MplbGpuError

pytestmark = pytest.mark.gpu


def both(oracle_mod, case, field, steps, phases=2):
    o = oracle_mod.Oracle(case)
    s = Solver(case)
    if field is not None:
        o.set_boundary_velocity(*field)
        s.set_boundary_velocity(*field)
    o.init_uniform()
    s.init_uniform()
    for _ in range(phases):
        o.step(steps)
        s.stream_collision(steps)
        o.update_macro()
        s.update_macro_vars()
        for b in case.block_ids:
            for got, want in zip(s.macro(b), o.macro(b)):
                assert np.array_equal(got, want)
            assert np.array_equal(s.f(b), o.f(b))
    return s


@pytest.mark.parametrize("shape", [(24, 12, 10), (14, 9, 7)])
def test_lchannel_perturbed_inlet_matches_oracle(gpu_lib, oracle_mod, shape):
    leg, side, depth = shape
    case = config.lchannel(leg=leg, side=side, depth=depth)
    k, comps = config.inlet_perturbation(case)
    s = both(oracle_mod, case, (k,) + comps, 25)
    s.close()


def test_cavity_lid_profile_hbb_matches_oracle(gpu_lib, oracle_mod):
    case = config.cavity(3, 12, 0.05, re=100, wall="HalfwayBounceBack")
    lid = [i for i, b in enumerate(case.boundaries)
           if any(abs(g) > 0 for g in b.given)][0]
    o = oracle_mod.Oracle(case)
    nx, ny, nz = o.boundary_extent(lid)
    x = np.linspace(0.0, 1.0, nx)[None, None, :]
    u = case.boundaries[lid].given[0] * np.sin(np.pi * x) * np.ones(
        (nz, ny, nx))
    v = 0.1 * u
    s = both(oracle_mod, case, (lid, u, v, None), 20)
    s.close()


def test_cavity2d_lid_profile_eqm_matches_oracle(gpu_lib, oracle_mod):
    case = config.cavity(2, 17, 0.05, re=100)
    lid = [i for i, b in enumerate(case.boundaries)
           if any(abs(g) > 0 for g in b.given)][0]
    o = oracle_mod.Oracle(case)
    nx, ny, nz = o.boundary_extent(lid)
    x = np.linspace(0.0, 1.0, nx)[None, None, :]
    u = case.boundaries[lid].given[0] * 4 * x * (1 - x) * np.ones(
        (nz, ny, nx))
    s = both(oracle_mod, case, (lid, u, None, None), 30)
    s.close()


def test_equal_field_is_uniform_bitwise(gpu_lib):
    case = config.lchannel(leg=20, side=10, depth=8)
    k = config.inlet_index(case)
    g = case.boundaries[k].given
    runs = []
    for field in (False, True):
        s = Solver(case)
        if field:
            nx, ny, nz = s.boundary_extent(k)
            s.set_boundary_velocity(k, *[np.full((nz, ny, nx), c) for c in g])
        s.init_uniform()
        s.stream_collision(30)
        runs.append([s.f(b) for b in case.block_ids])
        s.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_clearing_field_restores_given(gpu_lib):
    case = config.lchannel(leg=20, side=10, depth=8)
    k, comps = config.inlet_perturbation(case)
    out = []
    for perturb_then_clear in (False, True):
        s = Solver(case)
        if perturb_then_clear:
            s.set_boundary_velocity(k, *comps)
            s.set_boundary_velocity(k)
        s.init_uniform()
        s.stream_collision(30)
        out.append([s.f(b) for b in case.block_ids])
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_fp32_field_as_close_to_fp64_as_uniform(gpu_lib):
    """The FP32 form with the per-node inlet is as close to FP64 (with the
    same inlet) as the FP32 form with the uniform inlet is to its FP64
    run: the per-node wall constants lose nothing in the shifted form."""
    def velocity(prec, field):
        case = config.lchannel(leg=40, side=16, depth=12, precision=prec)
        s = Solver(case)
        if field:
            k, comps = config.inlet_perturbation(case)
            s.set_boundary_velocity(k, *comps)
        s.init_uniform()
        s.stream_collision(200)
        s.update_macro_vars()
        u = [s.macro(b)[1] for b in case.block_ids]
        s.close()
        return u

    def rel(a, b):
        return (sum(np.linalg.norm(x - y) for x, y in zip(a, b)) /
                sum(np.linalg.norm(y) for y in b))

    e_field = rel(velocity("fp32", True), velocity("fp64", True))
    e_unif = rel(velocity("fp32", False), velocity("fp64", False))
    assert e_field <= 1.5 * e_unif + 1e-7, (e_field, e_unif)


def test_field_rejections(gpu_lib):
    case = config.lchannel(leg=14, side=9, depth=7)
    s = Solver(case)
    vb = [i for i, b in enumerate(case.boundaries)
          if b.vertex_type == "VirtualBoundary"][0]
    with pytest.raises(MplbGpuError) as e:
        s.set_boundary_velocity(vb, 0.0)
    assert e.value.status == abi.ERR_UNSUPPORTED
    with pytest.raises(MplbGpuError) as e:
        s.boundary_extent(len(case.boundaries))
    assert e.value.status == abi.ERR_INVALID
    k = config.inlet_index(case)
    with pytest.raises(MplbGpuError) as e:
        s.set_boundary_velocity(k, np.nan)
    assert e.value.status == abi.ERR_INVALID
    s.close()
    sw = config.cavity(3, 10, 0.05, re=100,
                       scheme="Scheme_StreamCollision_Swap")
    t = Solver(sw)
    with pytest.raises(MplbGpuError) as e:
        t.set_boundary_velocity(0, 0.0)
    assert e.value.status == abi.ERR_UNSUPPORTED
    t.close()
