"""Per-node wall velocity (a new-build extension of the reference's uniform
GivenVars, used for the L-channel's perturbed inlet), on the CPU: the
seeded perturbation, and the oracle restatement with a field of equal
values against its uniform run (bit for bit), with a perturbed field
against the uniform one (it must differ, stay finite and keep the walls)."""
import numpy as np

from mplb_b200 import config
from oracle import pyoracle


def small_lchannel():
    return config.lchannel(leg=14, side=9, depth=7)


def test_inlet_perturbation_is_seeded_and_bounded():
    case = config.lchannel()
    k, (u, v, w) = config.inlet_perturbation(case)
    assert case.boundaries[k].vertex_type == "Inlet"
    assert u.shape == (128, 128, 1)
    u0 = case.boundaries[k].given[0]
    assert np.all(np.abs(u / u0 - 1.0) <= 0.01)
    assert abs(float(np.mean(u / u0 - 1.0))) < 1e-3
    assert not v.any() and not w.any()
    k2, (u2, _, _) = config.inlet_perturbation(case)
    assert k2 == k and np.array_equal(u, u2)
    _, (u3, _, _) = config.inlet_perturbation(case, seed=1)
    assert not np.array_equal(u, u3)


def test_oracle_extent_matches_face():
    case = small_lchannel()
    o = pyoracle.Oracle(case)
    k = config.inlet_index(case)
    assert o.boundary_extent(k) == config.face_extent(case, k)


def run(case, steps, field=None):
    o = pyoracle.Oracle(case)
    if field is not None:
        o.set_boundary_velocity(*field)
    o.init_uniform()
    o.step(steps)
    o.update_macro()
    return o


def test_oracle_equal_field_is_uniform_bitwise():
    case = small_lchannel()
    k = config.inlet_index(case)
    nx, ny, nz = config.face_extent(case, k)
    g = case.boundaries[k].given
    a = run(case, 30)
    b = run(case, 30, (k, np.full((nz, ny, nx), g[0]),
                       np.full((nz, ny, nx), g[1]),
                       np.full((nz, ny, nx), g[2])))
    for blk in case.block_ids:
        assert np.array_equal(a.f(blk), b.f(blk))


def test_oracle_perturbed_field_changes_inlet():
    case = small_lchannel()
    k, comps = config.inlet_perturbation(case)
    a = run(case, 30)
    b = run(case, 30, (k,) + comps)
    fa, fb = a.f(0), b.f(0)
    assert np.all(np.isfinite(fb))
    assert not np.array_equal(fa, fb)
    # the perturbation is +-1 % of the inlet speed: the fields stay close
    ua, ub = a.macro(0)[1], b.macro(0)[1]
    assert np.abs(ub - ua).max() < 0.05 * np.abs(ua).max()


def test_oracle_clearing_field_restores_given():
    case = small_lchannel()
    k, comps = config.inlet_perturbation(case)
    o = pyoracle.Oracle(case)
    o.set_boundary_velocity(k, *comps)
    o.set_boundary_velocity(k)
    o.init_uniform()
    o.step(20)
    a = run(case, 20)
    for blk in case.block_ids:
        assert np.array_equal(o.f(blk), a.f(blk))


def test_oracle_rejects_field_without_wall_kernel():
    case = small_lchannel()
    o = pyoracle.Oracle(case)
    vb = [i for i, b in enumerate(case.boundaries)
          if b.vertex_type == "VirtualBoundary"][0]
    try:
        o.set_boundary_velocity(vb, 0.0)
    except ValueError:
        return
    raise AssertionError("accepted a field on a VirtualBoundary surface")
