"""CPU checks of the oracle (the C restatement of the reference step):
bitwise against the golden fixtures made by the reference itself, and -
where the reference build is present - against the reference on more
cases."""
import dataclasses

import numpy as np
import pytest

import golden_cases
import random_cases
import special_cases
from mplb_b200 import config


def run_oracle(pyoracle, case, steps):
    o = pyoracle.Oracle(case)
    o.init_uniform()
    cp = case.check_period
    hist = []
    for _ in range(steps // cp):
        o.step(cp)
        o.update_macro()
        hist.append(o.residual(cp))
    o.step(steps % cp)
    o.update_macro()
    return o, hist


@pytest.mark.parametrize("name", golden_cases.names())
def test_oracle_matches_reference_golden(oracle_mod, name):
    g = golden_cases.load(name)
    o, hist = run_oracle(oracle_mod, g["case"], g["steps"])
    for b in g["case"].block_ids:
        for got, want in zip(o.macro(b), g["macro"][b]):
            assert np.array_equal(got, want)
        assert np.array_equal(o.f(b), g["f"][b])
    assert np.array_equal(np.array([h[0] for h in hist]), g["residual_max"])


def _swap_box():
    c = config.cavity(3, 13, 0.05, re=200,
                      scheme="Scheme_StreamCollision_Swap")
    return dataclasses.replace(c, block_sizes=[(13, 10, 9)],
                               body_force="BodyForce_1st",
                               accel=(-2e-3, 1e-3, 4e-3))


REF_CASES = {
    "cavity3d_13": (lambda: config.cavity(3, 13, 0.05, re=400), 40, 20),
    # the reference's one-array swap step, force without the shifted
    # velocity
    "swap_box_force": (_swap_box, 33, 11),
    # blocks of two nodes along an axis: no interior at all
    "tiny3d_3x2x4": (lambda: dataclasses.replace(
        config.cavity(3, 4, 0.05, re=50), block_sizes=[(3, 2, 4)]), 12, 4),
    "tiny3d_2x2x2": (lambda: dataclasses.replace(
        config.cavity(3, 2, 0.05, re=50), block_sizes=[(2, 2, 2)]), 12, 4),
    "tiny2d_7x2": (lambda: dataclasses.replace(
        config.cavity(2, 7, 0.05, re=50), block_sizes=[(7, 2)]), 12, 4),
    "cavity2d_lid_first": (lambda: config.cavity(
        2, 15, 0.1, re=30, order=("Top", "Left", "Right", "Bottom")), 120, 40),
    "lchannel_app_9": (lambda: config.lchannel_app(9), 50, 25),
    "poiseuille3d": (lambda: config.poiseuille(3, 7, 9, 6, g_lattice=1e-4),
                     60, 30),
}


@pytest.mark.parametrize("name", sorted(REF_CASES))
def test_oracle_matches_reference_built_here(oracle_mod, name):
    if not oracle_mod.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    build, steps, cp = REF_CASES[name]
    case = build()
    case.check_period = cp
    ref = oracle_mod.run_reference(case, steps)
    o, hist = run_oracle(oracle_mod, case, steps)
    for b in case.block_ids:
        for got, want in zip(o.macro(b), ref["macro"][b]):
            assert np.array_equal(got, want)
        assert np.array_equal(o.f(b), ref["f"][b])
    assert [h[0] for h in hist] == [r[1] for r in ref["residual"]]


def test_oracle_corner_populations_are_stale(oracle_mod):
    """3D corners: the six populations with all components pointing away
    from the corner's walls are neither streamed nor rewritten
    (Src/boundary_host_device.h:486-693 labels), so they keep f^0."""
    case = config.cavity(3, 8, 0.05, re=100)
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    f0 = o.f(0)[0, 0, 0].copy()
    o.step(25)
    f = o.f(0)[0, 0, 0]
    from csrc_tables import D3Q19_C
    stale = [i for i, c in enumerate(D3Q19_C) if c != (0, 0, 0)
             and all(v >= 0 for v in c)]
    assert len(stale) == 6
    assert np.array_equal(f[stale], f0[stale])


def test_oracle_mass_conserved_in_periodic_box(oracle_mod):
    """Fully periodic box (MDPeriodic on every face): total mass is
    conserved to round-off."""
    case = config.poiseuille(3, 6, 6, 6, g_lattice=0.0)
    case.boundaries = [b for b in case.boundaries
                       if b.surface not in ("Top", "Bottom")]
    case.boundaries += [config._bc(0, "Top", "MDPeriodic", "MDPeriodic"),
                        config._bc(0, "Bottom", "MDPeriodic", "MDPeriodic")]
    case.connections += [config.ConnectionDef(0, "Top", 0, "Bottom",
                                              "MDPeriodic"),
                         config.ConnectionDef(0, "Bottom", 0, "Top",
                                              "MDPeriodic")]
    o = oracle_mod.Oracle(case)
    rng = np.random.default_rng(7)
    shp = (6, 6, 6)
    o.init_macro(0, 1 + 0.01 * rng.standard_normal(shp),
                 0.01 * rng.standard_normal(shp),
                 0.01 * rng.standard_normal(shp),
                 0.01 * rng.standard_normal(shp))
    o.update_macro()
    m0 = o.macro(0)[0].sum()
    o.step(50)
    o.update_macro()
    assert abs(o.macro(0)[0].sum() - m0) < 1e-12 * m0


def test_json_round_trip():
    case = config.lchannel(leg=12, side=8, depth=6)
    back = config.CaseConfig.from_json(case.to_json())
    assert back.to_json() == case.to_json()


def test_oracle_rejects_swap_outside_its_scope(oracle_mod):
    """The swap scheme of this path: one 3D block, no connections,
    node-local boundary conditions on every face."""
    swap = "Scheme_StreamCollision_Swap"
    bad = [config.cavity(2, 9, 0.05, re=100, scheme=swap),
           config.cavity(3, 9, 0.05, re=100, scheme=swap,
                         wall="HalfwayBounceBack"),
           dataclasses.replace(config.lchannel(leg=9, side=6, depth=4),
                               scheme=swap)]
    for case in bad:
        with pytest.raises(ValueError):
            oracle_mod.Oracle(case)


@pytest.mark.parametrize("name", sorted(golden_cases.apps()))
def test_oracle_matches_reference_app_files(oracle_mod, name):
    """The reference's own case files (Apps/*/*.json), parsed by the JSON
    front end: the oracle reproduces the reference's run of the file bit
    for bit (digests of every block's f and moments)."""
    case, steps, want = golden_cases.apps()[name]
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    o.step(steps)
    o.update_macro()
    assert golden_cases.fingerprint(case, o.f, o.macro) == want


@pytest.mark.parametrize("seed", random_cases.SEEDS)
def test_oracle_matches_reference_random_cases(oracle_mod, seed):
    """Seeded random boxes (shapes, definition orders, moving and inflowing
    walls, outlets, periodic axes, body forces): the oracle is the
    reference bit for bit."""
    if not oracle_mod.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    case, steps = random_cases.random_case(seed)
    ref = oracle_mod.run_reference(case, steps)
    o, hist = run_oracle(oracle_mod, case, steps)
    for got, want in zip(o.macro(0), ref["macro"][0]):
        assert np.array_equal(got, want)
    assert np.array_equal(o.f(0), ref["f"][0])
    assert [h[0] for h in hist] == [r[1] for r in ref["residual"]]


@pytest.mark.parametrize("seed", random_cases.MULTI_SEEDS)
def test_oracle_matches_reference_random_two_blocks(oracle_mod, seed):
    """Seeded random pairs of blocks joined through VirtualBoundary
    connections (halo transfer between blocks, edge nodes of the joint):
    the oracle is the reference bit for bit."""
    if not oracle_mod.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    case, steps = random_cases.random_two_blocks(seed)
    ref = oracle_mod.run_reference(case, steps)
    o, hist = run_oracle(oracle_mod, case, steps)
    for b in case.block_ids:
        for got, want in zip(o.macro(b), ref["macro"][b]):
            assert np.array_equal(got, want)
        assert np.array_equal(o.f(b), ref["f"][b])
    assert [h[0] for h in hist] == [r[1] for r in ref["residual"]]


@pytest.mark.parametrize("seed", random_cases.SWAP_SEEDS)
def test_oracle_matches_reference_random_swap_boxes(oracle_mod, seed):
    """Seeded random boxes under the one-array swap scheme: the oracle's
    swap step is the reference's bit for bit."""
    if not oracle_mod.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    case, steps = random_cases.random_swap_box(seed)
    ref = oracle_mod.run_reference(case, steps)
    o, hist = run_oracle(oracle_mod, case, steps)
    for got, want in zip(o.macro(0), ref["macro"][0]):
        assert np.array_equal(got, want)
    assert np.array_equal(o.f(0), ref["f"][0])
    assert [h[0] for h in hist] == [r[1] for r in ref["residual"]]


@pytest.mark.parametrize("name", ["lchannel_app_9", "cavity2d_lid_first",
                                  "poiseuille3d"])
def test_parallel_parity_build_is_the_parity_build(oracle_mod, name):
    """ref_case_*_par (the parity build with OpenMP over loops without
    reductions, used for the full-size reference runs) gives the bits of
    the sequential parity build."""
    if not oracle_mod.reference_available("_par"):
        pytest.skip("reference build (oracle/_ref) not present")
    build, steps, cp = REF_CASES[name]
    case = build()
    case.check_period = cp
    seq = oracle_mod.run_reference(case, steps)
    par = oracle_mod.run_reference(case, steps, kind="_par")
    for b in case.block_ids:
        for got, want in zip(par["macro"][b], seq["macro"][b]):
            assert np.array_equal(got, want)
        assert np.array_equal(par["f"][b], seq["f"][b])
    assert par["residual"] == seq["residual"]


@pytest.mark.parametrize("name", sorted(golden_cases.bench_cases()))
def test_oracle_matches_reference_bench_cases(oracle_mod, name):
    """The benchmark cavity at 64^3 (300 steps) and the L-channel at
    96/32/32 (200 steps), fingerprinted from the reference's own run."""
    case, steps, residual, want = golden_cases.bench_cases()[name]
    o, hist = run_oracle(oracle_mod, case, steps)
    assert golden_cases.fingerprint(case, o.f, o.macro) == want
    assert [h[0] for h in hist] == [r[1] for r in residual]


def test_reference_fdperiodic_breaks_the_run(oracle_mod):
    """FDPeriodic as the reference runs it: KerCutCellPeriodic3D copies f
    from the halo of f, which its StreamCollision never transfers, so those
    nodes get zeros and the field turns to NaN within a few steps (10 steps
    of a forced channel made x-periodic through FDPeriodic instead of
    MDPeriodic).  The restatement copies from its own untouched halo of f the
    same way and gives the same field: zeros and NaNs at the same places,
    every other value bit for bit."""
    if not oracle_mod.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    case = special_cases.fdperiodic_channel()
    case.check_period = 5
    ref = oracle_mod.run_reference(case, 10)
    f = ref["f"][0]
    # FDPeriodic nodes of the Left face hold zeros, the interior is NaN
    assert np.all(f[:-1, 1:-1, 0] == 0.0)
    assert np.isnan(f[1:-1, 1:-1, 2:-2]).all()
    # the residual of rho is 0/0 (every interior rho is NaN but the sums
    # skip nothing): the reference reports NaN for u, v, w at least
    assert np.isnan(ref["residual"][-1][2][1:]).all()
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    o.step(10)
    got = o.f(0)
    assert np.array_equal(np.isnan(got), np.isnan(f))
    assert np.array_equal(got[~np.isnan(got)], f[~np.isnan(f)])


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_fdperiodic_edges_match_reference(oracle_mod, dim):
    """FDPeriodic and EQMDiffuseRefl mixed over a cavity's faces: the
    restatement's copies at faces, edges and corners (the reference's
    mislabelled edge and corner cases included) against the reference,
    NaNs at the same places and every other value bit for bit."""
    if not oracle_mod.reference_available():
        pytest.skip("reference build (oracle/_ref) not present")
    case = special_cases.fdperiodic_box(dim)
    case.check_period = 3
    ref = oracle_mod.run_reference(case, 3)
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    o.step(3)
    got, want = o.f(0), ref["f"][0]
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.array_equal(got[~np.isnan(got)], want[~np.isnan(want)])
    assert (got == 0.0).any()

