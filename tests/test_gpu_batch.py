"""Batched cavities: every cavity of an FP64 batch is bit-identical to the
same cavity run alone through the single-block path (halfway bounce-back
walls, lid on Top), in both launch styles (one CTA per tile, cooperative
persistent); residuals match the
single-block residual; converged cavities drop out; FP32 tracks FP64."""
import numpy as np
import pytest

from mplb_b200 import Solver, config
from mplb_b200.batch import Batch, CavitySpec

pytestmark = pytest.mark.gpu

SPECS = [CavitySpec(6, 30.0, 0.05), CavitySpec(9, 100.0, 0.08),
         CavitySpec(13, 60.0, 0.03), CavitySpec(20, 200.0, 0.06),
         CavitySpec(7, 15.0, 0.02)]


def single(spec, steps, check=None):
    case = config.cavity(2, spec.n, spec.lid, tau_lattice=spec.tau_lattice,
                         wall="HalfwayBounceBack")
    s = Solver(case)
    s.init_uniform()
    res = []
    if check:
        for _ in range(steps // check):
            s.stream_collision(check)
            s.update_macro_vars()
            res.append(s.calc_residual_error(check)[0])
    else:
        s.stream_collision(steps)
        s.update_macro_vars()
    m = s.macro(0)
    s.close()
    return [a[0] for a in m], res


@pytest.mark.parametrize("persistent", [0, 1])
@pytest.mark.parametrize("steps", [37, 100])
def test_batch_fp64_bitwise_vs_single(gpu_lib, persistent, steps):
    b = Batch(SPECS, "fp64")
    b.set_tuning(tile_nodes=64, persistent=persistent, chunk=10,
                 ctas_per_sm=2)
    b.init()
    b.step(steps)
    got = b.macro()
    for spec, g in zip(SPECS, got):
        want, _ = single(spec, steps)
        for a, w in zip(g, want):
            assert np.array_equal(a, w), (spec, persistent, steps)
    b.close()


def test_batch_residuals_vs_single(gpu_lib):
    b = Batch(SPECS, "fp64")
    b.set_tuning(tile_nodes=128, persistent=0, chunk=10, ctas_per_sm=4)
    b.init()
    steps, res, conv = b.run(max_steps=60, check_period=20, criterion=0.0)
    assert (steps == 60).all() and not conv.any()
    for spec, r in zip(SPECS, res):
        _, hist = single(spec, 60, check=20)
        np.testing.assert_allclose(r, hist[-1], rtol=1e-12)
    b.close()


def test_batch_convergence_drops_cavities(gpu_lib):
    specs = [CavitySpec(8, 5.0, 0.02), CavitySpec(24, 400.0, 0.08)]
    b = Batch(specs, "fp32")
    b.init()
    steps, res, conv = b.run(max_steps=20000, check_period=200,
                             criterion=1e-6)
    assert conv[0] and steps[0] < steps[1]
    assert res[0] < 1e-6
    b.close()


def test_batch_fp32_vs_fp64(gpu_lib):
    out = {}
    for prec in ("fp64", "fp32"):
        b = Batch(SPECS, prec)
        b.init()
        b.step(400)
        out[prec] = b.macro()
        b.close()
    for a, w in zip(out["fp32"], out["fp64"]):
        speed = np.hypot(a[1], a[2])
        ref = np.hypot(w[1], w[2])
        assert np.linalg.norm(speed - ref) / np.linalg.norm(ref) < 1e-4


def test_diverged_cavity_is_reported_not_converged(gpu_lib):
    """tau_L = 0.50015 with a fast lid: BGK blows up; the batch reports the
    cavity as diverged (NaN residual) and keeps solving the healthy one."""
    specs = [CavitySpec(64, 1.0e5, 0.08), CavitySpec(64, 100.0, 0.05)]
    b = Batch(specs, "fp32", lib=gpu_lib)
    b.init()
    steps, res, conv = b.run(max_steps=100000, check_period=1000,
                             criterion=1e-8)
    assert b.diverged.tolist() == [True, False]
    assert not conv[0] and np.isnan(res[0]) and steps[0] < 100000
    assert conv[1] and res[1] < 1e-8


@pytest.mark.parametrize("tile", [128, 256])
def test_batch_large_cavity_row_division(gpu_lib, tile):
    """A cavity above 1024 nodes per side takes the integer-division row
    index (the float reciprocal is exact only up to 1024): still bit for
    bit the single-block run, next to small ones."""
    specs = [CavitySpec(1030, 400.0, 0.05), CavitySpec(11, 50.0, 0.04)]
    b = Batch(specs, "fp64")
    b.set_tuning(tile_nodes=tile, persistent=0, chunk=2, ctas_per_sm=4)
    b.init()
    b.step(6)
    got = b.macro()
    for spec, g in zip(specs, got):
        want, _ = single(spec, 6)
        for a, w in zip(g, want):
            assert np.array_equal(a, w), spec
    b.close()


def test_autotune_valid_cached_and_bitwise(gpu_lib, tmp_path):
    """The autotuner times its candidates on the batch, keeps one of them,
    caches it (a second call reads the cache), and the batch it tunes gives
    the bits of the default tuning (FP64)."""
    from mplb_b200.batch import autotune, default_candidates
    cache = str(tmp_path / "tuning.json")
    b = Batch(SPECS, "fp64")
    best = autotune(b, steps=20, cache=cache)
    assert best["tuning"] in default_candidates()
    assert len(best["all"]) == len(default_candidates())
    assert all(r["mlups"] > 0 for r in best["all"])
    assert b.tuning() == best["tuning"]
    again = autotune(b, steps=20, cache=cache)
    assert again == best
    b.init()
    b.step(37)
    tuned = b.macro()
    b.close()
    d = Batch(SPECS, "fp64")
    d.init()
    d.step(37)
    for g, w in zip(tuned, d.macro()):
        for x, y in zip(g, w):
            assert np.array_equal(x, y)
    d.close()


def test_persistent_barrier_timeout_then_reinit(gpu_lib):
    """A grid barrier that gives up (a one-poll limit) ends the persistent
    launch with MPLBGPU_ERR_TIMEOUT instead of waiting on; the batch then
    refuses to step (MPLBGPU_ERR_STATE) until it is initialised again, after
    which it runs as a fresh batch, bit for bit."""
    from mplb_b200 import abi
    from mplb_b200.batch import BatchError
    b = Batch(SPECS, "fp64")
    b.set_tuning(tile_nodes=64, persistent=1, chunk=10, ctas_per_sm=2)
    b.init()
    b.set_wait_limit(1)
    with pytest.raises(BatchError) as e:
        b.step(10)
    assert e.value.status == abi.ERR_TIMEOUT
    with pytest.raises(BatchError) as e:
        b.step(10)
    assert e.value.status == abi.ERR_STATE
    b.set_wait_limit(1 << 26)
    b.init()
    b.step(37)
    got = b.macro()
    b.close()
    for spec, g in zip(SPECS, got):
        want, _ = single(spec, 37)
        for a, w in zip(g, want):
            assert np.array_equal(a, w), spec
