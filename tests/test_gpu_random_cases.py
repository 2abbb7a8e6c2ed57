"""The CUDA path (FP64, through the C ABI) against the oracle on the seeded
random cases of random_cases.py (single boxes, pairs of joined blocks and
swap-scheme boxes, all of which the CPU suite checks against the reference
itself): moments and distributions bit for bit, residuals within a relative
1e-12 (different summation order)."""
import numpy as np
import pytest

import random_cases
from mplb_b200 import Solver

pytestmark = pytest.mark.gpu


def compare(oracle_mod, case, steps, seed):
    cp = case.check_period
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    s = Solver(case)
    s.init_uniform()
    for _ in range(steps // cp):
        o.step(cp)
        o.update_macro()
        s.stream_collision(cp)
        s.update_macro_vars()
        np.testing.assert_allclose(s.calc_residual_error(cp)[0],
                                   o.residual(cp)[0], rtol=1e-12, atol=0)
    o.step(steps % cp)
    o.update_macro()
    s.stream_collision(steps % cp)
    s.update_macro_vars()
    for b in case.block_ids:
        for got, want in zip(s.macro(b), o.macro(b)):
            assert np.array_equal(got, want), seed
        assert np.array_equal(s.f(b), o.f(b)), seed
    s.close()


@pytest.mark.parametrize("seed", random_cases.SEEDS)
def test_gpu_matches_oracle_random_cases(gpu_lib, oracle_mod, seed):
    case, steps = random_cases.random_case(seed)
    compare(oracle_mod, case, steps, seed)


@pytest.mark.parametrize("seed", random_cases.MULTI_SEEDS)
def test_gpu_matches_oracle_random_two_blocks(gpu_lib, oracle_mod, seed):
    """Pairs of blocks joined through VirtualBoundary connections along a
    random axis (halo transfer, edge nodes of the joint)."""
    case, steps = random_cases.random_two_blocks(seed)
    compare(oracle_mod, case, steps, seed)


@pytest.mark.parametrize("seed", random_cases.SWAP_SEEDS)
def test_gpu_matches_oracle_random_swap_boxes(gpu_lib, oracle_mod, seed):
    """Boxes under the reference's one-array swap scheme."""
    case, steps = random_cases.random_swap_box(seed)
    compare(oracle_mod, case, steps, seed)
