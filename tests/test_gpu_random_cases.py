"""The CUDA path (FP64, through the C ABI) against the oracle on the seeded
random boxes of random_cases.py (which the CPU suite checks against the
reference itself): moments and distributions bit for bit, residuals within
a relative 1e-12 (different summation order)."""
import numpy as np
import pytest

import random_cases
from mplb_b200 import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", random_cases.SEEDS)
def test_gpu_matches_oracle_random_cases(gpu_lib, oracle_mod, seed):
    case, steps = random_cases.random_case(seed)
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
    for got, want in zip(s.macro(0), o.macro(0)):
        assert np.array_equal(got, want), seed
    assert np.array_equal(s.f(0), o.f(0)), seed
    s.close()
