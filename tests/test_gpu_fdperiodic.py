"""FDPeriodic on the GPU against the oracle restatement (pinned to the
reference's own build on CPU): the reference's KerCutCellPeriodic(3D)
copies every population from a halo cell of f that no step writes, so its
nodes get f = 0 and the field turns to NaN; the step gives the same field,
NaNs at the same places and every other value bit for bit."""
import numpy as np
import pytest

import special_cases
from mplb_b200 import Solver

pytestmark = pytest.mark.gpu

CASES = {
    "channel3d": (special_cases.fdperiodic_channel, 10),
    "box3d": (lambda: special_cases.fdperiodic_box(3), 3),
    "box2d": (lambda: special_cases.fdperiodic_box(2), 3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fdperiodic_matches_oracle(gpu_lib, oracle_mod, name):
    build, steps = CASES[name]
    case = build()
    o = oracle_mod.Oracle(case)
    o.init_uniform()
    o.step(steps)
    with Solver(case) as s:
        s.init_uniform()
        s.stream_collision(steps)
        for blk in case.block_ids:
            got, want = s.f(blk), o.f(blk)
            assert np.array_equal(np.isnan(got), np.isnan(want)), name
            assert np.array_equal(got[~np.isnan(got)], want[~np.isnan(want)])
            assert (got == 0.0).any()
