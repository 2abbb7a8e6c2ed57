"""The drop-in: the reference's own setup code (Src/*.cpp through the
sequential OPS stand-in) driving the B200 path through the C++ glue in
mplb_b200/dropin instead of its own StreamCollision, UpdateMacroVars and
CalcResidualError.  Results must equal the reference's golden fixtures bit
for bit (residuals to round-off of the summation order)."""
import os

import numpy as np
import pytest

import golden_cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", golden_cases.names())
def test_dropin_matches_reference(gpu_lib, oracle_mod, name):
    g = golden_cases.load(name)
    case = g["case"]
    exe = os.path.join(oracle_mod.REF_DIR, f"dropin_case_{case.space_dim}d")
    if not os.path.exists(exe):
        pytest.skip("drop-in driver (make -C oracle dropin) not built")
    out = oracle_mod.run_reference(case, g["steps"], program="dropin_case")
    for b in case.block_ids:
        for got, want in zip(out["macro"][b], g["macro"][b]):
            assert np.array_equal(got, want), name
        assert np.array_equal(out["f"][b], g["f"][b]), name
    np.testing.assert_allclose([r[1] for r in out["residual"]],
                               g["residual_max"], rtol=1e-12)
