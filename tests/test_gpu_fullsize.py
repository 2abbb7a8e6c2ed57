"""The benchmark workloads at their full sizes against the reference itself:
the 256^3 lid-driven cavity (D3Q19, Re 400, lid 0.05) for 5 steps and the
unperturbed 3-block L-channel (384 x 128 x 128, 128^3, 128 x 384 x 128,
z-periodic, pressure outlet) for 20 steps, bit for bit in f and in the
moments against the reference's own sources built here against the
sequential OPS stand-in (the parity build with OpenMP over loops without
reductions, oracle/_ref/ref_case_3d_par).  Each run holds a few GB of host
memory."""
import tempfile

import numpy as np
import pytest

from mplb_b200 import Solver, config

pytestmark = pytest.mark.gpu


def compare_with_reference(oracle_mod, case, steps):
    if not oracle_mod.reference_available("_par"):
        pytest.skip("reference build (oracle/_ref) not present")
    s = Solver(case)
    s.init_uniform()
    s.stream_collision(steps)
    s.update_macro_vars()
    with tempfile.TemporaryDirectory(prefix="mplb_full_") as tmp:
        ref = oracle_mod.run_reference(case, steps, kind="_par",
                                       workdir=tmp)
        for b in case.block_ids:
            for got, want in zip(s.macro(b), ref["macro"][b]):
                assert np.array_equal(got, want)
            want_f = ref["f"].pop(b)
            assert np.array_equal(s.f(b), want_f)
            del want_f
    s.close()


def test_bench_cavity_256_matches_reference(gpu_lib, oracle_mod):
    case = config.cavity(3, 256, 0.05, re=400)
    compare_with_reference(oracle_mod, case, 5)


def test_lchannel_full_size_matches_reference(gpu_lib, oracle_mod):
    case = config.lchannel()
    assert case.nodes() == 14_680_064
    compare_with_reference(oracle_mod, case, 20)
