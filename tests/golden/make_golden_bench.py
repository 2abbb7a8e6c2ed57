"""Fingerprints of the benchmark workloads at reduced size, run by the
reference itself.

The 3D lid-driven cavity of the benchmark (D3Q19, lid 0.05 lattice units
along +x on the z-max face, Re 400) at 64^3 for 300 steps, and the 3-block
L-channel (z-periodic, velocity inlet, pressure outlet, tau_L 0.6) at
96 x 32 x 32 / 32^3 / 32 x 96 x 32 for 200 steps, are run by the
reference's own sources built against the sequential OPS stand-in
(oracle/Makefile target "ref").  bench_cases.json stores per case the case
(reference JSON), the step count and check period, the residual history and
SHA-256 digests of every block's f and moments (float64, little-endian, the
reference driver's dump order).  Run where the reference sources are:

    make -C oracle ref && python tests/golden/make_golden_bench.py
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mplb_b200 import config  # noqa: E402
from oracle import pyoracle  # noqa: E402
from make_golden_apps import fingerprint  # noqa: E402

CASES = {
    # name: (builder, steps, check period)
    "cavity3d_64_re400": (lambda: config.cavity(3, 64, 0.05, re=400), 300,
                          100),
    "lchannel_96_32": (lambda: config.lchannel(leg=96, side=32, depth=32),
                       200, 100),
}


def main():
    res = {}
    for name, (build, steps, cp) in CASES.items():
        case = build()
        case.check_period = cp
        ref = pyoracle.run_reference(case, steps, kind="_par")
        res[name] = {"steps": steps, "check_period": cp,
                     "case_json": case.to_json(),
                     "residual": [[r[0], r[1], r[2]] for r in ref["residual"]],
                     "digest": fingerprint(case, ref["f"], ref["macro"])}
        print(name, steps, "steps")
    with open(os.path.join(HERE, "bench_cases.json"), "w") as fh:
        json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
