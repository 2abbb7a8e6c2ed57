"""Golden fixture of the 2D lid-driven cavity workload (D2Q9, FP64, 128x128
nodes, lid 0.05 lattice units on Top, Re = 100, reference walls
EQMDiffuseRefl), 20,000 steps with the residual every 1,000 steps, made by
the reference itself (oracle/_ref).  About 100 s of CPU.

    make -C oracle ref && python tests/golden/make_golden_config1.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mplb_b200 import config  # noqa: E402
from oracle import pyoracle  # noqa: E402


def main():
    case = config.cavity(2, 128, 0.05, re=100, check_period=1000)
    steps = 20000
    ref = pyoracle.run_reference(case, steps)
    arrays = {"steps": np.array(steps), "check_period": np.array(1000),
              "case_json": np.array(json.dumps(case.to_json()))}
    for n, a in zip(["rho", "u", "v"], ref["macro"][0]):
        arrays[f"{n}_b0"] = a
    arrays["f_b0"] = ref["f"][0]
    arrays["residual_steps"] = np.array([r[0] for r in ref["residual"]])
    arrays["residual_max"] = np.array([r[1] for r in ref["residual"]])
    arrays["residual_per_var"] = np.array([r[2] for r in ref["residual"]])
    out = os.path.join(HERE, "cavity2d_128_20k.npz")
    np.savez_compressed(out, **arrays)
    print(out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    main()
