"""Generates the golden fixtures in this directory from the reference itself.

The reference solver's own sources, built against the sequential OPS
stand-in (oracle/Makefile, target "ref"), are run on small cases written in
the reference's JSON format; the final moments, distributions and residual
history are saved as .npz.  Run in a checkout that has the reference
sources available:

    make -C oracle ref && python tests/golden/make_golden.py [name ...]

(all cases, or only the named ones).  The *_swap cases run the reference's
one-array swap step (SchemeType Scheme_StreamCollision_Swap).
"""
import dataclasses
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mplb_b200 import config  # noqa: E402
from oracle import pyoracle  # noqa: E402

CASES = {
    # name: (builder, steps, check period)
    "cavity2d_24": (lambda: config.cavity(2, 24, 0.05, re=100), 300, 100),
    "cavity2d_order": (lambda: config.cavity(
        2, 17, 0.08, re=50, order=("Top", "Bottom", "Left", "Right")), 200, 50),
    "cavity3d_10": (lambda: config.cavity(3, 10, 0.05, re=400), 60, 20),
    "lchannel_app_7": (lambda: config.lchannel_app(7, inflow=0.01), 60, 20),
    "lchannel_periodic": (lambda: config.lchannel(leg=10, side=6, depth=5),
                          60, 20),
    "poiseuille2d": (lambda: config.poiseuille(2, 12, 9, g_lattice=1e-4),
                     300, 100),
    "poiseuille3d": (lambda: config.poiseuille(3, 6, 8, 5, g_lattice=1e-4),
                     80, 40),
    "cavity3d_10_swap": (lambda: config.cavity(
        3, 10, 0.05, re=400, scheme="Scheme_StreamCollision_Swap"), 60, 20),
    # non-cubic box, first-order body force with the force-shifted velocity
    "box3d_force_swap": (lambda: dataclasses.replace(
        config.cavity(3, 10, 0.05, re=400,
                      scheme="Scheme_StreamCollision_Swap"),
        block_sizes=[(12, 9, 7)], body_force="BodyForce_1st",
        accel=(3e-3, -2e-3, 1e-3), force_velocity=True), 41, 10),
    # another definition order and a face whose scheme dispatches no kernel
    "box3d_order_swap": (lambda: _order_swap(), 25, 5),
}


def _order_swap():
    c = config.cavity(3, 8, 0.05, re=100, scheme="Scheme_StreamCollision_Swap",
                      order=("Front", "Back", "Top", "Bottom", "Left",
                             "Right"))
    b = list(c.boundaries)
    b[3] = dataclasses.replace(b[3], scheme="BounceBack")
    return dataclasses.replace(c, block_sizes=[(8, 11, 6)], boundaries=b)


def main(names=None):
    for name, (build, steps, cp) in CASES.items():
        if names and name not in names:
            continue
        case = build()
        case.check_period = cp
        ref = pyoracle.run_reference(case, steps)
        arrays = {"steps": np.array(steps), "check_period": np.array(cp),
                  "case_json": np.array(json.dumps(case.to_json()))}
        for b in case.block_ids:
            for n, a in zip(["rho", "u", "v", "w"], ref["macro"][b]):
                arrays[f"{n}_b{b}"] = a
            arrays[f"f_b{b}"] = ref["f"][b]
        arrays["residual_steps"] = np.array([r[0] for r in ref["residual"]])
        arrays["residual_max"] = np.array([r[1] for r in ref["residual"]])
        arrays["residual_per_var"] = np.array([r[2] for r in ref["residual"]])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, steps, "steps", os.path.getsize(
            os.path.join(HERE, name + ".npz")), "bytes")


if __name__ == "__main__":
    main(sys.argv[1:])
