"""Fingerprints of the reference's own app case files run by the reference.

The reference's JSON case files (Apps/2DCavity/Cavity2D.json,
Apps/3DCavity/Cavity3D.json, Apps/3DLChannel/LChannel.json) are read by the
reference's own configuration reader inside its solver (built against the
sequential OPS stand-in, oracle/Makefile target "ref") and run for a fixed
number of steps.  The final moments and distributions are too large to
keep, so apps.json stores, per case, the parse of the file by
mplb_b200.config (re-serialised, so the tests need no reference files), the
step count and SHA-256 digests of every block's f and moments (float64,
little-endian, the dump order of the reference driver).  Run where the
reference sources are available:

    make -C oracle ref && python tests/golden/make_golden_apps.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mplb_b200.config import CaseConfig  # noqa: E402
from oracle import pyoracle  # noqa: E402

APPS = {
    # name: (case file under the reference's Apps/, steps)
    "app_cavity2d": ("2DCavity/Cavity2D.json", 300),
    "app_cavity3d": ("3DCavity/Cavity3D.json", 100),
    "app_lchannel": ("3DLChannel/LChannel.json", 60),
}


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, "<f8").tobytes()).hexdigest()


def fingerprint(case, f, macro):
    names = ["rho", "u", "v", "w"][:case.space_dim + 1]
    out = {}
    for b in case.block_ids:
        out[f"f_b{b}"] = digest(f[b])
        for n, a in zip(names, macro[b]):
            out[f"{n}_b{b}"] = digest(a)
    return out


def main():
    res = {}
    for name, (rel, steps) in APPS.items():
        path = os.path.join(pyoracle.REF_ROOT, "Apps", rel)
        case = CaseConfig.load(path)
        ref = pyoracle.run_reference(case, steps, json_path=path)
        res[name] = {"file": "Apps/" + rel, "steps": steps,
                     "case_json": case.to_json(),
                     "digest": fingerprint(case, ref["f"], ref["macro"])}
        print(name, steps, "steps")
    with open(os.path.join(HERE, "apps.json"), "w") as fh:
        json.dump(res, fh, indent=1)


if __name__ == "__main__":
    main()
