"""Loads the golden fixtures made by tests/golden/make_golden.py."""
import json
import os

import numpy as np

from mplb_b200.config import CaseConfig

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# fixtures the CPU oracle replays in seconds; the rest (long runs of the
# benchmark workloads) are replayed on the GPU only
LONG = ("cavity2d_128_20k",)


def names(include_long=False):
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz")
                  and (include_long or f[:-4] not in LONG))


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    case = CaseConfig.from_json(json.loads(str(z["case_json"])))
    case.check_period = int(z["check_period"])
    out = {"case": case, "steps": int(z["steps"]), "macro": {}, "f": {},
           "residual_steps": z["residual_steps"],
           "residual_max": z["residual_max"],
           "residual_per_var": z["residual_per_var"]}
    vars_ = ["rho", "u", "v", "w"][:case.space_dim + 1]
    for b in case.block_ids:
        out["macro"][b] = [z[f"{n}_b{b}"] for n in vars_]
        out["f"][b] = z[f"f_b{b}"]
    return out


def apps():
    """The reference's own app case files, parsed and fingerprinted (made by
    tests/golden/make_golden_apps.py): name -> (case, steps, digests)."""
    with open(os.path.join(GOLDEN, "apps.json")) as fh:
        d = json.load(fh)
    return {k: (CaseConfig.from_json(v["case_json"]), v["steps"], v["digest"])
            for k, v in d.items()}


def fingerprint(case, f_of, macro_of):
    """SHA-256 digests in the layout of make_golden_apps.fingerprint."""
    import hashlib
    names = ["rho", "u", "v", "w"][:case.space_dim + 1]

    def dig(a):
        return hashlib.sha256(np.ascontiguousarray(a, "<f8").tobytes()
                              ).hexdigest()
    out = {}
    for b in case.block_ids:
        out[f"f_b{b}"] = dig(f_of(b))
        for n, a in zip(names, macro_of(b)):
            out[f"{n}_b{b}"] = dig(a)
    return out


def bench_cases():
    """The benchmark workloads at reduced size run by the reference (made
    by tests/golden/make_golden_bench.py): name -> (case, steps, residual
    history [(step, max, per-variable)], digests)."""
    with open(os.path.join(GOLDEN, "bench_cases.json")) as fh:
        d = json.load(fh)
    out = {}
    for k, v in d.items():
        case = CaseConfig.from_json(v["case_json"])
        case.check_period = v["check_period"]
        out[k] = (case, v["steps"], v["residual"], v["digest"])
    return out
