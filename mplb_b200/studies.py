"""Accuracy and throughput studies of the storage forms.

    python -m mplb_b200.studies precision [--quick]

Body-force Poiseuille channels (D2Q9 4096 x 1024 for 50,000 steps and
D3Q19 512 x 256 x 256 for 10,000 steps; tau_L = 0.8, g_L = 1e-6 along x;
walls at y-min/y-max, periodic in x and z) in the FP64 form (bit-identical
to the reference), the shifted FP32 form and the FP16-storage form.  The
channels' viscous times H^2/nu (10^7 and 6.6 x 10^5 steps) are far longer
than the prescribed runs, so a start from rest is far from developed at the
end.  Where the analytic profile is subsonic (peak below 0.3 lattice units:
the 3D channel, 0.082) the flow starts from it and the error against the
profile measures discretisation and storage error; the 2D channel's profile
would peak at 1.31 lattice units, so it starts from rest and its analytic
comparison only shows how far the flow has developed.  Each form
reports relative L2 and max errors of rho and u against the FP64 form and
of u against the profile, and its device-time MLUPS.  One JSON line per
run.
"""
import argparse
import json
import math
import sys

import numpy as np

from . import config
from .solver import Solver

SQRT3 = math.sqrt(3.0)


def analytic_u(ny, g, tau, wall):
    """Lattice-unit profile: walls half a spacing outside the first/last
    node for halfway bounce-back (H = ny), on the first/last node for
    EQMDiffuseRefl (H = ny - 1)."""
    nu = (tau - 0.5) / 3.0
    if wall == "HalfwayBounceBack":
        y = np.arange(ny) + 0.5
        h = ny
    else:
        y = np.arange(ny, dtype=float)
        h = ny - 1
    return g / (2.0 * nu) * y * (h - y)


def rel(a, b):
    d = a - b
    nb = np.linalg.norm(b)
    mb = np.abs(b).max()
    return (float(np.linalg.norm(d) / nb) if nb > 0 else float("nan"),
            float(np.abs(d).max() / mb) if mb > 0 else float("nan"))


def run_channel(dim, nx, ny, nz, steps, precision, wall, g=1e-6, tau=0.8):
    case = config.poiseuille(dim, nx, ny, nz, g_lattice=g, tau_lattice=tau,
                             wall=wall, precision=precision)
    ua = analytic_u(ny, g, tau, wall) * SQRT3
    shape = (nz, ny, nx) if dim == 3 else (1, ny, nx)
    start = "analytic" if ua.max() / SQRT3 < 0.3 else "rest"
    u0 = np.broadcast_to(ua[None, :, None], shape) if start == "analytic" \
        else 0.0
    with Solver(case) as s:
        s.init_macro(0, 1.0, u0, 0.0, 0.0 if dim == 3 else None)
        s.stream_collision(steps)
        ms = s.last_step_ms()
        s.update_macro_vars()
        m = s.macro(0)
    mlups = case.nodes() * steps / (ms * 1e-3) / 1e6
    return m, mlups, ua, start


def precision_study(quick=False):
    runs = [(2, 4096, 1024, 1, 50000), (3, 512, 256, 256, 10000)]
    if quick:
        runs = [(2, 256, 64, 1, 4000), (3, 64, 32, 32, 1000)]
    for dim, nx, ny, nz, steps in runs:
        for wall in ("HalfwayBounceBack", "EQMDiffuseRefl"):
            ref, ref_mlups, ua, start = run_channel(dim, nx, ny, nz, steps,
                                                    "fp64", wall)
            for prec in ("fp64", "fp32", "fp16"):
                if prec == "fp64":
                    m, mlups = ref, ref_mlups
                else:
                    m, mlups, _, _ = run_channel(dim, nx, ny, nz, steps,
                                                 prec, wall)
                u = m[1]
                prof = u.mean(axis=(0, 2)) / SQRT3
                line = {
                    "study": "precision", "dim": dim,
                    "grid": [nx, ny] + ([nz] if dim == 3 else []),
                    "steps": steps, "wall": wall, "precision": prec,
                    "start": start,
                    "mlups": mlups,
                    "rho_vs_fp64": rel(m[0], ref[0]),
                    "u_vs_fp64": rel(u, ref[1]),
                    "u_vs_analytic": rel(prof, ua / SQRT3),
                }
                print(json.dumps(line), flush=True)


def main(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("study", choices=["precision"])
    p.add_argument("--quick", action="store_true")
    a = p.parse_args(argv)
    if a.study == "precision":
        precision_study(a.quick)


if __name__ == "__main__":
    main(sys.argv[1:])
