"""Python access to the CPU checkers (TEST INFRASTRUCTURE ONLY).

* ``Oracle``: ctypes binding of liblbmoracle.so, the C restatement of the
  reference step (lbm_oracle.c).
* ``run_reference``: runs the reference solver itself (oracle/_ref, the
  reference's own sources built against the sequential OPS stand-in) on a
  case written in the reference's JSON format.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg and
reference arm (`--impl reference`) use this module.
"""
import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblbmoracle.so")
REF_DIR = os.path.join(HERE, "_ref")
# where the reference's sources are (only needed to build oracle/_ref)
REF_ROOT = os.environ.get("MPLB_REFERENCE_ROOT", "/root/reference")


def build_restatement():
    """Compiles the C restatement if it is missing or stale."""
    src = [os.path.join(HERE, "lbm_oracle.c"), os.path.join(HERE,
                                                             "lbm_oracle.h")]
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(s)
                                   for s in src):
        return LIB
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    return LIB


def reference_available(kind=""):
    return os.path.exists(os.path.join(REF_DIR, f"ref_case_2d{kind}")) and \
        os.path.exists(os.path.join(REF_DIR, f"ref_case_3d{kind}"))


def build_reference():
    """Builds oracle/_ref from the reference sources (only where they are)."""
    if not os.path.isdir(os.path.join(REF_ROOT, "Src")):
        return False
    subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref",
                    f"REF_ROOT={REF_ROOT}"], check=True)
    return True


class Oracle:
    def __init__(self, case):
        build_restatement()
        self.lib = ctypes.CDLL(LIB)
        L = self.lib
        vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.lbmo_create.argtypes = [vp, ctypes.POINTER(vp)]
        L.lbmo_create.restype = ip
        L.lbmo_error.restype = ctypes.c_char_p
        L.lbmo_destroy.argtypes = [vp]
        L.lbmo_init_macro.argtypes = [vp, ip, vp, vp, vp, vp]
        L.lbmo_set_f.argtypes = [vp, ip, vp]
        L.lbmo_step.argtypes = [vp, ip]
        L.lbmo_update_macro.argtypes = [vp]
        L.lbmo_residual.argtypes = [vp, ip, vp, vp]
        L.lbmo_get_macro.argtypes = [vp, ip, vp, vp, vp, vp]
        L.lbmo_get_f.argtypes = [vp, ip, vp]
        L.lbmo_get_node_info.argtypes = [vp, ip, vp, vp]
        L.lbmo_boundary_extent.argtypes = [vp, ip, vp]
        L.lbmo_set_boundary_velocity.argtypes = [vp, ip, vp, vp, vp]
        self.case = case
        desc, self._keep = case.to_desc()
        self._desc = desc
        h = ctypes.c_void_p()
        if L.lbmo_create(ctypes.byref(desc), ctypes.byref(h)) != 0:
            raise ValueError(L.lbmo_error().decode())
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lbmo_destroy(self.h)
            self.h = None

    def _shape(self, b):
        nx, ny, nz = self.case.size3(b)
        return (nz, ny, nx)

    def init_macro(self, block, rho=None, u=None, v=None, w=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64)
                for a in (rho, u, v, w)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self.lib.lbmo_init_macro(self.h, block, *ptrs)

    def init_uniform(self):
        rho, u, v, w = self.case.initial
        for b in self.case.block_ids:
            shp = self._shape(b)
            self.init_macro(b, np.full(shp, rho), np.full(shp, u),
                            np.full(shp, v), np.full(shp, w))

    def set_f(self, block, f):
        f = np.ascontiguousarray(f, np.float64)
        self.lib.lbmo_set_f(self.h, block, f.ctypes.data)

    def boundary_extent(self, boundary):
        ext = (ctypes.c_int * 3)()
        if self.lib.lbmo_boundary_extent(self.h, boundary, ext) != 0:
            raise ValueError(self.lib.lbmo_error().decode())
        return tuple(ext)

    def set_boundary_velocity(self, boundary, u=None, v=None, w=None):
        nx, ny, nz = self.boundary_extent(boundary)
        arrs = [None if a is None else np.ascontiguousarray(
            np.broadcast_to(a, (nz, ny, nx)), np.float64) for a in (u, v, w)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        if self.lib.lbmo_set_boundary_velocity(self.h, boundary, *ptrs) != 0:
            raise ValueError(self.lib.lbmo_error().decode())

    def step(self, n=1):
        self.lib.lbmo_step(self.h, n)

    def update_macro(self):
        self.lib.lbmo_update_macro(self.h)

    def residual(self, check_period):
        per = np.zeros(4)
        mx = ctypes.c_double()
        self.lib.lbmo_residual(self.h, check_period, per.ctypes.data,
                               ctypes.byref(mx))
        return mx.value, per[:self.case.space_dim + 1]

    def macro(self, block):
        shp = self._shape(block)
        out = [np.zeros(shp) for _ in range(4)]
        self.lib.lbmo_get_macro(self.h, block, *[a.ctypes.data for a in out])
        return out[:self.case.space_dim + 1]

    def f(self, block):
        shp = self._shape(block) + (self.case.q,)
        out = np.zeros(shp)
        self.lib.lbmo_get_f(self.h, block, out.ctypes.data)
        return out

    def node_info(self, block):
        shp = self._shape(block)
        vt = np.zeros(shp, np.int32)
        vg = np.zeros(shp, np.int32)
        self.lib.lbmo_get_node_info(self.h, block, vt.ctypes.data,
                                    vg.ctypes.data)
        return vt, vg


def run_reference(case, steps, kind="", workdir=None, program="ref_case",
                  json_path=None):
    """Runs oracle/_ref/{program}_{2d,3d}{kind}; returns dict with macro
    arrays per block, f per block and the residual history.  program
    "dropin_case" is the same driver with the B200 drop-in glue in place of
    the reference's step.  json_path: run that case file as it is (the
    reference's own JSON reader parses it) instead of case.to_json()."""
    exe = os.path.join(REF_DIR, f"{program}_{case.space_dim}d{kind}")
    tmp = workdir or tempfile.mkdtemp(prefix="mplbref_")
    cfg = os.path.join(tmp, "case.json")
    if json_path is not None:
        with open(json_path) as src, open(cfg, "w") as fh:
            fh.write(src.read())
    else:
        with open(cfg, "w") as fh:
            json.dump(case.to_json(), fh)
    env = dict(os.environ, OPS_SHIM_QUIET="1")
    subprocess.run([exe, cfg, tmp, str(steps)], check=True, env=env)
    names = ["rho", "u", "v", "w"][:case.space_dim + 1]
    out = {"macro": {}, "f": {}, "residual": []}
    for b in case.block_ids:
        nx, ny, nz = case.size3(b)
        out["macro"][b] = [np.fromfile(os.path.join(tmp, f"{n}_b{b}.f64"))
                           .reshape(nz, ny, nx) for n in names]
        out["f"][b] = np.fromfile(os.path.join(tmp, f"f_b{b}.f64")).reshape(
            nz, ny, nx, case.q)
    with open(os.path.join(tmp, "residual.txt")) as fh:
        for line in fh:
            vals = line.split()
            out["residual"].append((int(vals[0]), float(vals[1]),
                                    [float(v) for v in vals[2:]]))
    return out


def time_reference(case, warmup, steps, kind="_fast", threads=None):
    """Seconds for `steps` reference StreamCollision calls after `warmup`."""
    exe = os.path.join(REF_DIR, f"ref_case_{case.space_dim}d{kind}")
    tmp = tempfile.mkdtemp(prefix="mplbref_t_")
    cfg = os.path.join(tmp, "case.json")
    with open(cfg, "w") as fh:
        json.dump(case.to_json(), fh)
    env = dict(os.environ, OPS_SHIM_QUIET="1")
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    res = subprocess.run([exe, cfg, tmp, str(warmup), str(steps)], check=True,
                         env=env, capture_output=True, text=True)
    parts = res.stdout.split()
    return float(parts[1]), int(parts[3])
