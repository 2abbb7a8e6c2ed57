"""Python front end of the C ABI (include/mplbgpu.h).

``Solver`` mirrors the reference's iteration API for one case:

* ``Solver(case)`` - the state after the reference's Define* calls and
  ``Partition()`` (descriptor built from a ``CaseConfig``);
* ``init_uniform()`` / ``init_macro()`` - SetInitialMacrosVars followed by
  PreDefinedInitialCondition3D (f = feq);
* ``stream_collision(n)`` - n calls of StreamCollision()
  (Src/evolution.cpp:137-193);
* ``update_macro_vars()``, ``calc_residual_error()`` - UpdateMacroVars3D,
  CalcResidualError + GetMaximumResidual;
* ``iterate(steps=..)`` / ``iterate(criterion=..)`` - the two Iterate
  overloads (Src/evolution.cpp:71-135) without the HDF5 output.

Every call goes through libmplbgpu.so; there is no fallback path.
"""
import ctypes

import numpy as np

from . import abi


class MplbGpuError(RuntimeError):
    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")


class Solver:
    def __init__(self, case, lib=None):
        self.lib = lib or abi.load_library()
        self.case = case
        desc, self._keep = case.to_desc()
        self._desc = desc
        h = ctypes.c_void_p()
        rc = self.lib.mplbgpu_create(ctypes.byref(desc), ctypes.byref(h))
        if rc != abi.OK:
            raise MplbGpuError(rc, self.lib.mplbgpu_last_error(None).decode())
        self.h = h
        self.steps_done = 0

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.lib.mplbgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != abi.OK:
            raise MplbGpuError(rc, self.lib.mplbgpu_last_error(self.h).decode())

    def _shape(self, block):
        nx, ny, nz = self.case.size3(block)
        return (nz, ny, nx)

    # -- initial state ------------------------------------------------------
    def init_macro(self, block, rho=None, u=None, v=None, w=None):
        arrs = [None if a is None else
                np.ascontiguousarray(np.broadcast_to(a, self._shape(block)),
                                     np.float64) for a in (rho, u, v, w)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self._check(self.lib.mplbgpu_init_macro(self.h, block, *ptrs))
        self.steps_done = 0

    def init_uniform(self):
        rho, u, v, w = self.case.initial
        for b in self.case.block_ids:
            self.init_macro(b, rho, u, v, w)

    def upload_f(self, block, f):
        f = np.ascontiguousarray(f, np.float64)
        if f.shape != self._shape(block) + (self.case.q,):
            raise ValueError(f"f must have shape {self._shape(block)} + (Q,)")
        self._check(self.lib.mplbgpu_upload_f(self.h, block, f.ctypes.data))

    def boundary_extent(self, boundary):
        """(nx, ny, nz) of the node range of boundary `boundary` (index in
        definition order)."""
        ext = (ctypes.c_int * 3)()
        self._check(self.lib.mplbgpu_boundary_extent(self.h, int(boundary),
                                                     ext))
        return tuple(ext)

    def set_boundary_velocity(self, boundary, u=None, v=None, w=None):
        """Per-node wall velocity (MPLB units) of an EQMDiffuseRefl or
        halfway bounce-back boundary: arrays of shape (nz, ny, nx) over its
        node range (boundary_extent); all None restores the uniform given
        values.  No counterpart in the reference (uniform GivenVars)."""
        nx, ny, nz = self.boundary_extent(boundary)
        arrs = [None if a is None else np.ascontiguousarray(
            np.broadcast_to(a, (nz, ny, nx)), np.float64) for a in (u, v, w)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self._check(self.lib.mplbgpu_set_boundary_velocity(
            self.h, int(boundary), *ptrs))

    def set_step(self, step):
        """Positions the run at `step` (a restart's CurrentTimeStep): the
        check periods of iterate() and the FP16 rounding draws continue
        from there."""
        self._check(self.lib.mplbgpu_set_step(self.h, int(step)))
        self.steps_done = int(step)

    def step_kernel(self, block_id):
        """Which step kernel the block runs: "node", "split" or "swap"
        (mplbgpu_step_kernel)."""
        k = ctypes.c_int(-1)
        self._check(self.lib.mplbgpu_step_kernel(self.h, int(block_id),
                                                 ctypes.byref(k)))
        return ("node", "split", "swap")[k.value]

    # -- time stepping ------------------------------------------------------
    def stream_collision(self, n=1):
        self._check(self.lib.mplbgpu_step(self.h, int(n)))
        self.steps_done += int(n)

    step = stream_collision

    def update_macro_vars(self):
        self._check(self.lib.mplbgpu_update_macro(self.h))

    def calc_residual_error(self, check_period=None):
        """Returns (GetMaximumResidual, per-variable residuals)."""
        cp = check_period or self.case.check_period
        per = np.zeros(4)
        mx = ctypes.c_double()
        self._check(self.lib.mplbgpu_residual(self.h, int(cp), per.ctypes.data,
                                              ctypes.byref(mx)))
        return mx.value, per[:self.case.space_dim + 1].copy()

    def iterate(self, steps=None, criterion=None, check_period=None,
                max_steps=None, callback=None):
        """Iterate(steps, checkPeriod) or Iterate(criterion, checkPeriod).
        Returns the residual history [(step, max_residual, per_var)]."""
        cp = check_period or self.case.check_period
        history = []
        if steps is not None:
            done = 0
            while done < steps:
                n = min(cp - (self.steps_done % cp), steps - done)
                self.stream_collision(n)
                done += n
                if self.steps_done % cp == 0:
                    self.update_macro_vars()
                    if callback:
                        callback(self)
            return history
        if criterion is None:
            raise ValueError("give steps or criterion")
        res = 1.0
        while res >= criterion:
            self.stream_collision(cp - (self.steps_done % cp))
            self.update_macro_vars()
            res, per = self.calc_residual_error(cp)
            history.append((self.steps_done, res, per))
            if callback:
                callback(self)
            if max_steps is not None and self.steps_done >= max_steps:
                break
        return history

    # -- observation --------------------------------------------------------
    def macro(self, block):
        """Macro fields of one block (as of the last update_macro_vars)."""
        shp = self._shape(block)
        out = [np.zeros(shp) for _ in range(4)]
        self._check(self.lib.mplbgpu_download_macro(
            self.h, block, *[a.ctypes.data for a in out]))
        return out[:self.case.space_dim + 1]

    def f(self, block):
        out = np.zeros(self._shape(block) + (self.case.q,))
        self._check(self.lib.mplbgpu_download_f(self.h, block, out.ctypes.data))
        return out

    def mass(self):
        m = ctypes.c_double()
        self._check(self.lib.mplbgpu_mass(self.h, ctypes.byref(m)))
        return m.value

    def check_health(self):
        return self.lib.mplbgpu_check_health(self.h)

    def synchronize(self):
        self._check(self.lib.mplbgpu_synchronize(self.h))

    def launch_count(self):
        return int(self.lib.mplbgpu_launch_count(self.h))

    def last_step_ms(self):
        ms = ctypes.c_float()
        self._check(self.lib.mplbgpu_last_step_ms(self.h, ctypes.byref(ms)))
        return ms.value
