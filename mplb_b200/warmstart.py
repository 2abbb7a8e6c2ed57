"""Learned warm start of the batched cavities (include/mplbnn.h).

``Network`` wraps the tensor-core encoder-decoder: it maps a cavity's
conditioning (ln(Re/100)/ln 32, (U - 0.02)/0.06, (N - 64)/192) to its
normalised steady state on a 128 x 128 grid: (rho - 1) / (3 U^2), u / (sqrt3
U), v / (sqrt3 U) (MPLB units, U the lattice lid speed).  ``steady_states``
runs the batched solver cold to the residual criterion and resamples the
converged fields to the network grid (the training targets); ``train`` runs
Adam with a cosine learning-rate schedule; ``warm_fields`` predicts and
resamples back to each cavity's nodes for ``Batch.init``.

Device arrays are torch CUDA tensors (allocation only); every computation
on them is a kernel of libmplbgpu.so.  There is no CPU path.

    python -m mplb_b200.warmstart pipeline [--quick] [--out FILE]

runs the whole experiment: steady states of the training cavities, training,
then the held-out cavities cold-started and warm-started to the same
criterion, and prints one JSON line;

    python -m mplb_b200.warmstart trainbench [--steps K]

times training steps on a fixed synthetic batch of 32.
"""
import argparse
import ctypes
import json
import math
import os
import sys
import time
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .batch import SQRT3, Batch, CavitySpec, cavity_set

GRID = abi.NN_GRID


def conditioning(specs: Sequence[CavitySpec]) -> np.ndarray:
    return np.array([[math.log(s.re / 100.0) / math.log(32.0),
                      (s.lid - 0.02) / 0.06, (s.n - 64) / 192.0]
                     for s in specs], np.float32)


def scales(specs: Sequence[CavitySpec]):
    """(rho_scale, u_scale) per cavity: 3 U^2 and sqrt(3) U."""
    lid = np.array([s.lid for s in specs])
    return 3.0 * lid * lid, SQRT3 * lid


class NetworkError(RuntimeError):
    pass


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise NetworkError("the warm-start network needs a CUDA device")
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class Network:
    def __init__(self, batch: int = 32, lib=None):
        self.lib = lib or abi.load_library()
        h = ctypes.c_void_p()
        rc = self.lib.mplbnn_create(int(batch), ctypes.byref(h))
        if rc != abi.OK:
            raise NetworkError(self.lib.mplbnn_error().decode())
        self.h = h
        self.batch = int(batch)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mplbnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != abi.OK:
            raise NetworkError(f"{abi.STATUS_NAMES.get(rc, rc)}: " +
                               self.lib.mplbnn_last_error(self.h).decode())

    @property
    def param_count(self) -> int:
        return int(self.lib.mplbnn_param_count(self.h))

    def layers(self):
        out = []
        for l in range(self.lib.mplbnn_layer_count()):
            ci, co, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            wo, bo = ctypes.c_longlong(), ctypes.c_longlong()
            self.lib.mplbnn_layer_info(l, ctypes.byref(ci), ctypes.byref(co),
                                       ctypes.byref(t), ctypes.byref(wo),
                                       ctypes.byref(bo))
            out.append((ci.value, co.value, t.value, wo.value, bo.value))
        return out

    def init(self, seed: int = 1):
        self._check(self.lib.mplbnn_init_params(self.h, int(seed)))

    def params(self) -> np.ndarray:
        p = np.zeros(self.param_count, np.float32)
        self._check(self.lib.mplbnn_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.param_count
        self._check(self.lib.mplbnn_set_params(self.h, p.ctypes.data))

    def grads(self) -> np.ndarray:
        g = np.zeros(self.param_count, np.float32)
        self._check(self.lib.mplbnn_get_grads(self.h, g.ctypes.data))
        return g

    def forward(self, cond, out=None):
        """cond: (k, 3) float32 CUDA tensor -> (k, 128, 128, 3) predictions
        (processed in chunks of the network's batch)."""
        torch = _torch()
        k = cond.shape[0]
        if out is None:
            out = torch.empty((k, GRID, GRID, 3), dtype=torch.float32,
                              device=cond.device)
        torch.cuda.synchronize()
        for i in range(0, k, self.batch):
            n = min(self.batch, k - i)
            self._check(self.lib.mplbnn_forward(
                self.h, ctypes.c_void_p(cond[i:].data_ptr()), n,
                ctypes.c_void_p(out[i:].data_ptr())))
        return out

    def loss_grad(self, cond, target, index=None, want_loss=False):
        idx = None
        n = cond.shape[0]
        if index is not None:
            idx = np.ascontiguousarray(index, np.int32)
            n = idx.size
        loss = ctypes.c_double()
        self._check(self.lib.mplbnn_loss_grad(
            self.h, _ptr(cond), _ptr(target),
            idx.ctypes.data if idx is not None else None, int(n),
            ctypes.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self._check(self.lib.mplbnn_adam_step(self.h, float(lr), float(beta1),
                                              float(beta2), float(eps)))

    def synchronize(self):
        self._check(self.lib.mplbnn_synchronize(self.h))

    # -- fields <-> grid ------------------------------------------------------
    @staticmethod
    def _meta(specs):
        n = np.array([s.n for s in specs], np.int32)
        off = np.zeros(len(specs), np.int64)
        off[1:] = np.cumsum((n.astype(np.int64) ** 2))[:-1]
        rs, us = scales(specs)
        return n, off, np.ascontiguousarray(rs), np.ascontiguousarray(us)

    def fields_to_grid(self, specs, rho, u, v, grid=None):
        torch = _torch()
        if grid is None:
            grid = torch.empty((len(specs), GRID, GRID, 3),
                               dtype=torch.float32, device=rho.device)
        n, off, rs, us = self._meta(specs)
        torch.cuda.synchronize()
        self._check(self.lib.mplbnn_fields_to_grid(
            self.h, _ptr(rho), _ptr(u), _ptr(v), len(specs), n.ctypes.data,
            off.ctypes.data, rs.ctypes.data, us.ctypes.data, _ptr(grid)))
        return grid

    def grid_to_fields(self, specs, grid):
        torch = _torch()
        n, off, rs, us = self._meta(specs)
        total = int(off[-1] + int(n[-1]) ** 2)
        out = [torch.empty(total, dtype=torch.float64, device=grid.device)
               for _ in range(3)]
        torch.cuda.synchronize()
        self._check(self.lib.mplbnn_grid_to_fields(
            self.h, _ptr(grid), len(specs), n.ctypes.data, off.ctypes.data,
            rs.ctypes.data, us.ctypes.data, *[_ptr(t) for t in out]))
        return out


def device_macro(batch: Batch):
    """The batch's current moments as three CUDA float64 tensors."""
    torch = _torch()
    out = [torch.empty(batch.total_nodes, dtype=torch.float64, device="cuda")
           for _ in range(3)]
    torch.cuda.synchronize()
    batch._check(batch.lib.mplbgpu_batch_download_macro(
        batch.h, *[t.data_ptr() for t in out]))
    return out


def init_from_device(batch: Batch, rho, u, v):
    _torch().cuda.synchronize()
    batch._check(batch.lib.mplbgpu_batch_init(
        batch.h, rho.data_ptr(), u.data_ptr(), v.data_ptr()))


def solve(batch: Batch, max_steps, check_period, criterion, fields=None):
    """Initialise (rest, or the given device fields) and run to the
    criterion; returns (steps, residual, converged, wall seconds); the
    diverged cavities are in batch.diverged."""
    t0 = time.perf_counter()
    if fields is None:
        batch.init()
    else:
        init_from_device(batch, *fields)
    steps, res, conv = batch.run(max_steps, check_period, criterion)
    return steps, res, conv, time.perf_counter() - t0


def steady_states(specs, max_steps, check_period=1000, criterion=1e-8,
                  net: Optional[Network] = None, tuning=None):
    """Cold runs of `specs` to the criterion; returns (grid targets of the
    converged cavities, their indices, steps, converged, wall seconds)."""
    torch = _torch()
    b = Batch(specs, "fp32")
    if tuning:
        b.set_tuning(**tuning)
    steps, res, conv, wall = solve(b, max_steps, check_period, criterion)
    diverged = b.diverged
    rho, u, v = device_macro(b)
    b.close()
    own = net is None
    net = net or Network(1)
    grid = net.fields_to_grid(specs, rho, u, v)
    if own:
        net.close()
    del rho, u, v
    keep = np.nonzero(conv)[0]
    targets = grid[torch.from_numpy(keep).to(grid.device)].contiguous()
    del grid
    return targets, keep, steps, conv, diverged, wall


def train(net: Network, cond, target, epochs, lr_max=2e-3, lr_min=2e-5,
          seed=0, log_every=50, log=None):
    """Adam on (cond, target) CUDA tensors; cosine learning rate."""
    k = cond.shape[0]
    rng = np.random.default_rng(seed)
    per_epoch = max(1, math.ceil(k / net.batch))
    total = epochs * per_epoch
    hist = []
    step = 0
    _torch().cuda.synchronize()
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = rng.permutation(k)
        for i in range(0, k, net.batch):
            idx = perm[i:i + net.batch]
            lr = lr_min + 0.5 * (lr_max - lr_min) * (
                1.0 + math.cos(math.pi * step / max(1, total - 1)))
            want = (step % log_every == 0) or step == total - 1
            loss = net.loss_grad(cond, target, index=idx, want_loss=want)
            net.adam(lr)
            if want:
                hist.append((step, loss))
                if log:
                    log(f"step {step}/{total} epoch {ep} lr {lr:.2e} "
                        f"loss {loss:.4e} {time.perf_counter() - t0:.1f}s")
            step += 1
    net.synchronize()
    return hist, time.perf_counter() - t0


def warm_fields(net: Network, specs):
    """Predicted initial (rho, u, v) of each cavity, device float64."""
    torch = _torch()
    cond = torch.from_numpy(conditioning(specs)).cuda()
    pred = net.forward(cond)
    return net.grid_to_fields(specs, pred)


def rel_l2_per_cavity(specs, a, b):
    """Relative L2 difference of two packed fields, per cavity."""
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    out, o = [], 0
    for s in specs:
        m = s.n * s.n
        d = np.linalg.norm(a[o:o + m] - b[o:o + m])
        nb = np.linalg.norm(b[o:o + m])
        out.append(float(d / nb) if nb > 0 else float(d))
        o += m
    return np.array(out)


def pipeline(count=4096, seed=20261203, n_train=3072, max_steps=2_000_000,
             check_period=1000, criterion=1e-8, epochs=200, batch=32,
             log=print, tuning=None, lr_max=2e-3, details=None,
             reference_check=True, **cavity_kw):
    """The warm-start experiment; cavity_kw goes to cavity_set (sizes,
    re_range, lid_range).  Returns (summary dict, trained network); per-
    cavity arrays of the held-out set are added to `details` if given.
    With reference_check the held-out set is also run in FP64 to a 1000x
    tighter residual, and the cold- and warm-converged fields are compared
    with that reference (the same steady-state error on both sides)."""
    torch = _torch()
    specs = cavity_set(count, seed, **cavity_kw)
    train_specs, held = specs[:n_train], specs[n_train:]
    res = {"count": count, "n_train": n_train, "held_out": len(held),
           "criterion": criterion, "check_period": check_period,
           "max_steps": max_steps}
    net = Network(batch)
    t0 = time.perf_counter()
    targets, keep, tsteps, tconv, tdiv, twall = steady_states(
        train_specs, max_steps, check_period, criterion, net, tuning)
    res["train_converged"] = int(tconv.sum())
    res["train_diverged"] = int(tdiv.sum())
    res["train_solve_s"] = twall
    log(f"training set: {int(tconv.sum())}/{len(train_specs)} converged in "
        f"{twall:.1f}s")
    cond_all = torch.from_numpy(conditioning(train_specs)[keep]).cuda()
    net.init(seed)
    hist, train_s = train(net, cond_all, targets, epochs, lr_max=lr_max,
                          log=log)
    res["train_s"] = train_s
    res["loss_first"] = hist[0][1]
    res["loss_last"] = hist[-1][1]
    del targets
    # held-out: cold then warm, same batch object and tuning
    hb = Batch(held, "fp32")
    if tuning:
        hb.set_tuning(**tuning)
    csteps, cres, cconv, cwall = solve(hb, max_steps, check_period, criterion)
    cdiv = hb.diverged
    cold = device_macro(hb)
    tw = time.perf_counter()
    fields = warm_fields(net, held)
    infer_s = time.perf_counter() - tw
    wsteps, wres, wconv, wwall = solve(hb, max_steps, check_period, criterion,
                                       fields)
    wdiv = hb.diverged
    warm = device_macro(hb)
    init_err = rel_l2_per_cavity(held, fields[1], cold[1])
    final_diff = rel_l2_per_cavity(held, warm[1], cold[1])
    both = cconv & wconv
    ref_err = {}
    if reference_check:
        # the steady state to a 1000x tighter residual in FP64 (an FP32 run
        # may stall on its rounding noise above that), restarted from the
        # warm-converged fields: the error of each converged field against it
        rb = Batch(held, "fp64")
        rsteps, rres, rconv, rwall = solve(rb, max_steps, check_period,
                                           criterion * 1e-3, warm)
        ref = device_macro(rb)
        rb.close()
        err_cold = rel_l2_per_cavity(held, cold[1], ref[1])
        err_warm = rel_l2_per_cavity(held, warm[1], ref[1])
        sel = both & rconv
        ref_err = {
            "reference_criterion": criterion * 1e-3,
            "reference_converged": int(rconv.sum()),
            "reference_wall_s": rwall,
            "cold_u_error_vs_reference_median": float(np.median(err_cold[sel])),
            "warm_u_error_vs_reference_median": float(np.median(err_warm[sel])),
            "cold_u_error_vs_reference_p90": float(np.quantile(err_cold[sel], 0.9)),
            "warm_u_error_vs_reference_p90": float(np.quantile(err_warm[sel], 0.9)),
            "warm_error_le_cold_fraction": float(np.mean(err_warm[sel] <= err_cold[sel])),
        }
        if details is not None:
            details.update({"cold_u_error_vs_reference": err_cold.tolist(),
                            "warm_u_error_vs_reference": err_warm.tolist(),
                            "reference_conv": rconv.tolist()})
    res.update({
        "cold_wall_s": cwall, "warm_wall_s": wwall + infer_s,
        "warm_infer_s": infer_s, "speedup_wall": cwall / (wwall + infer_s),
        "cold_converged": int(cconv.sum()), "warm_converged": int(wconv.sum()),
        "cold_diverged": int(cdiv.sum()), "warm_diverged": int(wdiv.sum()),
        "cold_steps_total": int(csteps.sum()),
        "warm_steps_total": int(wsteps.sum()),
        "cold_node_steps": float(sum(s.n * s.n * int(k)
                                     for s, k in zip(held, csteps))),
        "warm_node_steps": float(sum(s.n * s.n * int(k)
                                     for s, k in zip(held, wsteps))),
        "steps_ratio_median": float(np.median(csteps[both] /
                                              np.maximum(wsteps[both], 1))),
        "warm_start_u_error_median": float(np.median(init_err[both])),
        "final_u_difference_max": float(final_diff[both].max())
        if both.any() else None,
        "final_u_difference_median": float(np.median(final_diff[both]))
        if both.any() else None,
        "total_s": time.perf_counter() - t0,
    })
    res.update(ref_err)
    if details is not None:
        details.update({
            "n": [s.n for s in held], "re": [s.re for s in held],
            "lid": [s.lid for s in held], "cold_steps": csteps.tolist(),
            "warm_steps": wsteps.tolist(), "cold_conv": cconv.tolist(),
            "warm_conv": wconv.tolist(), "init_u_error": init_err.tolist(),
            "final_u_difference": final_diff.tolist(),
            "loss_history": hist})
    return res, net


def train_bench(steps=50, warmup=3, batch=32, seed=0):
    """Time `steps` training steps (loss, gradients, Adam) on a fixed
    synthetic batch; returns (ms per step, convolution FLOPs per step)."""
    torch = _torch()
    net = Network(batch)
    net.init(1)
    rng = np.random.default_rng(seed)
    cond = torch.from_numpy(rng.uniform(0, 1, (batch, 3)).astype(
        np.float32)).cuda()
    tgt = torch.from_numpy((rng.standard_normal((batch, GRID, GRID, 3)) *
                            0.1).astype(np.float32)).cuda()
    torch.cuda.synchronize()
    for _ in range(warmup):
        net.loss_grad(cond, tgt)
        net.adam(1e-4)
    net.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        net.loss_grad(cond, tgt)
        net.adam(1e-4)
    net.synchronize()
    ms = (time.perf_counter() - t0) / steps * 1e3
    side = [128, 128, 64, 64, 32, 32, 16, 16, 32, 32, 64, 64, 128, 128, 128]
    flops = 0.0
    for l, (ci, co, t, _, _) in enumerate(net.layers()):
        f = 2.0 * batch * side[l] ** 2 * co * t * ci
        flops += f * (2 if l == 0 else 3)   # no data gradient of layer 0
    return ms, flops


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["pipeline", "trainbench"])
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--quick", action="store_true",
                    help="256 cavities of side 64/96, 20 epochs")
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--max-steps", type=int, default=2_000_000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=None)
    ap.add_argument("--details-out", default=None)
    ap.add_argument("--params-out", default=None)
    a = ap.parse_args(argv)
    if a.cmd == "trainbench":
        ms, flops = train_bench(a.steps)
        print(json.dumps({"train_step_ms": ms, "conv_flops_per_step": flops,
                          "tflops": flops / ms / 1e9}))
        return
    kw = dict(epochs=a.epochs, max_steps=a.max_steps, lr_max=a.lr)
    if a.quick:
        kw.update(count=256, n_train=192, sizes=(64, 96), epochs=20)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    details = {}
    res, net = pipeline(log=log, details=details, **kw)
    line = json.dumps(res)
    print(line, flush=True)
    if a.out:
        with open(a.out, "a") as fh:
            fh.write(line + "\n")
    if a.details_out:
        with open(a.details_out, "w") as fh:
            json.dump(details, fh)
    if a.params_out:
        np.save(a.params_out, net.params())


if __name__ == "__main__":
    main()
