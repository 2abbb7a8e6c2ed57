"""Benchmark of the fused stream-collision step.

Workload (N = 1): the 3D lid-driven cavity, D3Q19 BGK, FP64, 256^3 nodes,
lid 0.05 (lattice units) along +x on the z-max face, Re = 400 - MPLB's
StreamCollision step through the C ABI.  One "step" is one StreamCollision
over the whole 256^3 block.  Each population array is 2.7 GB, far larger
than the 126 MB L2, so consecutive timed steps cannot hit in L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --workload cavities [--gpus N]
    python bench.py --workload cavities-warmstart

With N > 1 (torchrun, one rank per GPU) every rank runs its own cavity (no
data-path exchange; weak scaling) and the value is the total node updates
of all ranks divided by the slowest rank's device time.

Printed (rank 0, one JSON line): MLUPS of the device-resident timed steps
(`value`), the end-to-end MLUPS through the C ABI with host buffers (`e2e`:
initial macroscopic fields uploaded from pinned host memory, K steps,
moments downloaded), the HBM roofline of the step kernel (304 algorithmic
bytes per node update), the reference's own CPU implementation timed on a
bounded sample on this host (`cpu_baseline`), SM clocks sampled during the
timed region and the number of kernel launches in it.

--impl reference times the reference solver's CPU implementation (built
from its own sources against the sequential OPS stand-in, OpenMP over all
host cores) on the same workload instead.
"""
import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_NODE = {("fp64", 3): 304, ("fp64", 2): 144, ("fp32", 3): 152,
                  ("fp32", 2): 72, ("fp16", 3): 76, ("fp16", 2): 36}
# DRAM bytes per node update of the step kernel measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum of SplitStepKernel on the
# 192^3 cavity, whose population arrays (1.08 GB FP64, 0.54 GB FP32,
# 0.27 GB FP16) are well beyond the 126 MB L2; mean of 2 launches over
# 7,077,888 nodes: FP64 2,152.4 MB = 304.1 B, FP32 1,087.0 MB = 153.6 B,
# FP16 585.8 MB = 82.8 B: its staged interior copies 16-byte-aligned
# windows, 6 % above the per-thread loads' 78.4 B), captured with
# `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,
# gpu__time_duration.sum --clock-control none -k regex:SplitStepKernel -s 3
# -c 2 python bench.py --size 192 --steps 10 --warmup 3 --no-cpu-baseline
# --no-forms --min-time 0 --precision fp64|fp32|fp16`.  Traffic grows with
# the node count, so a 256^3 launch moves this x 16,777,216 bytes.
TRAFFIC_PER_NODE = {("fp64", 3): 304.1, ("fp32", 3): 153.6,
                    ("fp16", 3): 82.8}
METRIC = "MLUPS (D3Q19 3D lid-driven cavity 256^3)"
DTYPES = {"fp64": "f64", "fp32": "f32 (shifted f - w)",
          "fp16": "f16 storage of (f - w)/w, f32 arithmetic"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="mplb", choices=["mplb", "reference"])
    p.add_argument("--size", type=int, default=256)
    p.add_argument("--precision", default="fp64",
                   choices=["fp64", "fp32", "fp16"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--min-time", type=float, default=1.0,
                   help="seconds of timed work: the K-step timed region is "
                        "repeated until this much has run, so that the clock "
                        "sampler sees the load (0: one repetition)")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the FP32/FP16 runs of the same case that the "
                        "FP64 line reports beside its own")
    p.add_argument("--workload", default="cavity3d",
                   choices=["cavity3d", "cavities", "cavities-warmstart",
                            "precision", "lchannel"],
                   help="cavities: throughput of the 4,096 batched D2Q9 "
                        "cavities split over the ranks; cavities-warmstart: "
                        "the learned warm start experiment (minutes; 1 GPU)")
    p.add_argument("--cavities", type=int, default=4096,
                   help="cavities: how many cavities of the seeded set "
                        "(its first ones; 4,096 is the workload, fewer "
                        "make a small case for profiling)")
    p.add_argument("--epochs", type=int, default=200)
    p.add_argument("--lsteps", type=int, default=10000,
                   help="lchannel: steps (checks every 1,000)")
    p.add_argument("--quick", action="store_true",
                   help="precision: small channels instead of the full ones")
    p.add_argument("--decomp", default="auto",
                   choices=["auto", "replicas", "slab"],
                   help="N > 1 on the cavity: one 256 x 256 x 256N cavity "
                        "cut into z slabs with a face exchange (NCCL) in "
                        "every step (auto, the default for N > 1), or "
                        "independent 256^3 replicas")
    p.add_argument("--scheme", default="stream", choices=["stream", "swap"],
                   help="swap: the reference's one-array swap step "
                        "(Scheme_StreamCollision_Swap), half the memory")
    return p.parse_args()


SCHEMES = {"stream": "Scheme_StreamCollision",
           "swap": "Scheme_StreamCollision_Swap"}


def workload(n, precision="fp64", scheme="stream"):
    from mplb_b200 import config
    case = config.cavity(3, n, 0.05, re=400, precision=precision,
                         scheme=SCHEMES[scheme])
    return case


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference(case, warmup, steps, budget_s, threads=None):
    """Times the reference's CPU implementation (oracle/_ref); returns
    (MLUPS, steps timed, threads, seconds)."""
    from oracle import pyoracle
    if not pyoracle.reference_available("_omp"):
        if not pyoracle.build_reference():
            return None
    threads = threads or os.cpu_count()
    kind = "_omp" if threads > 1 else "_fast"
    secs, cells = pyoracle.time_reference(case, warmup, 1, kind=kind,
                                          threads=threads)
    n = max(1, min(steps, int(budget_s / max(secs, 1e-6))))
    if n > 1:
        secs, cells = pyoracle.time_reference(case, warmup, n, kind=kind,
                                              threads=threads)
    return cells * n / secs / 1e6, n, threads, secs


def dist_setup(args):
    if args.gpus <= 1 or "RANK" not in os.environ:
        return 0, 1, 0
    import datetime
    import torch.distributed as dist
    rank = int(os.environ["RANK"])
    world = int(os.environ["WORLD_SIZE"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def repeat_timed(run_k, world, min_s=1.0, max_reps=2000):
    """Times run_k() - exactly K steps between a barrier and a device
    synchronize, returning its device milliseconds - again and again until
    at least min_s seconds of timed work have run, so that the clock
    sampler (200 ms period) sees the load.  Every rank runs the same number
    of repetitions (fixed from the slowest rank's first one).  Returns the
    per-repetition max-over-ranks device times."""
    first = max_over_ranks(run_k(), world)
    reps = int(min(max_reps, max(1, -(-min_s * 1e3 // max(first, 1e-3)))))
    times = [first]
    for _ in range(reps - 1):
        times.append(max_over_ranks(run_k(), world))
    return times


def cpu_model():
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True,
                             timeout=10).stdout
    except (OSError, subprocess.SubprocessError):
        return None
    for line in out.splitlines():
        if line.startswith("Model name:"):
            return line.split(":", 1)[1].strip()
    return None


def max_over_ranks(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cavity_config(args, world, nodes):
    """The `config` of the cavity workload's line (both arms)."""
    swap = args.scheme == "swap"
    return {"workload": f"3D lid-driven cavity D3Q19 {args.size}^3 "
                        f"{args.precision.upper()}, lid 0.05 (lattice), "
                        "Re 400" + (", swap scheme (one array)" if swap
                                    else ""),
            "nodes_per_gpu": nodes, "parallelism": f"replicas{world}",
            "l2": "population arrays of 0.7-2.7 GB each, larger than L2"}


def run_reference_arm(args, rank, world):
    """The reference's own CPU implementation of the step (oracle/_ref: its
    sources against the sequential OPS stand-in, OpenMP over every host
    core) on the same case, the same config and warm-up; K steps, or fewer
    where K would take more than a few minutes (the line says how many)."""
    case = workload(args.size, "fp64", args.scheme)
    swap = args.scheme == "swap"
    step_name = "SwapStreamCollision" if swap else "StreamCollision"
    if rank != 0:
        return
    if args.precision != "fp64":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference computes in FP64 only; its arm "
                          "runs with --precision fp64"}))
        return
    res = cpu_reference(case, args.warmup, args.steps, budget_s=150)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build (oracle/_ref) not present"}))
        return
    mlups, n, threads, secs = res
    line = {
        "impl": "reference",
        "metric": METRIC if not swap else METRIC[:-1] +
        ", one-array swap scheme)", "value": mlups,
        "unit": "MLUPS", "n_gpus": args.gpus, "steps": n,
        "warmup": args.warmup, "ms_per_step": secs / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": (slab_config(args, world, case.nodes())
                   if use_slab(args, world)
                   else cavity_config(args, world, case.nodes())),
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads,
                         "kind": "reference", "cpu_model": cpu_model(),
                         "sample": f"{n} {step_name} steps of the "
                                   f"{args.size}^3 cavity after "
                                   f"{args.warmup} warm-up steps (reference "
                                   "sources + sequential OPS stand-in, "
                                   "OpenMP)" +
                                   (f"; one slab's share of the {args.size}"
                                    f" x {args.size} x {args.size * world} "
                                    "cavity, the reference's cost per node "
                                    "being that of the whole block"
                                    if use_slab(args, world) else "")},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_cavities(args, rank, world, local):
    """Throughput of the batched workload: the 4,096 D2Q9 FP32 cavities
    (seed 20261203) split over the ranks by LPT on the node count, no
    exchange between ranks (strong scaling: the set is fixed).  K steps of
    every cavity after W warm-up steps, CUDA events on each batch's stream,
    max over ranks."""
    import torch
    from mplb_b200.batch import Batch, autotune, cavity_set, shard
    torch.cuda.set_device(local)
    specs = cavity_set(args.cavities)
    mine = [specs[i] for i in shard(specs, rank, world)]
    b = Batch(mine, "fp32")
    # the autotuner times every candidate on this rank's cavities and
    # leaves the fastest set (a fresh choice: the cache is not consulted)
    tuned = autotune(b, steps=200, force=True,
                     cache=os.path.join(tempfile.mkdtemp(), "tuning.json"))
    b.init()
    b.step(max(args.warmup, 50))
    s0 = b.stats()

    def run_k():
        barrier(world)
        a = b.stats()
        b.step(args.steps)        # CUDA events on the batch's stream
        z = b.stats()
        barrier(world)
        return z["device_ms"] - a["device_ms"]

    clocks = ClockSampler(local)
    clocks.start()
    times = repeat_timed(run_k, world, args.min_time)
    clk = clocks.stop()
    s1 = b.stats()
    ms = statistics.median(times)
    total_nodes = sum(s.n * s.n for s in specs)
    value = total_nodes * args.steps / (ms * 1e-3) / 1e6
    peak, peak_kind = measured_peaks()
    launches = (s1["launches"] - s0["launches"]) // len(times)
    b.close()
    if rank != 0:
        return
    per_gpu_ms = ms / args.steps
    achieved = 72.0 * total_nodes / world / (per_gpu_ms * 1e-3) / 1e9
    print(json.dumps({
        "metric": f"MLUPS ({len(specs):,} batched D2Q9 lid-driven "
                  "cavities, FP32)",
        "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 50),
        "ms_per_step": per_gpu_ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 (shifted f - w)", "data": "synthetic",
        "config": {"workload": f"{len(specs):,} D2Q9 cavities, N in "
                               "{64..256}, Re 100-3200, U 0.02-0.08, seed "
                               "20261203",
                   "nodes": total_nodes,
                   "parallelism": f"cavities split over {world} GPU(s) "
                                  "(LPT on nodes)"},
        "timing": {"repetitions": len(times),
                   "statistic": "median over repetitions of K timed steps"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_node": 72,
                     "traffic": None},
        "tuning": tuned["tuning"],
        "autotune": [{"mlups": round(r["mlups"], 1),
                      **{k: v for k, v in r.items() if k != "mlups"}}
                     for r in tuned["all"]],
        "clocks": clk, "gpu_launches": launches}))


def run_warmstart(args, rank, local):
    """The second half of the metric: wall time to residual 1e-8 of the
    1,024 held-out cavities of the 4,096-cavity batched workload, warm-
    started from the trained network (inference, resampling and the solve
    inside the timed region) against cold-started (the same batch object,
    same tuning).  One GPU; the other ranks of a multi-rank launch idle."""
    import torch
    from mplb_b200 import warmstart as ws
    if rank != 0:
        return
    torch.cuda.set_device(local)
    clocks = ClockSampler(local)
    clocks.start()
    res, _ = ws.pipeline(epochs=args.epochs, log=lambda m: None)
    clk = clocks.stop()
    line = {
        "metric": "wall-time to residual 1e-8, 1,024 held-out D2Q9 "
                  "cavities, learned warm start",
        "value": res["warm_wall_s"], "unit": "s", "n_gpus": 1,
        "steps": None, "warmup": None, "higher_is_better": False,
        "scaling": "none", "vs_baseline": None,
        "dtype": "f32 (shifted f - w) LBM; bf16 network", "data": "synthetic",
        "config": {"workload": "4,096 D2Q9 lid-driven cavities (N in "
                               "{64..256}, Re 100-3200, U 0.02-0.08, seed "
                               "20261203); first 3,072 train, last 1,024 "
                               "held out",
                   "parallelism": "single GPU"},
        "cold_wall_s": res["cold_wall_s"],
        "speedup_vs_cold": res["speedup_wall"],
        "warm_start": res,
        "clocks": clk,
    }
    print(json.dumps(line))


def interface_continuity(s):
    """Per interface of the L-channel (inlet leg | corner across x, corner |
    outlet leg across y) and per moment: the largest jump between the two
    blocks' nodes that face each other across the joint, and the largest
    difference between the same layer and the next one inside the first
    block (the size of one grid spacing's change where nothing is joined).
    A jump of the order of the in-block difference is a continuous field."""
    import numpy as np
    m = [s.macro(b) for b in (0, 1, 2)]
    names = ["rho", "u", "v", "w"]
    out = {}
    for label, a, b, axis in (("inlet_leg|corner", 0, 1, 2),
                              ("corner|outlet_leg", 1, 2, 1)):
        rec = {}
        for q, name in enumerate(names):
            qa, qb = m[a][q], m[b][q]
            last = np.take(qa, -1, axis=axis)
            prev = np.take(qa, -2, axis=axis)
            first = np.take(qb, 0, axis=axis)
            rec[name] = {"jump": float(np.abs(first - last).max()),
                         "in_block": float(np.abs(last - prev).max())}
        out[label] = rec
    return out


def run_lchannel(args, rank, local):
    """The 3-block L-channel (384 x 128 x 128 inlet leg, 128^3 corner,
    128 x 384 x 128 outlet leg = 14,680,064 nodes; D3Q19 BGK, tau_L 0.6,
    z-periodic, EQMDiffuseRefl walls, pressure outlet rho = 1) with the
    inlet at u_x = 0.03 lattice units plus a seeded uniform +-1 %
    perturbation per node (seed 20261203), from rest, for --lsteps steps
    (10,000) in periods of 1,000.  Device time of the steps (CUDA events
    on the library's stream; the check-period work outside it) gives the
    MLUPS; at each check: total mass (FP64 sum of rho), the residual and
    the continuity of the moments across the two block joints."""
    import torch
    from mplb_b200 import Solver, config
    if rank != 0:
        return
    torch.cuda.set_device(local)
    case = config.lchannel(precision=args.precision)
    k, comps = config.inlet_perturbation(case, seed=20261203, amplitude=0.01)
    s = Solver(case)
    s.set_boundary_velocity(k, *comps)
    s.init_uniform()
    nodes = case.nodes()
    mass0 = s.mass()
    cp = 1000
    launches0 = s.launch_count()
    device_ms, history = 0.0, []
    clocks = ClockSampler(local)
    clocks.start()
    done = 0
    while done < args.lsteps:
        n = min(cp, args.lsteps - done)
        s.stream_collision(n)
        device_ms += s.last_step_ms()
        done += n
        s.update_macro_vars()
        mass = s.mass()
        res, _ = s.calc_residual_error(n)
        history.append({"step": done, "mass": mass,
                        "mass_change": mass - mass0,
                        "residual": res,
                        "continuity": interface_continuity(s)})
    clk = clocks.stop()
    launches = s.launch_count() - launches0
    s.close()
    value = nodes * args.lsteps / (device_ms * 1e-3) / 1e6
    bpn = BYTES_PER_NODE[(args.precision, 3)]
    achieved = bpn * nodes / (device_ms / args.lsteps * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    line = {
        "metric": "MLUPS (3-block D3Q19 L-channel, 14,680,064 nodes)",
        "value": value, "unit": "MLUPS", "n_gpus": 1,
        "steps": args.lsteps, "warmup": 0,
        "ms_per_step": device_ms / args.lsteps, "higher_is_better": True,
        "scaling": "none", "vs_baseline": None,
        "dtype": DTYPES[args.precision], "data": "synthetic",
        "config": {"workload": "L-channel: 384x128x128 inlet leg, 128^3 "
                               "corner, 128x384x128 outlet leg, tau_L 0.6, "
                               "z-periodic, inlet u_x 0.03 (lattice) "
                               "+-1 % per node (seed 20261203), outlet "
                               "rho 1, from rest",
                   "nodes": nodes, "parallelism": "single GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_node": bpn,
                     "traffic": None},
        "mass_initial": mass0,
        "history": history,
        "clocks": clk,
        "gpu_launches": launches,
        "launches_per_step": launches / args.lsteps,
    }
    print(json.dumps(line))


# --- precision study of the storage forms (forced channels) --------------
SQRT3 = 3.0 ** 0.5


def analytic_u(ny, g, tau, wall):
    import numpy as np
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
    import numpy as np
    d = a - b
    nb = np.linalg.norm(b)
    mb = np.abs(b).max()
    return (float(np.linalg.norm(d) / nb) if nb > 0 else float("nan"),
            float(np.abs(d).max() / mb) if mb > 0 else float("nan"))


def run_channel(dim, nx, ny, nz, steps, precision, wall, g=1e-6, tau=0.8):
    from mplb_b200 import Solver, config
    case = config.poiseuille(dim, nx, ny, nz, g_lattice=g, tau_lattice=tau,
                             wall=wall, precision=precision)
    import numpy as np
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


def run_precision(args):
    """Body-force Poiseuille channels (D2Q9 4096 x 1024 for 50,000 steps and
    D3Q19 512 x 256 x 256 for 10,000 steps; tau_L = 0.8, g_L = 1e-6 along x;
    walls at y-min/y-max, periodic in x and z) in the FP64 form (bit-
    identical to the reference), the shifted FP32 form and the FP16-storage
    form.  The channels' viscous times H^2/nu (10^7 and 6.6 x 10^5 steps)
    are far longer than the prescribed runs: where the analytic profile is
    subsonic (the 3D channel, peak 0.082 lattice units) the flow starts
    from it and the error against it measures discretisation and storage
    error; the 2D profile would peak at 1.31 lattice units, so that channel
    starts from rest.  One JSON line per run: relative L2 and max errors of
    rho and u against the FP64 form, of u against the profile, and the
    device-time MLUPS.  --quick runs small channels."""
    quick = args.quick
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
                import numpy as np
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



def slab_config(args, world, local_nodes):
    """The `config` of the slab-decomposed cavity (both arms)."""
    n = args.size
    face = 5 * n * n * (8 if args.precision == "fp64" else
                        4 if args.precision == "fp32" else 2)
    return {"workload": f"3D lid-driven cavity D3Q19 {n} x {n} x "
                        f"{n * world} {args.precision.upper()}, lid 0.05 "
                        f"(lattice), Re 400, z slabs of {n}^3 per GPU",
            "nodes_per_gpu": local_nodes, "parallelism": f"slab{world}",
            "exchange_bytes_per_step_per_cut": 2 * face,
            "l2": "population arrays larger than L2"}


def use_slab(args, world):
    return args.workload == "cavity3d" and (
        args.decomp == "slab" or (args.decomp == "auto" and world > 1))


def run_slab(args, rank, world, local):
    """One 256 x 256 x 256N cavity cut into N z slabs, one per GPU (weak
    scaling: 256^3 nodes per GPU).  Every step: each rank exports the
    populations leaving its slab through its cut faces, queues the step's
    interior (which reads no halo), sends and receives the faces (NCCL, on
    a side stream, overlapping the interior), imports the neighbours' faces
    into its halos and finishes the step - no host wait inside the loop.
    Timed with CUDA events on the library's stream over K steps including
    the exchanges, repeated for at least a second, max over ranks."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    from mplb_b200 import config, slab
    torch.cuda.set_device(local)
    n = args.size
    case = config.cavity(3, n, 0.05, re=400, precision=args.precision)
    case = dataclasses.replace(case, block_sizes=[(n, n, n * world)])
    group = None
    if world > 1:
        group = dist.new_group(backend="nccl",
                               timeout=datetime.timedelta(seconds=300))
    s = slab.SlabSolver(case, world, [rank],
                        slab.DistExchange(group) if world > 1
                        else slab.LocalExchange())
    part = s.parts[0]
    nodes = case.nodes()
    local_nodes = slab.slab_case(case, world, rank).nodes()
    s.init_uniform()
    s.stream_collision(args.warmup)
    part.synchronize()
    ctx = torch.cuda.ExternalStream(part.stream_ptr())
    launches0 = part.solver.launch_count()

    def run_k():
        barrier(world)
        part.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(ctx)
        s.stream_collision(args.steps)
        ev1.record(ctx)
        ev1.synchronize()
        barrier(world)
        return ev0.elapsed_time(ev1)

    clocks = ClockSampler(local)
    clocks.start()
    times = repeat_timed(run_k, world, args.min_time)
    clk = clocks.stop()
    launches = (part.solver.launch_count() - launches0) // len(times)
    ms_max = statistics.median(times)
    value = nodes * args.steps / (ms_max * 1e-3) / 1e6
    bpn = BYTES_PER_NODE[(case.precision, 3)]
    achieved = bpn * local_nodes / (ms_max / args.steps * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    # end to end: initial fields from pinned host memory, K steps, moments
    # back to pinned host memory
    shp = slab.slab_case(case, world, rank).size3(0)[::-1]
    pinned = [torch.empty(shp, dtype=torch.float64, pin_memory=True)
              for _ in range(8)]
    pinned[0].fill_(1.0)
    for t in pinned[1:4]:
        t.zero_()
    lib = part.lib
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ptr = [t.data_ptr() for t in pinned]
    part._check(lib.mplbgpu_init_macro(part.solver.h, 0, *ptr[:4]))
    s.stream_collision(args.steps)
    s.update_macro_vars()
    part._check(lib.mplbgpu_download_macro(part.solver.h, 0, *ptr[4:]))
    t1 = time.perf_counter()
    barrier(world)
    e2e_s = max_over_ranks(t1 - t0, world)
    e2e = nodes * args.steps / e2e_s / 1e6
    ok = bool(np.isfinite(float(pinned[4].sum())))
    s.close()
    if group is not None:
        dist.destroy_process_group(group)
    if not ok:
        raise RuntimeError("non-finite density after the slab run")
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[args.precision], "data": "synthetic",
        "config": slab_config(args, world, local_nodes),
        "timing": {"repetitions": len(times),
                   "statistic": "median over repetitions of K timed steps "
                                "(max over ranks)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_node": bpn,
                     "traffic": None,
                     "note": "per-node bytes over the whole step, face "
                             "exchange included"},
        "e2e": {"value": e2e, "unit": "MLUPS",
                "h2d_bytes_per_step": 4 * 8 * nodes / args.steps,
                "d2h_bytes_per_step": 4 * 8 * nodes / args.steps},
        "cpu_baseline": None,
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference" and args.workload != "cavity3d":
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable":
                              "the reference has no batched or learned "
                              "solver; its CPU cavity solver is timed on "
                              "the default workload"}))
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.workload == "cavities-warmstart":
        run_warmstart(args, rank, local)
        return
    if args.workload == "lchannel":
        run_lchannel(args, rank, local)
        return
    if args.workload == "precision":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            run_precision(args)
        return
    if use_slab(args, world):
        run_slab(args, rank, world, local)
        return
    if args.workload == "cavities":
        run_cavities(args, rank, world, local)
        return
    import numpy as np
    import torch
    from mplb_b200 import Solver, abi
    torch.cuda.set_device(local)
    case = workload(args.size, args.precision, args.scheme)
    nodes = case.nodes()
    nx, ny, nz = case.size3(0)
    lib = abi.load_library()
    swap = args.scheme == "swap"

    # --- device-resident timing ------------------------------------------
    def device_run(prec):
        """K steps of the cavity in storage form `prec`, repeated for at
        least a second under the clock sampler; returns (median device ms of
        K steps, launches per K steps, clocks, per-repetition ms)."""
        c = workload(args.size, prec, args.scheme)
        s = Solver(c, lib)
        s.init_uniform()
        s.stream_collision(args.warmup)
        s.synchronize()
        launches0 = s.launch_count()

        def run_k():
            barrier(world)
            torch.cuda.synchronize()
            s.stream_collision(args.steps)   # CUDA events on its stream
            ms = s.last_step_ms()            # waits for the K steps
            barrier(world)
            return ms

        clocks = ClockSampler(local)
        clocks.start()
        times = repeat_timed(run_k, world, args.min_time)
        clk = clocks.stop()
        launches = (s.launch_count() - launches0) // len(times)
        s.close()
        return statistics.median(times), launches, clk, times

    ms_max, launches, clk, times = device_run(args.precision)
    value = world * nodes * args.steps / (ms_max * 1e-3) / 1e6
    kernel_ms = ms_max / args.steps      # one kernel launch per step
    bpn = BYTES_PER_NODE[(case.precision, 3)]
    achieved = bpn * nodes / (kernel_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    forms = {}
    if args.precision == "fp64" and not args.no_forms:
        # the shifted forms of the same case (precision target: FP32 at
        # >= 1.8x the FP64 node rate)
        for prec, key in (("fp32", "fp32_shifted"), ("fp16", "fp16_storage")):
            fms, _, fclk, _ = device_run(prec)
            fb = BYTES_PER_NODE[(prec, 3)]
            fach = fb * nodes / (fms / args.steps * 1e-3) / 1e9
            fv = world * nodes * args.steps / (fms * 1e-3) / 1e6
            ftr = TRAFFIC_PER_NODE.get((prec, 3))
            forms[key] = {"value": fv, "unit": "MLUPS",
                          "ms_per_step": fms / args.steps,
                          "vs_fp64": fv / value, "bytes_per_node": fb,
                          "achieved_gbs": fach, "frac": fach / peak,
                          "traffic": (ftr * nodes if ftr is not None and
                                      not swap else None),
                          "dtype": DTYPES[prec], "sm_mhz": fclk["sm_mhz"]}

    # --- end to end through the C ABI with host buffers ------------------
    shp = (nz, ny, nx)
    pinned = [torch.empty(shp, dtype=torch.float64, pin_memory=True)
              for _ in range(8)]
    pinned[0].fill_(1.0)
    for t in pinned[1:4]:
        t.zero_()
    e = Solver(case, lib)
    ptr = [t.data_ptr() for t in pinned]

    def end_to_end():
        """Initial fields up from pinned host memory, K steps, moments back
        to pinned host memory: seconds of wall time."""
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.mplbgpu_init_macro(e.h, 0, ptr[0], ptr[1], ptr[2], ptr[3])
        if rc != 0:
            raise RuntimeError(lib.mplbgpu_last_error(e.h).decode())
        e.stream_collision(args.steps)
        e.update_macro_vars()
        rc = lib.mplbgpu_download_macro(e.h, 0, ptr[4], ptr[5], ptr[6],
                                        ptr[7])
        if rc != 0:
            raise RuntimeError(lib.mplbgpu_last_error(e.h).decode())
        t1 = time.perf_counter()
        barrier(world)
        return t1 - t0

    end_to_end()    # warm-up pass, untimed (first-use costs of the context)
    e2e_s = max_over_ranks(end_to_end(), world)
    e2e = world * nodes * args.steps / e2e_s / 1e6
    rho_sum = float(pinned[4].sum())
    e.close()
    if not np.isfinite(rho_sum):
        raise RuntimeError("non-finite density after the end-to-end run")

    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline:
        res = cpu_reference(case, 1, 5, budget_s=25)
        if res is not None:
            mlups, n, threads, secs = res
            name = "SwapStreamCollision" if swap else "StreamCollision"
            cpu = {"value": mlups, "unit": "MLUPS", "cores": threads,
                   "kind": "reference", "cpu_model": cpu_model(),
                   "sample": f"{n} {name} steps of the same {args.size}^3 "
                             "cavity after 1 warm-up step (reference "
                             "sources + sequential OPS stand-in, OpenMP)"}
            one = cpu_reference(case, 1, 2, budget_s=10, threads=1)
            if one is not None:
                m1, n1, _, _ = one
                cpu["single_thread"] = {
                    "value": m1, "unit": "MLUPS", "cores": 1,
                    "sample": f"{n1} {name} steps after 1 warm-up step "
                              "(the same build without OpenMP: OPS seq)"}
    metric = METRIC if not swap else METRIC[:-1] + ", one-array swap scheme)"
    traffic = (TRAFFIC_PER_NODE[(case.precision, 3)] * nodes
               if (case.precision, 3) in TRAFFIC_PER_NODE and not swap
               else None)
    line = {
        "metric": metric, "value": value, "unit": "MLUPS",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[args.precision], "data": "synthetic",
        "config": cavity_config(args, world, nodes),
        "timing": {"repetitions": len(times),
                   "statistic": "median over repetitions of K timed steps",
                   "ms_per_step_min": min(times) / args.steps,
                   "ms_per_step_max": max(times) / args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     "bytes_per_node": bpn,
                     "traffic": traffic},
        "e2e": {"value": e2e, "unit": "MLUPS",
                "h2d_bytes_per_step": 4 * 8 * nodes / args.steps,
                "d2h_bytes_per_step": 4 * 8 * nodes / args.steps},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    if forms:
        line["forms"] = forms
    print(json.dumps(line))


if __name__ == "__main__":
    main()
