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
# (dram__bytes_read.sum + dram__bytes_write.sum of SplitStepKernel<3,double>
# on the 128^3 cavity, 2 launches: 615 MB / 2,097,152 nodes; FP32: 311 MB;
# captured with `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum
# --clock-control none -k regex:SplitStepKernel -s 5 -c 2 python bench.py
# --size 128 --steps 10 --warmup 3 --no-cpu-baseline --precision fp64`).
# Traffic grows with the node count, so a 256^3 launch moves this x
# 16,777,216 bytes.
TRAFFIC_PER_NODE = {("fp64", 3): 293.0, ("fp32", 3): 148.0}
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
    p.add_argument("--workload", default="cavity3d",
                   choices=["cavity3d", "cavities", "cavities-warmstart"],
                   help="cavities: throughput of the 4,096 batched D2Q9 "
                        "cavities split over the ranks; cavities-warmstart: "
                        "the learned warm start experiment (minutes; 1 GPU)")
    p.add_argument("--cavities", type=int, default=4096,
                   help="cavities: how many cavities of the seeded set "
                        "(its first ones; 4,096 is the workload, fewer "
                        "make a small case for profiling)")
    p.add_argument("--epochs", type=int, default=200)
    p.add_argument("--decomp", default="replicas",
                   choices=["replicas", "slab"],
                   help="N > 1 on the cavity: independent 256^3 replicas, or "
                        "one 256 x 256 x 256N cavity cut into z slabs with "
                        "a face exchange (NCCL) before every step")
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


def max_over_ranks(v, world):
    if world <= 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_arm(args, rank, world):
    case = workload(args.size, "fp64", args.scheme)
    swap = args.scheme == "swap"
    step_name = "SwapStreamCollision" if swap else "StreamCollision"
    if rank != 0:
        return
    res = cpu_reference(case, max(1, min(args.warmup, 1)), args.steps,
                        budget_s=120)
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
        "warmup": 1, "ms_per_step": secs / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3D lid-driven cavity D3Q19 {args.size}^3 "
                               "FP64, lid 0.05, Re 400" +
                               (", swap scheme (one array)" if swap else ""),
                   "nodes": case.nodes()},
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads,
                         "kind": "reference",
                         "sample": f"{n} {step_name} steps of the "
                                   f"{args.size}^3 cavity after 1 warm-up "
                                   "step (reference sources + sequential "
                                   "OPS stand-in, OpenMP)"},
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
    from mplb_b200.batch import Batch, cavity_set, shard
    torch.cuda.set_device(local)
    specs = cavity_set(args.cavities)
    mine = [specs[i] for i in shard(specs, rank, world)]
    b = Batch(mine, "fp32")
    b.set_tuning(tile_nodes=128, persistent=0, chunk=50, ctas_per_sm=8)
    b.init()
    b.step(max(args.warmup, 50))
    s0 = b.stats()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    b.step(args.steps)
    barrier(world)
    clk = clocks.stop()
    s1 = b.stats()
    ms = max_over_ranks(s1["device_ms"] - s0["device_ms"], world)
    total_nodes = sum(s.n * s.n for s in specs)
    value = total_nodes * args.steps / (ms * 1e-3) / 1e6
    peak, peak_kind = measured_peaks()
    launches = s1["launches"] - s0["launches"]
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
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_node": 72,
                     "traffic": None},
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


def run_slab(args, rank, world, local):
    """One 256 x 256 x 256N cavity cut into N z slabs, one per GPU (weak
    scaling: 256^3 nodes per GPU); before every step each rank exports the
    populations leaving its slab through each cut face and swaps them with
    its neighbour (NCCL send/recv), then imports the neighbour's into its
    halo.  Timed on the device over the K steps including the exchanges,
    max over ranks."""
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
    launches0 = part.solver.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    s.stream_collision(args.steps)
    part.synchronize()
    ev1.record()
    ev1.synchronize()
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    launches = part.solver.launch_count() - launches0
    ms_max = max_over_ranks(ms, world)
    value = nodes * args.steps / (ms_max * 1e-3) / 1e6
    step_kernel_ms = part.solver.last_step_ms()   # the last step's kernel
    bpn = BYTES_PER_NODE[(case.precision, 3)]
    achieved = bpn * local_nodes / (step_kernel_ms * 1e-3) / 1e9
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
    face = 5 * n * n * (8 if case.precision == "fp64" else
                        4 if case.precision == "fp32" else 2)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[args.precision], "data": "synthetic",
        "config": {"workload": f"3D lid-driven cavity D3Q19 {n} x {n} x "
                               f"{n * world} {args.precision.upper()}, lid "
                               "0.05 (lattice), Re 400, z slabs of "
                               f"{n}^3 per GPU",
                   "nodes_per_gpu": local_nodes,
                   "parallelism": f"slab{world}",
                   "exchange_bytes_per_step_per_cut": 2 * face,
                   "l2": "population arrays larger than L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "bytes_per_node": bpn,
                     "traffic": None},
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
    if args.decomp == "slab" and args.workload == "cavity3d":
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
    s = Solver(case, lib)
    s.init_uniform()
    s.stream_collision(args.warmup)
    s.synchronize()
    launches0 = s.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    barrier(world)
    torch.cuda.synchronize()
    s.stream_collision(args.steps)     # CUDA events on the library's stream
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = s.last_step_ms()
    launches = s.launch_count() - launches0
    ms_max = max_over_ranks(ms, world)
    value = world * nodes * args.steps / (ms_max * 1e-3) / 1e6
    kernel_ms = ms / args.steps          # one kernel launch per step
    bpn = BYTES_PER_NODE[(case.precision, 3)]
    achieved = bpn * nodes / (kernel_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    s.close()
    del s

    # --- end to end through the C ABI with host buffers ------------------
    shp = (nz, ny, nx)
    pinned = [torch.empty(shp, dtype=torch.float64, pin_memory=True)
              for _ in range(8)]
    pinned[0].fill_(1.0)
    for t in pinned[1:4]:
        t.zero_()
    e = Solver(case, lib)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ptr = [t.data_ptr() for t in pinned]
    rc = lib.mplbgpu_init_macro(e.h, 0, ptr[0], ptr[1], ptr[2], ptr[3])
    if rc != 0:
        raise RuntimeError(lib.mplbgpu_last_error(e.h).decode())
    e.stream_collision(args.steps)
    e.update_macro_vars()
    rc = lib.mplbgpu_download_macro(e.h, 0, ptr[4], ptr[5], ptr[6], ptr[7])
    if rc != 0:
        raise RuntimeError(lib.mplbgpu_last_error(e.h).decode())
    t1 = time.perf_counter()
    barrier(world)
    e2e_s = max_over_ranks(t1 - t0, world)
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
            cpu = {"value": mlups, "unit": "MLUPS", "cores": threads,
                   "kind": "reference",
                   "sample": f"{n} {'SwapStreamCollision' if swap else 'StreamCollision'} "
                             f"steps of the same "
                             f"{args.size}^3 cavity after 1 warm-up step "
                             "(reference sources + sequential OPS stand-in, "
                             "OpenMP)"}
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
        "config": {"workload": f"3D lid-driven cavity D3Q19 {args.size}^3 "
                               f"{args.precision.upper()}, lid 0.05 "
                               "(lattice), Re 400" +
                               (", swap scheme (one array)" if swap else ""),
                   "nodes_per_gpu": nodes, "parallelism": f"replicas{world}",
                   "l2": "population arrays of 0.7-2.7 GB each, larger "
                         "than L2"},
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
    print(json.dumps(line))


if __name__ == "__main__":
    main()
