"""Batched lid-driven cavities (mplbgpu_batch_* of the C ABI).

``cavity_set(count, seed)`` draws the benchmark's cavity population: side
N uniform in {64, 96, 128, 192, 256}, Reynolds number log-uniform in
[100, 3200] and lid speed uniform in [0.02, 0.08] (lattice units), drawn
cavity by cavity in the order N, Re, U from a 64-bit Mersenne twister
(MT19937-64, the generator of C++'s std::mt19937_64) with these mappings of
its raw 64-bit outputs r:  N = sizes[r mod 5],  Re = exp(ln 100 +
(r / 2^64) ln 32),  U = 0.02 + 0.06 r / 2^64.

``lpt_shards`` / ``shard`` partition the cavities over ranks (one GPU each;
the cavities are independent, so there is no data-path exchange).

``Batch`` wraps one batch on the GPU; ``autotune`` times tile size, launch
style (CUDA-graph chunks of one-step launches or a persistent multi-step
launch), CTAs per SM and chunk length on the batch itself and caches the
winner in a JSON file keyed by device, precision and the cavity sizes.
"""
import ctypes
import dataclasses
import hashlib
import json
import math
import os
from typing import List, Optional, Sequence

import numpy as np

from . import abi

SQRT3 = math.sqrt(3.0)
SIZES = (64, 96, 128, 192, 256)
DEFAULT_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                             "tuning_cache.json")


class MT19937_64:
    """64-bit Mersenne twister (Matsumoto & Nishimura, 2004)."""

    def __init__(self, seed: int):
        self.mt = [0] * 312
        self.mt[0] = seed & 0xFFFFFFFFFFFFFFFF
        for i in range(1, 312):
            prev = self.mt[i - 1]
            self.mt[i] = (6364136223846793005 * (prev ^ (prev >> 62)) + i) \
                & 0xFFFFFFFFFFFFFFFF
        self.idx = 312

    def _twist(self):
        um, lm = 0xFFFFFFFF80000000, 0x7FFFFFFF
        for i in range(312):
            x = (self.mt[i] & um) | (self.mt[(i + 1) % 312] & lm)
            xa = x >> 1
            if x & 1:
                xa ^= 0xB5026F5AA96619E9
            self.mt[i] = self.mt[(i + 156) % 312] ^ xa
        self.idx = 0

    def next(self) -> int:
        if self.idx >= 312:
            self._twist()
        y = self.mt[self.idx]
        self.idx += 1
        y ^= (y >> 29) & 0x5555555555555555
        y ^= (y << 17) & 0x71D67FFFEDA60000
        y ^= (y << 37) & 0xFFF7EEE000000000
        y ^= y >> 43
        return y & 0xFFFFFFFFFFFFFFFF


@dataclasses.dataclass
class CavitySpec:
    n: int
    re: float
    lid: float          # lattice units

    @property
    def tau_lattice(self) -> float:
        return 3.0 * self.lid * self.n / self.re + 0.5

    @property
    def dt(self) -> float:
        return 1.0 / ((self.n - 1) * SQRT3)

    @property
    def tau_ref(self) -> float:
        return (self.tau_lattice - 0.5) * self.dt


def cavity_set(count: int = 4096, seed: int = 20261203,
               sizes: Sequence[int] = SIZES, re_range=(100.0, 3200.0),
               lid_range=(0.02, 0.08)) -> List[CavitySpec]:
    g = MT19937_64(seed)
    out = []
    lr0, lr1 = math.log(re_range[0]), math.log(re_range[1])
    for _ in range(count):
        n = sizes[g.next() % len(sizes)]
        re = math.exp(lr0 + (g.next() / 2.0 ** 64) * (lr1 - lr0))
        lid = lid_range[0] + (lid_range[1] - lid_range[0]) * g.next() / 2.0 ** 64
        out.append(CavitySpec(n, re, lid))
    return out


def lpt_shards(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time partition of items over `world` ranks: items
    in decreasing cost (ties by index) each go to the least-loaded rank (ties
    to the lowest rank).  Deterministic, so every rank computes the same
    partition without communicating.  Returns each rank's item indices in
    increasing order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += costs[i]
        out[r].append(i)
    return [sorted(o) for o in out]


def shard(specs: Sequence[CavitySpec], rank: int, world: int,
          cost=lambda s: float(s.n * s.n)) -> List[int]:
    """Indices of the cavities rank `rank` of `world` runs (LPT on `cost`,
    by default the node count, i.e. the work of one step; weight by the
    expected steps to convergence to balance a solve to the criterion)."""
    if world <= 1:
        return list(range(len(specs)))
    return lpt_shards([cost(s) for s in specs], world)[rank]


class BatchError(RuntimeError):
    def __init__(self, message, status=None):
        self.status = status
        super().__init__(message)


class Batch:
    def __init__(self, specs: Sequence[CavitySpec], precision: str = "fp32",
                 lib=None):
        self.lib = lib or abi.load_library()
        self.specs = list(specs)
        arr = (abi.Cavity * len(self.specs))()
        for i, s in enumerate(self.specs):
            arr[i].n = s.n
            arr[i].lid_u = SQRT3 * s.lid
            arr[i].tau_ref = s.tau_ref
        h = ctypes.c_void_p()
        rc = self.lib.mplbgpu_batch_create(arr, len(self.specs),
                                           abi.PRECISIONS[precision],
                                           ctypes.byref(h))
        if rc != abi.OK:
            raise BatchError(self.lib.mplbgpu_batch_last_error(None).decode(),
                             rc)
        self.h = h
        self.precision = precision
        self.offsets = np.cumsum([0] + [s.n * s.n for s in self.specs])

    def close(self):
        if getattr(self, "h", None):
            self.lib.mplbgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != abi.OK:
            raise BatchError(f"{abi.STATUS_NAMES.get(rc, rc)}: " +
                             self.lib.mplbgpu_batch_last_error(self.h).decode(),
                             rc)

    @property
    def total_nodes(self) -> int:
        return int(self.offsets[-1])

    def set_tuning(self, tile_nodes=128, persistent=0, chunk=100,
                   ctas_per_sm=8):
        t = abi.BatchTuning(tile_nodes, persistent, chunk, ctas_per_sm)
        self._check(self.lib.mplbgpu_batch_set_tuning(self.h, ctypes.byref(t)))

    def set_wait_limit(self, polls):
        """Polls before a grid barrier of the persistent launch gives up
        (MPLBGPU_ERR_TIMEOUT, after which the batch needs init again)."""
        self._check(self.lib.mplbgpu_batch_set_wait_limit(self.h, int(polls)))

    def tuning(self):
        t = abi.BatchTuning()
        self._check(self.lib.mplbgpu_batch_get_tuning(self.h, ctypes.byref(t)))
        return dict(tile_nodes=t.tile_nodes, persistent=t.persistent,
                    chunk=t.chunk, ctas_per_sm=t.ctas_per_sm)

    def pack(self, fields: Optional[Sequence[np.ndarray]]):
        if fields is None:
            return None
        return np.ascontiguousarray(np.concatenate(
            [np.asarray(f, np.float64).reshape(-1) for f in fields]))

    def init(self, rho=None, u=None, v=None):
        """Per-cavity fields (lists of n x n arrays, MPLB units) or None."""
        packed = [self.pack(f) for f in (rho, u, v)]
        ptrs = [None if p is None else p.ctypes.data for p in packed]
        self._check(self.lib.mplbgpu_batch_init(self.h, *ptrs))

    def step(self, n):
        self._check(self.lib.mplbgpu_batch_step(self.h, int(n)))

    def run(self, max_steps, check_period=1000, criterion=1e-8):
        """Per cavity: steps, last residual, converged (bool); cavities whose
        residual turned NaN are in `self.diverged` afterwards."""
        k = len(self.specs)
        steps = np.zeros(k, np.int64)
        res = np.zeros(k)
        conv = np.zeros(k, np.int32)
        self._check(self.lib.mplbgpu_batch_run(
            self.h, int(max_steps), int(check_period), float(criterion),
            steps.ctypes.data, res.ctypes.data, conv.ctypes.data))
        self.diverged = conv == -1
        return steps, res, conv == 1

    def macro(self):
        """[(rho, u, v)] per cavity, n x n arrays (MPLB units)."""
        out = [np.zeros(self.total_nodes) for _ in range(3)]
        self._check(self.lib.mplbgpu_batch_download_macro(
            self.h, *[a.ctypes.data for a in out]))
        res = []
        for i, s in enumerate(self.specs):
            a, b = self.offsets[i], self.offsets[i + 1]
            res.append(tuple(f[a:b].reshape(s.n, s.n) for f in out))
        return res

    def stats(self):
        ms = ctypes.c_double()
        nu = ctypes.c_longlong()
        nl = ctypes.c_longlong()
        self._check(self.lib.mplbgpu_batch_stats(
            self.h, ctypes.byref(ms), ctypes.byref(nu), ctypes.byref(nl)))
        return dict(device_ms=ms.value, node_updates=nu.value,
                    launches=nl.value)


def _cache_key(batch: Batch) -> str:
    import torch
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "?"
    hist = {}
    for s in batch.specs:
        hist[s.n] = hist.get(s.n, 0) + 1
    h = hashlib.sha1(json.dumps(sorted(hist.items())).encode()).hexdigest()
    return f"{name}|{batch.precision}|{h[:12]}"


def default_candidates():
    """Tile size x launch style: one CTA per tile (persistent 0) or
    cooperative persistent steps (1, x CTAs per SM)."""
    graph = [dict(tile_nodes=t, persistent=0, chunk=50, ctas_per_sm=8)
             for t in (64, 128, 256)]
    persistent = [dict(tile_nodes=t, persistent=1, chunk=50, ctas_per_sm=k)
                  for t in (128, 256) for k in (4, 8)]
    return graph + persistent


def autotune(batch: Batch, steps: int = 200, cache: str = DEFAULT_CACHE,
             candidates=None, force=False):
    """Times each candidate tuning on `batch` (from its initial state) and
    keeps the fastest (MLUPS over `steps` steps); results are cached."""
    key = _cache_key(batch)
    table = {}
    if os.path.exists(cache):
        with open(cache) as fh:
            table = json.load(fh)
    if key in table and not force:
        batch.set_tuning(**table[key]["tuning"])
        return table[key]
    if candidates is None:
        candidates = default_candidates()
    results = []
    for cand in candidates:
        batch.set_tuning(**cand)
        batch.init()
        batch.step(cand["chunk"])            # warm-up (graph capture)
        s0 = batch.stats()
        batch.step(steps)
        s1 = batch.stats()
        ms = s1["device_ms"] - s0["device_ms"]
        mlups = batch.total_nodes * steps / (ms * 1e-3) / 1e6
        results.append((mlups, cand))
    results.sort(key=lambda r: -r[0])
    best = {"tuning": results[0][1], "mlups": results[0][0],
            "all": [{"mlups": m, **c} for m, c in results]}
    table[key] = best
    with open(cache, "w") as fh:
        json.dump(table, fh, indent=1)
    batch.set_tuning(**best["tuning"])
    return best
