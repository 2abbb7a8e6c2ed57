"""One block decomposed into slabs along its last axis, one per GPU.

The reference spreads a block over MPI ranks through OPS (``ops_partition``
in ``Partition()``, Src/flowfield.cpp); here each slab is a block of its own
context whose faces towards the neighbouring slabs are "cut"
(``mplbgpu_block.cut``): nodes there are interior, and before every step the
populations leaving each slab through a cut face are copied into the
neighbour's halo layer (``mplbgpu_export_face`` / ``mplbgpu_import_face``).
The decomposed run steps bit for bit as the whole block does.

    slab_bounds(n, parts)              -> [(start, stop), ...]
    slab_case(case, parts, index)      -> the slab's CaseConfig
    SlabSolver(case, parts, exchange)  -> steps, moments, residual

Exchanges: ``LocalExchange`` moves the faces between contexts of one
process (one device, device-to-device copies); ``DistExchange`` runs one
slab per rank of a torch.distributed process group (NCCL send/recv of the
face buffers between neighbouring ranks, CPU buffers through gloo).  Only
single blocks without connections are decomposed; the boundary conditions
of the cut faces belong to the slab at that end.
"""
import ctypes
import dataclasses
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import abi
from .config import CaseConfig
from .solver import MplbGpuError, Solver

# surfaces at the min / max end of each axis (BoundarySurface)
_LOW = {0: "Left", 1: "Bottom", 2: "Back"}
_HIGH = {0: "Right", 1: "Top", 2: "Front"}
# faces making up an edge surface
_EDGE_FACES = {
    "LeftBack": ("Left", "Back"), "LeftFront": ("Left", "Front"),
    "RightBack": ("Right", "Back"), "RightFront": ("Right", "Front"),
    "TopBack": ("Top", "Back"), "TopFront": ("Top", "Front"),
    "BottomBack": ("Bottom", "Back"), "BottomFront": ("Bottom", "Front"),
    "LeftTop": ("Left", "Top"), "LeftBottom": ("Left", "Bottom"),
    "RightTop": ("Right", "Top"), "RightBottom": ("Right", "Bottom"),
}


def slab_bounds(n: int, parts: int) -> List[Tuple[int, int]]:
    """Contiguous ranges of n nodes, sizes differing by at most one; every
    slab needs at least 2 nodes."""
    if parts < 1 or n < 2 * parts:
        raise ValueError(f"cannot cut {n} nodes into {parts} slabs")
    base, extra = divmod(n, parts)
    out, start = [], 0
    for k in range(parts):
        size = base + (1 if k < extra else 0)
        out.append((start, start + size))
        start += size
    return out


def _faces(surface: str) -> Tuple[str, ...]:
    return _EDGE_FACES.get(surface, (surface,))


def slab_case(case: CaseConfig, parts: int, index: int) -> CaseConfig:
    """The case of slab `index` of `parts` along the last axis."""
    if len(case.block_ids) != 1 or case.connections:
        raise ValueError("only a single block without connections is "
                         "decomposed")
    if case.swap:
        raise ValueError("the swap scheme is not decomposed")
    axis = case.space_dim - 1
    size = list(case.block_sizes[0])
    start, stop = slab_bounds(size[axis], parts)[index]
    size[axis] = stop - start
    cut_faces = set()
    if index > 0:
        cut_faces.add(_LOW[axis])
    if index < parts - 1:
        cut_faces.add(_HIGH[axis])
    bounds = [b for b in case.boundaries
              if not (set(_faces(b.surface)) & cut_faces)]
    cut = 0
    for f in cut_faces:
        cut |= 1 << abi.SURFACES[f]
    bid = case.block_ids[0]
    start_pos = dict(case._start_pos())
    pos = list(start_pos[bid])
    pos[axis] = pos[axis] + start * case.mesh_size
    return dataclasses.replace(
        case, case_name=f"{case.case_name}_slab{index}",
        block_sizes=[tuple(size)], boundaries=bounds,
        start_pos={bid: pos}, cuts={bid: cut})


class LocalExchange:
    """Face moves between slabs held by this process (device copies).  A
    step: every slab exports its faces, then begins its step (the interior,
    which reads no halo), imports its neighbours' faces and finishes the
    step."""

    def step(self, solver: "SlabSolver"):
        parts = solver.parts
        for p in parts:
            p.export_faces()
        for p in parts:
            p.synchronize()     # a neighbour's export is read by our import
        for p in parts:
            p.step_begin()
        for k in range(len(parts) - 1):
            lo, hi = parts[k], parts[k + 1]
            lo.import_face("high", hi.out["low"])
            hi.import_face("low", lo.out["high"])
        for p in parts:
            p.step_finish()


class DistExchange:
    """One slab per rank; neighbouring ranks swap their face buffers
    (torch.distributed point-to-point).  With NCCL the device buffers go
    GPU to GPU; with gloo they are staged through host memory, which also
    lets several ranks share one GPU (no kernel waits on another rank: the
    hosts wait)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.staged = dist.get_backend(group) == "gloo"
        self.host = {}

    def _wire(self, buf, key):
        """The tensor that travels: the buffer itself, or its host copy."""
        if not self.staged or not buf.is_cuda:
            return buf
        h = self.host.get(key)
        if h is None or h.numel() != buf.numel():
            h = self.host[key] = buf.new_empty(buf.shape, device="cpu")
        return h

    def _ops(self, p, rank):
        dist = self.dist
        peers = {"low": rank - 1, "high": rank + 1}
        ops, recv = [], []
        for side in ("low", "high"):
            if p.out[side] is None:
                continue
            send = self._wire(p.out[side], ("out", side))
            if send is not p.out[side]:
                send.copy_(p.out[side])
            into = self._wire(p.inb[side], ("in", side))
            ops.append(dist.P2POp(dist.isend, send, peers[side], self.group))
            ops.append(dist.P2POp(dist.irecv, into, peers[side], self.group))
            recv.append((side, into))
        return ops, recv

    def step(self, solver: "SlabSolver"):
        """One step: export the faces, begin the step (the interior), move
        the faces while it runs, import them, finish the step."""
        (p,) = solver.parts
        if not self.staged:
            return self._step_device(p, solver.index0)
        # gloo: the faces go through host memory while the interior runs
        p.export_faces()
        p.synchronize()
        p.step_begin()
        ops, recv = self._ops(p, solver.index0)
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        for side, into in recv:
            if into is not p.inb[side]:
                p.inb[side].copy_(into)
        if any(b is not None and b.is_cuda for b in p.inb.values()):
            import torch
            torch.cuda.current_stream().synchronize()
        for side, _ in recv:
            p.import_face(side, p.inb[side])
        p.step_finish()

    def _step_device(self, p, rank):
        """NCCL: nothing waits on the host.  The context's stream exports
        the faces and runs the interior; a side stream waits for the
        export, sends and receives; the context's stream waits for the
        transfer, imports and finishes the step."""
        import torch
        ctx = torch.cuda.ExternalStream(p.stream_ptr())
        if getattr(self, "comm", None) is None:
            self.comm = torch.cuda.Stream()
        p.export_faces()
        exported = torch.cuda.Event()
        exported.record(ctx)
        p.step_begin()
        ops, recv = self._ops(p, rank)
        moved = torch.cuda.Event()
        with torch.cuda.stream(self.comm):
            self.comm.wait_event(exported)
            if ops:
                for req in self.dist.batch_isend_irecv(ops):
                    req.wait()
            moved.record(self.comm)
        ctx.wait_event(moved)
        for side, _ in recv:
            p.import_face(side, p.inb[side])
        p.step_finish()


class _Part:
    """One slab: its solver and its face buffers (device tensors)."""

    def __init__(self, case: CaseConfig, index: int, parts: int, lib,
                 device: Optional[str]):
        import torch
        self.index = index
        self.case = case
        self.solver = Solver(case, lib)
        self.lib = self.solver.lib
        self.bid = case.block_ids[0]
        axis = case.space_dim - 1
        self.surface = {"low": abi.SURFACES[_LOW[axis]],
                        "high": abi.SURFACES[_HIGH[axis]]}
        self.out, self.inb = {}, {}
        for side, present in (("low", index > 0), ("high", index < parts - 1)):
            if not present:
                self.out[side] = self.inb[side] = None
                continue
            n = ctypes.c_longlong()
            eb = ctypes.c_int()
            self._check(self.lib.mplbgpu_face_size(
                self.solver.h, self.bid, self.surface[side], ctypes.byref(n),
                ctypes.byref(eb)))
            nbytes = n.value * eb.value
            self.out[side] = torch.empty(nbytes, dtype=torch.uint8,
                                         device=device)
            self.inb[side] = torch.empty(nbytes, dtype=torch.uint8,
                                         device=device)

    def _check(self, rc):
        if rc != abi.OK:
            raise MplbGpuError(rc, self.lib.mplbgpu_last_error(
                self.solver.h).decode())

    def export_faces(self):
        for side, buf in self.out.items():
            if buf is not None:
                self._check(self.lib.mplbgpu_export_face(
                    self.solver.h, self.bid, self.surface[side],
                    ctypes.c_void_p(buf.data_ptr())))

    def import_face(self, side, buf):
        self._check(self.lib.mplbgpu_import_face(
            self.solver.h, self.bid, self.surface[side],
            ctypes.c_void_p(buf.data_ptr())))

    def synchronize(self):
        self.solver.synchronize()

    def step_begin(self):
        self._check(self.lib.mplbgpu_step_begin(self.solver.h))

    def step_finish(self):
        self._check(self.lib.mplbgpu_step_finish(self.solver.h))
        self.solver.steps_done += 1

    def stream_ptr(self):
        st = ctypes.c_void_p()
        self._check(self.lib.mplbgpu_get_stream(self.solver.h,
                                                ctypes.byref(st)))
        return st.value or 0


class SlabSolver:
    """Slabs `indices` of a `parts`-way decomposition of `case`, held by
    this process (all of them with LocalExchange, one per rank with
    DistExchange)."""

    def __init__(self, case: CaseConfig, parts: int,
                 indices: Sequence[int], exchange, lib=None,
                 device: Optional[str] = "cuda"):
        self.case = case
        self.nparts = parts
        self.index0 = indices[0]
        self.exchange_impl = exchange
        self.parts = [_Part(slab_case(case, parts, k), k, parts, lib, device)
                      for k in indices]
        # arrays are (nz, ny, nx): the slabs follow one another along z in
        # 3D and along y in 2D
        self.join_axis = 0 if case.space_dim == 3 else 1

    def close(self):
        for p in self.parts:
            p.solver.close()

    # -- state ----------------------------------------------------------------
    def init_uniform(self):
        for p in self.parts:
            p.solver.init_uniform()

    def upload_f(self, f):
        """The distributions of the whole block (nz, ny, nx, Q); each slab
        held here takes its part (restart)."""
        f = np.asarray(f)
        axis = self.case.space_dim - 1
        n = self.case.block_sizes[0][axis]
        bounds = slab_bounds(n, self.nparts)
        for p in self.parts:
            lo, hi = bounds[p.index]
            part = f[lo:hi] if self.join_axis == 0 else f[:, lo:hi]
            p.solver.upload_f(p.bid, np.ascontiguousarray(part))

    def set_step(self, step):
        """Positions every slab held here at `step` (a restart)."""
        for p in self.parts:
            p.solver.set_step(step)

    def stream_collision(self, n=1):
        """n steps; the faces cross during each step (after its interior
        has been queued, before its boundary layers)."""
        for _ in range(int(n)):
            self.exchange_impl.step(self)

    def update_macro_vars(self):
        for p in self.parts:
            p.solver.update_macro_vars()

    def residual_sums(self):
        nv = self.case.space_dim + 1
        diff = np.zeros(4)
        tot = np.zeros(4)
        for p in self.parts:
            d = np.zeros(4)
            s = np.zeros(4)
            p._check(p.lib.mplbgpu_residual_sums(p.solver.h, d.ctypes.data,
                                                 s.ctypes.data))
            diff += d
            tot += s
        return diff[:nv], tot[:nv]

    def calc_residual_error(self, check_period=None, reduce=None):
        """(GetMaximumResidual, per-variable residuals) over all slabs;
        `reduce` sums the (diff, sum) arrays over processes."""
        cp = check_period or self.case.check_period
        diff, tot = self.residual_sums()
        if reduce is not None:
            diff, tot = reduce(diff, tot)
        per = diff / tot
        mx = 0.0
        for r in per:
            rel = r / (cp * self.case.dt)
            if mx <= rel:
                mx = rel
        return mx, per

    def macro(self):
        """Moments of the slabs held here, joined along the cut axis."""
        parts = [p.solver.macro(p.bid) for p in self.parts]
        return [np.concatenate([q[m] for q in parts], axis=self.join_axis)
                for m in range(len(parts[0]))]

    def f(self):
        return np.concatenate([p.solver.f(p.bid) for p in self.parts],
                              axis=self.join_axis)
