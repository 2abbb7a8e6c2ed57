"""Checkpoint and restart of the distributions, per block.

The reference dumps each block's distributions to HDF5 as
``<CaseName>_<blockId>_T<step>`` (``Field::WriteToHDF5``, Src/field.h:
166-205) and restarts from them when the case's ``CurrentTimeStep`` is
non-zero (Src/model.cpp:299-309).  HDF5 is not part of this build, so the
same per-block files are raw little-endian float64 arrays in the reference's
node layout (z, y, x slowest to fastest, the Q populations of a node
contiguous, halo excluded) with the suffix ``.f64``, plus one JSON manifest
``<CaseName>_T<step>.json`` naming the case, step, lattice and block shapes.

    save(solver, directory, step)        -> manifest path
    restart(case, directory, step, lib)  -> Solver positioned after `step`
    save_slabs / restart_slabs           -> the same for a run split into
                                            slabs (files of the whole block)

A restart uploads each block's f (``mplbgpu_upload_f``) and positions the
run at the checkpoint's step (``mplbgpu_set_step``: check periods and the
FP16 form's rounding draws continue from there); in FP64 the next step then
continues bit for bit as the uninterrupted run would.
"""
import json
import os
from typing import Dict, Optional

import numpy as np

from .solver import Solver

FORMAT = "mplb-b200 distributions v1"


def block_file(directory: str, case_name: str, block: int, step: int) -> str:
    return os.path.join(directory, f"{case_name}_{block}_T{step}.f64")


def manifest_file(directory: str, case_name: str, step: int) -> str:
    return os.path.join(directory, f"{case_name}_T{step}.json")


def write(directory: str, case, step: int,
          fields: Dict[int, np.ndarray]) -> str:
    """Writes the per-block distributions (arrays shaped (nz, ny, nx, Q))
    and the manifest; returns the manifest path."""
    os.makedirs(directory, exist_ok=True)
    blocks = {}
    for b in case.block_ids:
        f = np.ascontiguousarray(fields[b], dtype="<f8")
        nx, ny, nz = case.size3(b)
        if f.shape != (nz, ny, nx, case.q):
            raise ValueError(f"block {b}: shape {f.shape}, expected "
                             f"{(nz, ny, nx, case.q)}")
        path = block_file(directory, case.case_name, b, step)
        f.tofile(path)
        blocks[str(b)] = {"file": os.path.basename(path),
                          "shape": list(f.shape)}
    man = {"format": FORMAT, "case": case.case_name, "step": int(step),
           "space_dim": case.space_dim, "q": case.q,
           "precision": getattr(case, "precision", "fp64"),
           "blocks": blocks}
    mpath = manifest_file(directory, case.case_name, step)
    with open(mpath, "w") as fh:
        json.dump(man, fh, indent=1)
    return mpath


def read(directory: str, case, step: int) -> Dict[int, np.ndarray]:
    """Reads and checks the per-block distributions written by `write`."""
    with open(manifest_file(directory, case.case_name, step)) as fh:
        man = json.load(fh)
    if man.get("format") != FORMAT or man["q"] != case.q or \
            man["space_dim"] != case.space_dim:
        raise ValueError("checkpoint does not match the case")
    if man.get("precision", "fp64") != getattr(case, "precision", "fp64"):
        raise ValueError(f"checkpoint was written by a {man['precision']} "
                         f"run, the case is {case.precision}")
    out = {}
    for b in case.block_ids:
        ent = man["blocks"].get(str(b))
        if ent is None:
            raise ValueError(f"checkpoint has no block {b}")
        f = np.fromfile(os.path.join(directory, ent["file"]), dtype="<f8")
        shape = tuple(ent["shape"])
        if f.size != int(np.prod(shape)):
            raise ValueError(f"block {b}: truncated file")
        nx, ny, nz = case.size3(b)
        if shape != (nz, ny, nx, case.q):
            raise ValueError(f"block {b}: shape {shape} does not match case")
        out[b] = f.reshape(shape)
    return out


def save(solver: Solver, directory: str, step: int) -> str:
    """Checkpoint of a running solver (its current f per block)."""
    return write(directory, solver.case, step,
                 {b: solver.f(b) for b in solver.case.block_ids})


def save_slabs(solver, directory: str, step: int) -> str:
    """Checkpoint of a slab-decomposed run held by this process (every
    slab), in the files of the undivided block: it restarts as the whole
    block or as slabs."""
    if len(solver.parts) != solver.nparts:
        raise ValueError("every slab must be held by this process")
    bid = solver.case.block_ids[0]
    return write(directory, solver.case, step, {bid: solver.f()})


def restart_slabs(case, parts: int, directory: str, step: int, lib=None):
    """A slab-decomposed solver (all slabs in this process) holding the
    checkpointed f of the undivided block."""
    from . import slab
    fields = read(directory, case, step)
    s = slab.SlabSolver(case, parts, list(range(parts)), slab.LocalExchange(),
                        lib)
    s.upload_f(fields[case.block_ids[0]])
    s.set_step(step)
    return s


def restart(case, directory: str, step: int, lib=None) -> Solver:
    """A solver holding the checkpointed f of every block."""
    fields = read(directory, case, step)
    s = Solver(case, lib)
    for b in case.block_ids:
        s.upload_f(b, fields[b])
    s.set_step(step)
    return s
