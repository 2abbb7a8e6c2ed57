"""B200 lattice Boltzmann stream-collision path for MPLB cases.

    from mplb_b200 import config, Solver
    case = config.cavity(3, 256, 0.05, re=400)
    with Solver(case) as s:
        s.init_uniform()
        s.iterate(steps=5000)

The compute path is libmplbgpu.so (hand-written sm_100a CUDA behind the C
ABI in include/mplbgpu.h); ``mplb_b200.build`` compiles it in-tree.
"""
from . import abi, config
from .solver import MplbGpuError, Solver

__all__ = ["abi", "config", "Solver", "MplbGpuError"]
