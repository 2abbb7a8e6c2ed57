"""The C-ABI library: builds for sm_100a, loads, exports every entry point
include/mplbgpu.h and include/mplbnn.h declare; descriptor validation that
needs no device."""
import os
import re
import subprocess

import pytest

from mplb_b200 import abi, build, config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for h in ("mplbgpu.h", "mplbnn.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(mplb(?:gpu|nn)_[a-z_]+)\s*\(", text))
    return sorted(names)


def test_header_and_binding_agree():
    assert header_functions() == abi.exported_symbols()


def test_library_exports_every_declared_symbol():
    build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", build.OUT],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mplb(?:gpu|nn)_[a-z_]+)", out))
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    abi.load_library()  # loads without a device


def test_build_targets_sm100a_only():
    for obj, cmd in build.compile_commands():
        archs = [c for c in cmd if c.startswith("-gencode")]
        assert archs == ["-gencode=arch=compute_100a,code=sm_100a"]
        if obj.endswith(("mplbgpu.cu.o", "kernels_f64.cu.o")):
            assert "-fmad=false" in cmd


def test_descriptor_round_trip():
    case = config.cavity(3, 16, 0.05, re=400)
    d, keep = case.to_desc()
    assert d.abi_version == abi.ABI_VERSION
    assert d.nblocks == 1 and d.blocks[0].size[2] == 16
    assert d.nboundaries == 6
    assert [d.boundaries[i].surface for i in range(6)] == [0, 1, 2, 3, 4, 5]
    assert d.boundaries[4].given[0] == pytest.approx(0.05 * 3 ** 0.5)
