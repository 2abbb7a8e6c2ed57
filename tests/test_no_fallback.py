"""The product has no CPU fallback: a missing native library and a host
without a CUDA device both end in an error from every front end."""
import pytest

from mplb_b200 import abi, config, warmstart
from mplb_b200.batch import Batch, BatchError, cavity_set
from mplb_b200.solver import MplbGpuError, Solver


def _has_cuda():
    import torch
    return torch.cuda.is_available()


def test_missing_library_is_an_error(tmp_path):
    with pytest.raises(abi.NativeLibraryError, match="missing"):
        abi.load_library(str(tmp_path / "libmplbgpu.so"))


def test_unloadable_library_is_an_error(tmp_path):
    bad = tmp_path / "libmplbgpu.so"
    bad.write_bytes(b"not a shared object")
    with pytest.raises(abi.NativeLibraryError, match="cannot load"):
        abi.load_library(str(bad))


@pytest.mark.skipif(_has_cuda(), reason="needs a host without a GPU")
def test_no_device_solver():
    with pytest.raises(MplbGpuError, match="NO_DEVICE"):
        Solver(config.cavity(3, 8, 0.05, re=100))


@pytest.mark.skipif(_has_cuda(), reason="needs a host without a GPU")
def test_no_device_batch():
    with pytest.raises(BatchError, match="no CUDA device"):
        Batch(cavity_set(4))


@pytest.mark.skipif(_has_cuda(), reason="needs a host without a GPU")
def test_no_device_network():
    with pytest.raises(warmstart.NetworkError, match="no CUDA device"):
        warmstart.Network(32)
