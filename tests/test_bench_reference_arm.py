"""bench.py's reference arm on CPU: the reference's own CPU build of the step
(oracle/_ref) timed on a small cavity, the JSON line's keys, one line from
rank 0 under torchrun with two ranks, and the `unavailable` line for the
workloads the reference has no counterpart of."""
import json
import os
import socket
import subprocess
import sys
import types

import pytest

from oracle import pyoracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

needs_ref = pytest.mark.skipif(not pyoracle.reference_available("_omp"),
                               reason="reference CPU build not present")


def run(args, env=None, timeout=300):
    e = dict(os.environ)
    e.update(env or {})
    e.setdefault("OMP_NUM_THREADS", "2")
    p = subprocess.run(args, cwd=ROOT, env=e, capture_output=True, text=True,
                       timeout=timeout)
    assert p.returncode == 0, p.stderr[-2000:]
    return [json.loads(l) for l in p.stdout.splitlines()
            if l.startswith("{")]


@needs_ref
@pytest.mark.parametrize("scheme", ["stream", "swap"])
def test_reference_line_keys(scheme):
    lines = run([sys.executable, "bench.py", "--impl", "reference", "--size",
                 "20", "--steps", "3", "--warmup", "1", "--scheme", scheme])
    assert len(lines) == 1
    d = lines[0]
    assert d["impl"] == "reference"
    assert d["unit"] == "MLUPS" and d["value"] > 0
    assert d["higher_is_better"] is True
    assert d["steps"] == 3 and d["warmup"] == 1
    assert d["ms_per_step"] > 0
    # the same config as the B200 arm's line for the same arguments
    import bench
    args = types.SimpleNamespace(size=20, scheme=scheme, precision="fp64")
    assert d["config"] == bench.cavity_config(args, 1, 20 ** 3)
    assert d["cpu_baseline"]["sample"].count("1 warm-up") == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1
    assert cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "MLUPS",
                        "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    if scheme == "swap":
        assert "swap" in d["metric"] and "SwapStreamCollision" in cb["sample"]
    else:
        assert "swap" not in d["metric"]


@needs_ref
def test_reference_two_ranks_one_line():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    lines = run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                 "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                 "--master-port", str(port), "bench.py", "--impl",
                 "reference", "--gpus", "2", "--size", "16", "--steps", "2",
                 "--warmup", "1"])
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2


@pytest.mark.parametrize("workload", ["cavities", "cavities-warmstart"])
def test_reference_unavailable_for_new_workloads(workload):
    lines = run([sys.executable, "bench.py", "--impl", "reference",
                 "--workload", workload, "--steps", "1", "--warmup", "1"])
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and "unavailable" in lines[0]
