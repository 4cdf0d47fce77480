"""bench.py --impl reference on the request stream: the reference CPU pass
on the stream's first requests, in a process that never loads the GPU
library (its meshes come from the standalone builder and a numpy reader)."""
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_loads_no_gpu_library(tmp_path):
    from oracle.oracle import reference_available
    if not (reference_available(2) and reference_available(3)):
        pytest.skip("reference harness not built")
    code = ("import sys, bench\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--requests', '3', '--steps', '1',"
            " '--warmup', '1']\n"
            "bench.main()\n"
            "print('LOADED' if 'libsfxflux' in open('/proc/self/maps').read() else 'CLEAN')\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "CLEAN"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["steps"] == 1 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_reference_arm_on_two_ranks():
    """launched like the GPU arm on two ranks: rank 0 alone runs the sample
    and prints one line (n_gpus 2); the other rank exits at once, and no
    process group is formed"""
    from oracle.oracle import reference_available
    if not (reference_available(2) and reference_available(3)):
        pytest.skip("reference harness not built")
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--gpus", "2", "--requests", "3", "--steps", "1",
           "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["config"]["parallelism"].startswith("2 GPUs")
