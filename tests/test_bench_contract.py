"""bench.py's host-side contract on CPU: the reference arm under a 2-process torchrun launch
prints exactly one JSON line on rank 0 (the other rank exits 0 without output), with the
same metric string and config the CUDA arm prints for the workload, and the end-to-end
sample count rule."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_e2e_sample_count():
    assert bench.e2e_count(1325.0) == 3          # the headline: seconds per call
    assert bench.e2e_count(3.0) == 21            # millisecond calls span about a second
    assert bench.e2e_count(100.0) == 10
    assert bench.e2e_count(0.0) == 21


def test_headline_metric_string():
    # the 50-start x 200-step alignment workloads carry the headline metric verbatim
    assert bench.metric_of(bench.WORKLOADS["surf_esp"]) == bench.HEADLINE_METRIC
    assert bench.metric_of(bench.WORKLOADS["vol"]) == bench.HEADLINE_METRIC


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_once(tmp_path):
    import socket
    with socket.socket() as sk:      # a free port for the rendezvous
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    env = dict(os.environ, PYTHONPATH=ROOT, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--workload", "vol", "--pairs", "4", "--steps", "1", "--warmup", "0",
           "--cpu-seconds", "0.5"]
    out = subprocess.run(cmd, cwd=tmp_path, env=env, capture_output=True, text=True,
                         timeout=540)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, out.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.metric_of(bench.WORKLOADS["vol"])
    assert line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port"
