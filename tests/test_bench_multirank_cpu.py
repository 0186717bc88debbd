"""bench.py's multi-rank plumbing on host cores: world size 2 over gloo.
Replica runs reduce their step times with a max over ranks, and the
reference arm runs on rank 0 only while the other ranks exit cleanly."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _max_worker(rank, port, values, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2")
    dist.init_process_group("gloo", rank=rank, world_size=2)
    sys.path.insert(0, str(ROOT))
    import bench
    out[rank] = bench._max_over_ranks(values[rank], 2)
    bench._barrier(2)
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_max_worker, args=(_free_port(), [3.5, 7.25], out), nprocs=2, join=True)
    assert dict(out) == {0: 7.25, 1: 7.25}


@pytest.mark.skipif(not (ROOT / "oracle" / "_build" / "pi_cpu").exists(), reason="host restatement not built")
def test_reference_arm_under_torchrun():
    port = _free_port()
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), str(ROOT / "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, cwd=str(ROOT),
                       env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
