"""The N > 1 plumbing of bench.py on CPU ranks (gloo, world size 2).

The path has no exchange step: N GPUs run N independent replicas, and the
ranks only meet at the barriers around the timed region and in the max of
their times.  These tests run that host logic as two CPU processes: the
max-over-ranks reduction, and the reference arm launched the way the
multi-GPU benchmark launches it (torch.distributed.run, rendezvous on
127.0.0.1), where rank 0 alone works and prints one line.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    world, r, _ = bench.dist_setup("gloo")
    bench.dist_barrier(world)
    m = bench.dist_max(1.5 + r, world)  # each rank's time; the job's is the slowest
    (Path(out_dir) / f"rank{r}.json").write_text(json.dumps({"world": world, "max": m}))
    dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_rank_main, args=(free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        got = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert got == {"world": 2, "max": 2.5}


def test_reference_arm_under_torchrun():
    from oracle import build_ref
    if not build_ref.lib_path(8).exists():
        pytest.skip("reference build oracle/_ref/libgnref_L8_i0.so not present")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), str(ROOT / "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--L", "8"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
