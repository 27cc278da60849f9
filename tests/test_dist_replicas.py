"""The multi-process plumbing of bench.py, on CPU with two gloo ranks: one
simulation does not shard (every 2-D sine transform couples a whole level),
so N GPUs run N independent replicas and the ranks only meet at a barrier and
at the max of their timed regions."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    d = bench.Dist()
    d.barrier()
    m = d.max(1.5 + rank)             # a per-rank time; every rank gets the slowest
    d.barrier()
    d.close()
    with open(os.path.join(out, "rank%d.json" % rank), "w") as f:
        json.dump({"world": d.world, "rank": d.rank, "max": m}, f)


def test_barrier_and_max_over_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        with open(tmp_path / ("rank%d.json" % r)) as f:
            res = json.load(f)
        assert res == {"world": 2, "rank": r, "max": 2.5}


def test_reference_arm_under_torchrun():
    """`torch.distributed.run --nproc-per-node 2 bench.py --impl reference`:
    rank 0 alone times the CPU restatement and prints one JSON line; rank 1
    exits 0 without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()),
           "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout[-2000:]
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
