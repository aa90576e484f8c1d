"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): the timing is
the max over ranks, and the reference arm runs on rank 0 alone with every
rank exiting 0."""
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


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(1.5 + rank, dist, device="cpu")
        alone = bench.max_over_ranks(7.0, None)
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(f"{got} {alone}")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    for r in range(2):
        got, alone = open(tmp_path / f"r{r}.txt").read().split()
        assert float(got) == 2.5
        assert float(alone) == 7.0


def test_reference_arm_under_torchrun():
    """bench.py --impl reference launched as the driver does for N=2: rank 0
    prints one JSON line, the other rank exits 0 without work."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.reference_available(openmp=True):
        pytest.skip("the reference's OpenMP build is not compiled here")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "reference"
