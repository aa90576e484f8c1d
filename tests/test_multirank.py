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


# ---- the destination-range split of loopy BP (belief_propagation_b200.sharded)

class NumpyRangeEngine:
    """A rank's node range computed on the CPU with the reference's fp32
    operations in the reference's order (the checker side of the split: the
    test exercises the partition and the exchange; the CUDA range kernel is
    checked against bp_loopy in tests/test_gpu_sharded.py)."""

    def __init__(self, net, begin, end, chunk, world):
        import numpy as np
        from belief_propagation_b200.sharded import shard_edges
        eids = shard_edges(net, begin, end)
        order = eids[np.argsort(net.dst[eids], kind="stable")]     # position order
        self.begin, self.end, self.S = begin, end, int(net.s_max)
        self.pos_edge = order
        self.src = net.src[order].astype(np.int64)
        self.dst = net.dst[order].astype(np.int64)
        self.J = np.ascontiguousarray(net.joint[order][:, : self.S, : self.S], np.float32)
        counts = np.bincount(self.dst - begin, minlength=end - begin) if len(order) else np.zeros(end - begin, int)
        self.ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.q = [np.zeros((world * chunk, self.S), np.float32) for _ in range(2)]

    def _send(self, x):
        import numpy as np
        f32 = np.float32
        E, S = self.J.shape[0], self.S
        m = np.zeros((E, S), f32)
        tot = np.zeros(E, f32)
        for i in range(S):
            part = np.zeros(E, f32)
            for j in range(S):
                part = (part + (self.J[:, i, j] * x[:, j]).astype(f32)).astype(f32)
            m[:, i] = part
            tot = (tot + part).astype(f32)
        tot = np.where(tot <= 0, f32(1.0), tot)
        return (m / tot[:, None]).astype(np.float32)

    def _products(self, start, m):
        import numpy as np
        out = start.copy()
        deg = np.diff(self.ptr)
        for r in range(int(deg.max()) if len(deg) else 0):
            nodes = np.nonzero(deg > r)[0]
            mm = m[self.ptr[nodes] + r]
            out[nodes] = np.where(mm == mm, (out[nodes] * mm).astype(np.float32), out[nodes])
        return out

    def reset(self, beliefs):
        import numpy as np
        self.b = np.ascontiguousarray(beliefs[:, : self.S], np.float32).copy()
        self.m = self._send(self.b[self.src])

    def send_buffers(self, k):
        sl = slice(self.begin, self.end)
        self.q[k][sl] = self._products(self.b[sl], self.m)

    def iterate(self, k_in, k_out):
        import numpy as np
        f32 = np.float32
        m_new = self._send(self.q[k_in][self.src])
        d = (self.m - m_new).astype(f32)
        d = np.where(d != d, f32(0.0), np.abs(d))
        part = float(d.astype(np.float64).sum())
        sl = slice(self.begin, self.end)
        ones = np.ones((self.end - self.begin, self.S), f32)
        prod = self._products(ones, m_new)
        has = np.diff(self.ptr) > 0
        b = self.b[sl].copy()
        b[has] = (b[has] * prod[has]).astype(f32)
        tot = np.zeros(len(b), f32)
        for i in range(self.S):
            tot = (tot + b[:, i]).astype(f32)
        tot = np.where(tot <= 0, f32(1.0), tot)
        b = (b / tot[:, None]).astype(f32)
        self.b[sl] = b
        self.q[k_out][sl] = self._products(b, m_new)
        self.m = m_new
        import torch
        return torch.tensor([part], dtype=torch.float64)

    def beliefs(self):
        return self.b[self.begin:self.end]


class _NumpyTorchComm:
    """TorchComm over numpy send buffers (gloo moves CPU tensors)."""

    def __init__(self, dist, rank, chunk):
        from belief_propagation_b200.sharded import TorchComm
        self.inner = TorchComm(dist, rank, chunk)

    def exchange(self, engines, k):
        import torch
        (e,) = engines
        t = torch.from_numpy(e.q[k])
        self.inner.exchange([type("E", (), {"q": {k: t}})()], k)

    def deltas(self, engines, parts):
        return self.inner.deltas(engines, parts)


def _shard_rank(rank, world, port, out_dir):
    import numpy as np
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import belief_network_wrapper as W
    from belief_propagation_b200.sharded import node_ranges, sharded_loopy
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        net = W.bp.synth.random_loopy(1500, 6000, 3, 0.1, seed=77)
        ranges, chunk = node_ranges(net.V, world)
        eng = NumpyRangeEngine(net, *ranges[rank], chunk, world)
        r = sharded_loopy([eng], _NumpyTorchComm(dist, rank, chunk), net.beliefs, 1e-3, 40)
        np.savez(os.path.join(out_dir, f"shard{rank}.npz"), beliefs=eng.beliefs(), messages=eng.m,
                 edges=eng.pos_edge, iterations=r["iterations"], executed=r["executed"])
    finally:
        dist.destroy_process_group()


def test_destination_range_split_matches_one_rank(tmp_path):
    """Loopy BP split over 2 gloo ranks by destination-node ranges (each rank
    holds its nodes' in-edges; send buffers all-gathered, deltas summed in
    rank order after every iteration): the gathered beliefs and latest
    messages equal the oracle's single-process run bit for bit, with the same
    iteration count."""
    import numpy as np
    import torch.multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, ROOT)
    import belief_network_wrapper as W
    import oracle as O
    port = _free_port()
    mp.start_processes(_shard_rank, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    net = W.bp.synth.random_loopy(1500, 6000, 3, 0.1, seed=77)
    ora = O.Restatement().loopy(O.OracleGraph(net), 1e-3, 40)
    parts = [dict(np.load(tmp_path / f"shard{r}.npz")) for r in range(2)]
    b = np.concatenate([p["beliefs"] for p in parts])
    np.testing.assert_array_equal(b, ora["beliefs"][:, :3])
    for p in parts:
        np.testing.assert_array_equal(p["messages"], ora["latest"][p["edges"], :3])
        assert int(p["iterations"]) == ora["ret"] and int(p["executed"]) == ora["executed"]
