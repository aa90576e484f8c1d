"""Loopy BP split over ranks by destination-node ranges (one process per GPU).

Each rank owns the destination nodes [begin, end) of an equal split and holds
only their in-edges: a bp_graph of all V nodes whose edges are the network's
edges into its range, in edge order.  Per iteration of loopy_propagate_until
(graph.c:1278-1324) a rank

  1. runs the iteration for its nodes (bp_flood_range): their incoming
     messages from every node's send buffer Q_t, their beliefs, and their
     next send buffers Q_{t+1};
  2. exchanges send buffers: an all-gather of the ranks' Q_{t+1} slices gives
     every rank the full Q_{t+1} (the one data exchange of the schedule);
  3. sums the ranks' fp64 |diff| partials in rank order (an all-gather of one
     double per rank) and applies the reference's stopping rule to the sum,
     so every rank takes the same decision.

Messages, beliefs and iteration counts equal the single-GPU node schedule's
bit for bit (tests/test_multirank.py checks the partition and exchange on
2 gloo ranks against the oracle; tests/test_gpu_sharded.py runs the CUDA
kernels as 2 ranks in one process).

The compute of a rank is an `engine` object, so the same driver runs over
the CUDA library (RangeEngine, the product) or, in the CPU tests, over a
checker; the exchange is a `comm` object (torch.distributed, or in-process).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N


def node_ranges(V, world):
    """Equal node ranges (the last one shorter): [(begin, end)] per rank."""
    chunk = (V + world - 1) // world if world else V
    return [(min(r * chunk, V), min((r + 1) * chunk, V)) for r in range(world)], chunk


def shard_edges(net, begin, end):
    """Edge ids of the network's edges into [begin, end), in edge order."""
    return np.nonzero((net.dst >= begin) & (net.dst < end))[0]


class RangeEngine:
    """One rank's node range on the GPU (bp_send_buffers_range /
    bp_flood_range over a bp_graph of the range's in-edges)."""

    def __init__(self, net, begin, end, chunk, world, device="cuda", stream=None):
        import torch
        from .engine import BPGraph
        self.torch = torch
        self.lib = N.load()
        self.begin, self.end = begin, end
        eids = shard_edges(net, begin, end)
        self.eids = eids
        S = int(net.s_max)
        self.S = S
        uni = net.uniform_states
        # the library's kernels and torch's exchange on one stream
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        self.g = BPGraph(net.V, net.src[eids], net.dst[eids], net.joint[eids],
                         None if uni else net.num_states, uni, stream=stream)
        # send buffers padded to world * chunk nodes, so every rank's slice
        # has the same size for the all-gather
        self.q = [torch.zeros((world * chunk, S), dtype=torch.float32, device=device) for _ in range(2)]
        self.delta = torch.zeros(1, dtype=torch.float64, device=device)
        self.stream = stream

    def reset(self, beliefs):
        self.g.set_beliefs(beliefs)
        self.g.latest_slot = 1
        self.g.init_messages()

    def send_buffers(self, k):
        N.check(self.lib.bp_send_buffers_range(self.g.h, self.begin, self.end, C.c_void_p(self.q[k].data_ptr()),
                                               self._stream()))

    def iterate(self, k_in, k_out):
        N.check(self.lib.bp_flood_range(self.g.h, self.begin, self.end, C.c_void_p(self.q[k_in].data_ptr()),
                                        C.c_void_p(self.q[k_out].data_ptr()), C.c_void_p(self.delta.data_ptr()),
                                        self._stream()))
        return self.delta

    def _stream(self):
        return C.c_void_p(self.stream) if self.stream else None

    def synchronize(self):
        self.g.synchronize()

    def beliefs(self):
        return self.g.beliefs()[self.begin:self.end]

    def messages(self):
        """(edge ids, latest messages of those edges)."""
        return self.eids, self.g.messages(self.g.latest_slot)

    def close(self):
        self.g.close()


class TorchComm:
    """The exchange over torch.distributed (NCCL on GPUs, gloo on CPUs): this
    process drives one rank's engine."""

    def __init__(self, dist, rank, chunk, group=None):
        self.dist, self.rank, self.chunk, self.group = dist, rank, chunk, group

    def exchange(self, engines, k):
        """Every rank's slice of send-buffer array k to every rank."""
        (e,) = engines
        full, chunk = e.q[k], self.chunk
        world = self.dist.get_world_size(self.group)
        parts = [full[r * chunk:(r + 1) * chunk] for r in range(world)]
        mine = parts[self.rank].clone()
        self.dist.all_gather(parts, mine, group=self.group)

    def deltas(self, engines, parts):
        """Every rank's fp64 |diff| partial, in rank order."""
        import torch
        (x,) = parts
        world = self.dist.get_world_size(self.group)
        out = [torch.zeros_like(x) for _ in range(world)]
        self.dist.all_gather(out, x, group=self.group)
        return [float(t.item()) for t in out]


class LocalComm:
    """All ranks' engines in this process (one GPU, or a check): the exchange
    copies each engine's slice into the others' send buffers."""

    def __init__(self, chunk):
        self.chunk = chunk

    def exchange(self, engines, k):
        c = self.chunk
        for r, src in enumerate(engines):
            for dst in engines:
                if dst is not src:
                    dst.q[k][r * c:(r + 1) * c] = src.q[k][r * c:(r + 1) * c]

    def deltas(self, engines, parts):
        return [float(p.item()) for p in parts]


def sharded_loopy(engines, comm, beliefs, tol, max_iterations, verbose=False):
    """loopy_propagate_until (graph.c:1278-1324) split over ranks: `engines`
    are the ranks this process drives (one under torch.distributed, all of
    them with LocalComm).  The stopping rule is the reference's, on the fp64
    sum of the ranks' partials in rank order (BP_DELTA_F64's rule).  Returns
    the reference's return value, the iterations executed and the last two
    deltas."""
    for e in engines:
        e.reset(beliefs)
    cur = 0
    for e in engines:
        e.send_buffers(cur)
    comm.exchange(engines, cur)
    delta, prev = 0.0, -1.0
    i = 0
    executed = 0
    while i < max_iterations:
        parts = [e.iterate(cur, cur ^ 1) for e in engines]
        cur ^= 1
        comm.exchange(engines, cur)
        executed += 1
        delta = 0.0
        for p in comm.deltas(engines, parts):
            delta += p
        if delta < tol or abs(delta - prev) < tol:
            break
        if i < max_iterations - 1:
            prev = delta
        i += 1
    if i == max_iterations and verbose:
        print(f"No Convergence: previous: {prev:f} vs current: {delta:f}")
    return dict(iterations=i, executed=executed, delta=delta, previous_delta=prev)
