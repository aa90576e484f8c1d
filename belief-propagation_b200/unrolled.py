"""Differentiable T-step unrolled loopy BP (bp_unrolled in include/bp.h)
behind torch.autograd.Function.

    bp = UnrolledBP(num_nodes, src, dst, edge_table, states=4, iterations=30)
    beliefs = bp(log_unary, log_pair)       # [V, S], differentiable
    loss = torch.nn.functional.nll_loss(beliefs.log(), labels)
    loss.backward()                          # log_unary.grad, log_pair.grad

edge_table[e] names the shared table edge e uses (bit 0x80: transposed).
The forward is the reference's update (beliefs compound across iterations,
graph.c:1010, :1157); the backward is a hand-written adjoint kernel with
state checkpoints every `checkpoint_every` iterations recomputed per segment.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import native as N


class _UnrolledFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, log_unary, log_pair, engine):
        out = torch.empty_like(log_unary)
        engine._run(lambda h: engine.lib.bp_unrolled_forward(h, log_unary.data_ptr(), log_pair.data_ptr(),
                                                             out.data_ptr()))
        ctx.engine = engine
        ctx.shapes = (log_unary.shape, log_pair.shape)
        return out

    @staticmethod
    def backward(ctx, grad_b):
        eng = ctx.engine
        grad_b = grad_b.contiguous().float()
        gu = torch.empty(ctx.shapes[0], device=grad_b.device, dtype=torch.float32)
        gp = torch.empty(ctx.shapes[1], device=grad_b.device, dtype=torch.float32)
        eng._run(lambda h: eng.lib.bp_unrolled_backward(h, grad_b.data_ptr(), gu.data_ptr(), gp.data_ptr()))
        return gu, gp, None


class UnrolledBP:
    def __init__(self, num_nodes, src, dst, edge_table, states, iterations, checkpoint_every=5, num_tables=1):
        self.lib = N.load()
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        tab = np.ascontiguousarray(edge_table, np.uint8)
        self.V, self.S, self.T, self.K = int(num_nodes), int(states), int(iterations), int(num_tables)
        self.stream = torch.cuda.Stream()
        h = C.c_void_p()
        N.check(self.lib.bp_unrolled_create(C.byref(h), self.V, len(src), self.S, self.K, src.ctypes.data,
                                            dst.ctypes.data, tab.ctypes.data, self.T, int(checkpoint_every),
                                            C.c_void_p(self.stream.cuda_stream)))
        self.h = h

    def _run(self, call):
        cur = torch.cuda.current_stream()
        self.stream.wait_stream(cur)
        N.check(call(self.h))
        cur.wait_stream(self.stream)

    def __call__(self, log_unary, log_pair):
        if log_unary.dtype != torch.float32 or log_pair.dtype != torch.float32:
            raise TypeError("log-potentials must be float32 CUDA tensors")
        return _UnrolledFn.apply(log_unary.contiguous(), log_pair.contiguous(), self)

    def close(self):
        if getattr(self, "h", None):
            torch.cuda.synchronize()
            self.lib.bp_unrolled_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grid_tables(side):
    """Edges of a side x side 4-neighbour grid (synth.grid_edges order) and
    their table ids: forward edges use table 0, reverse edges its transpose."""
    from .synth import grid_edges
    src, dst, fwd = grid_edges(side)
    tab = np.where(fwd, 0, 0x80).astype(np.uint8)
    return src, dst, tab


def torch_unrolled(log_unary, log_pair, src, dst, edge_table, iterations):
    """Pure-torch unrolled reference of the same update (autograd through
    every step), any dtype; products over in-edges via index_add of logs."""
    V, S = log_unary.shape
    src = torch.as_tensor(np.asarray(src, np.int64), device=log_unary.device)
    dst = torch.as_tensor(np.asarray(dst, np.int64), device=log_unary.device)
    tab = np.asarray(edge_table)
    tid = torch.as_tensor((tab & 0x7F).astype(np.int64), device=log_unary.device)
    tr = torch.as_tensor((tab & 0x80) != 0, device=log_unary.device)
    E = torch.exp(log_pair)
    J = E[tid]
    J = torch.where(tr[:, None, None], J.transpose(1, 2), J)

    def send(x):
        r = torch.einsum("eij,ej->ei", J, x[src])
        return r / r.sum(1, keepdim=True)

    def prod_in(m):
        return torch.exp(torch.zeros(V, S, dtype=m.dtype, device=m.device).index_add(0, dst, torch.log(m)))

    b = torch.softmax(log_unary, dim=1)
    Q = b * prod_in(send(b))
    for _ in range(iterations):
        P = prod_in(send(Q))
        u = b * P
        b = u / u.sum(1, keepdim=True)
        Q = b * P
    return b
