"""Differentiable T-step unrolled loopy BP (bp_unrolled in include/bp.h)
behind torch.autograd.Function.

    bp = UnrolledBP(num_nodes, src, dst, edge_table, states=4, iterations=30)
    log_beliefs = bp(log_unary, log_pair)   # [V, S], differentiable
    loss = nll_loss(log_beliefs, labels)     # cross-entropy (fused)
    loss.backward()                          # log_unary.grad, log_pair.grad

edge_table[e] names the shared table edge e uses (bit 0x80: transposed).
The forward is the reference's update (beliefs compound across iterations,
graph.c:1010, :1157), run in the log domain; the backward is a hand-written
adjoint kernel with state checkpoints every `checkpoint_every` iterations
recomputed per segment.
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
        if grad_b.data_ptr() % 16:
            grad_b = grad_b.clone()
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
        def fresh(t):  # contiguous and 16-byte aligned (views with an offset are copied)
            t = t.contiguous()
            return t if t.data_ptr() % 16 == 0 else t.clone()
        return _UnrolledFn.apply(fresh(log_unary), fresh(log_pair), self)

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


class _NLLFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, log_beliefs, labels, scratch):
        lib = N.load()
        V, S = log_beliefs.shape
        loss = torch.empty((), device=log_beliefs.device, dtype=torch.float32)
        st = torch.cuda.current_stream().cuda_stream
        N.check(lib.bp_nll_f32(log_beliefs.data_ptr(), labels.data_ptr(), V, S, scratch.data_ptr(),
                               loss.data_ptr(), st))
        ctx.save_for_backward(labels)
        ctx.VS = (V, S)
        return loss

    @staticmethod
    def backward(ctx, g):
        (labels,) = ctx.saved_tensors
        V, S = ctx.VS
        g = g.contiguous().float()
        grad = torch.empty((V, S), device=g.device, dtype=torch.float32)
        N.check(N.load().bp_nll_grad_f32(labels.data_ptr(), V, S, g.data_ptr(), grad.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream))
        return grad, None, None


_nll_scratch = {}


def nll_loss(log_beliefs, labels):
    """Cross-entropy of log-beliefs [V, S] against int64 labels [V]: the value
    of torch.nn.functional.nll_loss(log_beliefs, labels) (mean over nodes),
    in one launch forward and one backward."""
    if log_beliefs.dtype != torch.float32 or labels.dtype != torch.int64:
        raise TypeError("float32 log-beliefs and int64 labels")
    dev = log_beliefs.device
    if dev not in _nll_scratch:
        _nll_scratch[dev] = torch.zeros(297, device=dev, dtype=torch.float64)
    return _NLLFn.apply(log_beliefs.contiguous(), labels.contiguous(), _nll_scratch[dev])


def grid_tables(side):
    """Edges of a side x side 4-neighbour grid (synth.grid_edges order) and
    their table ids: forward edges use table 0, reverse edges its transpose."""
    from .synth import grid_edges
    src, dst, fwd = grid_edges(side)
    tab = np.where(fwd, 0, 0x80).astype(np.uint8)
    return src, dst, tab


def torch_unrolled(log_unary, log_pair, src, dst, edge_table, iterations):
    """Pure-torch unrolled reference of the same update (autograd through
    every step), any dtype, log domain; returns log-beliefs."""
    V, S = log_unary.shape
    dev = log_unary.device
    src = torch.as_tensor(np.asarray(src, np.int64), device=dev)
    dst = torch.as_tensor(np.asarray(dst, np.int64), device=dev)
    tab = np.asarray(edge_table)
    tid = torch.as_tensor((tab & 0x7F).astype(np.int64), device=dev)
    tr = torch.as_tensor((tab & 0x80) != 0, device=dev)
    L = log_pair[tid]
    L = torch.where(tr[:, None, None], L.transpose(1, 2), L)

    def lmsg(x):
        r = torch.logsumexp(L + x[src][:, None, :], dim=2)
        return r - torch.logsumexp(r, dim=1, keepdim=True)

    def sum_in(lm):
        return torch.zeros(V, S, dtype=lm.dtype, device=dev).index_add(0, dst, lm)

    lb = torch.log_softmax(log_unary, dim=1)
    lq = lb + sum_in(lmsg(lb))
    for _ in range(iterations):
        lp = sum_in(lmsg(lq))
        a = lb + lp
        lb = a - torch.logsumexp(a, dim=1, keepdim=True)
        lq = lb + lp
    return lb
