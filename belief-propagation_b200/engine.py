"""Python front end of the device-resident engine (include/bp.h).

    g = BPGraph.from_network(net)          # upload + destination sort on the GPU
    g.set_beliefs(net.beliefs)
    g.init_messages()                      # init_previous_edge
    r = g.loopy(tol=1e-3, max_iterations=100)
    b = g.beliefs()                        # [V, S_max] numpy

Arrays may be numpy (host) or torch CUDA tensors (device pointers are passed
through without copies).  All work happens in lib/libbp.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N

_DELTA = {"auto": N.BP_DELTA_AUTO, "serial": N.BP_DELTA_SERIAL_F32, "f64": N.BP_DELTA_F64}
_SCHED = {"node": N.BP_SCHEDULE_NODE, "edge": N.BP_SCHEDULE_EDGE}


def _is_torch(a):
    return a is not None and not isinstance(a, np.ndarray) and hasattr(a, "data_ptr")


def _memory_of(*arrays):
    kinds = {("dev" if (_is_torch(a) and a.is_cuda) else "host") for a in arrays if a is not None}
    if len(kinds) > 1:
        raise ValueError("mix of host and device arrays")
    return N.BP_MEM_DEVICE if kinds == {"dev"} else N.BP_MEM_HOST


class BPGraph:
    """A graph resident in GPU memory (bp_graph)."""

    def __init__(self, num_nodes, src, dst, joint, num_states=None, uniform_states=0,
                 joint_row_stride=None, joint_edge_stride=None, dest_csr=None, stream=None, reorder=False):
        self.lib = N.load()
        V, E = int(num_nodes), int(len(src))
        if not _is_torch(src):
            src = np.ascontiguousarray(src, np.uint32)
            dst = np.ascontiguousarray(dst, np.uint32)
            joint = np.ascontiguousarray(joint, np.float32)
            if num_states is not None:
                num_states = np.ascontiguousarray(num_states, np.uint32)
        s_max = int(joint.shape[-1]) if joint.ndim == 3 else int(uniform_states)
        d = N.GraphDesc()
        d.num_nodes, d.num_edges = V, E
        d.uniform_states = int(uniform_states)
        d.node_num_states = N.ptr(num_states)
        d.edge_src, d.edge_dst, d.edge_joint = N.ptr(src), N.ptr(dst), N.ptr(joint)
        d.joint_row_stride = int(joint_row_stride or s_max)
        d.joint_edge_stride = int(joint_edge_stride or s_max * s_max)
        if dest_csr is not None:
            d.dest_node_list, d.dest_edge_list = N.ptr(dest_csr[0]), N.ptr(dest_csr[1])
        d.memory = _memory_of(src, dst, joint, num_states)
        d.flags = N.BP_GRAPH_REORDER_BY_OUT_DEGREE if reorder else 0
        self._keep = (src, dst, joint, num_states)
        h = C.c_void_p()
        N.check(self.lib.bp_graph_create(C.byref(h), C.byref(d), stream))
        self.h = h
        self._keep = None
        V_, E_, ms, uni = (C.c_uint32() for _ in range(4))
        N.check(self.lib.bp_graph_info(h, C.byref(V_), C.byref(E_), C.byref(ms), C.byref(uni)))
        self.V, self.E, self.ms, self.uniform = V_.value, E_.value, ms.value, uni.value

    @classmethod
    def from_network(cls, net, stream=None, with_beliefs=True, reorder=False):
        uni = net.uniform_states
        g = cls(net.V, net.src, net.dst, net.joint, None if uni else net.num_states, uni, stream=stream,
                reorder=reorder)
        if with_beliefs:
            g.set_beliefs(net.beliefs)
        return g

    def set_stream(self, stream):
        """Run this graph's later work on `stream` (a cudaStream_t as int);
        its pending work on the old stream is finished first."""
        N.check(self.lib.bp_set_stream(self.h, stream))

    def close(self):
        if getattr(self, "h", None):
            self.lib.bp_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state ----------------------------------------------------------
    def set_beliefs(self, b):
        if not _is_torch(b):
            b = np.ascontiguousarray(b, np.float32)
        ld = int(b.shape[1]) if b.ndim == 2 else self.ms
        N.check(self.lib.bp_set_beliefs(self.h, N.ptr(b), ld, _memory_of(b)))

    def beliefs(self, out=None, ld=None):
        ld = ld or self.ms
        if out is None:
            out = np.zeros((self.V, ld), np.float32)
        N.check(self.lib.bp_get_beliefs(self.h, N.ptr(out), out.shape[1], _memory_of(out)))
        return out

    def set_messages(self, slot, m):
        if not _is_torch(m):
            m = np.ascontiguousarray(m, np.float32)
        N.check(self.lib.bp_set_messages(self.h, int(slot), N.ptr(m), int(m.shape[1]), _memory_of(m)))

    def messages(self, slot=None, ld=None):
        if slot is None:
            slot = self.latest_slot
        ld = ld or self.ms
        out = np.zeros((self.E, ld), np.float32)
        N.check(self.lib.bp_get_messages(self.h, int(slot), N.ptr(out), ld, N.BP_MEM_HOST))
        return out

    @property
    def latest_slot(self):
        s = C.c_int()
        N.check(self.lib.bp_get_latest_slot(self.h, C.byref(s)))
        return s.value

    @latest_slot.setter
    def latest_slot(self, slot):
        N.check(self.lib.bp_set_latest_slot(self.h, int(slot)))

    def device_bytes(self):
        b = C.c_uint64()
        N.check(self.lib.bp_graph_device_bytes(self.h, C.byref(b)))
        return b.value

    def synchronize(self):
        N.check(self.lib.bp_synchronize(self.h))

    # ---- loopy -----------------------------------------------------------
    def init_messages(self):
        N.check(self.lib.bp_init_messages(self.h))

    def loopy(self, tol=1e-3, max_iterations=200, check_every=1, schedule="node", delta="auto",
              verbose=False, graph_chunk=0, kernel="auto"):
        o = N.LoopyOptions()
        self.lib.bp_loopy_default_options(C.byref(o))
        o.tolerance = float(tol)
        o.max_iterations = int(max_iterations)
        o.check_every = int(check_every)
        o.schedule = _SCHED[schedule]
        o.delta_mode = _DELTA[delta]
        o.verbose = int(bool(verbose))
        o.graph_chunk = int(graph_chunk)
        o.kernel_variant = {"auto": 0, "block": 1, "warp": 2, "staged": 3, "split": 4}[kernel]
        r = N.LoopyResult()
        N.check(self.lib.bp_loopy(self.h, C.byref(o), C.byref(r)))
        return r.as_dict()

    # ---- tree ------------------------------------------------------------
    def build_levels(self):
        lv = np.zeros(2 * max(self.V, 1), np.uint32)
        n = C.c_uint32(0)
        N.check(self.lib.bp_tree_build_levels(self.h, lv.ctypes.data, C.byref(n)))
        return lv[: 2 * self.V], n.value

    def set_levels(self, levels, num_levels):
        levels = np.ascontiguousarray(levels, np.uint32)
        N.check(self.lib.bp_tree_set_levels(self.h, levels.ctypes.data, int(num_levels)))

    def tree(self):
        r = N.TreeResult()
        N.check(self.lib.bp_tree(self.h, C.byref(r)))
        return {"num_levels": r.num_levels, "num_waves": r.num_waves, "elapsed_ms": r.elapsed_ms}

    def tree_start(self):
        N.check(self.lib.bp_tree_start(self.h))

    def tree_level(self, level):
        N.check(self.lib.bp_tree_level(self.h, int(level)))

    def tree_reset_visited(self):
        N.check(self.lib.bp_tree_reset_visited(self.h))

    def tree_marginalize(self):
        N.check(self.lib.bp_tree_marginalize(self.h))


class BPBatch:
    """Many independent networks solved together (bp_batch): one persistent
    launch per state count, each network with its own stopping rule."""

    def __init__(self, nets, stream=None):
        self.lib = N.load()
        self.nets = nets
        descs = (N.GraphDesc * len(nets))()
        keep = []
        for d, net in zip(descs, nets):
            S = net.uniform_states
            if S == 0:
                raise ValueError(f"{net.name}: batched networks need one state count per network")
            src = np.ascontiguousarray(net.src, np.uint32)
            dst = np.ascontiguousarray(net.dst, np.uint32)
            joint = np.ascontiguousarray(net.joint[:, :S, :S], np.float32)
            keep.append((src, dst, joint))
            d.num_nodes, d.num_edges, d.uniform_states = net.V, net.E, S
            d.edge_src, d.edge_dst, d.edge_joint = src.ctypes.data, dst.ctypes.data, joint.ctypes.data
            d.joint_row_stride, d.joint_edge_stride = S, S * S
            d.memory = N.BP_MEM_HOST
        h = C.c_void_p()
        N.check(self.lib.bp_batch_create(C.byref(h), len(nets), descs, stream))
        self.h = h
        n = len(nets)
        self.belief_off = np.zeros(n + 1, np.uint64)
        self.msg_off = np.zeros(n + 1, np.uint64)
        N.check(self.lib.bp_batch_layout(h, self.belief_off.ctypes.data, self.msg_off.ctypes.data))

    def close(self):
        if getattr(self, "h", None):
            self.lib.bp_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def pack_beliefs(self):
        out = np.zeros(int(self.belief_off[-1]), np.float32)
        for k, net in enumerate(self.nets):
            S = net.uniform_states
            a = int(self.belief_off[k])
            out[a:a + net.V * S] = net.beliefs[:, :S].ravel()
        return out

    def set_beliefs(self, flat=None):
        flat = self.pack_beliefs() if flat is None else flat
        mem = N.BP_MEM_DEVICE if (hasattr(flat, "is_cuda") and flat.is_cuda) else N.BP_MEM_HOST
        if mem == N.BP_MEM_HOST:
            flat = np.ascontiguousarray(flat, np.float32)
        N.check(self.lib.bp_batch_set_beliefs(self.h, N.ptr(flat), mem))

    def beliefs(self, k=None):
        flat = np.zeros(int(self.belief_off[-1]), np.float32)
        N.check(self.lib.bp_batch_get_beliefs(self.h, flat.ctypes.data, N.BP_MEM_HOST))
        if k is None:
            return flat
        net = self.nets[k]
        S = net.uniform_states
        a = int(self.belief_off[k])
        return flat[a:a + net.V * S].reshape(net.V, S)

    def messages(self, k=None):
        flat = np.zeros(max(int(self.msg_off[-1]), 1), np.float32)
        N.check(self.lib.bp_batch_get_messages(self.h, flat.ctypes.data, N.BP_MEM_HOST))
        if k is None:
            return flat
        net = self.nets[k]
        S = net.uniform_states
        a = int(self.msg_off[k])
        return flat[a:a + net.E * S].reshape(net.E, S)

    def options(self, tol=1e-4, max_iterations=200, delta="f64", block_threads=0, init=True):
        o = N.BatchOptions()
        self.lib.bp_batch_default_options(C.byref(o))
        o.tolerance, o.max_iterations = float(tol), int(max_iterations)
        o.delta_mode = _DELTA[delta]
        o.block_threads, o.init_messages = int(block_threads), int(bool(init))
        return o

    def autotune(self, **kw):
        N.check(self.lib.bp_batch_autotune(self.h, C.byref(self.options(**kw))))
        return self.block_threads()

    def groups(self):
        """The launch groups: state count, size bound (0 = the larger
        networks), threads per block and blocks in flight, launch order."""
        n = C.c_uint32(64)
        st, vm, bl, gr = (np.zeros(64, np.uint32) for _ in range(4))
        N.check(self.lib.bp_batch_get_groups(self.h, st.ctypes.data, vm.ctypes.data, bl.ctypes.data, gr.ctypes.data,
                                             C.byref(n)))
        return [{"states": int(st[i]), "max_nodes": int(vm[i]), "block": int(bl[i]), "grid": int(gr[i])}
                for i in range(min(n.value, 64))]

    def block_threads(self):
        """Threads per block by group: "S=<states>" for the larger networks
        of a state count, "S=<states>,V<=<bound>" for its small ones."""
        return {(f"S={g['states']}" + (f",V<={g['max_nodes']}" if g["max_nodes"] else "")): g["block"]
                for g in self.groups()}

    def loopy(self, **kw):
        r = N.BatchResult()
        N.check(self.lib.bp_batch_loopy(self.h, C.byref(self.options(**kw)), C.byref(r)))
        return r.as_dict()

    def results(self):
        n = len(self.nets)
        it = np.zeros(n, np.uint32)
        ex = np.zeros(n, np.uint32)
        cv = np.zeros(n, np.int32)
        dl = np.zeros(n, np.float32)
        N.check(self.lib.bp_batch_network_results(self.h, it.ctypes.data, ex.ctypes.data, cv.ctypes.data,
                                                  dl.ctypes.data))
        return dict(iterations=it, executed=ex, converged=cv, delta=dl)
