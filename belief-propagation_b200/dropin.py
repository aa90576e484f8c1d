"""The reference's C graph API (include/graph.h) driven from Python.

CGraph builds a struct graph through the same calls the reference's parsers
and drivers make (create_graph, graph_add_node, graph_set_node_state,
graph_add_edge, set_up_*_nodes_to_edges) and exposes the struct's fields as
numpy views, so code ported from the reference's drivers reads the same
fields it always did.  The propagate calls run on the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native as N

MS = N.MAX_STATES


class CGraph:
    def __init__(self, net, set_up=True, total_edges=None):
        self.lib = N.load()
        L = self.lib
        self.V, self.E = net.V, net.E
        self.g = L.create_graph(net.V, total_edges if total_edges is not None else net.E)
        b, j = net.padded()
        for v in range(net.V):
            s = int(net.num_states[v])
            L.graph_add_node(self.g, s, f"n{v}".encode())
        for v in range(net.V):
            s = int(net.num_states[v])
            row = np.ascontiguousarray(b[v], np.float32)
            L.graph_set_node_state(self.g, v, s, row.ctypes.data)
        for e in range(net.E):
            s, d = int(net.src[e]), int(net.dst[e])
            t = np.ascontiguousarray(j[e], np.float32)
            L.graph_add_edge(self.g, s, d, int(net.num_states[s]), int(net.num_states[d]), t.ctypes.data)
        if set_up:
            L.set_up_src_nodes_to_edges(self.g)
            L.set_up_dest_nodes_to_edges(self.g)

    @property
    def struct(self):
        return self.g.contents

    def _view(self, p, n, dtype=np.float32):
        return np.ctypeslib.as_array(p, shape=(n,)).view(dtype)

    def beliefs(self):
        return self._view(self.struct.node_states, self.V * MS).reshape(self.V, MS).copy()

    def messages(self, which):
        """which: 'edges_messages', 'last_edges_messages', 'previous', 'current'."""
        s = self.struct
        if which == "previous":
            p = s.previous_edge_messages.contents
        elif which == "current":
            p = s.current_edge_messages.contents
        else:
            p = getattr(s, which)
        return self._view(p, max(self.E, 1) * MS)[: self.E * MS].reshape(self.E, MS).copy()

    def levels(self):
        s = self.struct
        arr = self._view(s.levels_to_nodes, 2 * self.V, np.uint32).copy() if self.V else np.zeros(0, np.uint32)
        return arr, int(s.num_levels)

    # ---- the reference's entry points
    def init_previous_edge(self):
        self.lib.init_previous_edge(self.g)

    def loopy_propagate_until(self, tol, max_it):
        return int(self.lib.loopy_propagate_until(self.g, C.c_float(tol), int(max_it)))

    def loopy_propagate_until_edge(self, tol, max_it):
        return int(self.lib.loopy_propagate_until_edge(self.g, C.c_float(tol), int(max_it)))

    def loopy_progagate_until_acc(self, tol, max_it):
        return int(self.lib.loopy_progagate_until_acc(self.g, C.c_float(tol), int(max_it)))

    def loopy_progagate_until_edge_acc(self, tol, max_it):
        return int(self.lib.loopy_progagate_until_edge_acc(self.g, C.c_float(tol), int(max_it)))

    def loopy_propagate_one_iteration(self):
        self.lib.loopy_propagate_one_iteration(self.g)

    def init_levels_to_nodes(self):
        self.lib.init_levels_to_nodes(self.g)

    def tree_sequence(self):
        """c_benchmark/main.c:224-236"""
        L, g = self.lib, self.g
        L.init_levels_to_nodes(g)
        L.propagate_using_levels_start(g)
        n = int(self.struct.num_levels)
        for i in range(1, n - 1):
            L.propagate_using_levels(g, i)
        L.reset_visited(g)
        for i in range(n - 1, 0, -1):
            L.propagate_using_levels(g, i)
        L.marginalize(g)

    def set_sync_mode(self, mode):
        N.check(self.lib.bp_set_sync_mode(self.g, int(mode)))

    def sync_host(self):
        N.check(self.lib.bp_sync_host(self.g))

    def calculate_diameter(self):
        self.lib.calculate_diameter(self.g)
        return int(self.struct.diameter)

    def close(self):
        if self.g:
            self.lib.graph_destroy(self.g)
            self.g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
