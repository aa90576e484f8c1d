"""Python driver for the parity checker.  TEST INFRASTRUCTURE ONLY.

Two checkers, both on the reference's host layout (beliefs [V,10], joint
[E,10,10], messages [E,10], edge-id order):

* :class:`Restatement` -- this project's C restatement (bp_oracle.c), float
  and double builds.  Always available (builds with gcc alone).
* :class:`Reference`   -- the reference's own src/graph/graph.c compiled
  unmodified (oracle/_ref/libref_graph.so, plus the OpenMP build), driven
  through its own API exactly as its benchmark drivers do.  Available where
  oracle/_ref was built (this container, and any box the built files were
  copied to).

Only tests/, the smoke check and the bench's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference's sources lie (read-only); the same REF variable the
# Makefile takes.  Only building the checker and writing fixtures read it.
REF = os.environ.get("REF", "/root/reference")
MS = 10
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(reference=True):
    """Build the restatement (and the reference checker when its sources exist)."""
    targets = ["restatement"]
    if reference and reference_sources_present():
        targets.append("reference")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REF}"] + targets, check=True)


def reference_sources_present():
    return os.path.isdir(os.path.join(REF, "src", "graph"))


def reference_benchmark_files():
    """The reference's bundled network files (BIF / XMLBIF)."""
    return os.path.join(REF, "src", "benchmark_files")


def restatement_path(openmp=False):
    return os.path.join(HERE, "_build", "libbp_oracle_omp.so" if openmp else "libbp_oracle.so")


def reference_path(openmp=False):
    return os.path.join(HERE, "_ref", "libref_graph_omp.so" if openmp else "libref_graph.so")


def reference_available(openmp=False):
    return os.path.exists(reference_path(openmp))


def padded_arrays(net):
    b, j = net.padded()
    return np.ascontiguousarray(b), np.ascontiguousarray(j)


class _BpoGraph(C.Structure):
    _fields_ = [("V", C.c_uint32), ("E", C.c_uint32),
                ("num_states", C.c_void_p), ("edge_src", C.c_void_p), ("edge_dst", C.c_void_p),
                ("joint", C.c_void_p), ("in_ptr", C.c_void_p), ("in_edges", C.c_void_p),
                ("out_ptr", C.c_void_p), ("out_edges", C.c_void_p)]


class _BpoInfo(C.Structure):
    _fields_ = [("executed", C.c_uint32), ("swapped_odd", C.c_int),
                ("delta", C.c_double), ("prev_delta", C.c_double)]


def csr(V, key):
    """Stable counting sort (the reference's CSR order): (ptr[V+1], order[E])."""
    key = np.asarray(key, np.int64)
    counts = np.bincount(key, minlength=V) if key.size else np.zeros(V, np.int64)
    ptr = np.zeros(V + 1, np.uint32)
    ptr[1:] = np.cumsum(counts)
    order = np.argsort(key, kind="stable").astype(np.uint32)
    return ptr, order


class OracleGraph:
    """A network held in the checker's layout."""

    def __init__(self, net):
        self.net = net
        self.V, self.E = net.V, net.E
        self.num_states = np.ascontiguousarray(net.num_states, np.uint32)
        self.src = np.ascontiguousarray(net.src, np.uint32)
        self.dst = np.ascontiguousarray(net.dst, np.uint32)
        self.beliefs, self.joint = padded_arrays(net)
        self.in_ptr, self.in_edges = csr(self.V, self.dst)
        self.out_ptr, self.out_edges = csr(self.V, self.src)
        g = _BpoGraph()
        g.V, g.E = self.V, self.E
        for name in ("num_states", "joint", "in_ptr", "in_edges", "out_ptr", "out_edges"):
            setattr(g, name, getattr(self, name).ctypes.data)
        g.edge_src = self.src.ctypes.data
        g.edge_dst = self.dst.ctypes.data
        self.c = g


class Restatement:
    """ctypes front end of bp_oracle.c."""

    def __init__(self, openmp=False):
        """openmp: the build whose node loops run on all host cores (same
        results; the delta stays a serial sum)."""
        if not os.path.exists(restatement_path(openmp)):
            build(reference=False)
        self.lib = C.CDLL(restatement_path(openmp))
        L = self.lib
        for sfx, fp, real in (("f32", _f32p, C.c_float), ("f64", _f64p, C.c_double)):
            f = getattr(L, f"bpo_init_messages_{sfx}")
            f.argtypes = [C.POINTER(_BpoGraph), fp, fp]
            f = getattr(L, f"bpo_loopy_{sfx}")
            f.argtypes = [C.POINTER(_BpoGraph), fp, fp, fp, real, C.c_uint32, C.c_uint32, C.c_int,
                          C.POINTER(_BpoInfo)]
            f.restype = C.c_uint32
            f = getattr(L, f"bpo_loopy_edge_{sfx}")
            f.argtypes = [C.POINTER(_BpoGraph), fp, fp, fp, real, C.c_uint32, C.c_int, C.c_int,
                          C.POINTER(_BpoInfo)]
            f.restype = C.c_uint32
            f = getattr(L, f"bpo_tree_{sfx}")
            f.argtypes = [C.POINTER(_BpoGraph), _u32p, C.c_uint32, fp, fp]
        L.bpo_levels.argtypes = [C.POINTER(_BpoGraph), _u32p, C.POINTER(C.c_uint32)]
        L.bpo_levels.restype = C.c_int

    def loopy(self, og, tol, max_it, dtype=np.float32, check_every=1, schedule="node",
              init=True, verbose=False, beliefs=None, msgs=None):
        """Run a loopy schedule from the network's beliefs.

        Returns dict(beliefs [V,10], latest [E,10], older [E,10], ret, executed, delta,
        prev_delta).  `latest` is what *previous_edge_messages points at on return."""
        sfx = "f32" if dtype == np.float32 else "f64"
        b = np.ascontiguousarray((og.beliefs if beliefs is None else beliefs).astype(dtype))
        mp = np.zeros((og.E, MS), dtype) if msgs is None else np.ascontiguousarray(msgs[0].astype(dtype))
        mc = np.zeros((og.E, MS), dtype) if msgs is None else np.ascontiguousarray(msgs[1].astype(dtype))
        if init:
            getattr(self.lib, f"bpo_init_messages_{sfx}")(C.byref(og.c), b, mp)
        info = _BpoInfo()
        if schedule == "node":
            ret = getattr(self.lib, f"bpo_loopy_{sfx}")(C.byref(og.c), b, mp, mc, tol, max_it,
                                                        check_every, int(verbose), C.byref(info))
            latest, older = (mc, mp) if info.swapped_odd else (mp, mc)
        else:
            acc = 1 if check_every > 1 else 0
            ret = getattr(self.lib, f"bpo_loopy_edge_{sfx}")(C.byref(og.c), b, mp, mc, tol, max_it,
                                                             acc, int(verbose), C.byref(info))
            latest, older = mp, mc
        return dict(beliefs=b, latest=latest, older=older, ret=int(ret), executed=info.executed,
                    delta=info.delta, prev_delta=info.prev_delta, prev_arr=mp, cur_arr=mc)

    def levels(self, og):
        lv = np.zeros(2 * max(og.V, 1), np.uint32)
        n = C.c_uint32(0)
        rc = self.lib.bpo_levels(C.byref(og.c), lv, C.byref(n))
        if rc != 0:
            raise ValueError("graph has nodes unreachable from the in-degree<=2 seed set")
        return lv[: 2 * og.V], int(n.value)

    def tree(self, og, dtype=np.float32):
        lv, nl = self.levels(og)
        sfx = "f32" if dtype == np.float32 else "f64"
        b = np.ascontiguousarray(og.beliefs.astype(dtype))
        m = np.zeros((og.E, MS), dtype)
        getattr(self.lib, f"bpo_tree_{sfx}")(C.byref(og.c), lv if og.V else np.zeros(1, np.uint32), nl, b, m)
        return dict(beliefs=b, messages=m, levels=lv, num_levels=nl)


class Reference:
    """The reference's own graph.c (unmodified), driven through its C API."""

    def __init__(self, openmp=False):
        path = reference_path(openmp)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.refshim_build.argtypes = [C.c_uint32, C.c_uint32, _u32p, _f32p, _u8p, _u32p, _u32p, _f32p, C.c_int]
        L.refshim_build.restype = C.c_void_p
        L.refshim_get_beliefs.argtypes = [C.c_void_p, _f32p]
        L.refshim_set_beliefs.argtypes = [C.c_void_p, _f32p]
        L.refshim_get_messages.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.refshim_set_messages.argtypes = [C.c_void_p, C.c_int, _f32p]
        L.refshim_previous_is_edges_messages.argtypes = [C.c_void_p]
        L.refshim_used_direct_fill.argtypes = [C.c_void_p]
        L.refshim_num_levels.argtypes = [C.c_void_p]
        L.refshim_num_levels.restype = C.c_uint
        L.refshim_get_levels.argtypes = [C.c_void_p, _u32p]
        L.refshim_tree.argtypes = [C.c_void_p]
        for name in ("init_previous_edge", "graph_destroy", "init_levels_to_nodes",
                     "propagate_using_levels_start", "reset_visited", "marginalize",
                     "loopy_propagate_one_iteration"):
            getattr(L, name).argtypes = [C.c_void_p]
        L.propagate_using_levels.argtypes = [C.c_void_p, C.c_uint]
        for name in ("loopy_propagate_until", "loopy_propagate_until_edge",
                     "loopy_progagate_until_acc", "loopy_progagate_until_edge_acc"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_float, C.c_uint]
            getattr(L, name).restype = C.c_uint

    def build_graph(self, net, force_direct=False):
        b, j = padded_arrays(net)
        g = self.lib.refshim_build(net.V, net.E, np.ascontiguousarray(net.num_states, np.uint32), b,
                                   np.ascontiguousarray(net.observed, np.uint8),
                                   np.ascontiguousarray(net.src, np.uint32),
                                   np.ascontiguousarray(net.dst, np.uint32), j, int(force_direct))
        return g

    def read(self, g, V, E):
        b = np.zeros((V, MS), np.float32)
        self.lib.refshim_get_beliefs(g, b)
        out = dict(beliefs=b)
        for k, name in ((0, "edges_messages"), (1, "last_edges_messages"), (2, "latest"), (3, "older")):
            m = np.zeros((E, MS), np.float32)
            self.lib.refshim_get_messages(g, k, m)
            out[name] = m
        return out

    def loopy(self, net, tol, max_it, variant="until", init=True, force_direct=False):
        g = self.build_graph(net, force_direct)
        try:
            if init:
                self.lib.init_previous_edge(g)
            fn = {"until": "loopy_propagate_until", "edge": "loopy_propagate_until_edge",
                  "acc": "loopy_progagate_until_acc", "edge_acc": "loopy_progagate_until_edge_acc"}[variant]
            ret = getattr(self.lib, fn)(g, C.c_float(tol), max_it)
            out = self.read(g, net.V, net.E)
            out["ret"] = int(ret)
            return out
        finally:
            self.lib.graph_destroy(g)

    def tree(self, net, force_direct=False):
        g = self.build_graph(net, force_direct)
        try:
            self.lib.refshim_tree(g)
            out = self.read(g, net.V, net.E)
            nl = self.lib.refshim_num_levels(g)
            lv = np.zeros(2 * net.V, np.uint32)
            self.lib.refshim_get_levels(g, lv)
            out["levels"] = lv
            out["num_levels"] = int(nl)
            return out
        finally:
            self.lib.graph_destroy(g)
