"""CPU-only checks of the product's host side: the C-ABI library loads and
exports every declared symbol, the drop-in graph construction matches the
reference's struct graph field by field, the O(V+E) level lists match the
reference's O(V^2) ones, the reference's BIF parser builds identical graphs
inside libbp.so, and the synthetic generators keep their contracts.  No
propagate call is made here (they need a GPU)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
import oracle as O_  # the checker (conftest puts oracle/ on the path): where the reference files lie


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("#"))
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted({n for n in names if n not in ("sizeof",)})


def test_library_exports_every_declared_symbol(native):
    lib = native.load()
    missing = []
    headers = sorted(h for h in os.listdir(os.path.join(ROOT, "include")) if h.endswith(".h"))
    assert {"graph.h", "bp.h", "constants.h", "xml-expression.h"} <= set(headers)
    for header in headers:
        for name in _declared(header):
            try:
                getattr(lib, name)
            except AttributeError:
                missing.append(f"{header}:{name}")
    assert not missing, missing
    assert set(native.BP_SYMBOLS) <= set(_declared("bp.h"))
    assert set(native.GRAPH_SYMBOLS) <= set(_declared("graph.h"))


def test_library_is_sm100a_and_static_cudart(native):
    path = native.LIB_PATH
    blob = open(path, "rb").read()
    assert b"sm_100a" in blob
    out = os.popen(f"ldd {path}").read()
    assert "libcudart.so" not in out


def test_struct_graph_layout_matches_reference_header(native):
    """Field offsets of struct graph: the reference layout, plus one trailing
    pointer."""
    S = native.StructGraph
    assert S.total_num_vertices.offset == 0
    assert S.edges_src_index.offset == 24
    assert S.node_states.offset == 24 + 8 * 9
    assert S.bp_device.offset > S.edge_tables_created.offset


def test_errors_without_gpu_are_loud(native, synth):
    """Creating a device graph where there is no GPU fails with a status, not
    a silent fallback."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from belief_propagation_b200.engine import BPGraph
    net = synth.random_loopy(50, 100, 2, 0.1, seed=1)
    with pytest.raises(native.BPError) as e:
        BPGraph.from_network(net)
    assert e.value.status in (3, 5)


def _compare_struct_to_reference(cg, ref_lib, rg, V, E):
    s = cg.struct
    arr = lambda p, n, dt=np.uint32: np.ctypeslib.as_array(p, shape=(n,)).view(dt).copy()
    sp, se, dp, de = (np.zeros(V, np.uint32), np.zeros(E, np.uint32), np.zeros(V, np.uint32),
                      np.zeros(E, np.uint32))
    ref_lib.refshim_get_csr.argtypes = [C.c_void_p] * 5
    ref_lib.refshim_get_csr(rg, sp.ctypes.data, se.ctypes.data, dp.ctypes.data, de.ctypes.data)
    np.testing.assert_array_equal(arr(s.src_nodes_to_edges_node_list, V), sp)
    np.testing.assert_array_equal(arr(s.src_nodes_to_edges_edge_list, E), se)
    np.testing.assert_array_equal(arr(s.dest_nodes_to_edges_node_list, V), dp)
    np.testing.assert_array_equal(arr(s.dest_nodes_to_edges_edge_list, E), de)


def test_dropin_construction_and_levels_match_reference(native, synth, reference, O):
    from belief_propagation_b200.dropin import CGraph
    for net in (synth.random_tree(3000, (2,), 0.05, seed=2), synth.random_loopy(800, 2400, 3, 0.1, seed=3)):
        cg = CGraph(net)
        rg = reference.build_graph(net)
        try:
            _compare_struct_to_reference(cg, reference.lib, rg, net.V, net.E)
            reference.lib.init_levels_to_nodes(rg)
            nl_ref = reference.lib.refshim_num_levels(rg)
            lv_ref = np.zeros(2 * net.V, np.uint32)
            reference.lib.refshim_get_levels(rg, lv_ref)
            try:
                cg.init_levels_to_nodes()
            except Exception:
                raise
            lv, nl = cg.levels()
            assert nl == nl_ref
            np.testing.assert_array_equal(lv[:nl], lv_ref[:nl])
            np.testing.assert_array_equal(lv[net.V:], lv_ref[net.V:])
            assert cg.struct.max_degree == max(np.bincount(net.src, minlength=net.V))
        finally:
            reference.lib.graph_destroy(rg)
            cg.close()


def test_diameter_matches_reference(native, synth, reference):
    from belief_propagation_b200.dropin import CGraph
    reference.lib.calculate_diameter.argtypes = [C.c_void_p]
    for net in (synth.random_tree(60, (2,), 0.0, seed=9), synth.random_loopy(80, 200, 2, 0.0, seed=4)):
        cg = CGraph(net)
        rg = reference.build_graph(net)
        reference.lib.calculate_diameter(rg)
        d_ref = C.cast(rg, C.POINTER(native.StructGraph)).contents.diameter
        assert cg.calculate_diameter() == d_ref
        reference.lib.graph_destroy(rg)
        cg.close()


BIF = O_.reference_benchmark_files()


@pytest.mark.parametrize("rel", ["dog.bif", "small/asia.bif", "medium/alarm.bif", "medium/insurance.bif",
                                 "medium/water.bif", "large/hepar2.bif", "very_large/andes.bif"])
def test_reference_bif_parser_builds_same_graph_in_libbp(native, O, rel):
    """The reference's parser (its own objects, its own graph.h) linked against
    libbp.so builds the same struct graph as on the reference's graph.c."""
    on_bp = os.path.join(ROOT, "oracle", "_ref", "libbif_on_bp.so")
    on_ref = os.path.join(ROOT, "oracle", "_ref", "libref_bif.so")
    path = os.path.join(BIF, rel)
    if not (os.path.exists(on_bp) and os.path.exists(on_ref) and os.path.exists(path)):
        pytest.skip("reference parser or BIF files not available here")
    la, lb = C.CDLL(on_bp), C.CDLL(on_ref)
    for L in (la, lb):
        L.refbif_load.restype = C.c_void_p
        L.refbif_load.argtypes = [C.c_char_p]
    ga = C.cast(la.refbif_load(path.encode()), C.POINTER(native.StructGraph))
    gb = C.cast(lb.refbif_load(path.encode()), C.POINTER(native.StructGraph))
    a, b = ga.contents, gb.contents
    assert (a.current_num_vertices, a.current_num_edges) == (b.current_num_vertices, b.current_num_edges)
    V, E = a.current_num_vertices, a.current_num_edges
    u = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy()
    for f in ("edges_src_index", "edges_dest_index", "edges_x_dim", "edges_y_dim"):
        np.testing.assert_array_equal(u(getattr(a, f), E), u(getattr(b, f), E))
    np.testing.assert_array_equal(u(a.node_num_vars, V), u(b.node_num_vars, V))
    nv = u(a.node_num_vars, V)
    sa, sb = u(a.node_states, V * 10).reshape(V, 10), u(b.node_states, V * 10).reshape(V, 10)
    mask = np.arange(10)[None] < nv[:, None]
    np.testing.assert_array_equal(sa[mask], sb[mask])
    ja = u(a.edges_joint_probabilities, E * 100).reshape(E, 10, 10)
    jb = u(b.edges_joint_probabilities, E * 100).reshape(E, 10, 10)
    xd, yd = u(a.edges_x_dim, E), u(a.edges_y_dim, E)
    jm = (np.arange(10)[None, :, None] < xd[:, None, None]) & (np.arange(10)[None, None, :] < yd[:, None, None])
    np.testing.assert_array_equal(ja[jm], jb[jm])
    la.graph_destroy.argtypes = [C.c_void_p]
    lb.graph_destroy.argtypes = [C.c_void_p]
    la.graph_destroy(ga)
    lb.graph_destroy(gb)


def test_synth_random_loopy_contract(synth):
    net = synth.random_loopy(10000, 40000, 2, 0.10, seed=0)
    assert net.V == 10000 and net.E == 40000
    assert not np.any(net.src == net.dst)
    key = net.src.astype(np.int64) * net.V + net.dst
    assert len(np.unique(key)) == net.E
    np.testing.assert_allclose(net.joint.sum(axis=2), 1.0, rtol=1e-5)
    np.testing.assert_allclose(net.beliefs.sum(axis=1), 1.0, rtol=1e-5)
    assert net.observed.sum() == 1000


def test_synth_power_law_contract(synth):
    net = synth.power_law_loopy(1 << 16, 1 << 18, 2, 0.1, seed=1)
    deg = np.bincount(net.src, minlength=net.V)
    assert deg.min() >= 1 and deg.sum() == net.E
    assert abs(deg.mean() - 4.0) < 1e-9
    assert deg.max() > 100                       # heavy tail
    assert not np.any(net.src == net.dst)
    assert len(np.unique(net.src.astype(np.int64) * net.V + net.dst)) == net.E


def test_synth_tree_contract(synth):
    net = synth.random_tree(1000, (2, 3, 4, 8), 0.05, seed=1)
    assert net.E == 2 * (net.V - 1)
    assert set(np.unique(net.num_states)) <= {2, 3, 4, 8}
    par = net.src[0::2]
    assert np.all(par < net.dst[0::2])
    np.testing.assert_array_equal(net.joint[1::2], np.transpose(net.joint[0::2], (0, 2, 1)))


def test_bench_arguments_and_algorithmic_bytes(monkeypatch):
    """bench.py's documented defaults (the headline workload, N=1, W>=3, the
    e2e pipeline length, the batched delta) and the flooding kernel's
    algorithmic bytes: 44 B per edge + 28 B per node at 2 states, 3.42 GB for
    the 16.8M-node / 67.1M-edge graph."""
    import sys
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.gpus, a.impl, a.workload, a.iterations) == (1, "bp", "power_law", 100)
    assert a.warmup >= 3 and a.e2e_steps == 12 and a.batch_delta == "f64"
    assert (a.nodes, a.edges) == (1 << 24, 1 << 26)
    for d in ("serial", "f64"):
        monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "batched", "--batch-delta", d])
        assert bench.parse().batch_delta == d
    assert bench.flood_bytes_per_iteration(1, 1, 2) == 44 + 28
    assert abs(bench.flood_bytes_per_iteration(1 << 24, 1 << 26, 2) - 3.42e9) < 0.01e9
    assert a.configs == "all"


def test_bench_other_configs_collects_each_workload_line(monkeypatch):
    """The headline run's other_configs: one child `bench.py --workload W`
    per other workload, the fields of its JSON line kept, a failed child
    recorded as an error without failing the rest."""
    import json
    import subprocess
    import sys
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    calls = []

    def fake_run(cmd, **kw):
        w = cmd[cmd.index("--workload") + 1]
        calls.append((w, cmd[cmd.index("--warmup") + 1], kw["env"].get("RANK")))
        if w == "tree":
            return subprocess.CompletedProcess(cmd, 1, "", "boom")
        line = {"metric": w, "value": 1.5, "unit": "u", "clocks": {"sm_mhz": 1965}, "noise": 0}
        return subprocess.CompletedProcess(cmd, 0, "log line\n" + json.dumps(line) + "\n", "")

    monkeypatch.setattr(subprocess, "run", fake_run)
    monkeypatch.setenv("RANK", "0")
    out = bench.run_other_configs(a)
    assert [c[0] for c in calls] == list(bench.OTHER_WORKLOADS)
    assert all(int(c[1]) >= 3 and c[2] is None for c in calls)
    assert "boom" in out["tree"]["error"]
    assert out["batched"]["value"] == 1.5 and out["batched"]["clocks"] == {"sm_mhz": 1965}
    assert "noise" not in out["batched"] and "wall_s" in out["unrolled"]


def test_status_codes_and_thread_local_errors():
    """bp_status_string names every bp_status, argument errors come back as
    statuses before any device work, and bp_last_error is per thread."""
    import ctypes as C
    import threading
    from belief_propagation_b200 import native as N
    lib = N.load()
    names = [lib.bp_status_string(k) for k in range(9)]
    assert names[0] == b"ok" and len(set(names)) == 9 and all(names)
    assert lib.bp_status_string(99) == b"unknown status"
    assert lib.bp_version() >= 1
    dummy = (C.c_float * 4)()
    BP_ERR_INVALID, BP_ERR_SHAPE = 1, 2
    assert lib.bp_serial_sum_f32(None, C.c_uint64(5), C.addressof(dummy), 0, None) == BP_ERR_INVALID
    assert lib.bp_serial_sum_f32(C.addressof(dummy), C.c_uint64(4), C.addressof(dummy), 9, None) == BP_ERR_INVALID
    assert lib.bp_loopy(None, None, None) == BP_ERR_INVALID
    seen = {}

    def worker(name, call):
        seen[name] = (call(), lib.bp_last_error())

    t1 = threading.Thread(target=worker, args=("a", lambda: lib.bp_loopy(None, None, None)))
    t2 = threading.Thread(target=worker, args=("b", lambda: lib.bp_nll_f32(
        C.addressof(dummy), C.addressof(dummy), 0, 4, C.addressof(dummy), C.addressof(dummy), None)))
    t1.start(); t1.join(); t2.start(); t2.join()
    assert seen["a"] == (BP_ERR_INVALID, b"null argument")
    assert seen["b"][0] == BP_ERR_SHAPE and b"empty" in seen["b"][1]


@pytest.mark.parametrize("rel,V,E,ret", [("dog.bif", 5, 5, 6)])
def test_reference_parser_smoke_values(native, rel, V, E, ret):
    """The reference's own parser smoke run (bnf-parser/main.c:230-242: build,
    both CSRs, init_previous_edge, loopy_propagate_until(graph, 1e-3, 200)) on
    the serial reference build: dog, 5 nodes / 5 edges, returns 6."""
    on_ref = os.path.join(ROOT, "oracle", "_ref", "libref_bif.so")
    path = os.path.join(BIF, rel)
    if not (os.path.exists(on_ref) and os.path.exists(path)):
        pytest.skip("reference parser or BIF files not available here")
    L = C.CDLL(on_ref)
    L.refbif_load.restype = C.c_void_p
    L.refbif_load.argtypes = [C.c_char_p]
    for f in ("init_previous_edge", "set_up_src_nodes_to_edges", "set_up_dest_nodes_to_edges"):
        getattr(L, f).argtypes = [C.c_void_p]
    L.loopy_propagate_until.argtypes = [C.c_void_p, C.c_float, C.c_uint]
    L.loopy_propagate_until.restype = C.c_uint
    L.graph_destroy.argtypes = [C.c_void_p]
    g = L.refbif_load(path.encode())
    s = C.cast(g, C.POINTER(native.StructGraph)).contents
    assert (s.current_num_vertices, s.current_num_edges) == (V, E)
    L.set_up_src_nodes_to_edges(g)
    L.set_up_dest_nodes_to_edges(g)
    L.init_previous_edge(g)
    assert L.loopy_propagate_until(g, C.c_float(1e-3), 200) == ret
    L.graph_destroy(g)


def test_synth_batch_contract(synth):
    """Config 2's generator: node counts log-uniform in [32, 4096], edges
    U(2, 6) x nodes, one state count per network from {2, 3, 4, 8}, no
    self-loops or duplicate edges, normalised priors and tables."""
    nets = synth.batch_of_networks(count=64, seed=2)
    assert len(nets) == 64
    for n in nets:
        assert 32 <= n.V <= 4096 and 2 * n.V - 1 <= n.E <= 6 * n.V + 1
        assert len(set(np.asarray(n.num_states).tolist())) == 1 and int(n.num_states[0]) in (2, 3, 4, 8)
        assert not np.any(n.src == n.dst)
        assert len(np.unique(n.src.astype(np.int64) * n.V + n.dst)) == n.E
        np.testing.assert_allclose(n.beliefs[:, : n.s_max].sum(axis=1), 1.0, rtol=1e-5)
    sizes = np.log([n.V for n in nets])
    assert sizes.min() < np.log(128) and sizes.max() > np.log(1024)   # spread over the log range


def test_synth_grid_edges_contract(synth):
    """Configs 3-4's grid: side x side nodes, 4-neighbour, both directions
    (512 x 512 gives 1,046,528 directed edges), each forward edge followed by
    its reverse."""
    for side in (2, 7, 512):
        src, dst, fwd = synth.grid_edges(side)
        assert len(src) == 4 * side * (side - 1)
        np.testing.assert_array_equal(src[0::2], dst[1::2])
        np.testing.assert_array_equal(dst[0::2], src[1::2])
        assert fwd[0::2].all() and not fwd[1::2].any()
        d = np.abs(src.astype(np.int64) - dst.astype(np.int64))
        assert np.all((d == 1) | (d == side))
    assert len(synth.grid_edges(512)[0]) == 1_046_528
