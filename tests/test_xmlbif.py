"""XMLBIF readers (no libxml2) and the py3 generator.  CPU only.

parse_xml_file (csrc/xmlbif.c, exported by libbp.so) is the drop-in for the
reference's src/bnf-xml-parser/xml-expression.c:441-466; read_xmlbif
(xmlbif.py) restates the same construction in Python.  The reference's XML
parser needs libxml2, which is not installed here, so it cannot run.  The
readers are pinned instead through the reference's own BIF parser: dog.xml
and dog.bif describe the same network (the reference's XML check,
src/bnf-xml-parser/main.c:33-40, asserts equal counts), and the C reader's
graph of dog.xml equals the reference parser's graph of dog.bif node for
node and edge for edge by name -- state counts, observed flags, priors and
every joint table bit for bit.  The two readers agree on every bundled
XMLBIF file, and the reference's c_benchmark/main.c links against libbp.so
with the C reader."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as _O  # noqa: E402  (the checker: where the reference files lie)

BENCH = _O.reference_benchmark_files()


def _graph_fields(g):
    from belief_propagation_b200 import native as N
    a = C.cast(g, C.POINTER(N.StructGraph)).contents
    V, E = a.current_num_vertices, a.current_num_edges
    u = lambda p, n: np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0)
    b8 = lambda p, n: np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(n,)).copy()
    names = b8(a.node_names, V * 50).reshape(V, 50)
    return dict(V=V, E=E, src=u(a.edges_src_index, E), dst=u(a.edges_dest_index, E), x=u(a.edges_x_dim, E),
                y=u(a.edges_y_dim, E), nv=u(a.node_num_vars, V), states=u(a.node_states, V * 10).reshape(V, 10),
                joint=u(a.edges_joint_probabilities, E * 100).reshape(E, 10, 10), obs=b8(a.observed_nodes, V),
                names=[bytes(r).split(b"\0")[0].decode() for r in names])


def _by_name(f):
    nodes = {f["names"][v]: (int(f["nv"][v]), int(f["obs"][v]), f["states"][v, : f["nv"][v]].tobytes())
             for v in range(f["V"])}
    edges = {}
    for e in range(f["E"]):
        key = (f["names"][f["src"][e]], f["names"][f["dst"][e]])
        edges.setdefault(key, []).append(f["joint"][e, : f["x"][e], : f["y"][e]].tobytes())
    return nodes, edges


def _c_reader():
    from belief_propagation_b200 import native as N
    lib = N.load()
    lib.parse_xml_file.restype = C.c_void_p
    lib.parse_xml_file.argtypes = [C.c_char_p]
    lib.graph_destroy.argtypes = [C.c_void_p]
    return lib


def test_c_xml_reader_dog_equals_reference_bif_parser(bp):
    """libbp.so's parse_xml_file on dog.xml against the reference's own BIF
    parser (compiled from its sources, oracle/_ref/libref_bif.so) on
    dog.bif: the same nodes (state counts, observed flags, priors) and the
    same edges with the same joint tables, matched by node name; the two
    files list the nodes in different orders."""
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libref_bif.so")
    if not (os.path.exists(os.path.join(BENCH, "dog.xml")) and os.path.exists(ref_so)):
        pytest.skip("reference benchmark files or the reference BIF parser not available here")
    lib = _c_reader()
    ref = C.CDLL(ref_so)
    ref.refbif_load.restype = C.c_void_p
    ref.refbif_load.argtypes = [C.c_char_p]
    ref.graph_destroy.argtypes = [C.c_void_p]
    gx = lib.parse_xml_file(os.path.join(BENCH, "dog.xml").encode())
    gb = ref.refbif_load(os.path.join(BENCH, "dog.bif").encode())
    x, b = _graph_fields(gx), _graph_fields(gb)
    assert (x["V"], x["E"]) == (b["V"], b["E"])
    nx, ex = _by_name(x)
    nb, eb = _by_name(b)
    assert nx == nb
    assert ex == eb
    lib.graph_destroy(gx)
    ref.graph_destroy(gb)


@pytest.mark.parametrize("rel", ["dog.xml"] + [f"xml/bf_{n}_{2 * n}_{k}.xml" for n in (1000, 2000, 5000)
                                               for k in (1, 2, 3)])
def test_c_xml_reader_matches_python_reader(bp, rel):
    """parse_xml_file (C) and read_xmlbif (Python) build the same graph from
    every bundled XMLBIF file: node order, state counts, priors, observed
    flags, edge order and joint tables, bit for bit."""
    from belief_propagation_b200.xmlbif import read_xmlbif
    path = os.path.join(BENCH, rel)
    if not os.path.exists(path):
        pytest.skip("reference benchmark file not available here")
    lib = _c_reader()
    g = lib.parse_xml_file(path.encode())
    f = _graph_fields(g)
    n = read_xmlbif(path)
    S = n.s_max
    assert (f["V"], f["E"]) == (n.V, n.E)
    np.testing.assert_array_equal(f["nv"], n.num_states)
    np.testing.assert_array_equal(f["obs"], n.observed)
    np.testing.assert_array_equal(f["src"], n.src)
    np.testing.assert_array_equal(f["dst"], n.dst)
    np.testing.assert_array_equal(f["states"][:, :S], n.beliefs[:, :S])
    np.testing.assert_array_equal(f["joint"][:, :S, :S], n.joint[:, :S, :S])
    assert f["names"] == n.meta["names"]
    lib.graph_destroy(g)


def test_reference_c_benchmark_links_against_libbp():
    """The reference's c_benchmark/main.c -- its BIF and XML drivers,
    run_tests_with_xml_file included -- links against libbp.so with no
    libxml2: parse_xml_file and the graph API resolve to this library."""
    exe = os.path.join(ROOT, "oracle", "_ref", "c_benchmark_on_bp")
    if not os.path.exists(exe):
        pytest.skip("drop-in link check not built here (needs the reference sources)")
    out = subprocess.run(["nm", "-D", "--undefined-only", exe], capture_output=True, text=True).stdout
    for sym in ("parse_xml_file", "create_graph", "loopy_propagate_until", "init_levels_to_nodes"):
        assert sym in out, sym
    deps = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert "libbp.so" in deps and "libxml2" not in deps


def test_dog_xml_matches_dog_bif_counts(bp):
    from belief_propagation_b200.xmlbif import read_xmlbif
    if not os.path.exists(os.path.join(BENCH, "dog.xml")):
        pytest.skip("reference benchmark files not available here")
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_bif.so")):
        pytest.skip("reference BIF parser not built here")
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as M
    x = read_xmlbif(os.path.join(BENCH, "dog.xml"))
    b = M.bif_network(os.path.join(BENCH, "dog.bif"))
    assert (x.V, x.E) == (b.V, b.E)
    assert sorted(x.num_states.tolist()) == sorted(b.num_states.tolist())
    assert int(x.observed.sum()) == int(b.observed.sum())


@pytest.mark.parametrize("name", ["bf_1000_2000_1.xml", "bf_2000_4000_2.xml"])
def test_bundled_xml_networks_parse(bp, name):
    from belief_propagation_b200.xmlbif import read_xmlbif
    path = os.path.join(BENCH, "xml", name)
    if not os.path.exists(path):
        pytest.skip("reference benchmark files not available here")
    n = read_xmlbif(path)
    nodes = int(name.split("_")[1])
    assert n.V == nodes
    assert set(np.unique(n.num_states).tolist()) == {2}
    # each arc adds child<-parent plus parent<-child unless the parent is observed
    np.testing.assert_allclose(n.joint[:, :2, :2].sum(axis=0).sum(), n.joint.sum())
    assert n.E >= nodes - 1


def test_generator_round_trip(bp, tmp_path):
    from belief_propagation_b200.xmlbif import read_xmlbif
    out = tmp_path / "net.xml"
    r = subprocess.run([sys.executable, os.path.join(ROOT, "generate_belief_network.py"), "--nodes", "300",
                        "--arcs", "600", "--seed", "4", "--file", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n = read_xmlbif(str(out))
    assert n.V == 300
    assert int(n.observed.sum()) == int(0.3 * 300)
    # arcs = definitions with GIVEN; edges = 2 * arcs - arcs whose parent is observed
    fwd = n.src < n.dst
    assert fwd.sum() + (~fwd).sum() == n.E
    assert 600 <= n.E <= 1200
    # single-parent CPTs: the marginalised table of a parent->child edge holds
    # P(child state i | parent state j) at [i][j] (the reference parser's
    # indexing, xml-expression.c:381-395), so it sums to 1 over i
    rows = n.joint[fwd][:, :2, :2].sum(axis=1)
    np.testing.assert_allclose(rows, 1.0, rtol=1e-5)


def test_generator_rejects_bad_arguments(tmp_path):
    r = subprocess.run([sys.executable, os.path.join(ROOT, "generate_belief_network.py"), "--nodes", "10",
                        "--arcs", "5", "--file", str(tmp_path / "x.xml")], capture_output=True, text=True)
    assert r.returncode != 0
