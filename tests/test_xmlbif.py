"""XMLBIF reader (no libxml2) and the py3 generator.  CPU only.

The reference's own XML check (src/bnf-xml-parser/main.c:33-40) asserts that
dog.xml and dog.bif give the same node and edge counts; the same is checked
here against the reference's BIF parser, plus the generator's output
contract.  The reference's XML parser itself needs libxml2, which is not
installed here, so graph construction from XML is pinned only through that
count check and the generator round trip."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as _O  # noqa: E402  (the checker: where the reference files lie)

BENCH = _O.reference_benchmark_files()


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
