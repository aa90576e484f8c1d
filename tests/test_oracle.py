"""The checker itself: the C restatement (oracle/bp_oracle.c) against the
reference's own graph.c compiled unmodified, and against exact answers.

CPU only.  Where the reference library is not built (a box without the
reference sources) the reference-pinned cases skip and the fixture-pinned
ones still run."""
import itertools

import numpy as np
import pytest

from conftest import load_golden
import golden_nets as GN


def _nets(synth):
    yield synth.random_loopy(2000, 8000, 2, 0.10, seed=11)
    yield synth.random_loopy(500, 3000, 3, 0.10, seed=12)
    yield synth.random_loopy(300, 1500, 4, 0.20, seed=13)
    yield synth.random_loopy(301, 1201, 8, 0.10, seed=14)   # odd E: the byte-copy quirk splits a float
    yield synth.random_loopy(200, 700, 10, 0.0, seed=15)


@pytest.mark.parametrize("variant,check,sched", [("until", 1, "node"), ("acc", 10, "node"),
                                                  ("edge", 1, "edge"), ("edge_acc", 10, "edge")])
def test_restatement_matches_reference_loopy(synth, restatement, reference, O, variant, check, sched):
    for net in _nets(synth):
        og = O.OracleGraph(net)
        for tol, max_it in ((1e-3, 60), (0.0, 25), (1e-1, 200)):
            a = restatement.loopy(og, tol, max_it, check_every=check, schedule=sched)
            b = reference.loopy(net, tol, max_it, variant=variant)
            assert a["ret"] == b["ret"], (net.name, variant, tol)
            np.testing.assert_array_equal(a["beliefs"], b["beliefs"])
            np.testing.assert_array_equal(a["prev_arr"], b["last_edges_messages"])
            np.testing.assert_array_equal(a["cur_arr"], b["edges_messages"])


def test_restatement_matches_reference_large_degree(synth, restatement, reference, O):
    """Nodes above MAX_DEGREE: the reference graph is filled directly."""
    net = synth.power_law_loopy(4000, 16000, 2, 0.1, seed=21)
    assert net.meta["max_out_degree"] > 20
    og = O.OracleGraph(net)
    a = restatement.loopy(og, 1e-3, 30)
    b = reference.loopy(net, 1e-3, 30)
    assert a["ret"] == b["ret"]
    np.testing.assert_array_equal(a["beliefs"], b["beliefs"])


def test_restatement_matches_reference_tree(synth, restatement, reference, O):
    for seed, n in ((1, 3000), (2, 500), (3, 50)):
        net = synth.random_tree(n, (2,), 0.05, seed=seed)
        og = O.OracleGraph(net)
        a = restatement.tree(og)
        b = reference.tree(net)
        V, nl = net.V, a["num_levels"]
        assert nl == b["num_levels"]
        np.testing.assert_array_equal(a["levels"][:nl], b["levels"][:nl])
        np.testing.assert_array_equal(a["levels"][V:], b["levels"][V:])
        np.testing.assert_array_equal(a["beliefs"], b["beliefs"])
        np.testing.assert_array_equal(a["messages"], b["edges_messages"])


def test_restatement_tree_on_loopy_graph(synth, restatement, reference, O):
    """Tree BP on a graph with cycles: exercises same-level sends (the
    visited order inside a level)."""
    net = synth.random_loopy(400, 1200, 2, 0.1, seed=5)
    og = O.OracleGraph(net)
    try:
        a = restatement.tree(og)
    except ValueError:
        pytest.skip("unreachable nodes for this seed")
    b = reference.tree(net)
    np.testing.assert_array_equal(a["beliefs"], b["beliefs"])
    np.testing.assert_array_equal(a["messages"], b["edges_messages"])


def test_known_answer_example(restatement, O, bp):
    """example-belief-propagation.c:72-107: tree BP marginals to 1e-4."""
    net = GN.example_network()
    a = restatement.tree(O.OracleGraph(net))
    b = a["beliefs"]
    expect = GN.EXAMPLE_MARGINALS
    np.testing.assert_allclose(b[:, :2], expect, atol=1e-4)


def test_golden_fixtures_against_restatement(restatement, O, bp):
    """Fixtures made by running the reference itself (tests/golden/make_golden.py)."""
    for name in ("loopy_random_10000_40000.npz", "example_4node.npz", "tree_random_2000.npz",
                 "loopy_random_s3_500.npz", "bif_asia.npz", "bif_cancer.npz", "bif_earthquake.npz",
                 "bif_sachs.npz"):
        fx = load_golden(name)
        net = GN.network_from_fixture(fx)
        og = O.OracleGraph(net)
        if "tree_beliefs" in fx:
            a = restatement.tree(og)
            S = fx["tree_beliefs"].shape[1]
            np.testing.assert_array_equal(a["beliefs"][:, :S], fx["tree_beliefs"])
            np.testing.assert_array_equal(a["messages"][:, :S], fx["tree_messages"])
        if "loopy_beliefs" in fx:
            tol, max_it = float(fx["loopy_tol"]), int(fx["loopy_max_it"])
            a = restatement.loopy(og, tol, max_it)
            assert a["ret"] == int(fx["loopy_ret"])
            S = fx["loopy_beliefs"].shape[1]
            np.testing.assert_array_equal(a["beliefs"][:, :S], fx["loopy_beliefs"])
            np.testing.assert_array_equal(a["latest"][:, :S], fx["loopy_latest"])


def _enumerate_marginals(net):
    """Exact marginals of the pairwise model prod_v prior_v(x_v) prod_e J_e[x_dst, x_src]
    over tree-shaped networks where each undirected pair carries J and J^T."""
    V = net.V
    S = [int(s) for s in net.num_states]
    pairs = {}
    for e in range(net.E):
        s, d = int(net.src[e]), int(net.dst[e])
        if (d, s) not in pairs:
            pairs[(s, d)] = net.joint[e]
    total = np.zeros((V, max(S)))
    for x in itertools.product(*[range(s) for s in S]):
        w = 1.0
        for v in range(V):
            w *= float(net.beliefs[v, x[v]])
        for (s, d), J in pairs.items():
            w *= float(J[x[d], x[s]])
        for v in range(V):
            total[v, x[v]] += w
    return total / total.sum(axis=1, keepdims=True)


def test_tree_bp_exact_on_chain_with_leaf_evidence(bp, restatement, O):
    """Tree BP equals exact enumeration when the only priors sit on the
    in-degree<=2 senders and every other node starts flat (the condition under
    which the reference's schedule is exact)."""
    net = GN.example_network()
    ex = _enumerate_marginals(net)
    a = restatement.tree(O.OracleGraph(net), dtype=np.float64)
    np.testing.assert_allclose(a["beliefs"][:, :2], ex[:, :2], atol=1e-9)
