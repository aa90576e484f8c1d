"""Tree BP on the GPU (level-synchronous waves) against the oracle."""
import numpy as np
import pytest

from conftest import load_golden
import golden_nets as GN

pytestmark = pytest.mark.gpu


def gpu_tree(net, levels=None):
    from belief_propagation_b200.engine import BPGraph
    g = BPGraph.from_network(net)
    try:
        if levels is not None:
            g.set_levels(*levels)
        else:
            lv, nl = g.build_levels()
            levels = (lv, nl)
        r = g.tree()
        return dict(r, beliefs=g.beliefs(), messages=g.messages(0), levels=levels[0], num_levels=levels[1])
    finally:
        g.close()


def test_tree_example_known_answer(bp):
    """example-belief-propagation.c:72-107 on the GPU: marginals to 1e-4."""
    r = gpu_tree(GN.example_network())
    np.testing.assert_allclose(r["beliefs"][:, :2], GN.EXAMPLE_MARGINALS, atol=1e-4)


@pytest.mark.parametrize("name", ["tree_random_2000.npz", "example_4node.npz", "bif_asia.npz",
                                  "bif_cancer.npz", "bif_earthquake.npz", "bif_sachs.npz"])
def test_tree_fixtures(bp, name):
    fx = load_golden(name)
    net = GN.network_from_fixture(fx)
    r = gpu_tree(net)
    nl = int(fx["tree_num_levels"])
    assert r["num_levels"] == nl
    np.testing.assert_array_equal(r["levels"][: nl], fx["tree_levels_offsets"])
    np.testing.assert_array_equal(r["levels"][net.V:], fx["tree_levels_nodes"])
    S = fx["tree_beliefs"].shape[1]
    np.testing.assert_array_equal(r["beliefs"][:, :S], fx["tree_beliefs"])
    np.testing.assert_array_equal(r["messages"][:, :S], fx["tree_messages"])


@pytest.mark.parametrize("n,states,seed", [(5000, (2,), 1), (3000, (2, 3, 4, 8), 2), (20000, (3,), 3),
                                           (1, (2,), 4), (2, (4,), 5)])
def test_tree_random_trees(bp, synth, restatement, O, n, states, seed):
    net = synth.random_tree(n, states, 0.05, seed=seed)
    ora = restatement.tree(O.OracleGraph(net))
    r = gpu_tree(net)
    S = net.s_max
    assert r["num_levels"] == ora["num_levels"]
    np.testing.assert_array_equal(r["levels"][net.V:], ora["levels"][net.V:])
    np.testing.assert_array_equal(r["beliefs"][:, :S], ora["beliefs"][:, :S])
    np.testing.assert_array_equal(r["messages"][:, :S], ora["messages"][:, :S])


def test_tree_on_graph_with_cycles(bp, synth, restatement, O):
    """Same-level neighbours exercise the wave split (graph.c:508-521)."""
    done = 0
    for seed in range(5, 40):
        net = synth.random_loopy(600, 1500, 2, 0.1, seed=seed)
        og = O.OracleGraph(net)
        try:
            ora = restatement.tree(og)
        except ValueError:
            continue
        r = gpu_tree(net)
        np.testing.assert_array_equal(r["beliefs"][:, :2], ora["beliefs"][:, :2])
        np.testing.assert_array_equal(r["messages"][:, :2], ora["messages"][:, :2])
        done += 1
        if done == 3:
            break
    assert done > 0


def test_tree_unreachable_reports_error(bp, synth):
    """Nodes unreachable from the in-degree<=2 seeds: the reference loops
    forever; the engine returns BP_ERR_GRAPH."""
    from belief_propagation_b200.engine import BPGraph
    from belief_propagation_b200.native import BPError
    # a complete directed graph on 4 nodes: every in-degree is 3, so no node
    # qualifies as a level-0 seed and nothing is ever reached
    src = [u for u in range(4) for w in range(4) if u != w]
    dst = [w for u in range(4) for w in range(4) if u != w]
    V = 4
    src = np.array(src, np.uint32)
    dst = np.array(dst, np.uint32)
    net = synth.Network(np.full(V, 2, np.uint32), np.ones((V, 2), np.float32), np.zeros(V, np.uint8), src, dst,
                        np.full((len(src), 2, 2), 0.5, np.float32))
    g = BPGraph.from_network(net)
    try:
        indeg = np.bincount(dst, minlength=V)
        if (indeg <= 2).any():
            pytest.skip("construction has a seed node")
        with pytest.raises(BPError):
            g.build_levels()
    finally:
        g.close()
