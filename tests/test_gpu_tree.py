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


def _path_network(synth, V, seed):
    """A path 0-1-2-...: every node has in-degree <= 2, so the whole path is
    level 0 and each node waits on its predecessor (V waves)."""
    rng = np.random.default_rng(seed)
    a = np.arange(V - 1, dtype=np.uint32)
    src = np.empty(2 * (V - 1), np.uint32)
    dst = np.empty(2 * (V - 1), np.uint32)
    src[0::2], dst[0::2] = a, a + 1
    src[1::2], dst[1::2] = a + 1, a
    j = rng.random((len(src), 2, 2), dtype=np.float32)
    j /= j.sum(axis=2, keepdims=True)
    b = rng.random((V, 2), dtype=np.float32)
    b /= b.sum(axis=1, keepdims=True)
    return synth.Network(np.full(V, 2, np.uint32), b, np.zeros(V, np.uint8), src, dst, j)


@pytest.mark.parametrize("V", [40, 700])
def test_tree_long_wave_chains(bp, synth, restatement, O, V):
    """Waves as long as the level (the device split hands chains longer than
    its round cap to the host split): same results as the reference."""
    net = _path_network(synth, V, seed=V)
    ora = restatement.tree(O.OracleGraph(net))
    r = gpu_tree(net)
    assert r["num_levels"] == ora["num_levels"]
    np.testing.assert_array_equal(r["levels"][net.V:], ora["levels"][net.V:])
    np.testing.assert_array_equal(r["beliefs"][:, :2], ora["beliefs"][:, :2])
    np.testing.assert_array_equal(r["messages"][:, :2], ora["messages"][:, :2])


def test_tree_device_and_host_level_builds_agree(bp, synth, monkeypatch):
    """The device level build gives the host build's lists, level count and
    wave count, on trees and on graphs with cycles."""
    nets = [synth.random_tree(30000, (2, 3), 0.05, seed=11)]
    for seed in range(50, 80):
        net = synth.random_loopy(500, 1200, 2, 0.1, seed=seed)
        if (np.bincount(net.dst, minlength=net.V) <= 2).any():
            nets.append(net)
        if len(nets) == 4:
            break
    from belief_propagation_b200.native import BPError
    compared = 0
    for net in nets:
        try:
            dev = gpu_tree(net)
        except BPError:
            dev = None
        monkeypatch.setenv("BP_TREE_LEVELS", "host")
        try:
            host = gpu_tree(net)
        except BPError:
            host = None
        monkeypatch.delenv("BP_TREE_LEVELS")
        assert (dev is None) == (host is None)
        if dev is None:
            continue
        compared += 1
        assert dev["num_levels"] == host["num_levels"]
        assert dev["num_waves"] == host["num_waves"]
        np.testing.assert_array_equal(dev["levels"][: dev["num_levels"]], host["levels"][: host["num_levels"]])
        np.testing.assert_array_equal(dev["levels"][net.V:], host["levels"][net.V:])
        np.testing.assert_array_equal(dev["beliefs"], host["beliefs"])
    assert compared >= 2


@pytest.mark.parametrize("n,states,seed", [(60000, (2, 3, 4, 8), 5), (30000, (2,), 6)])
def test_tree_small_waves_in_one_launch(bp, synth, restatement, O, monkeypatch, n, states, seed):
    """The runs of small waves go through one cooperative launch with a grid
    barrier between waves (BP_TREE_TAIL=1) or one launch per wave (the
    default): the same beliefs and messages, the oracle's."""
    net = synth.random_tree(n, states, 0.05, seed=seed)
    ora = restatement.tree(O.OracleGraph(net))
    S = net.s_max
    sep = gpu_tree(net)
    monkeypatch.setenv("BP_TREE_TAIL", "1")
    coop = gpu_tree(net)
    for r in (coop, sep):
        np.testing.assert_array_equal(r["beliefs"], ora["beliefs"][:, :S])
        np.testing.assert_array_equal(r["messages"][:, :S], ora["messages"][:, :S])


def _visited(g):
    import ctypes as C
    from belief_propagation_b200 import native as N
    out = np.zeros(g.V, np.uint8)
    N.check(g.lib.bp_get_visited(g.h, C.c_void_p(out.ctypes.data)))
    return out


@pytest.mark.parametrize("case", ["mixed_tree", "cycles", "path"])
def test_tree_whole_schedule_matches_step_calls(bp, synth, case):
    """bp_tree derives each step's visited flags from the levels; the graph.h
    steps (start, levels 1 .. L-2, reset_visited, levels L-1 .. 1,
    marginalize) read and write the flags.  Both leave the same messages,
    beliefs and visited flags, after stale flags were set beforehand."""
    from belief_propagation_b200.engine import BPGraph
    import ctypes as C
    from belief_propagation_b200 import native as N
    if case == "mixed_tree":
        net = synth.random_tree(4000, (2, 3, 4, 8), 0.05, seed=21)
    elif case == "path":
        net = _path_network(synth, 300, seed=3)
    else:
        net = None
        for seed in range(5, 40):
            cand = synth.random_loopy(600, 1500, 2, 0.1, seed=seed)
            g = BPGraph.from_network(cand)
            try:
                g.build_levels()
                net = cand
                break
            except Exception:
                continue
            finally:
                g.close()
        assert net is not None
    rng = np.random.default_rng(0)
    stale = (rng.random(net.V) < 0.5).astype(np.uint8)
    res = []
    for whole in (True, False):
        g = BPGraph.from_network(net)
        try:
            lv, L = g.build_levels()
            N.check(g.lib.bp_set_visited(g.h, C.c_void_p(stale.ctypes.data)))
            if whole:
                g.tree()
            else:
                g.tree_reset_visited()
                g.tree_start()
                for l in range(1, L - 1):
                    g.tree_level(l)
                g.tree_reset_visited()
                for l in range(L - 1, 0, -1):
                    g.tree_level(l)
                g.tree_marginalize()
            res.append((g.messages(0), g.beliefs(), _visited(g)))
        finally:
            g.close()
    for a, b in zip(*res):
        np.testing.assert_array_equal(a, b)
