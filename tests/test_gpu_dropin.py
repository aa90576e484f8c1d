"""The drop-in: the reference's C graph API (include/graph.h) on the GPU,
driven exactly as the reference's drivers drive it, compared with the
reference's own outputs (fixtures) and with the restatement."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, load_golden
import golden_nets as GN

pytestmark = pytest.mark.gpu


def test_dropin_loopy_driver_sequence(bp):
    """c_benchmark/main.c:277-281: init_previous_edge + loopy_propagate_until
    through struct graph; fields read back as the driver does."""
    from belief_propagation_b200.dropin import CGraph
    fx = load_golden("loopy_random_s3_500.npz")
    net = GN.network_from_fixture(fx)
    g = CGraph(net)
    g.init_previous_edge()
    ret = g.loopy_propagate_until(float(fx["loopy_tol"]), int(fx["loopy_max_it"]))
    assert ret == int(fx["loopy_ret"])
    S = fx["loopy_beliefs"].shape[1]
    np.testing.assert_array_equal(g.beliefs()[:, :S], fx["loopy_beliefs"])
    np.testing.assert_array_equal(g.messages("previous")[:, :S], fx["loopy_latest"])
    np.testing.assert_array_equal(g.messages("current")[:, :S], fx["loopy_older"])
    g.close()


def test_dropin_tree_driver_sequence(bp):
    """c_benchmark/main.c:224-236 through struct graph."""
    from belief_propagation_b200.dropin import CGraph
    fx = load_golden("tree_random_2000.npz")
    net = GN.network_from_fixture(fx)
    g = CGraph(net)
    g.tree_sequence()
    lv, nl = g.levels()
    assert nl == int(fx["tree_num_levels"])
    np.testing.assert_array_equal(lv[net.V:], fx["tree_levels_nodes"])
    S = fx["tree_beliefs"].shape[1]
    np.testing.assert_array_equal(g.beliefs()[:, :S], fx["tree_beliefs"])
    np.testing.assert_array_equal(g.messages("edges_messages")[:, :S], fx["tree_messages"])
    g.close()


@pytest.mark.parametrize("variant", ["until", "acc", "edge", "edge_acc", "one_iteration"])
def test_dropin_loopy_variants(bp, synth, restatement, O, variant):
    from belief_propagation_b200.dropin import CGraph
    net = synth.random_loopy(700, 2800, 2, 0.1, seed=61)
    g = CGraph(net)
    g.init_previous_edge()
    if variant == "one_iteration":
        g.loopy_propagate_one_iteration()
        g.loopy_propagate_one_iteration()
        ora = restatement.loopy(O.OracleGraph(net), -1.0, 2)
        ret = ora["ret"]
    else:
        fn = {"until": g.loopy_propagate_until, "acc": g.loopy_progagate_until_acc,
              "edge": g.loopy_propagate_until_edge, "edge_acc": g.loopy_progagate_until_edge_acc}[variant]
        ret = fn(1e-3, 60)
        check = 10 if "acc" in variant else 1
        sched = "edge" if "edge" in variant else "node"
        ora = restatement.loopy(O.OracleGraph(net), 1e-3, 60, check_every=check, schedule=sched)
    assert ret == ora["ret"]
    np.testing.assert_array_equal(g.beliefs()[:, :2], ora["beliefs"][:, :2])
    np.testing.assert_array_equal(g.messages("last_edges_messages")[:, :2], ora["prev_arr"][:, :2])
    np.testing.assert_array_equal(g.messages("edges_messages")[:, :2], ora["cur_arr"][:, :2])
    g.close()


def test_dropin_lazy_sync_mode(bp, synth, restatement, O):
    """Lazy mode: the device copy stays authoritative across the per-level
    calls; the host fields are refreshed by marginalize."""
    from belief_propagation_b200.dropin import CGraph
    from belief_propagation_b200 import native as N
    net = synth.random_tree(3000, (2, 3), 0.05, seed=8)
    g = CGraph(net)
    g.set_sync_mode(N.BP_SYNC_LAZY)
    g.tree_sequence()
    ora = restatement.tree(O.OracleGraph(net))
    np.testing.assert_array_equal(g.beliefs()[:, :3], ora["beliefs"][:, :3])
    g.close()


def _run_prebuilt(name, *args):
    exe = os.path.join(ROOT, "oracle", "_ref", name)
    if not os.path.exists(exe):
        pytest.skip(f"{name} not prebuilt (needs the reference sources at build time)")
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)


def test_reference_example_program_on_bp(bp):
    """The reference's own example-belief-propagation.c, compiled unchanged
    against its own graph.h and linked against libbp.so: its asserts (tree-BP
    marginals to 1e-4) run on the GPU."""
    r = _run_prebuilt("example_on_bp")
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "x1" in r.stdout


