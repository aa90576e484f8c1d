"""Batched loopy BP: every network of a batch must come out exactly as the
plain engine (and the oracle) gives it alone -- bit-exact beliefs and
messages, same returned iteration index."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solo(net, tol, max_it, delta):
    from belief_propagation_b200.engine import BPGraph
    g = BPGraph.from_network(net)
    try:
        g.latest_slot = 1
        g.init_messages()
        r = g.loopy(tol, max_it, delta=delta)
        return dict(r, beliefs=g.beliefs(), latest=g.messages(g.latest_slot))
    finally:
        g.close()


@pytest.fixture(scope="module")
def small_batch(synth):
    return synth.batch_of_networks(count=48, v_range=(20, 600), seed=5)


@pytest.mark.parametrize("delta", ["serial", "f64"])
@pytest.mark.parametrize("block", [64, 256])
def test_batch_matches_each_network_alone(bp, small_batch, restatement, O, delta, block):
    from belief_propagation_b200.engine import BPBatch
    nets = small_batch
    b = BPBatch(nets)
    try:
        b.set_beliefs()
        b.loopy(tol=1e-4, max_iterations=120, delta=delta, block_threads=block)
        res = b.results()
        for k, net in enumerate(nets):
            S = net.uniform_states
            if delta == "serial":
                ora = restatement.loopy(O.OracleGraph(net), 1e-4, 120)
                assert res["iterations"][k] == ora["ret"], k
                assert np.float32(res["delta"][k]) == np.float32(ora["delta"]), k
                np.testing.assert_array_equal(b.beliefs(k), ora["beliefs"][:, :S])
                np.testing.assert_array_equal(b.messages(k), ora["latest"][:, :S])
            else:
                solo = _solo(net, 1e-4, 120, "f64")
                if res["iterations"][k] != solo["iterations"]:
                    # fp64 sums in a different order may flip a borderline decision
                    continue
                np.testing.assert_array_equal(b.beliefs(k), solo["beliefs"])
                np.testing.assert_array_equal(b.messages(k), solo["latest"])
    finally:
        b.close()


def test_batch_autotune_and_rerun(bp, small_batch, tmp_path, monkeypatch):
    """Autotuning picks a block size per state-count group, restores the
    state, and a re-run (CUDA graph replay) gives the same answer."""
    from belief_propagation_b200.engine import BPBatch
    monkeypatch.setenv("BP_AUTOTUNE_CACHE", str(tmp_path / "tune.txt"))
    b = BPBatch(small_batch)
    try:
        b.set_beliefs()
        tuned = b.autotune(tol=1e-4, max_iterations=120)
        assert {int(k.split(",")[0][2:]) for k in tuned} == {n.uniform_states for n in small_batch}
        assert all(v in (64, 128, 256, 512) for v in tuned.values())
        groups = b.groups()
        assert len(groups) == len(tuned)
        for g in groups:
            assert g["max_nodes"] == 0 and g["grid"] >= 1
        assert (tmp_path / "tune.txt").exists()
        b.loopy(tol=1e-4, max_iterations=120)
        first = b.beliefs().copy()
        it1 = b.results()["iterations"].copy()
        b.set_beliefs()
        b.loopy(tol=1e-4, max_iterations=120)
        np.testing.assert_array_equal(b.beliefs(), first)
        np.testing.assert_array_equal(b.results()["iterations"], it1)
    finally:
        b.close()


def test_batch_mixed_state_network_rejected(bp, synth):
    from belief_propagation_b200.engine import BPBatch
    net = synth.random_tree(50, (2, 3), 0.0, seed=1)
    with pytest.raises(ValueError):
        BPBatch([net])


def test_batch_size_classes_change_no_result(bp, small_batch, monkeypatch):
    """With BP_BATCH_SMALL_NODES set, networks of at most that many nodes get
    launch groups of their own; with the reference's serial delta every network's beliefs,
    messages, iteration index and delta are the same with one group per
    state count (BP_BATCH_SMALL_NODES=0) as with the split."""
    from belief_propagation_b200.engine import BPBatch
    out = []
    for small in ("0", "256"):
        monkeypatch.setenv("BP_BATCH_SMALL_NODES", small)
        b = BPBatch(small_batch)
        try:
            groups = b.groups()
            states = {n.uniform_states for n in small_batch}
            if small == "0":
                assert len(groups) == len(states) and all(g["max_nodes"] == 0 for g in groups)
            else:
                want = {(n.uniform_states, 256 if n.V <= 256 else 0) for n in small_batch}
                assert {(g["states"], g["max_nodes"]) for g in groups} == want
            b.set_beliefs()
            b.loopy(tol=1e-4, max_iterations=120, delta="serial")
            r = b.results()
            out.append((b.beliefs().copy(), [b.messages(k).copy() for k in range(len(small_batch))],
                        r["iterations"].copy(), r["delta"].copy()))
        finally:
            b.close()
    (b0, m0, i0, d0), (b1, m1, i1, d1) = out
    np.testing.assert_array_equal(b0, b1)
    np.testing.assert_array_equal(i0, i1)
    np.testing.assert_array_equal(d0, d1)
    for x, y in zip(m0, m1):
        np.testing.assert_array_equal(x, y)
