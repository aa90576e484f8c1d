"""The destination-range split of loopy BP on the GPU: the CUDA range
iteration (bp_send_buffers_range / bp_flood_range) as 2 and 3 ranks driven
from one process with the in-process exchange (the ranks do not wait on one
another: each rank's kernels finish before the exchange), against the
single-GPU node schedule with the same fp64 stopping rule and against the
oracle, bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _split_run(net, world, tol, max_it):
    import torch
    from belief_propagation_b200.sharded import LocalComm, RangeEngine, node_ranges, sharded_loopy
    ranges, chunk = node_ranges(net.V, world)
    engines = [RangeEngine(net, b, e, chunk, world) for b, e in ranges]
    try:
        r = sharded_loopy(engines, LocalComm(chunk), net.beliefs, tol, max_it)
        torch.cuda.synchronize()
        beliefs = np.concatenate([e.beliefs() for e in engines])
        latest = np.zeros((net.E, int(net.s_max)), np.float32)
        for e in engines:
            eids, m = e.messages()
            latest[eids] = m
    finally:
        for e in engines:
            e.close()
    return r, beliefs, latest


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case", [dict(V=3000, E=12000, S=2, seed=5), dict(V=1200, E=6000, S=4, seed=6),
                                  dict(V=700, E=3000, S=8, seed=7)], ids=lambda c: f"S{c['S']}")
def test_range_split_matches_single_gpu(bp, synth, restatement, O, case, world):
    from belief_propagation_b200.engine import BPGraph
    net = synth.random_loopy(case["V"], case["E"], case["S"], 0.1, seed=case["seed"])
    for tol, max_it in ((1e-3, 50), (0.0, 12)):
        r, b, latest = _split_run(net, world, tol, max_it)
        g = BPGraph.from_network(net)
        try:
            g.latest_slot = 1
            g.init_messages()
            want = g.loopy(tol, max_it, delta="f64")
            wb, wl = g.beliefs(), g.messages(g.latest_slot)
        finally:
            g.close()
        assert r["iterations"] == want["iterations"] and r["executed"] == want["executed"]
        np.testing.assert_array_equal(b, wb)
        np.testing.assert_array_equal(latest, wl)
        if tol == 0.0:
            ora = restatement.loopy(O.OracleGraph(net), tol, max_it)
            np.testing.assert_array_equal(b, ora["beliefs"][:, : case["S"]])


def test_range_split_mixed_states_and_empty_range(bp, synth, restatement, O):
    """Mixed state counts, and more ranks than some ranges have edges (a rank
    whose nodes have no in-edges still exchanges its send buffers)."""
    base = synth.random_loopy(500, 2000, 2, 0.1, seed=8)
    rng = np.random.default_rng(9)
    ns = rng.choice(np.array([2, 3, 5], np.uint32), size=base.V)
    S = 5
    b = rng.random((base.V, S), dtype=np.float32) * (np.arange(S)[None] < ns[:, None])
    j = rng.random((base.E, S, S), dtype=np.float32)
    j *= (np.arange(S)[None, :, None] < ns[base.src][:, None, None])
    j *= (np.arange(S)[None, None, :] < ns[base.dst][:, None, None])
    keep = base.dst < 400                        # nodes 400.. receive nothing
    net = synth.Network(ns, b.astype(np.float32), base.observed, base.src[keep], base.dst[keep],
                        j[keep].astype(np.float32))
    r, bel, _ = _split_run(net, 4, 0.0, 9)
    ora = restatement.loopy(O.OracleGraph(net), 0.0, 9)
    np.testing.assert_array_equal(bel, ora["beliefs"][:, :S])
    assert r["executed"] == 9
