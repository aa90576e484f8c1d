"""Loopy BP on the GPU against the oracle: bit-exact beliefs and messages and
the same returned iteration index as the reference on the same inputs.

Slot convention: slot 0 = struct graph's edges_messages, slot 1 =
last_edges_messages; the reference starts with *previous_edge_messages ->
last_edges_messages, so init_previous_edge writes slot 1."""
import numpy as np
import pytest

from conftest import load_golden
import golden_nets as GN

pytestmark = pytest.mark.gpu


def gpu_loopy(bp, net, tol, max_it, check_every=1, schedule="node", delta="serial", init=True,
              msgs=None, graph_chunk=0, reorder=False, kernel="auto"):
    from belief_propagation_b200.engine import BPGraph
    g = BPGraph.from_network(net, reorder=reorder)
    try:
        if msgs is not None:
            g.set_messages(1, msgs[0][:, : net.s_max])
            g.set_messages(0, msgs[1][:, : net.s_max])
        g.latest_slot = 1
        if init:
            g.init_messages()
        r = g.loopy(tol, max_it, check_every=check_every, schedule=schedule, delta=delta,
                    graph_chunk=graph_chunk, kernel=kernel)
        out = dict(r, beliefs=g.beliefs(), slot1=g.messages(1), slot0=g.messages(0), latest=g.latest_slot)
    finally:
        g.close()
    return out


def assert_same(gpu, ora, S, deltas=True):
    """Bit-exact beliefs and messages, the same return value and iterations;
    with the serial delta (gpu_loopy's default) also the reference's returned
    fp32 delta and previous delta."""
    np.testing.assert_array_equal(gpu["beliefs"][:, :S], ora["beliefs"][:, :S])
    np.testing.assert_array_equal(gpu["slot1"][:, :S], ora["prev_arr"][:, :S])
    np.testing.assert_array_equal(gpu["slot0"][:, :S], ora["cur_arr"][:, :S])
    assert gpu["iterations"] == ora["ret"]
    assert gpu["executed"] == ora["executed"]
    if deltas:
        assert np.float32(gpu["delta"]) == np.float32(ora["delta"]), (gpu["delta"], ora["delta"])
        assert np.float32(gpu["previous_delta"]) == np.float32(ora["prev_delta"]), \
            (gpu["previous_delta"], ora["prev_delta"])


def test_loopy_random_10k_matches_reference_fixture(bp):
    """The reference-runnable workload: 10,000 nodes, 40,000 edges, 2 states,
    tol 1e-3, max 100 -- against the reference's own outputs."""
    fx = load_golden("loopy_random_10000_40000.npz")
    net = GN.network_from_fixture(fx)
    for delta in ("serial", "f64"):
        r = gpu_loopy(bp, net, float(fx["loopy_tol"]), int(fx["loopy_max_it"]), delta=delta)
        assert r["iterations"] == int(fx["loopy_ret"])
        np.testing.assert_array_equal(r["beliefs"], fx["loopy_beliefs"])
        latest = r["slot1"] if r["latest"] == 1 else r["slot0"]
        older = r["slot0"] if r["latest"] == 1 else r["slot1"]
        np.testing.assert_array_equal(latest, fx["loopy_latest"])
        np.testing.assert_array_equal(older, fx["loopy_older"])


@pytest.mark.parametrize("name", ["loopy_random_s3_500.npz", "bif_asia.npz", "bif_cancer.npz",
                                  "bif_earthquake.npz", "bif_sachs.npz", "example_4node.npz",
                                  "tree_random_2000.npz"])
def test_loopy_fixtures(bp, name):
    fx = load_golden(name)
    net = GN.network_from_fixture(fx)
    r = gpu_loopy(bp, net, float(fx["loopy_tol"]), int(fx["loopy_max_it"]))
    assert r["iterations"] == int(fx["loopy_ret"])
    S = fx["loopy_beliefs"].shape[1]
    np.testing.assert_array_equal(r["beliefs"][:, :S], fx["loopy_beliefs"])


CASES = [
    dict(V=3000, E=12000, S=2, seed=31),
    dict(V=1000, E=5000, S=3, seed=32),
    dict(V=800, E=4000, S=4, seed=33),
    dict(V=500, E=2500, S=5, seed=34),
    dict(V=400, E=2000, S=8, seed=35),
    dict(V=300, E=1201, S=10, seed=36),
]


@pytest.mark.parametrize("reorder", [False, True], ids=["ids", "renumbered"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"S{c['S']}")
@pytest.mark.parametrize("tol,max_it", [(1e-3, 40), (0.0, 15)])
def test_loopy_node_parity(bp, synth, restatement, O, case, tol, max_it, reorder):
    net = synth.random_loopy(case["V"], case["E"], case["S"], 0.1, seed=case["seed"])
    ora = restatement.loopy(O.OracleGraph(net), tol, max_it)
    gpu = gpu_loopy(bp, net, tol, max_it, reorder=reorder)
    assert_same(gpu, ora, case["S"])


def test_loopy_renumbered_power_law_and_mixed(bp, synth, restatement, O):
    """Renumbering by out-degree changes nothing in the results: a power-law
    graph and a mixed-state graph, bit for bit."""
    net = synth.power_law_loopy(1 << 15, 1 << 17, 2, 0.1, seed=3)
    ora = restatement.loopy(O.OracleGraph(net), 1e-3, 30)
    assert_same(gpu_loopy(bp, net, 1e-3, 30, reorder=True), ora, 2)
    base = synth.random_loopy(400, 1600, 2, 0.1, seed=8)
    rng = np.random.default_rng(4)
    ns = rng.choice(np.array([2, 3, 5], np.uint32), size=base.V)
    S = 5
    b = rng.random((base.V, S), dtype=np.float32) * (np.arange(S)[None] < ns[:, None])
    j = rng.random((base.E, S, S), dtype=np.float32)
    j *= (np.arange(S)[None, :, None] < ns[base.src][:, None, None])
    j *= (np.arange(S)[None, None, :] < ns[base.dst][:, None, None])
    mixed = synth.Network(ns, b.astype(np.float32), base.observed, base.src, base.dst, j.astype(np.float32))
    ora = restatement.loopy(O.OracleGraph(mixed), 1e-3, 20)
    assert_same(gpu_loopy(bp, mixed, 1e-3, 20, reorder=True), ora, S)


def test_renumbered_graph_refuses_tree_and_edge_schedule(bp, synth):
    from belief_propagation_b200.engine import BPGraph
    from belief_propagation_b200.native import BPError
    net = synth.random_loopy(100, 300, 2, 0.1, seed=1)
    g = BPGraph.from_network(net, reorder=True)
    try:
        with pytest.raises(BPError):
            g.build_levels()
        with pytest.raises(BPError):
            g.loopy(1e-3, 5, schedule="edge")
    finally:
        g.close()


@pytest.mark.parametrize("check,sched", [(10, "node"), (1, "edge"), (10, "edge")])
@pytest.mark.parametrize("case", CASES[:3] + CASES[4:5], ids=lambda c: f"S{c['S']}")
def test_loopy_variants_parity(bp, synth, restatement, O, case, check, sched):
    net = synth.random_loopy(case["V"], case["E"], case["S"], 0.1, seed=case["seed"])
    for tol, max_it in ((1e-3, 60), (0.0, 25)):
        ora = restatement.loopy(O.OracleGraph(net), tol, max_it, check_every=check, schedule=sched)
        gpu = gpu_loopy(bp, net, tol, max_it, check_every=check, schedule=sched)
        assert_same(gpu, ora, case["S"])


def test_loopy_edge_byte_copy_odd_edges(bp, synth, restatement, O):
    """E odd: the reference's byte-count memcpy copies half of one float."""
    net = synth.random_loopy(101, 401, 2, 0.1, seed=40)
    ora = restatement.loopy(O.OracleGraph(net), 0.0, 7, schedule="edge")
    gpu = gpu_loopy(bp, net, 0.0, 7, schedule="edge")
    assert_same(gpu, ora, 2)


def test_loopy_mixed_states(bp, synth, restatement, O):
    """Nodes with different state counts: the zero-padding convention, same
    as the restatement."""
    nets = synth.batch_of_networks(count=1, v_range=(300, 300), seed=3)
    net = nets[0]
    rng = np.random.default_rng(5)
    ns = rng.choice(np.array([2, 3, 4, 8], np.uint32), size=net.V)
    S = 8
    b = rng.random((net.V, S), dtype=np.float32) * (np.arange(S)[None] < ns[:, None])
    j = rng.random((net.E, S, S), dtype=np.float32)
    j *= (np.arange(S)[None, :, None] < ns[net.src][:, None, None])
    j *= (np.arange(S)[None, None, :] < ns[net.dst][:, None, None])
    mixed = synth.Network(ns, b.astype(np.float32), net.observed, net.src, net.dst, j.astype(np.float32))
    for check, sched in ((1, "node"), (10, "node"), (1, "edge")):
        ora = restatement.loopy(O.OracleGraph(mixed), 1e-3, 30, check_every=check, schedule=sched)
        gpu = gpu_loopy(bp, mixed, 1e-3, 30, check_every=check, schedule=sched)
        assert_same(gpu, ora, S)


def test_loopy_hub_node_chunked(bp, synth, restatement, O):
    """A node with far more in-edges than one tile's shared memory holds."""
    V = 9000
    src = np.arange(1, V, dtype=np.uint32)
    dst = np.zeros(V - 1, np.uint32)
    rng = np.random.default_rng(9)
    extra_s = rng.integers(0, V, 4000).astype(np.uint32)
    extra_d = rng.integers(1, V, 4000).astype(np.uint32)
    keep = extra_s != extra_d
    src = np.concatenate([src, extra_s[keep]])
    dst = np.concatenate([dst, extra_d[keep]])
    key = src.astype(np.int64) * V + dst
    _, first = np.unique(key, return_index=True)
    first.sort()
    src, dst = src[first], dst[first]
    E = len(src)
    j = rng.random((E, 2, 2), dtype=np.float32)
    j /= j.sum(axis=2, keepdims=True)
    b = rng.random((V, 2), dtype=np.float32) + 0.5
    net = synth.Network(np.full(V, 2, np.uint32), b, np.zeros(V, np.uint8), src, dst, j)
    ora = restatement.loopy(O.OracleGraph(net), 0.0, 6)
    gpu = gpu_loopy(bp, net, 0.0, 6)
    assert_same(gpu, ora, 2)


def test_loopy_nan_messages_skipped(bp, synth, restatement, O):
    """NaN entries in incoming messages are skipped by combine (graph.c:455)
    and count 0 in the delta."""
    net = synth.random_loopy(200, 800, 2, 0.1, seed=41)
    rng = np.random.default_rng(2)
    prev = rng.random((net.E, 10), dtype=np.float32)
    prev[rng.random(net.E) < 0.05, 0] = np.nan
    cur = np.zeros((net.E, 10), np.float32)
    ora = restatement.loopy(O.OracleGraph(net), 1e-3, 5, init=False, msgs=(prev, cur))
    gpu = gpu_loopy(bp, net, 1e-3, 5, init=False, msgs=(prev, cur))
    np.testing.assert_array_equal(gpu["beliefs"][:, :2], ora["beliefs"][:, :2])
    assert gpu["iterations"] == ora["ret"]


@pytest.mark.parametrize("V,E", [(1, 0), (5, 0), (2, 1), (2, 2)])
def test_loopy_degenerate_graphs(bp, synth, restatement, O, V, E):
    rng = np.random.default_rng(V * 10 + E)
    src = np.array([0, 1][:E], np.uint32)
    dst = np.array([1, 0][:E], np.uint32)
    j = rng.random((E, 2, 2), dtype=np.float32)
    b = rng.random((V, 2), dtype=np.float32)
    net = synth.Network(np.full(V, 2, np.uint32), b, np.zeros(V, np.uint8), src, dst, j)
    for tol, max_it, check in ((1e-3, 10, 1), (0.0, 3, 1), (1e-3, 0, 1), (1e-3, 25, 10)):
        ora = restatement.loopy(O.OracleGraph(net), tol, max_it, check_every=check)
        gpu = gpu_loopy(bp, net, tol, max_it, check_every=check)
        assert_same(gpu, ora, 2)


def test_loopy_graph_chunks_agree(bp, synth):
    """The CUDA-graph chunk size changes nothing but launch grouping."""
    net = synth.random_loopy(2000, 8000, 2, 0.1, seed=42)
    a = gpu_loopy(bp, net, 1e-3, 50, graph_chunk=1)
    b = gpu_loopy(bp, net, 1e-3, 50, graph_chunk=7)
    c = gpu_loopy(bp, net, 1e-3, 50, graph_chunk=64)
    for x in (b, c):
        assert x["iterations"] == a["iterations"]
        np.testing.assert_array_equal(x["beliefs"], a["beliefs"])


def test_loopy_power_law_scale(bp, synth, restatement, O):
    """Power-law out-degree graph, fixed iterations, 1M edges."""
    net = synth.power_law_loopy(1 << 18, 1 << 20, 2, 0.1, seed=1)
    ora = restatement.loopy(O.OracleGraph(net), 0.0, 5)
    gpu = gpu_loopy(bp, net, 0.0, 5, delta="f64")
    np.testing.assert_array_equal(gpu["beliefs"][:, :2], ora["beliefs"][:, :2])
    np.testing.assert_array_equal(gpu["slot1"][:, :2], ora["prev_arr"][:, :2])
    # the GPU's fp64 delta against an fp64 sum of the oracle's own |m_t - m_(t-1)|
    # (the reference's fp32 serial sum of 2M terms carries ~1e-3 relative error)
    d = np.abs(ora["prev_arr"][:, :2].astype(np.float64) - ora["cur_arr"][:, :2].astype(np.float64))
    d64 = float(np.nan_to_num(d).sum())
    assert abs(gpu["delta_f64"] - d64) <= 1e-9 * max(1.0, d64)


@pytest.fixture(scope="module")
def headline_sample(synth, O):
    """The headline workload's generator at 1,048,576 nodes / 4,194,304 edges
    (power-law out-degree, 2 states, seed 1) and the oracle's beliefs and
    latest messages after 10 and 100 fixed iterations from the priors.  The
    100-iteration run uses the reference's own graph.c (OpenMP build: with a
    fixed iteration count its thread-scaled delta changes nothing) where it
    was built, else the restatement."""
    net = synth.power_law_loopy(1 << 20, 1 << 22, 2, 0.1, seed=1)
    R = O.Restatement()
    og = O.OracleGraph(net)
    out = {10: R.loopy(og, 0.0, 10)}
    if O.reference_available(openmp=True):
        r = O.Reference(openmp=True).loopy(net, 0.0, 100)
        out[100] = dict(beliefs=r["beliefs"], latest=r["latest"])
    else:
        out[100] = R.loopy(og, 0.0, 100)
    return net, out


@pytest.mark.parametrize("path", ["block", "block_outdeg", "split"])
@pytest.mark.parametrize("iterations", [10, 100])
def test_loopy_headline_path_bit_exact(bp, headline_sample, monkeypatch, iterations, path):
    """The benchmark's code paths -- nodes renumbered by out-degree, fp64
    delta, tolerance 0 -- on the headline generator at 1M nodes / 4M edges:
    block: the persistent-grid block-tile kernel with the source id loaded
    one round ahead and the evict-last send-buffer prefix cut to 1 MB, so
    most sources take the plain-load side;
    block_outdeg: the same with out-degree ties broken by id only
    (BP_REORDER_INDEG=0);
    split: the send pass over source ranges (cut to 2 MB of send buffers
    here, 4 ranges) + node pass.
    Bit-exact beliefs and latest messages against the oracle after 10 and
    100 iterations."""
    net, ora = headline_sample
    monkeypatch.setenv("BP_REORDER_INDEG", "0" if path == "block_outdeg" else "1")
    if path in ("block", "block_outdeg"):
        monkeypatch.setenv("BP_FLOOD_SPLIT", "0")
        monkeypatch.setenv("BP_FLOOD_HOT_MB", "1")
        monkeypatch.setenv("BP_FLOOD_PIPE", "1")
    else:
        monkeypatch.setenv("BP_FLOOD_SPLIT", "1")
        monkeypatch.setenv("BP_FLOOD_RANGE_MB", "2")
    gpu = gpu_loopy(bp, net, 0.0, iterations, delta="f64", reorder=True, kernel="split" if path == "split" else "auto")
    assert gpu["executed"] == iterations
    latest = gpu["slot1"] if gpu["latest"] == 1 else gpu["slot0"]
    np.testing.assert_array_equal(gpu["beliefs"][:, :2], ora[iterations]["beliefs"][:, :2])
    np.testing.assert_array_equal(latest[:, :2], ora[iterations]["latest"][:, :2])


SPLIT_CASES = [
    dict(V=3000, E=12000, S=2, seed=41),
    dict(V=1000, E=5000, S=3, seed=42),
    dict(V=800, E=4000, S=4, seed=43),
    dict(V=2500, E=9000, S=1, seed=44),
]


@pytest.mark.parametrize("reorder", [False, True], ids=["ids", "renumbered"])
@pytest.mark.parametrize("case", SPLIT_CASES, ids=lambda c: f"S{c['S']}")
@pytest.mark.parametrize("range_nodes", ["97", "100000"], ids=["many_ranges", "one_range"])
def test_loopy_split_schedule_parity(bp, synth, restatement, O, monkeypatch, case, reorder, range_nodes):
    """The split schedule (send pass over source ranges + node pass) forced
    on small graphs: with one range, and with ranges of 97 nodes
    (BP_FLOOD_RANGE_NODES); the reference's serial delta and the fp64 delta, check every iteration and
    every 10 (_acc): beliefs, both message arrays, iteration count and
    returned deltas equal the oracle's."""
    monkeypatch.setenv("BP_FLOOD_SPLIT", "1")
    monkeypatch.setenv("BP_FLOOD_RANGE_NODES", range_nodes)
    net = synth.random_loopy(case["V"], case["E"], case["S"], 0.1, seed=case["seed"])
    S = case["S"]
    for tol, max_it, check in ((1e-3, 40, 1), (0.0, 15, 1), (1e-3, 45, 10)):
        ora = restatement.loopy(O.OracleGraph(net), tol, max_it, check_every=check)
        gpu = gpu_loopy(bp, net, tol, max_it, check_every=check, reorder=reorder, kernel="split")
        assert_same(gpu, ora, S)
        f64 = gpu_loopy(bp, net, tol, max_it, check_every=check, reorder=reorder, kernel="split", delta="f64")
        blk = gpu_loopy(bp, net, tol, max_it, check_every=check, reorder=reorder, kernel="block", delta="f64")
        for k in ("iterations", "executed", "latest"):
            assert f64[k] == blk[k], k
        for k in ("beliefs", "slot0", "slot1"):
            np.testing.assert_array_equal(f64[k], blk[k])


@pytest.mark.parametrize("nodes_form", ["0", "1", "2", "3"])
@pytest.mark.parametrize("range_nodes", ["1", "4096"])
def test_loopy_split_schedule_ragged_power_law(bp, synth, restatement, O, monkeypatch, range_nodes, nodes_form):
    """The split schedule on a 2-state power-law graph whose edge count fills
    no whole round of the send pass, with one node per range and with ranges
    of 4096 nodes (BP_FLOOD_RANGE_NODES): the oracle's results."""
    monkeypatch.setenv("BP_FLOOD_SPLIT", "1")
    monkeypatch.setenv("BP_FLOOD_RANGE_NODES", range_nodes)
    monkeypatch.setenv("BP_SPLIT_NODES", nodes_form)
    net = synth.power_law_loopy(20_011, 80_021, 2, 0.1, seed=13)
    ora = restatement.loopy(O.OracleGraph(net), 0.0, 12)
    assert_same(gpu_loopy(bp, net, 0.0, 12, reorder=True, kernel="split", delta="f64"), ora, 2, deltas=False)


def test_loopy_split_schedule_power_law_serial_delta(bp, synth, restatement, O, monkeypatch):
    """A power-law graph through the split schedule with four source ranges
    and the reference's serial delta at a tolerance it converges under."""
    monkeypatch.setenv("BP_FLOOD_SPLIT", "1")
    monkeypatch.setenv("BP_FLOOD_RANGE_NODES", "4096")
    net = synth.power_law_loopy(1 << 14, 1 << 16, 2, 0.1, seed=9)
    ora = restatement.loopy(O.OracleGraph(net), 1e-2, 60)
    assert_same(gpu_loopy(bp, net, 1e-2, 60, reorder=True, kernel="split"), ora, 2)


def test_loopy_split_schedule_refuses_or_falls_back(bp, synth, restatement, O, monkeypatch):
    """Graphs the split layout does not hold -- mixed state counts, more than
    4 states -- are refused by kernel="split" and run k_flood in the default
    loop (split wanted), with the oracle's results; a hub with 5000 in-edges
    runs split, with the oracle's results."""
    from belief_propagation_b200.native import BPError
    from belief_propagation_b200.engine import BPGraph
    rng = np.random.default_rng(3)
    base = synth.random_loopy(400, 1600, 2, 0.1, seed=8)
    ns = rng.choice(np.array([2, 3], np.uint32), size=base.V)
    S = 3
    b = rng.random((base.V, S), dtype=np.float32) * (np.arange(S)[None] < ns[:, None])
    j = rng.random((base.E, S, S), dtype=np.float32)
    j *= (np.arange(S)[None, :, None] < ns[base.src][:, None, None])
    j *= (np.arange(S)[None, None, :] < ns[base.dst][:, None, None])
    mixed = synth.Network(ns, b.astype(np.float32), base.observed, base.src, base.dst, j.astype(np.float32))
    five = synth.random_loopy(300, 1200, 5, 0.1, seed=2)
    V = 3000
    src = rng.integers(1, V, 5000).astype(np.uint32)
    dst = np.zeros(5000, np.uint32)          # node 0's tile: 5000 in-edges > 2048
    hub = synth.Network(np.full(V, 2, np.uint32), rng.random((V, 2), dtype=np.float32), np.zeros(V, np.uint8),
                        src, dst, rng.random((5000, 2, 2), dtype=np.float32))
    monkeypatch.setenv("BP_FLOOD_SPLIT", "1")
    for net in (mixed, five):
        g = BPGraph.from_network(net)
        try:
            with pytest.raises(BPError):
                g.loopy(0.0, 3, delta="f64", kernel="split")
        finally:
            g.close()
        ora = restatement.loopy(O.OracleGraph(net), 1e-3, 20)
        gpu = gpu_loopy(bp, net, 1e-3, 20)
        assert_same(gpu, ora, int(net.s_max))
    ora = restatement.loopy(O.OracleGraph(hub), 1e-3, 20)
    assert_same(gpu_loopy(bp, hub, 1e-3, 20, kernel="split"), ora, 2)


def _staged_cases(synth):
    rng = np.random.default_rng(17)
    out = {"power_law": synth.power_law_loopy(1 << 16, 1 << 18, 2, 0.1, seed=5),
           "ragged_tail": synth.random_loopy(257, 1000, 2, 0.1, seed=6),
           "one_tile": synth.random_loopy(40, 150, 2, 0.1, seed=7)}
    V = 300
    out["no_edges"] = synth.Network(np.full(V, 2, np.uint32), rng.random((V, 2), dtype=np.float32),
                                    np.zeros(V, np.uint8), np.zeros(0, np.uint32), np.zeros(0, np.uint32),
                                    np.zeros((0, 2, 2), np.float32))
    # a hub whose in-edges overflow a stage, beside ordinary tiles
    V = 6000
    src = np.arange(1, 3001, dtype=np.uint32)
    dst = np.zeros(3000, np.uint32)
    es = rng.integers(0, V, 12000).astype(np.uint32)
    ed = rng.integers(1, V, 12000).astype(np.uint32)
    keep = es != ed
    src = np.concatenate([src, es[keep]])
    dst = np.concatenate([dst, ed[keep]])
    key = src.astype(np.int64) * V + dst
    _, first = np.unique(key, return_index=True)
    first.sort()
    src, dst = src[first], dst[first]
    j = rng.random((len(src), 2, 2), dtype=np.float32)
    j /= j.sum(axis=2, keepdims=True)
    out["hub"] = synth.Network(np.full(V, 2, np.uint32), rng.random((V, 2), dtype=np.float32) + 0.5,
                               np.zeros(V, np.uint8), src, dst, j)
    return out


@pytest.mark.parametrize("name", ["power_law", "ragged_tail", "one_tile", "no_edges", "hub"])
def test_loopy_staged_kernel_parity(bp, synth, restatement, O, name):
    """The bulk-copy staged kernel (explicitly selected): the same beliefs and
    messages, bit for bit, as the reference; fixed iterations, the _acc
    variant's every-10 check (stages without the old messages), renumbered
    ids, a partial last tile, a graph without edges and a hub tile that
    overflows a stage."""
    net = _staged_cases(synth)[name]
    for tol, max_it, check, reorder in ((0.0, 7, 1, False), (0.0, 25, 10, False), (0.0, 6, 1, True)):
        ora = restatement.loopy(O.OracleGraph(net), tol, max_it, check_every=check)
        gpu = gpu_loopy(bp, net, tol, max_it, check_every=check, delta="f64", kernel="staged", reorder=reorder)
        assert_same(gpu, ora, 2, deltas=False)


def test_loopy_staged_matches_block_kernel_with_tolerance(bp, synth):
    """Stopping on a tolerance: the staged and block kernels stop at the same
    iteration with identical beliefs (their f64 deltas differ only in
    summation order)."""
    net = synth.power_law_loopy(1 << 15, 1 << 17, 2, 0.1, seed=9)
    a = gpu_loopy(bp, net, 1e-3, 100, delta="f64", kernel="block")
    b = gpu_loopy(bp, net, 1e-3, 100, delta="f64", kernel="staged")
    assert a["iterations"] == b["iterations"] and a["executed"] == b["executed"]
    np.testing.assert_array_equal(a["beliefs"], b["beliefs"])
    np.testing.assert_array_equal(a["slot0"], b["slot0"])
    assert abs(a["delta_f64"] - b["delta_f64"]) <= 1e-12 * max(1.0, abs(a["delta_f64"]))


def test_loopy_staged_refuses_inapplicable_graphs(bp, synth):
    from belief_propagation_b200.engine import BPGraph
    from belief_propagation_b200.native import BPError
    for net, delta in ((synth.random_loopy(300, 1200, 3, 0.1, seed=1), "f64"),
                       (synth.random_loopy(300, 1200, 2, 0.1, seed=1), "serial"),
                       (synth.random_loopy(300, 3000, 2, 0.1, seed=1), "f64")):
        g = BPGraph.from_network(net)
        try:
            with pytest.raises(BPError):
                g.loopy(0.0, 3, delta=delta, kernel="staged")
        finally:
            g.close()


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"S{c['S']}")
def test_loopy_fused_loop_matches_launch_loop(bp, synth, restatement, O, monkeypatch, case):
    """Small graphs run every iteration in one cooperative launch (grid
    barrier between iterations); the launch-per-iteration loop
    (BP_FLOOD_FUSED=0) gives the same beliefs, messages, iteration count and
    f64 delta bit for bit, and the beliefs match the reference's."""
    net = synth.random_loopy(case["V"], case["E"], case["S"], 0.1, seed=case["seed"] + 100)
    S = case["S"]
    for tol, max_it, check, reorder in ((1e-3, 60, 1, False), (0.0, 12, 1, True), (1e-3, 45, 10, False)):
        fused = gpu_loopy(bp, net, tol, max_it, check_every=check, delta="f64", reorder=reorder)
        monkeypatch.setenv("BP_FLOOD_FUSED", "0")
        loop = gpu_loopy(bp, net, tol, max_it, check_every=check, delta="f64", reorder=reorder)
        monkeypatch.delenv("BP_FLOOD_FUSED")
        for k in ("iterations", "executed", "delta_f64", "latest"):
            assert fused[k] == loop[k], k
        for k in ("beliefs", "slot0", "slot1"):
            np.testing.assert_array_equal(fused[k], loop[k])
        if tol == 0.0:
            ora = restatement.loopy(O.OracleGraph(net), tol, max_it, check_every=check)
            np.testing.assert_array_equal(fused["beliefs"][:, :S], ora["beliefs"][:, :S])
            assert fused["iterations"] == ora["ret"]


def test_loopy_fused_loop_mixed_states(bp, synth, restatement, O, monkeypatch):
    """Mixed state counts through the fused (one-launch) loop: the same
    results as the launch-per-iteration loop, and the reference's beliefs."""
    base = synth.random_loopy(700, 2800, 2, 0.1, seed=77)
    rng = np.random.default_rng(12)
    S = 6
    ns = rng.choice(np.array([2, 3, 6], np.uint32), size=base.V)
    b = rng.random((base.V, S), dtype=np.float32) * (np.arange(S)[None] < ns[:, None])
    j = rng.random((base.E, S, S), dtype=np.float32)
    j *= (np.arange(S)[None, :, None] < ns[base.src][:, None, None])
    j *= (np.arange(S)[None, None, :] < ns[base.dst][:, None, None])
    net = synth.Network(ns, b.astype(np.float32), base.observed, base.src, base.dst, j.astype(np.float32))
    fused = gpu_loopy(bp, net, 0.0, 9, delta="f64")
    monkeypatch.setenv("BP_FLOOD_FUSED", "0")
    loop = gpu_loopy(bp, net, 0.0, 9, delta="f64")
    monkeypatch.delenv("BP_FLOOD_FUSED")
    assert fused["delta_f64"] == loop["delta_f64"] and fused["executed"] == loop["executed"]
    np.testing.assert_array_equal(fused["beliefs"], loop["beliefs"])
    np.testing.assert_array_equal(fused["slot0"], loop["slot0"])
    ora = restatement.loopy(O.OracleGraph(net), 0.0, 9)
    np.testing.assert_array_equal(fused["beliefs"][:, :S], ora["beliefs"][:, :S])


@pytest.mark.parametrize("delta", ["f64", "serial"])
def test_fused_loop_barrier_wait_runs_out_and_graph_stays_usable(bp, synth, restatement, O, monkeypatch, delta):
    """The one-launch loop's grid barrier waits a bounded time.  With block 1
    held back from the first barrier (BP_DEBUG_BARRIER_SKIP) and the limit cut
    to 50 ms (BP_DEBUG_WAIT_MS), every other block's wait runs out and so does
    block 1's next one: bp_loopy returns BP_ERR_TIMEOUT instead of hanging,
    the context stays usable, and the same graph then solves bit-exactly."""
    from belief_propagation_b200.engine import BPGraph
    from belief_propagation_b200.native import BPError
    net = synth.random_loopy(3000, 12000, 2, 0.1, seed=91)   # 24 tiles: the fused loop runs
    g = BPGraph.from_network(net)
    try:
        monkeypatch.setenv("BP_DEBUG_WAIT_MS", "50")
        monkeypatch.setenv("BP_DEBUG_BARRIER_SKIP", "1")
        g.latest_slot = 1
        g.init_messages()
        with pytest.raises(BPError) as err:
            g.loopy(1e-3, 40, delta=delta)
        assert err.value.status == 8, err.value    # BP_ERR_TIMEOUT
        monkeypatch.delenv("BP_DEBUG_WAIT_MS")
        monkeypatch.delenv("BP_DEBUG_BARRIER_SKIP")
        g.set_beliefs(net.beliefs)
        g.set_messages(0, np.zeros((net.E, 2), np.float32))
        g.latest_slot = 1
        g.init_messages()
        r = g.loopy(1e-3, 40, delta="serial")
        gpu = dict(r, beliefs=g.beliefs(), slot1=g.messages(1), slot0=g.messages(0), latest=g.latest_slot)
    finally:
        g.close()
    assert_same(gpu, restatement.loopy(O.OracleGraph(net), 1e-3, 40), 2)


def _oracle_deltas(restatement, O, net, n, schedule="node", check=1):
    """The reference's fp32 delta after each of the first n checks."""
    og = O.OracleGraph(net)
    return [np.float32(restatement.loopy(og, 0.0, k * check, check_every=check, schedule=schedule)["delta"])
            for k in range(1, n + 1)]


def _straddling_tolerances(restatement, O, net, deltas, sched, check):
    """Tolerances whose stopping decision at some check k is certain to need
    the serial sum: the serial sum's rounding bound (about 0.1 % of the delta
    here) straddles the tolerance in one comparison while the other is decided
    by a wide margin, and the reference's loop does reach check k."""
    out = []
    for k in range(1, len(deltas)):
        dk, dp = deltas[k], deltas[k - 1]
        diff = np.float32(abs(np.float32(dk - dp)))
        cands = []
        if diff > np.float32(1.05) * dk:      # delta < tol straddles, |delta - prev| >= tol surely
            cands = [dk, np.nextafter(dk, np.float32(np.inf))]
        elif dk > np.float32(1.05) * diff:    # |delta - prev| < tol straddles, delta >= tol surely
            cands = [diff, np.nextafter(diff, np.float32(np.inf))]
        for tol in cands:
            ora = restatement.loopy(O.OracleGraph(net), float(tol), 200, check_every=check, schedule=sched)
            if ora["executed"] >= (k + 1) * check:
                out.append((float(tol), ora))
        if len(out) >= 4:
            break
    return out


@pytest.mark.parametrize("path", ["fused", "launch_loop", "warp", "edge", "node_acc"])
def test_serial_delta_bound_straddling_tolerance(bp, synth, restatement, O, monkeypatch, path):
    """The serial fp32 delta is decided from the f64 sum and the serial sum's
    rounding bound, and formed only when that interval straddles the
    tolerance.  Tolerances at the reference's own delta (or its step) at a
    check make the interval straddle on purpose: the stop, iteration count,
    beliefs, messages and returned deltas are still the reference's, and
    those decisions formed the serial sum."""
    net = synth.random_loopy(2000, 8000, 2, 0.1, seed=71)
    sched = "edge" if path == "edge" else "node"
    check = 10 if path == "node_acc" else 1
    kernel = "warp" if path == "warp" else "auto"
    if path == "launch_loop":
        monkeypatch.setenv("BP_FLOOD_FUSED", "0")
    d = _oracle_deltas(restatement, O, net, 12, sched, check)
    cases = _straddling_tolerances(restatement, O, net, d, sched, check)
    assert cases, d
    for tol, ora in cases:
        gpu = gpu_loopy(bp, net, tol, 200, check_every=check, schedule=sched, kernel=kernel)
        assert_same(gpu, ora, 2)
        assert gpu["serial_sums"] + gpu["serial_refines"] >= 1, (tol, d)


@pytest.mark.parametrize("case", CASES[:2] + CASES[4:5], ids=lambda c: f"S{c['S']}")
def test_serial_delta_fused_matches_launch_loop(bp, synth, restatement, O, monkeypatch, case):
    """The serial delta through the one-launch (fused) loop and the
    launch-per-iteration loop: identical results, equal to the reference's."""
    net = synth.random_loopy(case["V"], case["E"], case["S"], 0.1, seed=case["seed"] + 200)
    S = case["S"]
    for tol, max_it, check in ((1e-3, 60, 1), (1e-3, 45, 10)):
        ora = restatement.loopy(O.OracleGraph(net), tol, max_it, check_every=check)
        fused = gpu_loopy(bp, net, tol, max_it, check_every=check)
        monkeypatch.setenv("BP_FLOOD_FUSED", "0")
        loop = gpu_loopy(bp, net, tol, max_it, check_every=check)
        monkeypatch.delenv("BP_FLOOD_FUSED")
        assert_same(fused, ora, S)
        assert_same(loop, ora, S)


def _serial_sum_cases():
    rng = np.random.default_rng(123)
    f32 = np.float32
    out = {
        "empty": np.zeros(0, f32),
        "one": np.array([3.5], f32),
        "zeros": np.zeros(5000, f32),
        "uniform_80k": rng.random(80_000, dtype=f32),
        "tiny_terms": (rng.random(200_000, dtype=f32) * f32(1e-4)),
        "wide_exponents": (rng.random(50_000) * 10.0 ** rng.uniform(-40, 30, 50_000)).astype(f32),
        "subnormals": (rng.integers(0, 1 << 20, 30_000).astype(np.uint32)).view(f32),
        # powers of two: every add an exact tie or exact, ties to even
        "ties": np.ldexp(f32(1.0), rng.integers(-30, -10, 100_000)).astype(f32),
        "half_ulp_runs": np.concatenate([np.array([1.0], f32), np.full(70_000, np.ldexp(f32(1.0), -24), f32),
                                         np.full(3000, np.ldexp(f32(1.0), -23), f32)]),
        "large_then_small": np.concatenate([np.full(10, 1e30, f32), rng.random(20_000, dtype=f32)]),
        "growing": (np.arange(1, 60_001, dtype=np.float64) ** 2).astype(f32),
        "with_inf": np.concatenate([rng.random(9000, dtype=f32), np.array([np.inf], f32),
                                    rng.random(9000, dtype=f32)]),
        "overflow": np.full(40, 3.0e38, f32),
        "ragged_1793": rng.random(1793, dtype=f32),
        "max_float_mix": np.concatenate([rng.random(4000, dtype=f32),
                                         np.full(4, np.finfo(f32).max / f32(8), f32)]),
    }
    # |diff| terms as the iteration kernels write them: messages of 2 states
    a = rng.random((40_000, 2), dtype=f32)
    b = a + (rng.standard_normal((40_000, 2)) * 1e-3).astype(f32)
    out["message_diffs"] = np.abs(a - b).ravel()
    return out


@pytest.mark.parametrize("name", list(_serial_sum_cases()))
def test_serial_sum_parallel_is_the_one_by_one_sum(bp, name):
    """The parallel serial fp32 sum (a scan of per-term increments inside each
    binade of the running sum) equals the one-add-at-a-time fp32 sum bit for
    bit -- the device chain and numpy's sequential accumulate -- for every
    block shape, on ties, subnormals, exponent ranges, inf and overflow."""
    import ctypes as C
    import torch
    from belief_propagation_b200 import native as N
    x = _serial_sum_cases()[name]
    ref = np.add.accumulate(x, dtype=np.float32)[-1] if len(x) else np.float32(0.0)
    xd = torch.from_numpy(x.copy()).cuda() if len(x) else torch.zeros(1, device="cuda")
    out = torch.full((5,), -7.0, device="cuda")
    lib = N.load()
    for method in range(5):
        rc = lib.bp_serial_sum_f32(C.c_void_p(xd.data_ptr()), C.c_uint64(len(x)),
                                   C.c_void_p(out.data_ptr() + 4 * method), method, None)
        assert rc == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for method in range(5):
        assert got[method].tobytes() == np.float32(ref).tobytes(), (name, method, got[method], ref)


@pytest.mark.parametrize("name", list(_serial_sum_cases()))
def test_serial_sum_bounds_hold_the_sum(bp, name):
    """The interval narrowed from the terms' own rounding errors holds the
    one-by-one fp32 sum on every input (ties, subnormals, binade crossings),
    and is far narrower than the worst-case bound n u S on plain data."""
    import ctypes as C
    import torch
    from belief_propagation_b200 import native as N
    x = _serial_sum_cases()[name]
    with np.errstate(over="ignore"):
        ref = float(np.add.accumulate(x, dtype=np.float32)[-1]) if len(x) else 0.0
    xd = torch.from_numpy(x.copy()).cuda() if len(x) else torch.zeros(1, device="cuda")
    lohi = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert N.load().bp_serial_sum_bounds(C.c_void_p(xd.data_ptr()), C.c_uint64(len(x)),
                                         C.c_void_p(lohi.data_ptr()), None) == 0
    torch.cuda.synchronize()
    lo, hi = lohi.cpu().numpy()
    assert lo <= ref <= hi, (name, lo, ref, hi)
    if name in ("uniform_80k", "message_diffs", "tiny_terms"):
        worst = len(x) * 2.0 ** -24 * float(np.sum(x, dtype=np.float64))
        assert hi - lo < 0.05 * worst, (name, hi - lo, worst)


def test_reserve_cached_memory_then_build_and_solve(bp, synth, restatement, O):
    """bp_reserve_cached_memory grows the stream-ordered pool once (a second
    call with a smaller size does nothing); graphs built afterwards solve as
    before, and bp_release_cached_memory hands the memory back."""
    from belief_propagation_b200 import native as N
    lib = N.load()
    assert lib.bp_reserve_cached_memory(256 << 20) == 0
    assert lib.bp_reserve_cached_memory(16 << 20) == 0
    net = synth.random_loopy(2000, 8000, 2, 0.1, seed=4)
    ora = restatement.loopy(O.OracleGraph(net), 1e-3, 30)
    assert_same(gpu_loopy(bp, net, 1e-3, 30), ora, 2)
    assert lib.bp_release_cached_memory() == 0


@pytest.mark.parametrize("reorder", [False, True], ids=["ids", "renumbered"])
def test_loopy_long_runs_of_nodes_without_in_edges(bp, synth, restatement, O, reorder):
    """Row pointers from the sorted destinations when long runs of nodes have
    no in-edges: the first 3000 nodes, 2500 in the middle and the last 2000
    receive none (renumbered, such nodes of one out-degree are also grouped
    together).  The oracle's results, and the edge schedule's."""
    rng = np.random.default_rng(23)
    V = 10000
    receivers = np.concatenate([np.arange(3000, 5000), np.arange(7500, 8000)]).astype(np.uint32)
    E = 24000
    src = rng.integers(0, V, E).astype(np.uint32)
    dst = rng.choice(receivers, E).astype(np.uint32)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    j = rng.random((len(src), 2, 2), dtype=np.float32)
    j /= j.sum(axis=2, keepdims=True)
    b = rng.random((V, 2), dtype=np.float32)
    b /= b.sum(axis=1, keepdims=True)
    net = synth.Network(np.full(V, 2, np.uint32), b, np.zeros(V, np.uint8), src, dst, j)
    ora = restatement.loopy(O.OracleGraph(net), 1e-3, 30)
    assert_same(gpu_loopy(bp, net, 1e-3, 30, reorder=reorder), ora, 2)
    if not reorder:
        ora_e = restatement.loopy(O.OracleGraph(net), 1e-3, 30, schedule="edge")
        assert_same(gpu_loopy(bp, net, 1e-3, 30, schedule="edge"), ora_e, 2)
