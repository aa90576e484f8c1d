"""bp_loopy_noalloc: loopy BP for callers that must not allocate GPU memory
while they run (a host application that owns the device allocator, a loop
that cannot afford cudaMalloc/cudaFree, a process at its memory cap).

It is called here through the C-ABI with caller-owned device arrays (torch
allocates them: the test is the caller) and must give exactly what the
allocating entry point bp_loopy gives (the repository's parity tolerance is
exact equality), on two calls in a row -- the second call finds the first
call's leftovers in the library's fixed working array.  Kept in a file that
pytest collects last."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _caller_arrays(net, torch):
    """The destination-sorted layout, built by the caller on the host."""
    S = net.s_max
    order = np.argsort(net.dst, kind="stable")
    counts = np.bincount(net.dst, minlength=net.V)
    in_ptr = np.zeros(net.V + 1, np.uint32)
    in_ptr[1:] = np.cumsum(counts)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    return dict(order=order, in_ptr=dev(in_ptr), in_src=dev(net.src[order].astype(np.uint32)),
                joint=dev(net.joint[order].astype(np.float32)), S=S)


def _allocating_result(net, tol, max_it, latest_slot=1, init=True, start=None):
    """bp_loopy on the same network with the fp64 delta, the stopping rule
    bp_loopy_noalloc uses; `start` = messages (edge order) for slot
    latest_slot when init is off."""
    from belief_propagation_b200.engine import BPGraph
    g = BPGraph.from_network(net)
    try:
        if start is not None:
            g.set_messages(latest_slot, start)
        g.latest_slot = latest_slot
        if init:
            g.init_messages()
        r = g.loopy(tol, max_it, delta="f64")
        return dict(r, beliefs=g.beliefs(), latest=g.messages(g.latest_slot), latest_slot=g.latest_slot)
    finally:
        g.close()


def _noalloc_call(lib, N, net, arrs, tol, max_it, torch, latest_slot=1, init=True, start=None):
    beliefs = torch.from_numpy(np.ascontiguousarray(net.beliefs)).cuda()
    messages = torch.zeros((2, net.E, arrs["S"]), dtype=torch.float32, device="cuda")
    if start is not None:
        messages[latest_slot] = torch.from_numpy(np.ascontiguousarray(start[arrs["order"]])).cuda()
    torch.cuda.synchronize()
    res = N.LoopyResult()
    latest = C.c_int(-1)
    st = lib.bp_loopy_noalloc(net.V, net.E, arrs["S"], arrs["in_ptr"].data_ptr(), arrs["in_src"].data_ptr(),
                              arrs["joint"].data_ptr(), beliefs.data_ptr(), messages.data_ptr(), latest_slot,
                              int(init), C.c_float(tol), max_it, None, C.byref(res), C.byref(latest))
    N.check(st)
    m_pos = messages[latest.value].cpu().numpy()
    m_edge = np.empty_like(m_pos)
    m_edge[arrs["order"]] = m_pos
    return dict(res.as_dict(), beliefs=beliefs.cpu().numpy(), latest=m_edge, latest_slot=latest.value)


def _assert_same_run(got, want, call):
    for k in ("iterations", "executed", "converged", "delta", "previous_delta", "delta_f64", "latest_slot"):
        assert got[k] == want[k], (k, call, got[k], want[k])
    np.testing.assert_array_equal(got["beliefs"], want["beliefs"])
    np.testing.assert_array_equal(got["latest"], want["latest"])


@pytest.mark.parametrize("V,E,S,tol,max_it", [(20000, 80000, 2, 1e-3, 100), (3000, 15000, 4, 0.0, 25),
                                              (500, 2000, 8, 1e-3, 60)])
def test_noalloc_matches_allocating_entry_point(synth, V, E, S, tol, max_it):
    """Two calls in a row give what bp_loopy (fp64 delta) gives: beliefs,
    latest messages, iteration counts, stop flag, deltas and latest slot."""
    import torch
    from belief_propagation_b200 import native as N
    lib = N.load()
    net = synth.random_loopy(V, E, S, 0.1, seed=V + S)
    want = _allocating_result(net, tol, max_it)
    arrs = _caller_arrays(net, torch)
    for call in range(2):
        _assert_same_run(_noalloc_call(lib, N, net, arrs, tol, max_it, torch), want, call)


def test_noalloc_caller_initialised_messages_in_slot_0(synth):
    """init_messages = 0 with the caller's own messages in slot 0: the loop
    starts from them, as bp_loopy does from the same slot."""
    import torch
    from belief_propagation_b200 import native as N
    lib = N.load()
    net = synth.random_loopy(4000, 16000, 3, 0.1, seed=17)
    rng = np.random.default_rng(5)
    start = rng.random((net.E, 3), dtype=np.float32)
    start /= start.sum(1, keepdims=True)
    want = _allocating_result(net, 1e-3, 50, latest_slot=0, init=False, start=start)
    arrs = _caller_arrays(net, torch)
    for call in range(2):
        got = _noalloc_call(lib, N, net, arrs, 1e-3, 50, torch, latest_slot=0, init=False, start=start)
        _assert_same_run(got, want, call)


def test_noalloc_zero_iterations_still_initialises(synth):
    """max_iterations = 0: the loop body never runs, but init_messages still
    fills the latest slot (init_previous_edge), and nothing else changes."""
    import torch
    from belief_propagation_b200 import native as N
    from belief_propagation_b200.engine import BPGraph
    lib = N.load()
    net = synth.random_loopy(2000, 8000, 2, 0.1, seed=23)
    g = BPGraph.from_network(net)
    try:
        g.latest_slot = 1
        g.init_messages()
        init_msgs = g.messages(1)
    finally:
        g.close()
    arrs = _caller_arrays(net, torch)
    got = _noalloc_call(lib, N, net, arrs, 1e-3, 0, torch)
    assert got["iterations"] == 0 and got["executed"] == 0 and got["latest_slot"] == 1
    np.testing.assert_array_equal(got["latest"], init_msgs)
    np.testing.assert_array_equal(got["beliefs"], net.beliefs)


def test_noalloc_rejects_a_malformed_layout(synth):
    """A row pointer past num_edges or a source id >= num_nodes is caught on
    the device before any kernel reads through it (BP_ERR_INVALID)."""
    import torch
    from belief_propagation_b200 import native as N
    lib = N.load()
    net = synth.random_loopy(1000, 4000, 2, 0.1, seed=29)
    arrs = _caller_arrays(net, torch)
    for name, bad in (("in_ptr", lambda a: a["in_ptr"].__setitem__(500, net.E + 7)),
                      ("in_src", lambda a: a["in_src"].__setitem__(123, net.V))):
        a = dict(arrs, in_ptr=arrs["in_ptr"].clone(), in_src=arrs["in_src"].clone())
        bad(a)
        with pytest.raises(N.BPError) as err:
            _noalloc_call(lib, N, net, a, 1e-3, 10, torch)
        assert err.value.status == 1, name   # BP_ERR_INVALID
    got = _noalloc_call(lib, N, net, arrs, 1e-3, 10, torch)   # the well-formed arrays still run
    assert got["executed"] >= 1


def test_noalloc_rejects_graphs_beyond_its_working_memory():
    from belief_propagation_b200 import native as N
    lib = N.load()
    res = N.LoopyResult()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.bp_loopy_noalloc(4_000_000, 1, 2, dummy, dummy, dummy, dummy, dummy, 1, 0, C.c_float(0.0), 5,
                              None, C.byref(res), None)
    assert st == 2  # BP_ERR_SHAPE
    assert b"BP_NOALLOC_SCRATCH_BYTES" in lib.bp_last_error()
