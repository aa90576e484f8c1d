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


def _allocating_result(net, tol, max_it):
    from belief_propagation_b200.engine import BPGraph
    g = BPGraph.from_network(net)
    try:
        g.latest_slot = 1
        g.init_messages()
        r = g.loopy(tol, max_it, delta="f64")
        return dict(r, beliefs=g.beliefs(), latest=g.messages(g.latest_slot))
    finally:
        g.close()


def _noalloc_call(lib, N, net, arrs, tol, max_it, torch):
    beliefs = torch.from_numpy(np.ascontiguousarray(net.beliefs)).cuda()
    messages = torch.zeros((2, net.E, arrs["S"]), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    res = N.LoopyResult()
    latest = C.c_int(-1)
    st = lib.bp_loopy_noalloc(net.V, net.E, arrs["S"], arrs["in_ptr"].data_ptr(), arrs["in_src"].data_ptr(),
                              arrs["joint"].data_ptr(), beliefs.data_ptr(), messages.data_ptr(), 1, 1,
                              C.c_float(tol), max_it, None, C.byref(res), C.byref(latest))
    N.check(st)
    m_pos = messages[latest.value].cpu().numpy()
    m_edge = np.empty_like(m_pos)
    m_edge[arrs["order"]] = m_pos
    return dict(res.as_dict(), beliefs=beliefs.cpu().numpy(), latest=m_edge)


@pytest.mark.parametrize("V,E,S,tol,max_it", [(20000, 80000, 2, 1e-3, 100), (3000, 15000, 4, 0.0, 25),
                                              (500, 2000, 8, 1e-3, 60)])
def test_noalloc_matches_allocating_entry_point(synth, V, E, S, tol, max_it):
    import torch
    from belief_propagation_b200 import native as N
    lib = N.load()
    net = synth.random_loopy(V, E, S, 0.1, seed=V + S)
    want = _allocating_result(net, tol, max_it)
    arrs = _caller_arrays(net, torch)
    for call in range(2):
        got = _noalloc_call(lib, N, net, arrs, tol, max_it, torch)
        assert got["iterations"] == want["iterations"], call
        assert got["executed"] == want["executed"], call
        np.testing.assert_array_equal(got["beliefs"], want["beliefs"])
        np.testing.assert_array_equal(got["latest"], want["latest"])


def test_noalloc_rejects_graphs_beyond_its_working_memory():
    from belief_propagation_b200 import native as N
    lib = N.load()
    res = N.LoopyResult()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.bp_loopy_noalloc(4_000_000, 1, 2, dummy, dummy, dummy, dummy, dummy, 1, 0, C.c_float(0.0), 5,
                              None, C.byref(res), None)
    assert st == 2  # BP_ERR_SHAPE
    assert b"BP_NOALLOC_SCRATCH_BYTES" in lib.bp_last_error()
