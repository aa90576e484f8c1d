"""Differentiable unrolled BP: forward against a pure-torch unrolled
reference of the same update, gradients against that reference's autograd
and against FP64 finite differences on a 16x16 grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(side, S, T, seed, ck=5):
    import torch
    from belief_propagation_b200.unrolled import UnrolledBP, grid_tables
    src, dst, tab = grid_tables(side)
    rng = np.random.default_rng(seed)
    V = side * side
    theta = torch.tensor(rng.normal(0, 1, (V, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    W = torch.tensor(rng.normal(0, 0.5, (1, S, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    labels = torch.tensor(rng.integers(0, S, V), device="cuda")
    eng = UnrolledBP(V, src, dst, tab, S, T, checkpoint_every=ck)
    return eng, theta, W, labels, (src, dst, tab)


def _loss(lb, labels):
    import torch
    return torch.nn.functional.nll_loss(lb, labels)


@pytest.mark.parametrize("side,S,T,ck", [(16, 4, 30, 5), (32, 8, 20, 5), (24, 3, 7, 3), (16, 4, 30, 1),
                                         (16, 2, 6, 100), (20, 5, 8, 3), (18, 7, 6, 2), (12, 10, 5, 2)])
def test_unrolled_matches_torch_reference(bp, side, S, T, ck):
    import torch
    from belief_propagation_b200.unrolled import torch_unrolled
    eng, theta, W, labels, (src, dst, tab) = _setup(side, S, T, seed=side * 7 + S, ck=ck)
    b = eng(theta, W)
    loss = _loss(b, labels)
    loss.backward()
    g_theta, g_W = theta.grad.detach().clone(), W.grad.detach().clone()
    th64 = theta.detach().double().requires_grad_(True)
    W64 = W.detach().double().requires_grad_(True)
    b64 = torch_unrolled(th64, W64, src, dst, tab, T)
    _loss(b64, labels).backward()
    lb, lb64 = b.detach().cpu().numpy(), b64.detach().cpu().numpy()
    # fp32 against fp64 after up to 30 compounding iterations
    np.testing.assert_allclose(np.exp(lb), np.exp(lb64), atol=1e-4)
    live = lb64 > -20.0
    np.testing.assert_allclose(lb[live], lb64[live], atol=2e-3)
    scale_t = th64.grad.abs().max().item()
    scale_w = W64.grad.abs().max().item()
    np.testing.assert_allclose(g_theta.cpu().numpy(), th64.grad.cpu().numpy(), atol=1e-3 * scale_t + 1e-7)
    np.testing.assert_allclose(g_W.cpu().numpy(), W64.grad.cpu().numpy(), rtol=1e-3, atol=1e-3 * scale_w + 1e-7)
    eng.close()


def test_unrolled_gradient_fp64_finite_differences(bp):
    """16x16 grid, 4 states, T = 30: central differences in FP64 through the
    torch reference, on a sample of coordinates of both parameters."""
    import torch
    from belief_propagation_b200.unrolled import torch_unrolled
    side, S, T = 16, 4, 30
    eng, theta, W, labels, (src, dst, tab) = _setup(side, S, T, seed=3)
    _loss(eng(theta, W), labels).backward()
    th0, W0 = theta.detach().double(), W.detach().double()

    def f(th, w):
        with torch.no_grad():
            return _loss(torch_unrolled(th, w, src, dst, tab, T), labels).item()

    h = 1e-5
    rng = np.random.default_rng(0)
    for _ in range(12):
        v, i = int(rng.integers(0, side * side)), int(rng.integers(0, S))
        tp, tm = th0.clone(), th0.clone()
        tp[v, i] += h
        tm[v, i] -= h
        fd = (f(tp, W0) - f(tm, W0)) / (2 * h)
        assert abs(theta.grad[v, i].item() - fd) <= 1e-4 * max(1e-3, abs(fd)) + 2e-6, (v, i)
    for i in range(S):
        for j in range(S):
            wp, wm = W0.clone(), W0.clone()
            wp[0, i, j] += h
            wm[0, i, j] -= h
            fd = (f(th0, wp) - f(th0, wm)) / (2 * h)
            assert abs(W.grad[0, i, j].item() - fd) <= 2e-4 * max(1e-3, abs(fd)) + 2e-6, (i, j)
    eng.close()


def test_unrolled_forward_equals_plain_engine_update(bp, synth):
    """The unrolled forward is the reference's update: with the same tables
    and priors the plain engine (tolerance 0, T fixed iterations, linear
    domain) gives the same beliefs up to fp32 rounding."""
    import torch
    from belief_propagation_b200.engine import BPGraph
    side, S, T = 20, 4, 12
    eng, theta, W, labels, (src, dst, tab) = _setup(side, S, T, seed=11)
    b = np.exp(eng(theta, W).detach().cpu().numpy())
    E = np.exp(W.detach().cpu().numpy()[0])
    joint = np.where((tab & 0x80)[:, None, None] != 0, E.T[None], E[None]).astype(np.float32)
    prior = torch.softmax(theta.detach(), 1).cpu().numpy()
    net = synth.Network(np.full(side * side, S, np.uint32), prior, np.zeros(side * side, np.uint8), src, dst, joint)
    g = BPGraph.from_network(net)
    g.latest_slot = 1
    g.init_messages()
    g.loopy(0.0, T, delta="f64")
    np.testing.assert_allclose(g.beliefs(), b, atol=1e-5)
    g.close()
    eng.close()


def test_unrolled_gradient_is_a_descent_direction(bp):
    """A small step against the gradient lowers the loss (8-state grid)."""
    import torch
    eng, theta, W, labels, _ = _setup(24, 8, 20, seed=9)
    loss0 = _loss(eng(theta, W), labels)
    loss0.backward()
    with torch.no_grad():
        W2 = W - 1e-3 * W.grad / (W.grad.norm() + 1e-30)
        th2 = theta - 1e-3 * theta.grad / (theta.grad.norm() + 1e-30)
        loss1 = _loss(eng(th2.contiguous(), W2.contiguous()), labels)
    assert loss1.item() < loss0.item()
    eng.close()


def test_unrolled_repeated_calls_are_deterministic(bp):
    """The forward and backward replay captured CUDA graphs over the engine's
    own buffers: the same inputs give the same bits every call."""
    import torch
    eng, theta, W, labels, _ = _setup(16, 4, 12, seed=21)
    out = []
    for _ in range(3):
        theta.grad = None
        W.grad = None
        lb = eng(theta, W)
        _loss(lb, labels).backward()
        out.append((lb.detach().clone(), theta.grad.clone(), W.grad.clone()))
    for o in out[1:]:
        for x, y in zip(o, out[0]):
            assert torch.equal(x, y)
    eng.close()


@pytest.mark.parametrize("S,K", [(4, 3), (8, 2)])
def test_unrolled_several_tables(bp, S, K):
    """Several shared tables (edge e uses table tab[e] & 0x7f): forward and
    both gradients against the fp64 torch reference."""
    import torch
    from belief_propagation_b200.unrolled import UnrolledBP, grid_tables, torch_unrolled
    side, T = 20, 9
    src, dst, tab = grid_tables(side)
    rng = np.random.default_rng(S * 10 + K)
    tab = (tab & 0x80) | rng.integers(0, K, len(tab)).astype(np.uint8)
    V = side * side
    theta = torch.tensor(rng.normal(0, 1, (V, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    W = torch.tensor(rng.normal(0, 0.5, (K, S, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    labels = torch.tensor(rng.integers(0, S, V), device="cuda")
    eng = UnrolledBP(V, src, dst, tab, S, T, checkpoint_every=4, num_tables=K)
    _loss(eng(theta, W), labels).backward()
    th64 = theta.detach().double().requires_grad_(True)
    W64 = W.detach().double().requires_grad_(True)
    b64 = torch_unrolled(th64, W64, src, dst, tab, T)
    _loss(b64, labels).backward()
    np.testing.assert_allclose(np.exp(eng(theta, W).detach().cpu().numpy()), np.exp(b64.detach().cpu().numpy()),
                               atol=1e-4)
    scale_t = th64.grad.abs().max().item()
    scale_w = W64.grad.abs().max().item()
    np.testing.assert_allclose(theta.grad.cpu().numpy(), th64.grad.cpu().numpy(), atol=1e-3 * scale_t + 1e-7)
    np.testing.assert_allclose(W.grad.cpu().numpy(), W64.grad.cpu().numpy(), rtol=1e-3, atol=1e-3 * scale_w + 1e-7)
    eng.close()


def test_fused_nll_loss_matches_torch():
    """The fused cross-entropy head: torch's nll_loss value (mean over nodes)
    and its gradient, -1/V at each node's label."""
    import torch
    from belief_propagation_b200.unrolled import nll_loss
    g = torch.Generator(device="cpu").manual_seed(5)
    for V, S in ((1, 2), (1000, 4), (262_144, 4), (70_001, 8)):
        lb = torch.log_softmax(torch.randn(V, S, generator=g), 1).cuda().requires_grad_(True)
        labels = torch.randint(0, S, (V,), generator=g).cuda()
        loss = nll_loss(lb, labels)
        loss.backward()
        ref = torch.nn.functional.nll_loss(lb.detach().double(), labels)
        assert abs(float(loss) - float(ref)) <= 1e-6 * max(1.0, abs(float(ref)))
        ref_lb = lb.detach().clone().requires_grad_(True)
        torch.nn.functional.nll_loss(ref_lb, labels).backward()
        torch.testing.assert_close(lb.grad, ref_lb.grad, rtol=1e-7, atol=0)
    bad = torch.zeros(4, 3, device="cuda")
    assert torch.isnan(nll_loss(bad, torch.tensor([0, 1, 3, 2], device="cuda")))


def test_unrolled_batch_of_grids_of_different_sides(bp):
    """The batched + differentiable workload's shape: a disjoint union of
    grids of sides 9, 16 and 23 (one engine, one launch sequence forward and
    one backward), 8 states, one shared 8x8 table, T = 20, checkpoints every
    5.  Forward and both gradients against the fp64 torch reference, and one
    coordinate of the shared table against an fp64 central difference."""
    import torch
    from belief_propagation_b200.unrolled import UnrolledBP, torch_unrolled
    from belief_propagation_b200.synth import grid_edges
    S, T = 8, 20
    srcs, dsts, tabs, off = [], [], [], 0
    for side in (9, 16, 23):
        s_, d_, fwd = grid_edges(side)
        srcs.append(s_.astype(np.int64) + off)
        dsts.append(d_.astype(np.int64) + off)
        tabs.append(np.where(fwd, 0, 0x80).astype(np.uint8))
        off += side * side
    V = off
    src = np.concatenate(srcs).astype(np.uint32)
    dst = np.concatenate(dsts).astype(np.uint32)
    tab = np.concatenate(tabs)
    rng = np.random.default_rng(4)
    theta = torch.tensor(rng.normal(0, 1, (V, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    W = torch.tensor(rng.normal(0, 0.5, (1, S, S)), dtype=torch.float32, device="cuda", requires_grad=True)
    labels = torch.tensor(rng.integers(0, S, V), device="cuda")
    eng = UnrolledBP(V, src, dst, tab, S, T, checkpoint_every=5)
    lb = eng(theta, W)
    _loss(lb, labels).backward()
    th64 = theta.detach().double().requires_grad_(True)
    W64 = W.detach().double().requires_grad_(True)
    lb64 = torch_unrolled(th64, W64, src, dst, tab, T)
    _loss(lb64, labels).backward()
    np.testing.assert_allclose(np.exp(lb.detach().cpu().numpy()), np.exp(lb64.detach().cpu().numpy()), atol=1e-4)
    scale_t = th64.grad.abs().max().item()
    scale_w = W64.grad.abs().max().item()
    np.testing.assert_allclose(theta.grad.cpu().numpy(), th64.grad.cpu().numpy(), atol=1e-3 * scale_t + 1e-7)
    np.testing.assert_allclose(W.grad.cpu().numpy(), W64.grad.cpu().numpy(), rtol=1e-3, atol=1e-3 * scale_w + 1e-7)
    th0, W0 = theta.detach().double(), W.detach().double()

    def f(w):
        with torch.no_grad():
            return _loss(torch_unrolled(th0, w, src, dst, tab, T), labels).item()

    h = 1e-5
    i, j = 2, 5
    wp, wm = W0.clone(), W0.clone()
    wp[0, i, j] += h
    wm[0, i, j] -= h
    fd = (f(wp) - f(wm)) / (2 * h)
    assert abs(W.grad[0, i, j].item() - fd) <= 2e-4 * max(1e-3, abs(fd)) + 2e-6, (W.grad[0, i, j].item(), fd)
    eng.close()


@pytest.mark.parametrize("side,S,T,ck", [(24, 4, 7, 3), (32, 8, 20, 5), (17, 5, 6, 6), (15, 1, 4, 2)])
def test_unrolled_pull_adjoint_matches_scatter_adjoint(bp, side, S, T, ck, monkeypatch):
    """One shared table and up to 8 states: the adjoint in pull form (each
    source gathers the destinations' Pbar over its out-edges) against the
    scatter form (each destination writes per-edge x adjoint terms into the
    sources' slots, BP_UBWD_PULL=0).  Same forward bits, gradients equal to
    fp32 rounding of the two summation orders."""
    res = []
    for pull in ("1", "0"):
        monkeypatch.setenv("BP_UBWD_PULL", pull)
        eng, theta, W, labels, _ = _setup(side, S, T, seed=side + S, ck=ck)
        lb = eng(theta, W)
        _loss(lb, labels).backward()
        res.append((lb.detach().clone(), theta.grad.detach().clone(), W.grad.detach().clone()))
        eng.close()
    (lb1, gt1, gw1), (lb0, gt0, gw0) = res
    assert np.array_equal(lb1.cpu().numpy(), lb0.cpu().numpy())
    st = gt0.abs().max().item()
    sw = gw0.abs().max().item()
    np.testing.assert_allclose(gt1.cpu().numpy(), gt0.cpu().numpy(), rtol=1e-4, atol=1e-5 * st + 1e-9)
    np.testing.assert_allclose(gw1.cpu().numpy(), gw0.cpu().numpy(), rtol=1e-4, atol=1e-5 * sw + 1e-9)


@pytest.mark.parametrize("S,T,ck", [(3, 5, 2), (6, 4, 4), (8, 1, 1), (2, 7, 3)])
def test_unrolled_pull_adjoint_on_irregular_graph(bp, S, T, ck, monkeypatch):
    """One shared table on a random graph that is not a grid: sources with no
    in-edges, sinks with no out-edges, isolated nodes, repeated edges, both
    table orientations mixed at random, T = 1 included.  The pull-form adjoint
    against the scatter form and against the fp64 torch reference."""
    import torch
    from belief_propagation_b200.unrolled import UnrolledBP, torch_unrolled
    rng = np.random.default_rng(100 + S * 10 + T)
    V, E = 300, 900
    src = rng.integers(0, 200, E).astype(np.uint32)          # nodes 200.. send nothing
    dst = rng.integers(40, 260, E).astype(np.uint32)         # nodes < 40 receive nothing, 260.. are isolated or sources
    src[:20] = src[20:40]                                     # repeated edges
    dst[:20] = dst[20:40]
    tab = np.where(rng.random(E) < 0.5, 0, 0x80).astype(np.uint8)
    theta0 = rng.normal(0, 1, (V, S))
    W0 = rng.normal(0, 0.5, (1, S, S))
    labels = torch.tensor(rng.integers(0, S, V), device="cuda")
    res = []
    for pull in ("1", "0"):
        monkeypatch.setenv("BP_UBWD_PULL", pull)
        theta = torch.tensor(theta0, dtype=torch.float32, device="cuda", requires_grad=True)
        W = torch.tensor(W0, dtype=torch.float32, device="cuda", requires_grad=True)
        eng = UnrolledBP(V, src, dst, tab, S, T, checkpoint_every=ck)
        lb = eng(theta, W)
        _loss(lb, labels).backward()
        res.append((lb.detach().cpu().numpy(), theta.grad.cpu().numpy(), W.grad.cpu().numpy()))
        eng.close()
    (lb1, gt1, gw1), (lb0, gt0, gw0) = res
    assert np.array_equal(lb1, lb0)
    th64 = torch.tensor(theta0, dtype=torch.float64, device="cuda", requires_grad=True)
    W64 = torch.tensor(W0, dtype=torch.float64, device="cuda", requires_grad=True)
    _loss(torch_unrolled(th64, W64, src, dst, tab, T), labels).backward()
    st = th64.grad.abs().max().item()
    sw = W64.grad.abs().max().item()
    for gt, gw in ((gt1, gw1), (gt0, gw0)):
        np.testing.assert_allclose(gt, th64.grad.cpu().numpy(), atol=1e-3 * st + 1e-7)
        np.testing.assert_allclose(gw, W64.grad.cpu().numpy(), rtol=1e-3, atol=1e-3 * sw + 1e-7)
    np.testing.assert_allclose(gt1, gt0, rtol=1e-4, atol=1e-5 * st + 1e-9)
    np.testing.assert_allclose(gw1, gw0, rtol=1e-4, atol=1e-5 * sw + 1e-9)
