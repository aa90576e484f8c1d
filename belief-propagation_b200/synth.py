"""Seeded synthetic belief networks for the benchmark workloads.

Every workload is a :class:`Network`: a directed graph whose edge ``e`` carries
a joint table ``joint[e, i, j]`` read as in the reference's
``send_message_for_edge`` (src/graph/graph.c:884-910): the message on ``e`` is
``m[i] = sum_j joint[e, i, j] * buf_src[j]`` for ``i < S_src``, ``j < S_dst``.
Arrays are zero-padded to ``S_max`` states; node ``v`` uses the first
``num_states[v]`` slots.  Edge ids are insertion order, which fixes the
order of every per-node product exactly as ``graph_add_edge`` does
(graph.c:149-211).

Workloads (sizes as named in the project's benchmark configuration):

* :func:`random_loopy`     -- uniform random directed graph (10,000 nodes,
  40,000 edges, 2 states, 10% evidence), the reference-runnable case.
* :func:`power_law_loopy`  -- 16,777,216 nodes, 67,108,864 edges, out-degree
  power law (exponent 2.5, min 1, mean 4), destinations uniform, 2 states.
* :func:`random_tree`      -- random recursive tree (parent of node i uniform in
  [0, i)), both directions, states per node uniform in {2, 3, 4, 8}.
* :func:`batch_of_networks` -- many independent random networks.
* :func:`grid_mrf`          -- 4-neighbour grid pairwise MRF from log-potentials.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

MAX_STATES = 10


@dataclass
class Network:
    num_states: np.ndarray          # uint32 [V]
    beliefs: np.ndarray             # float32 [V, S_max] (zero beyond num_states)
    observed: np.ndarray            # uint8 [V]
    src: np.ndarray                 # uint32 [E]
    dst: np.ndarray                 # uint32 [E]
    joint: np.ndarray               # float32 [E, S_max, S_max]
    name: str = "network"
    meta: dict = field(default_factory=dict)

    @property
    def V(self) -> int:
        return int(self.num_states.shape[0])

    @property
    def E(self) -> int:
        return int(self.src.shape[0])

    @property
    def s_max(self) -> int:
        return int(self.beliefs.shape[1])

    @property
    def uniform_states(self) -> int:
        """The common state count, or 0 when nodes differ."""
        if self.V == 0:
            return self.s_max
        lo, hi = int(self.num_states.min()), int(self.num_states.max())
        return lo if lo == hi else 0

    def padded(self):
        """(beliefs [V,10], joint [E,10,10]) in the reference's host layout."""
        b = np.zeros((self.V, MAX_STATES), np.float32)
        b[:, : self.s_max] = self.beliefs
        j = np.zeros((self.E, MAX_STATES, MAX_STATES), np.float32)
        j[:, : self.s_max, : self.s_max] = self.joint
        return b, j


def _row_normalised_uniform(rng, n, s):
    t = rng.random((n, s, s), dtype=np.float32)
    return (t / t.sum(axis=2, keepdims=True)).astype(np.float32)


def _dirichlet1(rng, n, s):
    t = rng.exponential(size=(n, s)).astype(np.float32)
    return (t / t.sum(axis=1, keepdims=True)).astype(np.float32)


def _apply_evidence(rng, beliefs, num_states, fraction):
    V = beliefs.shape[0]
    k = int(round(fraction * V))
    observed = np.zeros(V, np.uint8)
    if k == 0:
        return observed
    idx = rng.choice(V, size=k, replace=False)
    state = (rng.random(k) * num_states[idx]).astype(np.int64)
    beliefs[idx] = 0.0
    beliefs[idx, state] = 1.0
    observed[idx] = 1
    return observed


def _dedup_edges(rng, V, src, dst):
    """Redraw destinations until there are no self-loops and no duplicate
    (src, dst) pairs; src (and so each node's out-degree) is kept."""
    src = src.astype(np.int64)
    dst = dst.astype(np.int64)
    for _ in range(64):
        key = src * V + dst
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(len(ks), bool)
        dup[1:] = ks[1:] == ks[:-1]
        bad = np.zeros(len(src), bool)
        bad[order[dup]] = True
        bad |= src == dst
        nbad = int(bad.sum())
        if nbad == 0:
            return src.astype(np.uint32), dst.astype(np.uint32)
        d = rng.integers(0, V - 1, size=nbad)
        s = src[bad]
        d = d + (d >= s)
        dst[bad] = d
    raise RuntimeError("could not remove duplicate edges")


def _uniform_edges(rng, V, E):
    if V < 2 and E > 0:
        raise ValueError("need at least 2 nodes for edges without self-loops")
    if E > V * (V - 1):
        raise ValueError("too many edges for a simple directed graph")
    src = rng.integers(0, V, size=E)
    dst = rng.integers(0, V - 1, size=E)
    dst = dst + (dst >= src)
    src, dst = _dedup_edges(rng, V, src, dst)
    order = np.lexsort((np.arange(E), src))  # group by source, keep draw order
    return src[order], dst[order]


def random_loopy(num_nodes=10_000, num_edges=40_000, states=2, evidence=0.10, seed=0,
                 name="random_loopy"):
    """Uniform random directed graph: endpoints uniform, no self-loops, no
    duplicate edges; row-normalised U(0,1) joint tables; Dirichlet(1) priors;
    a fraction of nodes observed as one-hot evidence."""
    rng = np.random.default_rng(seed)
    V, E, S = int(num_nodes), int(num_edges), int(states)
    src, dst = _uniform_edges(rng, V, E)
    joint = _row_normalised_uniform(rng, E, S)
    num_states = np.full(V, S, np.uint32)
    beliefs = _dirichlet1(rng, V, S)
    observed = _apply_evidence(rng, beliefs, num_states, evidence)
    return Network(num_states, beliefs, observed, src, dst, joint, name=name,
                   meta=dict(seed=seed, kind="random_loopy"))


def power_law_out_degrees(rng, V, E, exponent=2.5):
    """Out-degrees with P(k) ~ k^-exponent, min 1, rescaled to sum exactly E.

    Draws a continuous Pareto (shape exponent-1) with x_min chosen so the mean
    is E/V before flooring, floors, caps at V-1, then adds or removes single
    edges at random nodes (never below 1) until the total is exactly E."""
    a = exponent - 1.0
    mean = E / V
    x_min = mean * (a - 1.0) / a + 0.5  # +0.5 compensates the floor
    deg = np.floor(x_min * (rng.pareto(a, size=V) + 1.0)).astype(np.int64)
    deg = np.clip(deg, 1, V - 1)
    diff = E - int(deg.sum())
    while diff != 0:
        if diff > 0:
            idx = rng.integers(0, V, size=diff)
            np.add.at(deg, idx, 1)
            deg = np.minimum(deg, V - 1)
        else:
            cand = np.flatnonzero(deg > 1)
            idx = rng.choice(cand, size=min(-diff, cand.size), replace=False)
            deg[idx] -= 1
        diff = E - int(deg.sum())
    return deg


def power_law_loopy(num_nodes=1 << 24, num_edges=1 << 26, states=2, evidence=0.10, seed=1,
                    exponent=2.5, name="power_law_loopy"):
    """Power-law out-degree loopy graph (destinations uniform, no self-loops,
    no duplicates), tables and priors as in :func:`random_loopy`."""
    rng = np.random.default_rng(seed)
    V, E, S = int(num_nodes), int(num_edges), int(states)
    deg = power_law_out_degrees(rng, V, E, exponent)
    src = np.repeat(np.arange(V, dtype=np.int64), deg)
    dst = rng.integers(0, V - 1, size=E)
    dst = dst + (dst >= src)
    src, dst = _dedup_edges(rng, V, src, dst)
    joint = _row_normalised_uniform(rng, E, S)
    num_states = np.full(V, S, np.uint32)
    beliefs = _dirichlet1(rng, V, S)
    observed = _apply_evidence(rng, beliefs, num_states, evidence)
    return Network(num_states, beliefs, observed, src, dst, joint, name=name,
                   meta=dict(seed=seed, kind="power_law_loopy", max_out_degree=int(deg.max())))


def random_tree(num_nodes=2_000_000, state_choices=(2, 3, 4, 8), evidence=0.05, seed=1,
                name="random_tree"):
    """Random recursive tree: parent(i) uniform in [0, i).  For every child the
    parent->child edge (table S_parent x S_child) is added, then the
    child->parent edge with the transposed table, the order the BIF parser
    inserts a CPT's two edges (expression.c:756-759)."""
    rng = np.random.default_rng(seed)
    V = int(num_nodes)
    choices = np.asarray(state_choices, np.uint32)
    num_states = choices[rng.integers(0, len(choices), size=V)]
    S = int(choices.max())
    child = np.arange(1, V, dtype=np.int64)
    parent = (rng.random(V - 1) * child).astype(np.int64)
    E = 2 * (V - 1)
    src = np.empty(E, np.uint32)
    dst = np.empty(E, np.uint32)
    src[0::2], dst[0::2] = parent, child
    src[1::2], dst[1::2] = child, parent
    t = rng.random((V - 1, S, S), dtype=np.float32)
    sp = num_states[parent][:, None, None]
    sc = num_states[child][:, None, None]
    ii = np.arange(S)[None, :, None]
    jj = np.arange(S)[None, None, :]
    t = np.where((ii < sp) & (jj < sc), t, 0.0).astype(np.float32)
    t = t / np.maximum(t.sum(axis=2, keepdims=True), np.float32(1e-30))
    joint = np.empty((E, S, S), np.float32)
    joint[0::2] = t
    joint[1::2] = np.transpose(t, (0, 2, 1))
    beliefs = _dirichlet1(rng, V, S)
    beliefs = np.where(np.arange(S)[None, :] < num_states[:, None], beliefs, 0.0).astype(np.float32)
    beliefs /= beliefs.sum(axis=1, keepdims=True)
    observed = _apply_evidence(rng, beliefs, num_states, evidence)
    return Network(num_states, beliefs, observed, src, dst, joint, name=name,
                   meta=dict(seed=seed, kind="random_tree"))


def batch_of_networks(count=4096, v_range=(32, 4096), e_factor=(2.0, 6.0),
                      state_choices=(2, 3, 4, 8), evidence=0.10, seed=2):
    """Independent random networks of uneven size and state count: node
    counts log-uniform in v_range, edge count U(e_factor)*V, one state count per
    network."""
    rng = np.random.default_rng(seed)
    nets = []
    lo, hi = np.log(v_range[0]), np.log(v_range[1])
    for n in range(count):
        V = int(round(np.exp(rng.uniform(lo, hi))))
        E = int(round(rng.uniform(*e_factor) * V))
        S = int(rng.choice(state_choices))
        sub = int(rng.integers(0, 2**31 - 1))
        nets.append(random_loopy(V, E, S, evidence, seed=sub, name=f"net{n}"))
    return nets


def grid_edges(side):
    """Directed 4-neighbour grid edges, right/down edges first as (a, b) then
    the reverse (b, a) right after each, so each undirected pair is a CPT-like
    pair of edges; returns (src, dst, forward_mask)."""
    idx = np.arange(side * side, dtype=np.int64).reshape(side, side)
    a = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel()])
    b = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()])
    E = 2 * a.size
    src = np.empty(E, np.uint32)
    dst = np.empty(E, np.uint32)
    src[0::2], dst[0::2] = a, b
    src[1::2], dst[1::2] = b, a
    fwd = np.zeros(E, bool)
    fwd[0::2] = True
    return src, dst, fwd


def grid_mrf(side=512, states=4, unary_sigma=1.0, pair_sigma=0.5, seed=3):
    """Grid pairwise MRF from log-potentials: priors = softmax(unary), the
    shared table J = exp(W) on forward edges and exp(W)^T on reverse edges.
    Returns (network, unary [V,S], W [S,S], labels [V])."""
    rng = np.random.default_rng(seed)
    V, S = side * side, states
    unary = rng.normal(0.0, unary_sigma, size=(V, S)).astype(np.float32)
    W = rng.normal(0.0, pair_sigma, size=(S, S)).astype(np.float32)
    labels = rng.integers(0, S, size=V).astype(np.int64)
    src, dst, fwd = grid_edges(side)
    J = np.exp(W).astype(np.float32)
    joint = np.where(fwd[:, None, None], J[None], J.T[None]).astype(np.float32)
    pri = np.exp(unary - unary.max(axis=1, keepdims=True))
    pri = (pri / pri.sum(axis=1, keepdims=True)).astype(np.float32)
    net = Network(np.full(V, S, np.uint32), pri, np.zeros(V, np.uint8), src, dst, joint,
                  name=f"grid{side}", meta=dict(seed=seed, kind="grid_mrf", side=side))
    return net, unary, W, labels
