"""Networks and expected values the tests pin against.

* example_network(): the 4-node MRF of the reference's known-answer test
  (src/example-belief-propagation/example-belief-propagation.c:17-70), built
  the way that program builds it; EXAMPLE_MARGINALS are the marginals its
  validate_nodes() asserts to 1e-4 (:72-107).
* network_from_fixture(): rebuilds a Network from a fixture written by
  make_golden.py (either stored arrays or the seeded generator call).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import belief_network_wrapper as W  # noqa: E402

synth = W.bp.synth

EXAMPLE_MARGINALS = np.array([[0.521531100478469, 0.47846889952153115],
                              [0.9090909090909091, 0.09090909090909091],
                              [0.1652892561983471, 0.8347107438016529],
                              [1.0, 0.0]])


def example_network():
    """x1, x2, x3 flat (DEFAULT_STATE 1.0), y2 observed (1, 0); edges
    x1->x2, x2->x1 (phi12), x2->x3, x3->x2 (phi23), y2->x2 (phi24)."""
    phi12 = np.array([[1.0, 0.9], [0.9, 1.0]], np.float32)
    phi23 = np.array([[0.1, 1.0], [1.0, 0.1]], np.float32)
    phi24 = np.array([[1.0, 0.1], [0.1, 1.0]], np.float32)
    beliefs = np.array([[1, 1], [1, 1], [1, 1], [1, 0]], np.float32)
    src = np.array([0, 1, 1, 2, 3], np.uint32)
    dst = np.array([1, 0, 2, 1, 1], np.uint32)
    joint = np.stack([phi12, phi12, phi23, phi23, phi24]).astype(np.float32)
    return synth.Network(np.full(4, 2, np.uint32), beliefs, np.array([0, 0, 0, 1], np.uint8), src, dst, joint,
                         name="example_4node")


def generate(kind, **kw):
    return getattr(synth, kind)(**kw)


def network_from_fixture(fx):
    if "gen_kind" in fx:
        kw = {k[4:]: (v.item() if v.ndim == 0 else tuple(v.tolist())) for k, v in fx.items()
              if k.startswith("gen_") and k != "gen_kind"}
        net = generate(str(fx["gen_kind"]), **kw)
        digest = input_digest(net)
        if "input_sha" in fx and str(fx["input_sha"]) != digest:
            raise AssertionError("seeded generator output changed: fixture no longer matches its inputs")
        return net
    return synth.Network(fx["num_states"], fx["beliefs"], fx["observed"], fx["src"], fx["dst"], fx["joint"],
                         name=str(fx.get("name", "fixture")))


def input_digest(net):
    import hashlib
    h = hashlib.sha256()
    for a in (net.num_states, net.beliefs, net.observed, net.src, net.dst, net.joint):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()
