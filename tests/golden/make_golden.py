"""Write the golden fixtures of tests/golden/ by running the REFERENCE ITSELF:
its src/graph/graph.c compiled unmodified into oracle/_ref/libref_graph.so
(oracle/Makefile), and its vendored BIF parser (libref_bif.so) for the
bundled networks.  Needs the reference sources (REF, as oracle/oracle.py
reads it; run in the build container):

    make -C oracle reference && python tests/golden/make_golden.py

Each .npz holds the inputs (or the seeded generator call plus a digest of
its output) and the reference's outputs: beliefs, the latest message array,
the returned iteration index, tree-BP beliefs/messages/levels.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import golden_nets as GN  # noqa: E402
import oracle as O  # noqa: E402

BENCH = O.reference_benchmark_files()


def _pack(net):
    s = net.s_max
    return dict(num_states=net.num_states, beliefs=net.beliefs, observed=net.observed, src=net.src,
                dst=net.dst, joint=net.joint[:, :s, :s], name=np.array(net.name))


def _outputs(ref, net, tol, max_it, tree=True, loopy=True):
    out = {}
    S = net.s_max
    if loopy:
        r = ref.loopy(net, tol, max_it)
        out.update(loopy_tol=np.float32(tol), loopy_max_it=np.int64(max_it), loopy_ret=np.int64(r["ret"]),
                   loopy_beliefs=r["beliefs"][:, :S], loopy_latest=r["latest"][:, :S], loopy_older=r["older"][:, :S])
    if tree:
        t = ref.tree(net)
        out.update(tree_beliefs=t["beliefs"][:, :S], tree_messages=t["edges_messages"][:, :S],
                   tree_num_levels=np.int64(t["num_levels"]),
                   tree_levels_nodes=t["levels"][net.V:], tree_levels_offsets=t["levels"][: t["num_levels"]])
    return out


def bif_network(path):
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_bif.so"))
    lib.refbif_load.restype = C.c_void_p
    lib.refbif_load.argtypes = [C.c_char_p]
    g = lib.refbif_load(path.encode())
    if not g:
        raise RuntimeError(f"parse failed: {path}")
    V, E = C.c_uint(), C.c_uint()
    lib.refshim_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    lib.refshim_sizes(g, C.byref(V), C.byref(E))
    V, E = V.value, E.value
    ns = np.zeros(V, np.uint32)
    b = np.zeros((V, 10), np.float32)
    ob = np.zeros(V, np.uint8)
    src = np.zeros(E, np.uint32)
    dst = np.zeros(E, np.uint32)
    j = np.zeros((E, 10, 10), np.float32)
    lib.refshim_dump.argtypes = [C.c_void_p] + [C.c_void_p] * 6
    lib.refshim_dump(g, ns.ctypes.data, b.ctypes.data, ob.ctypes.data, src.ctypes.data, dst.ctypes.data,
                     j.ctypes.data)
    lib.graph_destroy.argtypes = [C.c_void_p]
    lib.graph_destroy(g)
    s = int(ns.max())
    return GN.synth.Network(ns, b[:, :s].copy(), ob, src, dst, j[:, :s, :s].copy(),
                            name=os.path.basename(path).replace(".bif", ""))


def main():
    ref = O.Reference()
    fixtures = {}

    net = GN.example_network()
    fixtures["example_4node.npz"] = dict(_pack(net), **_outputs(ref, net, 1e-9, 10000))

    gen = dict(kind="random_loopy", num_nodes=10000, num_edges=40000, states=2, evidence=0.10, seed=0)
    net = GN.generate(gen["kind"], **{k: v for k, v in gen.items() if k != "kind"})
    fx = {f"gen_{k}": np.array(v) for k, v in gen.items()}
    fx["input_sha"] = np.array(GN.input_digest(net))
    fx.update(_outputs(ref, net, 1e-3, 100, tree=False))
    fixtures["loopy_random_10000_40000.npz"] = fx

    net = GN.synth.random_loopy(500, 2500, 3, 0.1, seed=7)
    fixtures["loopy_random_s3_500.npz"] = dict(_pack(net), **_outputs(ref, net, 1e-3, 50, tree=False))

    net = GN.synth.random_tree(2000, (2,), 0.05, seed=4)
    fixtures["tree_random_2000.npz"] = dict(_pack(net), **_outputs(ref, net, 1e-3, 50, loopy=True))

    # bundled BIF networks whose nodes all have the same state count (the
    # reference's arithmetic is defined there), parsed by the reference parser
    for rel in ("small/asia.bif", "small/cancer.bif", "small/earthquake.bif", "small/sachs.bif"):
        path = os.path.join(BENCH, rel)
        if not os.path.exists(path):
            continue
        net = bif_network(path)
        if net.uniform_states == 0:
            continue
        fixtures[f"bif_{net.name}.npz"] = dict(_pack(net), **_outputs(ref, net, 1e-3, 200))

    for name, fx in fixtures.items():
        np.savez_compressed(os.path.join(HERE, name), **fx)
        print(name, os.path.getsize(os.path.join(HERE, name)))


if __name__ == "__main__":
    main()
