#!/usr/bin/env python3
"""Random Bayesian-network generator writing XMLBIF 0.3, the format the
reference's XML parser reads (src/bnf-xml-parser/xml-expression.c).

Same command line as the reference's generate_belief_network.py:69-80
(--nodes, --arcs, --seed, --file, --observed-probability) and the same kind of
network: every node has two outcomes (Value1, Value2); a random spanning
structure connects all nodes, then extra arcs are added between random
distinct pairs (always from the lower to the higher id, no repeats) until
`arcs` arcs exist; each arc is a DEFINITION with one GIVEN and a 2x2 table
whose rows sum to 1; a fraction `observed-probability` of the nodes gets a
prior DEFINITION without GIVEN.  The reference's script only runs under
Python 2 (`random.choice(dict.keys())`); this one is Python 3, and draws its
structure with its own seeded generator, so a given --seed gives a different
(equally distributed) network than the reference's.
"""
from __future__ import annotations

import argparse
import random
import sys

HEADER = """<?xml version="1.0"?>
<!-- DTD for the XMLBIF 0.3 format -->
<!DOCTYPE BIF [
    <!ELEMENT BIF ( NETWORK )*>
          <!ATTLIST BIF VERSION CDATA #REQUIRED>
    <!ELEMENT NETWORK ( NAME, ( PROPERTY | VARIABLE | DEFINITION )* )>
    <!ELEMENT NAME (#PCDATA)>
    <!ELEMENT VARIABLE ( NAME, ( OUTCOME |  PROPERTY )* ) >
          <!ATTLIST VARIABLE TYPE (nature|decision|utility) "nature">
    <!ELEMENT OUTCOME (#PCDATA)>
    <!ELEMENT DEFINITION ( FOR | GIVEN | TABLE | PROPERTY )* >
    <!ELEMENT FOR (#PCDATA)>
    <!ELEMENT GIVEN (#PCDATA)>
    <!ELEMENT TABLE (#PCDATA)>
    <!ELEMENT PROPERTY (#PCDATA)>
]>


<BIF VERSION="0.3">
<NETWORK>
<NAME>RandomNet</NAME>"""

FOOTER = """</NETWORK>
</BIF>"""


def parse_arguments(argv=None):
    p = argparse.ArgumentParser(description="Generate a random bayesian network")
    p.add_argument("--nodes", type=int, required=True, help="The number of nodes to generate")
    p.add_argument("--arcs", type=int, required=True, help="The number of arcs to generate")
    p.add_argument("--seed", type=int, default=1, help="The seed to use for generation")
    p.add_argument("--file", type=str, required=True, help="The file to write to")
    p.add_argument("--observed-probability", type=float, default=0.3,
                   help="The probability that a given node is observed")
    a = p.parse_args(argv)
    if a.nodes <= 0:
        p.error(f"The number of nodes ({a.nodes}) must be greater than 0.")
    if a.arcs < a.nodes - 1:
        p.error(f"Arcs ({a.arcs}) must be >= Nodes - 1 ({a.nodes - 1})")
    if a.arcs > a.nodes * (a.nodes - 1) // 2:
        p.error(f"Arcs ({a.arcs}) must be <= Nodes * (Nodes - 1) / 2 ({a.nodes * (a.nodes - 1) // 2})")
    return a


def variable(i):
    return (f'<VARIABLE TYPE="nature">\n<NAME>Node{i}</NAME>\n<OUTCOME>Value1</OUTCOME>\n'
            f'<OUTCOME>Value2</OUTCOME>\n<PROPERTY>position = (0,0)</PROPERTY>\n</VARIABLE>')


def prior(i, p):
    return f"<DEFINITION>\n<FOR>Node{i}</FOR>\n<TABLE>\n{p} {1.0 - p}\n</TABLE>\n</DEFINITION>"


def arc(src, dst, rng):
    a, b = rng.random(), rng.random()
    return (f"<DEFINITION>\n<FOR>Node{dst}</FOR>\n<GIVEN>Node{src}</GIVEN>\n<TABLE>\n"
            f"{a} {1 - a}\n{b} {1 - b}\n</TABLE>\n</DEFINITION>")


def structure(n, arcs, rng):
    """Arcs (src < dst): a random spanning tree over a random node order, then
    random extra pairs without repeats."""
    order = list(range(n))
    rng.shuffle(order)
    edges = []
    seen = set()
    for k in range(1, n):
        u, w = order[k], order[rng.randrange(k)]
        e = (min(u, w), max(u, w))
        seen.add(e)
        edges.append(e)
    while len(edges) < arcs:
        u, w = rng.randrange(n), rng.randrange(n)
        if u == w:
            continue
        e = (min(u, w), max(u, w))
        if e in seen:
            continue
        seen.add(e)
        edges.append(e)
    return edges


def generate_file(a, out=None):
    rng = random.Random(a.seed)
    close = out is None
    out = out or open(a.file, "w")
    try:
        out.write(HEADER)
        for i in range(a.nodes):
            out.write(variable(i))
        k = int(a.observed_probability * a.nodes)
        for i in rng.sample(range(a.nodes), k):
            out.write(prior(i, rng.random()))
        for src, dst in structure(a.nodes, a.arcs, rng):
            out.write(arc(src, dst, rng))
        out.write(FOOTER)
    finally:
        if close:
            out.close()


def main(argv=None):
    generate_file(parse_arguments(argv))
    return 0


if __name__ == "__main__":
    sys.exit(main())
