"""XMLBIF 0.3 reader without libxml2.

Builds the same graph the reference's parse_xml_file
(src/bnf-xml-parser/xml-expression.c:441-466) builds, as a
:class:`synth.Network`:

* one node per VARIABLE in document order, its state count = number of
  OUTCOMEs, belief DEFAULT_STATE (1.0) per state (add_nodes_to_graph,
  :200-214);
* first pass over DEFINITIONs: each one without GIVEN sets its FOR node's
  belief to the TABLE values and marks it observed (graph_set_node_state,
  :290-317);
* second pass: each DEFINITION with GIVENs walks its parents from the last
  GIVEN to the first, marginalises the CPT onto (parent state, child state)
  with the reference's strided sum (:345-404, float accumulation in the same
  order), and adds the edge parent -> child, then child -> parent with the
  transposed table unless the parent is observed (:408-411).

The TABLE text is the last text node of the element (:236, :258).  Numbers
are parsed to float32 (the reference uses sscanf "%f").
"""
from __future__ import annotations

import xml.etree.ElementTree as ET

import numpy as np

from .synth import Network

MAX_STATES = 10


def _table_values(defn):
    t = defn.find(".//TABLE")
    text = (t.text or "") if t is not None else ""
    # the last text node: text after the last child element, if any
    if t is not None and len(t):
        text = t[-1].tail or ""
    return [np.float32(tok) for tok in text.split()]


def _marginalise(total, slice_, s_src, s_dst, offset):
    """sub_graph[j][k], j < S_src, k < S_dst (xml-expression.c:381-395)."""
    sub = np.zeros((MAX_STATES, MAX_STATES), np.float32)
    n = len(total)
    for k in range(s_dst):
        for j in range(s_src):
            acc = np.float32(0.0)
            diff = 0
            index = j * offset + diff
            while index <= slice_:
                index = j * offset + diff
                nxt = (j + 1) * offset + diff
                while index < nxt:
                    pos = index + k * slice_
                    acc = np.float32(acc + (total[pos] if pos < n else np.float32(0.0)))
                    index += 1
                index += s_src * offset
                diff += s_src * offset
            sub[j, k] = acc
    return sub


def read_xmlbif(path):
    root = ET.parse(path).getroot()
    net = root.find(".//NETWORK")
    variables = net.findall("VARIABLE")
    names = [v.find("NAME").text.strip() for v in variables]
    states = [len(v.findall("OUTCOME")) for v in variables]
    index = {n: i for i, n in enumerate(names)}
    V = len(names)
    S = max(states) if states else 1
    beliefs = np.zeros((V, S), np.float32)
    for i, s in enumerate(states):
        beliefs[i, :s] = 1.0
    observed = np.zeros(V, np.uint8)
    defs = net.findall("DEFINITION")
    for d in defs:
        if d.find("GIVEN") is not None:
            continue
        vals = _table_values(d)
        v = index[d.find("FOR").text.strip()]
        if len(vals) > states[v]:
            raise ValueError(f"prior of {names[v]} has {len(vals)} entries for {states[v]} states")
        beliefs[v, : len(vals)] = vals
        observed[v] = 1
    src, dst, joints = [], [], []
    for d in defs:
        givens = d.findall("GIVEN")
        if not givens:
            continue
        total = _table_values(d)
        dest = index[d.find("FOR").text.strip()]
        slice_ = len(total) // states[dest]
        offset = 1
        for g in reversed(givens):
            s = index[g.text.strip()]
            sub = _marginalise(total, slice_, states[s], states[dest], offset)
            src.append(s)
            dst.append(dest)
            joints.append(sub[:S, :S])
            if observed[s] != 1:
                src.append(dest)
                dst.append(s)
                joints.append(sub.T[:S, :S].copy())
            offset *= states[s]
    joint = np.stack(joints).astype(np.float32) if joints else np.zeros((0, S, S), np.float32)
    return Network(np.asarray(states, np.uint32), beliefs, observed, np.asarray(src, np.uint32),
                   np.asarray(dst, np.uint32), joint, name=str(path),
                   meta=dict(kind="xmlbif", names=names))
