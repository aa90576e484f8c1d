#!/usr/bin/env python3
"""belief_network_wrapper.py -- drop-in for the reference's
belief_network_wrapper.py, plus the Python front end of the CUDA engine.

Run as a script it keeps the reference's behaviour
(belief_network_wrapper.py:5-14): for node counts 200k..900k in steps of
100k (skipping 500k) it calls generate_belief_network.py with
arcs = 2 * nodes and writes src/benchmark_files/xml2/<nodes>_<arcs>.xml.

Imported, it registers the engine package (directory
``belief-propagation_b200/``) as ``belief_propagation_b200`` and exposes it as
``bp``.
"""
from __future__ import annotations

import importlib.util
import os
import subprocess
import sys

_HERE = os.path.dirname(os.path.abspath(__file__))
PACKAGE_DIR = os.path.join(_HERE, "belief-propagation_b200")
PACKAGE_NAME = "belief_propagation_b200"


def load_package():
    """Import the engine package from its (hyphenated) directory."""
    if PACKAGE_NAME in sys.modules:
        return sys.modules[PACKAGE_NAME]
    spec = importlib.util.spec_from_file_location(
        PACKAGE_NAME, os.path.join(PACKAGE_DIR, "__init__.py"),
        submodule_search_locations=[PACKAGE_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[PACKAGE_NAME] = mod
    try:
        spec.loader.exec_module(mod)
    except BaseException:
        del sys.modules[PACKAGE_NAME]
        raise
    return mod


bp = load_package()


def main():
    i = 100000
    while i < 1000000:
        if i != 100000 and i != 500000:
            num_nodes = int(i)
            num_arcs = 2 * num_nodes
            file_name = 'src/benchmark_files/xml2/%d_%d.xml' % (num_nodes, num_arcs)
            subprocess.call([sys.executable, os.path.join(_HERE, 'generate_belief_network.py'),
                             '--nodes', str(num_nodes), '--arcs', str(num_arcs), '--file', file_name])
        i += 100000


if __name__ == '__main__':
    main()
