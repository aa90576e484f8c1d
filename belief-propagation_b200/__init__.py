"""belief_propagation_b200 -- B200-native belief propagation.

The product is the C-ABI library ``lib/libbp.so`` (sources in ``csrc/``): a
drop-in implementation of the reference's C graph API (``include/graph.h``)
plus an extended device-resident API (``include/bp.h``), both running
hand-written sm_100a CUDA kernels.  This Python package is the thin wrapper
over that library (ctypes; PyTorch only for device memory and autograd).

The directory name contains a hyphen, so it is registered under the module
name ``belief_propagation_b200`` by ``belief_network_wrapper.load_package()``
(or by anything that loads it from its path).
"""
from . import synth  # noqa: F401

__all__ = ["synth"]
