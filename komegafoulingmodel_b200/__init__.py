"""B200-native D2Q9 + k-omega time step of kOmegaFoulingModel.

The hot path (collide-stream, k-omega assembly, implicit k/omega solve,
diagnostics) is hand-written sm_100a CUDA in csrc/, exposed through the C ABI
of include/kofm.h and built into libkofm.so next to this file.  This package
is the Python handle on that library (ctypes) plus host-side set-up.
"""
from . import _abi, geometry
from ._abi import KofmDesc, KofmError, KofmStats
from .lattice import Lattice, desc_default

__all__ = ["Lattice", "desc_default", "KofmDesc", "KofmStats", "KofmError", "geometry", "_abi"]
