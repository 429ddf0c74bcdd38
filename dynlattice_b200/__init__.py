"""B200-native explicit dynamics of geometrically exact Cosserat rod lattices.

The engine is ``libdynlattice_b200.so`` (C++ host + sm_100a CUDA kernels,
C ABI in ``include/dynlattice.h``); this package holds its ctypes binding,
workload generators and the torch autograd wrapper of its adjoint.
"""
from .abi import (BC, Contact, Material, ModelSpec, DL_PLAIN_FP64, DL_MIXED)  # noqa: F401

__all__ = ["BC", "Contact", "Material", "ModelSpec", "DL_PLAIN_FP64", "DL_MIXED"]
