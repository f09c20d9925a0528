"""B200-native Total-FETI dual iteration behind ESPRESO's FETI4I C API.

The solver is libfeti4i_b200.so (C++ host preprocessing + sm_100a CUDA
kernels, built in-tree by ``espreso_b200.build``); ``espreso_b200.feti4i``
binds its C ABI and ``espreso_b200.problems`` generates synthetic callers.
"""
from . import feti4i, problems  # noqa: F401
