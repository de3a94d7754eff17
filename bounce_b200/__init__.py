"""B200-native collision pipeline for the Bounce physics engine.

The compute path is the CUDA library ``libb3g.so`` (C ABI in include/b3g.h);
this package holds its Python host mirror (``pipeline``), the seeded scene
generators and kinematic driver (``scene``) and the ctypes loader.
"""
from . import _native  # noqa: F401
from ._native import B3GError, MANIFOLD_DTYPE, POINT_DTYPE, load  # noqa: F401
