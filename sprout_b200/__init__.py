"""sprout_b200: B200-native (sm_100a) ray-cast hot path of the sprout renderer.

The native library (``libsprout_b200.so``, built from ``csrc/`` by ``build.py``) carries
the CUDA kernels and the C ABI declared in ``include/sprout_b200.h``; this package is a thin
ctypes layer over it.
"""

from ._lib import SproutError, load  # noqa: F401
from .cast import MISS, Tree, random_rays, sphere_mesh  # noqa: F401

__all__ = ["Tree", "MISS", "SproutError", "load", "sphere_mesh", "random_rays"]
