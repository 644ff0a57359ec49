"""B200-native (sm_100a, FP64) spatial discretization of the 2D Euler ALE equations.

A drop-in for PyEulerALE's ``SpatialDiscretization`` (``src/py_euler_ale/__init__.py``):
the same class API, backed by hand-written CUDA kernels reached through the C ABI of
``include/euler_b200.h``.
"""

from .grid import HEAT_RATIO, NUM_DIM, NUM_VAR

__all__ = ["HEAT_RATIO", "NUM_DIM", "NUM_VAR", "SpatialDiscretization"]


def __getattr__(name):
    if name == "SpatialDiscretization":
        from .core import SpatialDiscretization

        return SpatialDiscretization
    raise AttributeError(name)
