"""krigekit_b200 -- the krigekit kriging solve path on one NVIDIA B200.

Drop-in replacements for krigekit's ``Kriging`` and ``SpaceTimeKriging`` (and
helper functions) whose
search, covariance assembly and solves run as hand-written sm_100a CUDA
kernels in ``libkrigecuda.so``, called through the krige_* C-ABI.
"""
from .kriging import Kriging, cokriging, ordinary_kriging, sequential_gaussian_simulation  # noqa: F401
from .kriging_indicator import IndicatorKriging  # noqa: F401
from .kriging_st import SpaceTimeKriging, spacetime_cokriging, spacetime_kriging  # noqa: F401

__all__ = ["Kriging", "ordinary_kriging", "cokriging", "sequential_gaussian_simulation", "IndicatorKriging",
           "SpaceTimeKriging",
           "spacetime_kriging", "spacetime_cokriging"]
__version__ = "0.1.0"
