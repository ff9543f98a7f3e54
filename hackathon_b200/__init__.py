"""B200-native (sm_100a) implementation of motility-ddm's DDM analysis path.

The compute path is the CUDA library hackathon_b200/_lib/libddm_b200.so
(sources in csrc/, C ABI in include/ddm_b200.h); ``DdmEngine`` mirrors the
reference's engine API over that ABI.
"""
from .engine import DdmEngine, DdmError, DdmArgError  # noqa: F401
from .radial import Radial  # noqa: F401
