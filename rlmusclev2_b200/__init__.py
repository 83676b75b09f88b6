"""B200-native (sm_100a) XPBD muscle substep: a drop-in for the XpbdEngine path
of chunleili/rlmuscleV2 (MuscleSim / MultiGridSim).

Python host code keeps the reference's engine API and JSON configs; all
compute runs in libxpbd_b200.so (hand-written CUDA for sm_100a) through the
C ABI in include/xpbd_b200.h.
"""
from .defs import ConstraintType, FemFlag
from .engine import XpbdEngine, XpbdSolver
from .musclesim import MuscleSim

__all__ = ["ConstraintType", "FemFlag", "XpbdEngine", "XpbdSolver", "MuscleSim"]
