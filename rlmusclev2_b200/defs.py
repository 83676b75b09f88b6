"""Constraint-type tags and FEM flags (values of src/muscle/defs.py:20-42).

The integer values are the reference's, so a constraint table sorted by tag
visits types in the same order as the reference's per-type dispatch.
"""
from __future__ import annotations

from enum import IntEnum, IntFlag


class ConstraintType(IntEnum):
    PIN = 157323
    ATTACH = 1650556
    PINTOTARGET = 771624311
    TETVOLUME = -215389979
    TETFIBERNORM = -303462111
    DISTANCELINE = 1621136047
    TETARAP = -92199131
    TETARAPSVD = -92199132
    TETARAPNORM = -885573303
    TETARAPANISO = -92199133
    TETFIBERDGF = -403562211
    TETSNH = -503462311
    TETFIBERMILLARD = -503662411
    DISTANCE = 1621136100
    TETVOLUMEHARD = -215389990
    TETINVERSION = -215389991


class FemFlag(IntFlag):
    LINEARENERGY = 1 << 0
    NORMSTIFFNESS = 1 << 1


# Types the sm_100a path projects (the rest of the reference's catalogue is
# outside this project's hot path).
SUPPORTED_TET_TYPES = (ConstraintType.TETARAPSVD, ConstraintType.TETVOLUME, ConstraintType.TETARAPANISO,
                       ConstraintType.TETSNH)
