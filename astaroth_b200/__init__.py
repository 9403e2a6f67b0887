"""B200-native single-device Astaroth MHD solver.

The product is the C-ABI library built from astaroth_b200/csrc (see
include/astaroth.h, astaroth_utils.h, astaroth_b200.h); this package holds its
build script and a thin Python mirror of the reference's Device interface.
"""
from . import abi  # noqa: F401
from .device import AcError, Device, Ensemble  # noqa: F401

__all__ = ["abi", "Device", "Ensemble", "AcError"]
