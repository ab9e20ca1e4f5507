"""tdse_nd_mpi_b200 — B200-native split-operator TDSE engine (QuantumND hot path).

The compute path is libqnd_b200.so (hand-written sm_100a CUDA behind the C ABI in
include/qnd.h); this package is a thin host-side mirror of the reference's
interface over that ABI. See :mod:`tdse_nd_mpi_b200.engine`.
"""
from ._lib import LIB_PATH, QndError
from .engine import DeviceState, Grid, obs_width

__all__ = ["Grid", "DeviceState", "QndError", "obs_width", "LIB_PATH"]
