"""B200 (sm_100a) implementation of k-Wave's first-order k-space time loop.

Drop-in entry points mirroring the reference's MATLAB API:
``kspaceFirstOrder2D``, ``kspaceFirstOrder3D`` and ``kWaveGrid``, plus the
input helpers the reference provides (``makeDisc``, ``makeBall``,
``makeCartCircle``, ``cart2grid``, ``smooth``, ``getWin``).  The loop runs in
the in-tree C-ABI library ``libkwave_b200.so`` (include/kwave_b200.h); there
is no CPU fallback.
"""
from .kgrid import kWaveGrid
from .helpers import (makeDisc, makeBall, makeCartCircle, cart2grid, smooth, getWin, reorderBinarySensorData,
                      TransducerSource)
from .solver import Simulation, Server, kspaceFirstOrder2D, kspaceFirstOrder3D, KWaveInputError
from ._abi import KWaveError, load_library, LIB_PATH

__all__ = [
    "kWaveGrid", "makeDisc", "makeBall", "makeCartCircle", "cart2grid", "smooth", "getWin",
    "reorderBinarySensorData", "TransducerSource", "Simulation", "Server", "kspaceFirstOrder2D", "kspaceFirstOrder3D",
    "KWaveInputError", "KWaveError", "load_library", "LIB_PATH",
]
