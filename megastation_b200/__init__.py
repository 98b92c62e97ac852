"""B200-native (sm_100a) MegaStation per-slot baseband hot path.

The compute lives in libmegastation_b200.so behind the C ABI of
include/megastation_b200.h; this package binds it (ops) and sequences it per
slot (slot).  Importing raises when the shared library is missing.
"""
from . import _lib  # noqa: F401  (loads the shared library or raises)
from .ops import (Beamform, DownlinkIFFT, Equalize, Ldpc, Modulation, PilotFFT, Precode,  # noqa: F401
                  Scrambler, UplinkFFT, dmrs_table, ldpc_sizes, pilot_sign)

__version__ = "0.1.0"
