"""B200 FlexMesh hot path: Neo-Hookean tet assembly -> CSR -> ILU(0)-PCG -> Newton.

The compute lives in libflexmesh_b200.so (sm_100a kernels behind the C ABI of
include/fm_api.h); this package binds it for Python callers and mirrors the
reference's solver API (see ``solver``).
"""
from ._lib import (FLAG_BREAKDOWN, FLAG_INVERTED, FLAG_J_CLAMPED, FLAG_NONFINITE, FLAG_PIVOT,
                   FLAG_TIMEOUT, FM_FP64, FM_MIXED, FM_PATTERN_REFERENCE, FM_PATTERN_SOLVE,
                   Context, FMError, lib, unit_cube)

__all__ = ["Context", "FMError", "lib", "unit_cube", "FM_FP64", "FM_MIXED",
           "FM_PATTERN_REFERENCE", "FM_PATTERN_SOLVE", "FLAG_NONFINITE", "FLAG_INVERTED",
           "FLAG_J_CLAMPED", "FLAG_PIVOT", "FLAG_TIMEOUT", "FLAG_BREAKDOWN"]
