"""virtualcbct_b200: VirtualCBCT's MBFPA forward projection and FDK
reconstruction as hand-written sm_100a CUDA behind a C ABI (include/vcbct.h).

The compute path is libvcbct.so only; there is no CPU fallback.
"""
from . import _native
from ._native import FILTER_BF16X3, FILTER_DIRECT_F32, VcbctError
from .fdk import Fdk, redundancy_weights
from .geometry import FdkGeometry, ProjGeometry, attenuation_table, trig_tables
from .projector import Batch, Projector

__all__ = ["Projector", "Batch", "Fdk", "ProjGeometry", "FdkGeometry", "trig_tables", "attenuation_table",
           "VcbctError", "FILTER_DIRECT_F32", "FILTER_BF16X3", "lib", "redundancy_weights"]


def lib():
    """The loaded C library (raises if it is not built)."""
    return _native.lib()

