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
           "VcbctError", "FILTER_DIRECT_F32", "FILTER_BF16X3", "lib", "probe_gather", "redundancy_weights"]


def lib():
    """The loaded C library (raises if it is not built)."""
    return _native.lib()


def probe_gather(kind: int, stream=None) -> float:
    """Measured gather roofline (vcbct_probe_gather): kind 0 = forward
    projector pattern, lane-records/s; kind 1 / 2 = backprojector pattern
    from shared memory / through L1, voxel updates/s."""
    import ctypes as C

    from .projector import _stream_ptr
    r = C.c_double(0.0)
    _native.check(_native.lib().vcbct_probe_gather(int(kind), C.byref(r), _stream_ptr(stream)))
    return float(r.value)
