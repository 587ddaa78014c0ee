"""Measurement support for bench.py and the profiler captures in profiles/.

Not part of the product library: ``libgather_probe.so`` (built from
``gather_probe.cu`` by ``measure/Makefile``) replays the two gather-bound
kernels' access patterns without arithmetic, giving the measured gather
rooflines; ``profile_cases`` holds the small launches the ncu captures run.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "libgather_probe.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        _LIB = C.CDLL(path)
        _LIB.gather_probe_run.restype = C.c_int
        _LIB.gather_probe_run.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_void_p]
        _LIB.gather_probe_error.restype = C.c_char_p
    return _LIB


def probe_gather(kind: int, stream=None) -> float:
    """Measured gather roofline on the current device: kind 0 / 3 = the
    forward projector's ray-front pattern over 16-byte uint16 / 32-byte float
    records (lane-records/s); kind 1 / 2 = the backprojector's bilinear
    pattern from shared memory / through L1 (voxel updates/s)."""
    L = _lib()
    r = C.c_double(0.0)
    sp = None if stream is None else C.c_void_p(stream.cuda_stream)
    rc = L.gather_probe_run(int(kind), C.byref(r), sp)
    if rc != 0:
        raise RuntimeError(f"gather probe failed ({rc}): {L.gather_probe_error().decode()}")
    return float(r.value)
