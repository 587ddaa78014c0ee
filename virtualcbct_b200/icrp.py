"""Organ-labelled voxel phantoms to element volumes, the conversion of
ICRPphantoms_2mmslice/To_material_distribution_for512_random.cpp: jittered
media and organ tables read by the C library (``vcbct_phantom_tables_read``)
and a GPU table lookup (``vcbct_organs_to_elements``) producing the
projector's uint16 [Z][6][rows][cols] input."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .projector import _is_torch_cuda, _stream_ptr


class PhantomTables:
    """Jittered media (H, C, N, O, P, Ca mass percentages), organ rows and
    the per-organ-number element table (uint16 [256][6])."""

    def __init__(self, media_csv, organs_csv, seed: int = 1):
        self._c = N.PhantomTablesC()
        N.check(N.lib().vcbct_phantom_tables_read(str(media_csv).encode(), str(organs_csv).encode(),
                                                   int(seed), C.byref(self._c)))

    @property
    def table(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._c.table).reshape(256, 6).copy()

    @property
    def media(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._c.media).reshape(100, 6)[: self._c.n_media].copy()


def organs_to_elements(ids, tables: PhantomTables, out=None, stream=None):
    """uint8 organ numbers [Z][rows][cols] (numpy or CUDA tensor) ->
    uint16 element values [Z][6][rows][cols] (int16 bits for a tensor)."""
    Z = ids.shape[0]
    slice_voxels = int(np.prod(ids.shape[1:]))
    L = N.lib()
    if _is_torch_cuda(ids):
        import torch
        src = ids.contiguous()
        if src.dtype != torch.uint8:
            raise ValueError("organ numbers must be uint8")
        if out is None:
            out = torch.empty((Z, 6) + tuple(ids.shape[1:]), dtype=torch.int16, device=src.device)
        N.check(L.vcbct_organs_to_elements(C.c_void_p(src.data_ptr()), slice_voxels, Z, C.byref(tables._c),
                                           C.c_void_p(out.data_ptr()), 1, _stream_ptr(stream)))
        return out
    src = np.ascontiguousarray(ids, np.uint8)
    out = np.empty((Z, 6) + tuple(ids.shape[1:]), np.uint16) if out is None else out
    N.check(L.vcbct_organs_to_elements(C.c_void_p(src.ctypes.data), slice_voxels, Z, C.byref(tables._c),
                                       C.c_void_p(out.ctypes.data), 0, None))
    return out
