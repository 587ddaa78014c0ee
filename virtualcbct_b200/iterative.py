"""The iterative-reconstruction update of the projector program
(IR_ImageCBCT.cpp:19-93) on the GPU; the sensitivity backprojection that
feeds it is ``Projector.lengthproj``."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .projector import _is_torch_cuda, _stream_ptr


def ir_update(before, npf, npf_re, scale: float, wbefore: float, weight_tv: float = 0.0,
              weight_prior: float = 0.0, out=None, stream=None):
    """out = before * (wbefore + (1 - wbefore) * npf_re / (npf + weight_tv *
    TV(before) + 1e-6)), clamped and masked as the reference does.
    ``before`` short [Z][N][N]; ``npf``, ``npf_re`` float [Z][N][N]; all host
    (numpy) or all CUDA tensors."""
    Z, n1, n2 = before.shape
    if n1 != n2:
        raise ValueError("volumes must be [Z][N][N]")
    L = N.lib()
    if _is_torch_cuda(before):
        import torch
        b, a, r = before.contiguous(), npf.contiguous(), npf_re.contiguous()
        if out is None:
            out = torch.empty((Z, n1, n1), dtype=torch.float32, device=b.device)
        N.check(L.vcbct_ir_update(n1, Z, float(scale), C.c_void_p(b.data_ptr()), C.c_void_p(out.data_ptr()),
                                  C.c_void_p(a.data_ptr()), C.c_void_p(r.data_ptr()), float(wbefore),
                                  float(weight_tv), float(weight_prior), 1, _stream_ptr(stream)))
        return out
    b = np.ascontiguousarray(before, np.int16)
    a = np.ascontiguousarray(npf, np.float32)
    r = np.ascontiguousarray(npf_re, np.float32)
    out = np.empty((Z, n1, n1), np.float32) if out is None else out
    N.check(L.vcbct_ir_update(n1, Z, float(scale), C.c_void_p(b.ctypes.data), C.c_void_p(out.ctypes.data),
                              C.c_void_p(a.ctypes.data), C.c_void_p(r.ctypes.data), float(wbefore),
                              float(weight_tv), float(weight_prior), 0, None))
    return out
