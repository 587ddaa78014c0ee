"""Host mirror of the MBFPA projector interface.

``Projector`` owns a ``vcbct_projector`` handle (the state the reference keeps
in file-scope globals after ``initializeGPU``, reprojectionOnGPU.cu:710-825)
and exposes the forward projection, per-element path integrals, segment count
and adjoint.  Buffers are numpy arrays (host) or CUDA torch tensors (device);
device calls run on the current torch stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .geometry import ProjGeometry


def _is_torch_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def _dp(a):
    return np.ascontiguousarray(a, np.float64).ctypes.data_as(C.POINTER(C.c_double))


def _volume_key(kind, t):
    """Identity of a loaded device volume: storage, version counter, shape."""
    return (kind, t.data_ptr(), t._version, tuple(t.shape))


class Projector:
    """Polychromatic material-based forward projector on one GPU."""

    def __init__(self, geom: ProjGeometry, cos_table, sin_table, xcenter, ycenter):
        self.geom = geom
        self._keep = [np.ascontiguousarray(t, np.float64) for t in (cos_table, sin_table, xcenter, ycenter)]
        for t in self._keep:
            if t.shape[0] < geom.V:
                raise ValueError("view tables shorter than the number of views")
        h = C.c_void_p()
        gc = geom.to_c()
        L = N.lib()
        N.check(L.vcbct_projector_create(C.byref(gc), *[t.ctypes.data_as(C.POINTER(C.c_double)) for t in self._keep],
                                         C.byref(h)))
        self._h = h
        self.NE = 0
        self.loaded = None  # key of the device volume last loaded, if any

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().vcbct_projector_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- inputs --
    def set_spectrum(self, mu, pdf, xfactor: float):
        mu = np.ascontiguousarray(mu, np.float32)
        pdf = np.ascontiguousarray(pdf, np.float32)
        if mu.ndim != 2 or mu.shape[0] != self.geom.nmat or mu.shape[1] != pdf.shape[0]:
            raise ValueError("mu must be [nmat][NE] and pdf [NE]")
        N.check(N.lib().vcbct_projector_set_spectrum(self._h, mu.ctypes.data_as(C.POINTER(C.c_float)),
                                                     pdf.ctypes.data_as(C.POINTER(C.c_float)),
                                                     int(pdf.shape[0]), float(xfactor)))
        self.NE = int(pdf.shape[0])

    def _check_vol(self, vol, dtype_name):
        g = self.geom
        shape = (g.Z, g.nmat, g.N, g.N)
        if tuple(vol.shape) != shape:
            raise ValueError(f"volume must be {dtype_name} {shape}, got {tuple(vol.shape)}")

    def load_volume(self, vol, stream=None):
        """uint16 [Z][nmat][N][N] element volume (host numpy or CUDA torch)."""
        self._check_vol(vol, "uint16")
        L = N.lib()
        if _is_torch_cuda(vol):
            import torch
            if vol.dtype not in (torch.uint16, torch.int16):
                raise ValueError("device volume must be uint16/int16 bits")
            v = vol.contiguous()
            N.check(L.vcbct_projector_load_volume(self._h, C.c_void_p(v.data_ptr()), 1, _stream_ptr(stream)))
            self._vol_ref = v
            self.loaded = _volume_key("u16", v)
        else:
            v = np.ascontiguousarray(vol, np.uint16)
            N.check(L.vcbct_projector_load_volume(self._h, C.c_void_p(v.ctypes.data), 0, None))
            self.loaded = None

    def load_deck(self, deck: dict, stream=None) -> int:
        """Stream a projector deck's slice files (``decks.read_proj_deck``)
        into the device volume; returns the number of missing or short
        slice files."""
        bad = C.c_int(0)
        N.check(N.lib().vcbct_projector_load_deck(self._h, C.byref(deck["_c"]), C.byref(bad), _stream_ptr(stream)))
        self.loaded = None
        return int(bad.value)

    def load_volume_f32(self, vol, stream=None):
        """float32 [Z][nmat][N][N] element volume (host numpy or CUDA torch)."""
        self._check_vol(vol, "float32")
        L = N.lib()
        if _is_torch_cuda(vol):
            v = vol.contiguous()
            N.check(L.vcbct_projector_load_volume_f32(self._h, C.c_void_p(v.data_ptr()), 1, _stream_ptr(stream)))
            self._vol_ref = v
            self.loaded = _volume_key("f32", v)
        else:
            v = np.ascontiguousarray(vol, np.float32)
            N.check(L.vcbct_projector_load_volume_f32(self._h, C.c_void_p(v.ctypes.data), 0, None))
            self.loaded = None

    # ------------------------------------------------------------ outputs --
    def forward(self, out=None, stream=None):
        """Spectral projection float [V][H][W].  With a CUDA torch ``out`` (or
        out=None and torch available) the result stays on the device; with a
        numpy ``out`` it is copied to the host."""
        g = self.geom
        L = N.lib()
        if out is None:
            import torch
            out = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device="cuda")
        if _is_torch_cuda(out):
            N.check(L.vcbct_projector_forward(self._h, C.c_void_p(out.data_ptr()), 1, _stream_ptr(stream)))
        else:
            if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != g.V * g.H * g.W:
                raise ValueError("host out must be contiguous float32 [V][H][W]")
            N.check(L.vcbct_projector_forward(self._h, C.c_void_p(out.ctypes.data), 0, None))
        return out

    def project(self, vol, out=None):
        """Host uint16 volume [Z][nmat][N][N] in, host projections float
        [V][H][W] out, in one call (``vcbct_projector_project``): the volume's
        upload overlaps the projection.  Bitwise ``load_volume`` + ``forward``;
        the volume stays loaded."""
        g = self.geom
        self._check_vol(vol, "uint16")
        v = np.ascontiguousarray(vol, np.uint16)
        if out is None:
            out = np.empty((g.V, g.H, g.W), np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != g.V * g.H * g.W:
            raise ValueError("host out must be contiguous float32 [V][H][W]")
        N.check(N.lib().vcbct_projector_project(self._h, C.c_void_p(v.ctypes.data), C.c_void_p(out.ctypes.data),
                                                None))
        self.loaded = None
        return out

    def path_integrals(self, stream=None):
        import torch
        g = self.geom
        Lb = torch.empty((g.V, g.H, g.W, g.nmat), dtype=torch.float32, device="cuda")
        N.check(N.lib().vcbct_projector_path_integrals(self._h, C.c_void_p(Lb.data_ptr()), _stream_ptr(stream)))
        return Lb

    def count_segments(self, stream=None) -> int:
        tot = C.c_ulonglong(0)
        N.check(N.lib().vcbct_projector_count_segments(self._h, C.byref(tot), _stream_ptr(stream)))
        return int(tot.value)

    def autotune(self, stream=None) -> int:
        """Pick the fastest launch shape for this geometry (see vcbct.h)."""
        import torch
        g = self.geom
        tmp = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device="cuda")
        c = C.c_int(0)
        N.check(N.lib().vcbct_projector_autotune(self._h, C.c_void_p(tmp.data_ptr()), _stream_ptr(stream),
                                                 C.byref(c)))
        return c.value

    def forward_state(self, out=None, L=None, stream=None):
        """Device projection [V][H][W] and per-ray path integrals
        L [V][H][W][nmat] in one launch (for adjoint_state)."""
        import torch
        g = self.geom
        if out is None:
            out = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device="cuda")
        if L is None:
            L = torch.empty((g.V, g.H, g.W, g.nmat), dtype=torch.float32, device="cuda")
        N.check(N.lib().vcbct_projector_forward_state(self._h, C.c_void_p(out.data_ptr()),
                                                      C.c_void_p(L.data_ptr()), _stream_ptr(stream)))
        return out, L

    def adjoint_state(self, L, grad_out, grad=None, stream=None):
        """adjoint() with the path integrals L of forward_state instead of a
        recomputing march."""
        import torch
        g = self.geom
        if grad is None:
            grad = torch.zeros((g.Z, g.nmat, g.N, g.N), dtype=torch.float32, device="cuda")
        go = grad_out.contiguous()
        N.check(N.lib().vcbct_projector_adjoint_state(self._h, C.c_void_p(L.data_ptr()),
                                                      C.c_void_p(go.data_ptr()),
                                                      C.c_void_p(grad.data_ptr()), _stream_ptr(stream)))
        return grad

    def set_noise(self, i0: float = 0.0, max_counts: float = 65535.0, seed: int = 0, model: str = "gaussian"):
        """Detector noise on the projections (i0 = counts of an unattenuated
        ray; i0 = 0 turns it off): model "gaussian" (the reference's n +
        sqrt(n) z) or "poisson" (exact Poisson counts)."""
        if model not in ("gaussian", "poisson"):
            raise ValueError("model must be 'gaussian' or 'poisson'")
        kind = 0 if i0 <= 0 else (1 if model == "gaussian" else 2)
        N.check(N.lib().vcbct_projector_set_noise(self._h, kind, float(i0), float(max_counts), int(seed)))

    def lengthproj(self, proj, ite: int = 0, views=None, npf=None, stream=None):
        """Sensitivity backprojection of uint16 projections [V][H][W]
        (lengthproj.cpp:10-131): float [Z][N][N], host or device like proj."""
        g = self.geom
        v0, v1 = (0, g.V) if views is None else views
        L = N.lib()
        if _is_torch_cuda(proj):
            import torch
            pr = proj.contiguous()
            if pr.dtype not in (torch.int16, torch.uint16):
                raise ValueError("device projections must be uint16/int16 bits")
            if npf is None:
                npf = torch.empty((g.Z, g.N, g.N), dtype=torch.float32, device=pr.device)
            N.check(L.vcbct_projector_lengthproj(self._h, int(ite), int(v0), int(v1), C.c_void_p(pr.data_ptr()), 1,
                                                 C.c_void_p(npf.data_ptr()), 1, _stream_ptr(stream)))
            return npf
        pr = np.ascontiguousarray(proj, np.uint16)
        if pr.shape != (g.V, g.H, g.W):
            raise ValueError("projections must be uint16 [V][H][W]")
        if npf is None:
            npf = np.empty((g.Z, g.N, g.N), np.float32)
        N.check(L.vcbct_projector_lengthproj(self._h, int(ite), int(v0), int(v1), C.c_void_p(pr.ctypes.data), 0,
                                             C.c_void_p(npf.ctypes.data), 0, None))
        return npf

    def adjoint(self, grad_out, grad=None, stream=None):
        """Accumulate d loss / d volume (float [Z][nmat][N][N], device) for a
        device d loss / d projection ``grad_out`` [V][H][W]."""
        import torch
        g = self.geom
        if grad is None:
            grad = torch.zeros((g.Z, g.nmat, g.N, g.N), dtype=torch.float32, device="cuda")
        go = grad_out.contiguous()
        N.check(N.lib().vcbct_projector_adjoint(self._h, C.c_void_p(go.data_ptr()),
                                                C.c_void_p(grad.data_ptr()), _stream_ptr(stream)))
        return grad


class Batch:
    """Several projectors (uneven phantoms, view sets and detectors) projected
    by one persistent launch, optionally replayed from a captured CUDA graph."""

    def __init__(self):
        h = C.c_void_p()
        N.check(N.lib().vcbct_batch_create(C.byref(h)))
        self._h = h
        self._items = []

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            N.lib().vcbct_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, projector: Projector, out=None):
        """Add a projector (volume and spectrum loaded); returns its
        device output tensor [V][H][W]."""
        import torch
        g = projector.geom
        if out is None:
            out = torch.empty((g.V, g.H, g.W), dtype=torch.float32, device="cuda")
        N.check(N.lib().vcbct_batch_add(self._h, projector._h, C.c_void_p(out.data_ptr())))
        self._items.append((projector, out))
        return out

    def forward(self, use_graph: bool = True, stream=None):
        N.check(N.lib().vcbct_batch_forward(self._h, int(bool(use_graph)), _stream_ptr(stream)))
        return [o for _, o in self._items]

    PERSISTENT, PER_ITEM, FLAT = 0, 1, 2

    def configure(self, strategy: int = 0, cols_per_block: int = 4):
        """Fix the launch strategy: Batch.PERSISTENT (one persistent launch),
        Batch.PER_ITEM (per-item launches on two graph branches) or
        Batch.FLAT (one launch, a block per tile); and the columns per block."""
        N.check(N.lib().vcbct_batch_configure(self._h, int(strategy), int(cols_per_block)))

    def autotune(self, stream=None) -> int:
        """Time the three strategies x {2, 4, 8} columns per block and keep
        the fastest; returns columns per block + 100 x strategy."""
        c = C.c_int(0)
        N.check(N.lib().vcbct_batch_autotune(self._h, _stream_ptr(stream), C.byref(c)))
        return c.value
