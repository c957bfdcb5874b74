"""``make_sht("cuda", ...)``: the Gauss-Legendre transform on the GPU behind the reference's
transform interface (SLEvolve ``python/slevolve/sht.py:43-46``, ``sht_ducc.py:206-217``).

``CudaSHT(nlat, nlon, lmax)``
    ``analysis(grid[nlat, nlon] float64, out=None) -> coeffs[lmax+1, lmax+1] complex128``
    ``synthesis(coeffs, out=None) -> grid``

``raw=True`` is the sign-free convention of the reference's ducc backend (sht_ducc.py:101-110):
``analysis`` returns V[l, m] = (-1)^m U[l, m] and ``synthesis`` reads V.  The ``*_device`` entry
points always use U.

``precision="mixed"`` runs the Legendre contractions as split-TF32 tensor-core GEMMs with FP32
accumulation (FP64 recurrence, row FFTs and degree-0 coefficient); the default ``"fp64"`` matches
the reference to round-off.

Inputs may be NumPy arrays (copied to the device and back) or CUDA ``torch`` tensors (used in
place, results stay on the device).  With ``out=None`` the NumPy path returns an internal buffer
that the next call overwrites, exactly like the reference (sht.py:297-302, 339-343).
Attributes read by the reference callers: ``gaulats``, ``weights``, ``table_bytes``, ``raw``,
``nthreads``, ``mean00_weights()``.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

SQRT2_LEGACY = 1.41421356


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("slevolve_b200 needs a CUDA device; none is available")
    return torch


def _stream_ptr(torch):
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class CudaSHT:
    """Pseudo-spectral transform on a Gauss-Legendre grid, legacy conventions, on the GPU."""

    backend = "cuda"

    def __init__(self, nlat: int, nlon: int, lmax: int, workers: int = 1, chunk: int = 16,
                 raw: bool = False, precision: str = "fp64"):
        if nlat % 2 != 0:
            raise ValueError("nlat must be even")
        if lmax > nlon // 2:
            raise ValueError("lmax must be <= nlon/2")
        L = _lib.lib()
        torch = _torch()
        h = C.c_void_p()
        _lib.check(L.sle_sht_create(int(nlat), int(nlon), int(lmax), C.byref(h)), "sle_sht_create")
        self._h = h
        self._L = L
        self.precision = "mixed" if _lib.precision_code(precision) == _lib.PREC_MIXED else "fp64"
        _lib.check(L.sle_sht_set_precision(h, _lib.precision_code(precision)), "sle_sht_set_precision")
        self.nlat, self.nlon, self.lmax = int(nlat), int(nlon), int(lmax)
        self.nm = self.lmax + 1
        self.nh = self.nlat // 2
        self.raw = bool(raw)
        self.workers = int(workers)
        self.nthreads = int(workers)
        nc = C.c_longlong()
        _lib.check(L.sle_sht_info(h, None, None, None, C.byref(nc)), "sle_sht_info")
        self.ncoef = int(nc.value)
        mu = np.empty(self.nlat)
        w = np.empty(self.nlat)
        _lib.check(L.sle_sht_gauss(h, mu.ctypes.data, w.ctypes.data), "sle_sht_gauss")
        self.gaulats, self.weights = mu, w
        frac = C.c_double()
        _lib.check(L.sle_sht_work_fraction(h, C.byref(frac)), "sle_sht_work_fraction")
        self.work_fraction = float(frac.value)
        self.device_index = torch.cuda.current_device()
        dev = torch.device("cuda", self.device_index)
        self._grid_d = torch.empty((self.nlat, self.nlon), dtype=torch.float64, device=dev)
        self._coef_d = torch.empty((self.nm, self.nm), dtype=torch.complex128, device=dev)
        self._grid_h = torch.empty((self.nlat, self.nlon), dtype=torch.float64).pin_memory()
        self._coef_h = torch.empty((self.nm, self.nm), dtype=torch.complex128).pin_memory()
        self._coef_out = self._coef_h.numpy()
        self._grid_out = self._grid_h.numpy()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.sle_sht_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def table_bytes(self) -> int:
        """Device bytes of the Legendre seed and coefficient tables (no full P table is stored)."""
        nseg = sum((self.lmax - m) // 64 + 1 for m in range(self.nm))
        return int(nseg * self.nh * 16 + self.ncoef * 16)

    # ------------------------------------------------------------- device paths
    def _check_device_args(self, grids, coeffs, layout, torch):
        """Equal counts, and every tensor a contiguous CUDA tensor on the plan's device holding what
        the library reads or writes through its pointer: nlat * nlon float64 per grid, (lmax+1)^2
        (dense) or the packed count of complex128 per spectrum."""
        if len(grids) != len(coeffs):
            raise ValueError(f"{len(grids)} grids but {len(coeffs)} spectra")
        ncoef = self.nm * self.nm if layout == _lib.LAYOUT_DENSE else self.ncoef
        for g in grids:
            if not (isinstance(g, torch.Tensor) and g.is_cuda and g.dtype == torch.float64 and g.is_contiguous()
                    and g.numel() == self.nlat * self.nlon):
                raise ValueError(f"grids must be contiguous CUDA float64 tensors of {self.nlat} x {self.nlon}")
            self._check_on_device(g)
        for c in coeffs:
            if not (isinstance(c, torch.Tensor) and c.is_cuda and c.dtype == torch.complex128
                    and c.is_contiguous() and c.numel() == ncoef):
                raise ValueError(f"spectra must be contiguous CUDA complex128 tensors of {ncoef} values")
            self._check_on_device(c)

    def _check_on_device(self, t):
        """The library dereferences the tensor's pointer on the plan's device: a tensor on another
        GPU is refused rather than read through a foreign address."""
        if t.device.index != self.device_index:
            raise ValueError(f"tensor on cuda:{t.device.index}, but this transform plan lives on "
                             f"cuda:{self.device_index}")

    def analysis_device(self, grids, coeffs, layout=_lib.LAYOUT_DENSE):
        """Analyse CUDA float64 grids into CUDA complex128 tensors (in place): up to four with the
        dense layout, up to 256 with the packed one."""
        torch = _torch()
        self._check_device_args(grids, coeffs, layout, torch)
        n = len(grids)
        gp = (C.c_void_p * n)(*[g.data_ptr() for g in grids])
        cp = (C.c_void_p * n)(*[c.data_ptr() for c in coeffs])
        _lib.check(self._L.sle_sht_analysis(self._h, n, gp, cp, int(layout), _stream_ptr(torch)),
                   "sle_sht_analysis")

    def synthesis_device(self, coeffs, grids, layout=_lib.LAYOUT_DENSE):
        """Synthesise CUDA complex128 spectra into CUDA float64 grids (in place): up to four with
        the dense layout, up to 256 with the packed one."""
        torch = _torch()
        self._check_device_args(grids, coeffs, layout, torch)
        n = len(grids)
        cp = (C.c_void_p * n)(*[c.data_ptr() for c in coeffs])
        gp = (C.c_void_p * n)(*[g.data_ptr() for g in grids])
        _lib.check(self._L.sle_sht_synthesis(self._h, n, cp, int(layout), gp, _stream_ptr(torch)),
                   "sle_sht_synthesis")

    # --------------------------------------------------------- reference API
    def analysis(self, grid, out=None):
        """grid[nlat, nlon] float64 -> coeffs[lmax+1, lmax+1] complex128 ([l, m])."""
        torch = _torch()
        if isinstance(grid, torch.Tensor) and grid.is_cuda:
            g = grid.to(torch.float64).contiguous()
            if tuple(g.shape) != (self.nlat, self.nlon):
                raise ValueError(f"grid shape {tuple(g.shape)} != {(self.nlat, self.nlon)}")
            res = out if out is not None else torch.empty((self.nm, self.nm), dtype=torch.complex128,
                                                        device=g.device)
            self._check_device_out(res, (self.nm, self.nm), torch.complex128, torch)
            self.analysis_device([g], [res])
            if self.raw:
                res[:, 1::2].neg_()
            return res
        a = np.ascontiguousarray(grid, dtype=np.float64)
        if a.shape != (self.nlat, self.nlon):
            raise ValueError(f"grid shape {a.shape} != {(self.nlat, self.nlon)}")
        self._grid_h.numpy()[...] = a
        self._grid_d.copy_(self._grid_h, non_blocking=True)
        self.analysis_device([self._grid_d], [self._coef_d])
        if self.raw:
            self._coef_d[:, 1::2].neg_()
        self._coef_h.copy_(self._coef_d)
        if out is None:
            return self._coef_out
        out[...] = self._coef_out
        return out

    def synthesis(self, coeffs, out=None):
        """coeffs[lmax+1, lmax+1] complex128 ([l, m]) -> grid[nlat, nlon] float64."""
        torch = _torch()
        if isinstance(coeffs, torch.Tensor) and coeffs.is_cuda:
            c = coeffs.to(torch.complex128).contiguous()
            if tuple(c.shape) != (self.nm, self.nm):
                raise ValueError(f"coeffs shape {tuple(c.shape)} != {(self.nm, self.nm)}")
            if self.raw:
                c = c.clone()
                c[:, 1::2].neg_()
            res = out if out is not None else torch.empty((self.nlat, self.nlon), dtype=torch.float64,
                                                        device=c.device)
            self._check_device_out(res, (self.nlat, self.nlon), torch.float64, torch)
            self.synthesis_device([c], [res])
            return res
        a = np.ascontiguousarray(coeffs, dtype=np.complex128)
        if a.shape != (self.nm, self.nm):
            raise ValueError(f"coeffs shape {a.shape} != {(self.nm, self.nm)}")
        self._coef_h.numpy()[...] = a
        self._coef_d.copy_(self._coef_h, non_blocking=True)
        if self.raw:
            self._coef_d[:, 1::2].neg_()
        self.synthesis_device([self._coef_d], [self._grid_d])
        self._grid_h.copy_(self._grid_d)
        if out is None:
            return self._grid_out
        out[...] = self._grid_out
        return out

    def _check_device_out(self, t, shape, dtype, torch):
        if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and tuple(t.shape) == shape
                and t.is_contiguous()):
            raise ValueError(f"out must be a contiguous CUDA {dtype} tensor of shape {shape}")
        self._check_on_device(t)

    def mean00_weights(self):
        """Row weights with ``analysis(g)[0, 0].real == mean00_weights() @ g.sum(axis=1)`` up to
        round-off: P~_00 w_j / (nlon * 1.41421356), P~_00 = sqrt(0.5)."""
        return np.sqrt(0.5) * self.weights / self.nlon / SQRT2_LEGACY


def make_sht(backend: str, nlat: int, nlon: int, lmax: int, workers: int = 1, chunk: int = 16,
             raw: bool = False, precision: str = "fp64"):
    """Transform factory with the reference's signature (sht_ducc.py:206-217); this package
    provides the ``"cuda"`` backend only and raises ValueError for any other name."""
    if backend == "cuda":
        return CudaSHT(nlat, nlon, lmax, workers=workers, chunk=chunk, raw=raw, precision=precision)
    raise ValueError(f"unknown SHT backend {backend!r} (slevolve_b200 provides 'cuda'; the 'numpy' "
                     "and 'ducc' backends belong to the reference package)")
