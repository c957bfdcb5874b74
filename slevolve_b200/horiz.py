"""Grid components of the horizontal displacement from its potential Psi_lm (the step dict's
``horiz``), behind the reference's ``horiz.gradient(U, nlat, nlon, nthreads=1)``
(SLEvolve python/slevolve/horiz.py:39-60):

    u_theta = dPsi/dtheta  (theta = colatitude, positive southward),
    u_phi   = (1 / sin theta) dPsi/dphi  (positive eastward),

on the Gauss-Legendre grid, rows north -> south, first column at phi = 0, U[l, m] in the legacy
(spharmt U) convention of the other spectral outputs.

The reference calls ducc0's spin-1 gradient synthesis.  Here the gradient is formed from three
scalar syntheses on the package's FP64 CUDA transform, by the recurrence of the orthonormal
Legendre functions P~_lm (normalised to 1 over x in [-1, 1]):

    sin theta dP~_lm/dtheta = l cos theta P~_lm - e_lm P~_{l-1,m},
    e_lm = sqrt((2l + 1)(l^2 - m^2) / (2l - 1)),

so that, with A_lm = l U_lm, B_{l-1,m} = e_lm U_lm and C_lm = i m U_lm,

    u_theta = (cos theta  synth(A) - synth(B)) / sin theta,   u_phi = synth(C) / sin theta.

The coefficient arrays are formed on the host (O(L^2)), the three transforms run on the GPU and
the row combine runs on the device before the two grids come back.  One transform plan per
(nlat, nlon, lmax) is kept for the calls that follow; ``release_plans()`` frees them.
"""

from __future__ import annotations

import numpy as np

_SHT_CACHE = {}


def gradient_coeffs(U):
    """(A, B, C) of the recurrence above from U[l, m] (complex, (L+1) x (L+1)); the imaginary
    part of the m = 0 column is dropped first, as the reference drops it (horiz.py:34)."""
    U = np.array(U, dtype=np.complex128)
    nl = U.shape[0]
    if U.ndim != 2 or U.shape[1] != nl:
        raise ValueError(f"U must be square [l, m], got shape {U.shape}")
    U[:, 0] = U[:, 0].real
    l = np.arange(nl, dtype=np.float64)[:, None]
    m = np.arange(nl, dtype=np.float64)[None, :]
    A = U * l
    with np.errstate(invalid="ignore", divide="ignore"):
        e = np.sqrt(np.where(l >= m, (2.0 * l + 1.0) * (l * l - m * m), 0.0) / np.where(l > 0, 2.0 * l - 1.0, 1.0))
    B = np.zeros_like(U)
    B[:-1] = U[1:] * e[1:]
    C = U * (1j * m)
    return A, B, C


def combine_rows(gA, gB, gC, x):
    """u_theta, u_phi from the three synthesised grids and the row nodes x = cos theta (works on
    NumPy arrays and on torch tensors alike)."""
    s = (1.0 - x * x) ** 0.5
    return (x * gA - gB) / s, gC / s


def _sht(nlat, nlon, lmax):
    key = (int(nlat), int(nlon), int(lmax))
    sh = _SHT_CACHE.get(key)
    if sh is None:
        from .sht import CudaSHT

        sh = CudaSHT(nlat, nlon, lmax)
        _SHT_CACHE[key] = sh
    return sh


def release_plans():
    """Drop the cached transform plans (their device tables are freed with them)."""
    _SHT_CACHE.clear()


def gradient(U, nlat: int, nlon: int, nthreads: int = 1):
    """(u_theta, u_phi) as float64 NumPy arrays (nlat, nlon) from Psi coefficients U[l, m]
    (lmax <= nlat - 1 and lmax <= (nlon - 1) // 2, as the reference requires).  ``nthreads`` is
    accepted for the reference's signature; the work runs on the GPU."""
    import torch

    U = np.asarray(U, dtype=np.complex128)
    lmax = U.shape[0] - 1
    if lmax > nlat - 1 or lmax > (nlon - 1) // 2:
        raise ValueError(f"lmax {lmax} needs lmax <= nlat - 1 and lmax <= (nlon - 1) // 2")
    return _gradient_with(_sht(nlat, nlon, lmax), U, torch.device("cuda"))


def _gradient_with(sh, U, dev):
    """The three syntheses of ``sh`` (which takes and returns torch tensors on ``dev``) and the
    row combine on ``dev``; returns NumPy grids."""
    import torch

    grids = []
    for c in gradient_coeffs(U):
        cd = torch.from_numpy(np.ascontiguousarray(c)).to(dev)
        grids.append(sh.synthesis(cd))
    x = torch.from_numpy(np.ascontiguousarray(sh.gaulats)).to(dev)[:, None]
    ut, up = combine_rows(grids[0], grids[1], grids[2], x)
    return ut.cpu().numpy(), up.cpu().numpy()


__all__ = ["gradient", "gradient_coeffs", "combine_rows", "release_plans"]
