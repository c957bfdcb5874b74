"""Oracle (test infrastructure only): NumPy restatement of the reference's grid conversion of the
horizontal-displacement potential (SLEvolve python/slevolve/horiz.py:39-60):

    u_theta = dPsi/dtheta,   u_phi = (1 / sin theta) dPsi/dphi

on the Gauss-Legendre grid (rows north -> south, first column at phi = 0, theta = colatitude),
Psi given by its coefficients U[l, m] in the legacy (spharmt U) convention that
``oracle.sht.OracleSHT.synthesis`` evaluates.  The reference does this with ducc0's spin-1
gradient synthesis (``mode="GRAD_ONLY"``); ducc0 is not installed here, so this restatement works
from the definition instead: dP~_lm/dtheta is carried through the same recursion that
``legendre_rows`` uses (forward-mode differentiation, with x = cos theta and
dx/dtheta = -sin theta), and the grid is evaluated row by row without the north/south fold.
Pinned, as the reference's own self-test is (python/slevolve/tools/horiz_grad.py:27-42), to
analytic fields whose gradients are known in closed form, to 1e-10.
"""

from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from .sht import SQRT2_LEGACY, gauss_nodes


def legendre_dtheta_rows(x: np.ndarray, lmax: int):
    """Yield ``(m, P, dP)`` with ``P[l - m, j] = P~_lm(x_j)`` and ``dP[l - m, j]`` its derivative in
    theta (x = cos theta), carried through the recursion of ``legendre_rows``:
    P~_mm = sqrt(0.5 C_m) sin^m theta, so dP~_mm = m cos theta / sin theta P~_mm;
    P~_{m+1,m} = sqrt(2m+3) x P~_mm; P~_n = (x P~_{n-1} - eps_{n-1} P~_{n-2}) / eps_n."""
    x = np.asarray(x, dtype=np.float64)
    s = np.sqrt(1.0 - x * x)
    one_minus = 1.0 - x * x
    num, den = 1.0, 0.0
    prod = np.ones(x.size)
    for m in range(lmax + 1):
        nl = lmax + 1 - m
        if m > 0:
            num += 2.0
            den += 2.0
            prod = prod * one_minus * num / den
        P = np.zeros((nl, x.size))
        dP = np.zeros((nl, x.size))
        p0 = np.sqrt(0.5 * prod)
        d0 = m * x / s * p0
        P[0], dP[0] = p0, d0
        c = np.sqrt(float(2 * m + 3))
        p1 = c * x * p0
        d1 = c * (-s * p0 + x * d0)
        if nl >= 2:
            P[1], dP[1] = p1, d1
        for r in range(2, nl):
            n = m + r
            e = np.sqrt(float(n * n - m * m) / float(4 * n * n - 1))
            e1 = np.sqrt(float((n - 1) ** 2 - m * m) / float(4 * (n - 1) ** 2 - 1))
            pn = (x * p1 - e1 * p0) / e
            dn = (-s * p1 + x * d1 - e1 * d0) / e
            P[r], dP[r] = pn, dn
            p0, d0, p1, d1 = p1, d1, pn, dn
        yield m, P, dP


def gradient(U: np.ndarray, nlat: int, nlon: int):
    """(u_theta, u_phi) on the (nlat, nlon) Gauss-Legendre grid from Psi coefficients U[l, m]."""
    U = np.asarray(U, dtype=np.complex128)
    lmax = U.shape[0] - 1
    x, _ = gauss_nodes(nlat)
    s = np.sqrt(1.0 - x * x)
    scale = SQRT2_LEGACY * nlon
    nf = nlon // 2 + 1
    ft = np.zeros((nlat, nf), dtype=np.complex128)
    fp = np.zeros((nlat, nf), dtype=np.complex128)
    for m, P, dP in legendre_dtheta_rows(x, lmax):
        u = U[m:, m] * scale
        if m == 0:
            u = u.real.astype(np.complex128)
        ft[:, m] = dP.T @ u
        fp[:, m] = (1j * m) * (P.T @ u) / s
    ut = sfft.irfft(ft, n=nlon, axis=1)
    up = sfft.irfft(fp, n=nlon, axis=1)
    return ut, up
