"""Oracle spherical-harmonic transform (test infrastructure only; see ``oracle/__init__``).

NumPy restatement of the reference transform ``python/slevolve/sht.py``:

* ``gauss_nodes``   restates ``gaulw`` (sht.py:65-101): Newton on P_N from the
                    asymptotic guess, at most 10 sweeps, per-node latch at
                    |dz| < 1e-15, weights 2/((1-z^2) P_N'^2).  Rows run north->south.
* ``legendre_rows`` restates ``legend_columns`` (sht.py:105-144), the exact
                    ``LEGEND`` recursion: orthonormal P~_lm without the
                    Condon-Shortley phase.  The arithmetic is kept in the same
                    order so that the values agree with the reference bit for bit.
* ``OracleSHT``     restates ``SHT.analysis`` / ``SHT.synthesis``
                    (sht.py:274-343): rFFT along longitude, north/south fold with
                    the Gauss weights divided by nlon, a parity-split Legendre
                    contraction per order m, and the legacy 1.41421356 factor
                    (sht.py:60-61).  The contraction is done per order m as one
                    (n_l x nh) @ (nh x 2) matrix product instead of the
                    reference's padded 16-order blocks; sums therefore agree to
                    round-off, not bit for bit.
"""

from __future__ import annotations

import numpy as np
import scipy.fft as sfft

# legacy literal used by spat2spec/spec2spat instead of sqrt(2) (sht.py:60-61)
SQRT2_LEGACY = 1.41421356


def gauss_nodes(nlat: int):
    """Gauss-Legendre nodes mu_j (north -> south, mu_0 > 0) and weights (sht.py:65-101)."""
    n = int(nlat)
    tol = 0.1 ** 15
    pi = 4.0 * np.arctan(1.0)
    z = np.cos(pi * (np.arange(1, n + 1, dtype=np.float64) - 0.25) / (n + 0.5))
    z_fin = np.zeros(n)
    dp_fin = np.zeros(n)
    latched = np.zeros(n, dtype=bool)
    for _sweep in range(10):
        p_cur = np.ones(n)
        p_prev = np.zeros(n)
        for k in range(1, n + 1):
            p_old = p_prev
            p_prev = p_cur
            p_cur = ((2.0 * k - 1.0) * z * p_prev - (k - 1.0) * p_old) / k
        dp = n * (z * p_cur - p_prev) / (z * z - 1.0)
        z_before = z
        z = z_before - p_cur / dp
        ok = np.abs(z - z_before) < tol
        new = ok & ~latched
        z_fin[new] = z[new]
        dp_fin[new] = dp[new]
        latched |= ok
        if latched.all():
            break
    if not latched.all():
        raise RuntimeError("gauss_nodes: Newton iteration did not converge")
    w = 2.0 / ((1.0 - z_fin * z_fin) * dp_fin * dp_fin)
    return z_fin, w


def legendre_rows(x: np.ndarray, lmax: int):
    """Yield ``(m, P)`` with ``P[l - m, j] = P~_lm(x_j)`` for m = 0..lmax (sht.py:105-144).

    P~_mm = sqrt(0.5 * prod_m), prod_m = prod_{i<=m} (1 - x^2) (2i+1)/(2i) accumulated in
    order; P~_{m+1,m} = sqrt(2m+3) x P~_mm; then
    P~_n = (x P~_{n-1} - eps_{n-1} P~_{n-2}) / eps_n with eps_n = sqrt((n^2-m^2)/(4n^2-1)).
    """
    x = np.asarray(x, dtype=np.float64)
    nj = x.size
    one_minus = 1.0 - x * x
    num = 1.0
    den = 0.0
    prod = np.ones(nj)
    for m in range(lmax + 1):
        nl = lmax + 1 - m
        if m > 0:
            num += 2.0
            den += 2.0
            prod = prod * one_minus * num / den
        P = np.zeros((nl, nj))
        p0 = np.sqrt(0.5 * prod)
        P[0] = p0
        p1 = np.sqrt(float(2 * m + 3)) * x * p0
        if nl >= 2:
            P[1] = p1
        n1 = m + 1
        e_prev = np.sqrt(float(n1 * n1 - m * m) / float(4 * n1 * n1 - 1))
        t = x * p1 - e_prev * p0
        for r in range(2, nl):
            n = m + r
            e = np.sqrt(float(n * n - m * m) / float(4 * n * n - 1))
            pn = t / e
            P[r] = pn
            t = x * pn - e * p1
            p0 = p1
            p1 = pn
        yield m, P


class OracleSHT:
    """Gauss-Legendre pseudo-spectral transform in the legacy conventions (sht.py:148-343).

    ``analysis(grid[nlat, nlon]) -> U[lmax+1, lmax+1]`` (dense ``[l, m]``, zero for m > l) and
    ``synthesis(U) -> grid``.  Both return a fresh array unless ``out`` is given.
    """

    def __init__(self, nlat: int, nlon: int, lmax: int, workers: int = 1):
        if nlat % 2 != 0:
            raise ValueError("nlat must be even")
        if lmax > nlon // 2:
            raise ValueError("lmax must be <= nlon/2")
        self.nlat, self.nlon, self.lmax = int(nlat), int(nlon), int(lmax)
        self.nm = self.lmax + 1
        self.nh = self.nlat // 2
        self.workers = int(workers)
        self.gaulats, self.weights = gauss_nodes(self.nlat)
        nh = self.nh
        # weights folded with the power-of-two 1/nlon of the FFT normalisation (sht.py:168-170)
        self._wn = self.weights[:nh] / self.nlon
        self._ws = self.weights[self.nlat - 1: nh - 1: -1] / self.nlon
        self._Pe = []
        self._Po = []
        for m, P in legendre_rows(self.gaulats[:nh], self.lmax):
            self._Pe.append(np.ascontiguousarray(P[0::2]))   # l - m even
            self._Po.append(np.ascontiguousarray(P[1::2]))   # l - m odd

    @property
    def table_bytes(self) -> int:
        return int(sum(a.nbytes for a in self._Pe) + sum(a.nbytes for a in self._Po))

    def analysis(self, grid: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        nh, nm, nlat = self.nh, self.nm, self.nlat
        F = sfft.rfft(np.asarray(grid, dtype=np.float64), axis=1, workers=self.workers)
        A = F[:nh, :nm] * self._wn[:, None]
        B = F[nlat - 1: nh - 1: -1, :nm] * self._ws[:, None]
        S = A + B
        D = A - B
        if out is None:
            out = np.zeros((nm, nm), dtype=np.complex128)
        else:
            out[...] = 0.0
        for m in range(nm):
            rs = np.stack((S[:, m].real, S[:, m].imag), axis=1)
            rd = np.stack((D[:, m].real, D[:, m].imag), axis=1)
            ce = self._Pe[m] @ rs
            co = self._Po[m] @ rd
            out[m::2, m] = (ce[:, 0] + 1j * ce[:, 1]) / SQRT2_LEGACY
            out[m + 1::2, m] = (co[:, 0] + 1j * co[:, 1]) / SQRT2_LEGACY
        return out

    def synthesis(self, coeffs: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        nh, nm, nlat = self.nh, self.nm, self.nlat
        scale = SQRT2_LEGACY * self.nlon
        E = np.zeros((nh, nm), dtype=np.complex128)
        O = np.zeros((nh, nm), dtype=np.complex128)
        for m in range(nm):
            ce = coeffs[m::2, m] * scale
            co = coeffs[m + 1::2, m] * scale
            ve = self._Pe[m].T @ np.stack((ce.real, ce.imag), axis=1)
            vo = self._Po[m].T @ np.stack((co.real, co.imag), axis=1)
            E[:, m] = ve[:, 0] + 1j * ve[:, 1]
            O[:, m] = vo[:, 0] + 1j * vo[:, 1]
        spec = np.zeros((nlat, self.nlon // 2 + 1), dtype=np.complex128)
        spec[:nh, :nm] = E + O
        spec[nlat - 1: nh - 1: -1, :nm] = E - O
        g = sfft.irfft(spec, n=self.nlon, axis=1, workers=self.workers)
        if out is not None:
            out[...] = g
            return out
        return g

    def degree0(self, grid: np.ndarray) -> float:
        """Real part of ``analysis(grid)[0, 0]`` by a row-sum quadrature (the degree-0 term only).

        U_00 = sum_j P~_00 w_j rowsum_j / (nlon * 1.41421356), P~_00 = sqrt(0.5)."""
        rs = np.asarray(grid, dtype=np.float64).sum(axis=1)
        return float(np.sqrt(0.5) * (self.weights * rs).sum() / self.nlon / SQRT2_LEGACY)
