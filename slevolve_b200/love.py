"""Earth models: the SLEvolve Love-number text format and the seeded synthetic Earth.

Both produce an object with the attribute set the solver reads from the reference's
``LoveNumbers`` (SLEvolve ``python/slevolve/solver.py:114-225``): ``nmod[l]``, ``s[k, l]`` (inverse
relaxation times in 1/kyr), elastic ``he, ke, hTE, kTE`` (k already divided by the degree),
residues ``r`` (h), ``rprime`` (k / l), ``rT``, ``rprimeT`` (tidal), and ``max_modes``.  A
``LoveNumbers`` object of the reference itself is accepted everywhere as well.
"""

from __future__ import annotations

import numpy as np

NPAM = 500  # row capacity of the mode arrays (solver.py:39)


class _Records:
    """Fortran list-directed reads: every read starts a new record (line)."""

    def __init__(self, path):
        with open(path, "r") as fh:
            self.lines = fh.read().split("\n")
        self.i = 0

    def skip(self):
        self.i += 1

    def take(self, n):
        vals = []
        while len(vals) < n:
            if self.i >= len(self.lines):
                raise ValueError("Love-number file ended early")
            vals.extend(self.lines[self.i].split())
            self.i += 1
        return vals[:n]

    def floats(self, n):
        return [float(v) for v in self.take(n)]


class LoveNumbers:
    """Reader for the SLEvolve Love-number text file (format of solver.py:150-186).

    Per degree block: ``l nmodes``; nmodes inverse relaxation times; elastic line
    (h, l*l, ., ., l*k); fluid line; nmodes h, l*l, l*k residues; for l >= 2 the same five
    records for the tidal numbers.  k and l values are stored multiplied by the degree.
    """

    def __init__(self, path, norder):
        self.norder = int(norder)
        nl = self.norder + 1
        rd = _Records(path)
        rd.skip()
        nmod = np.zeros(nl, dtype=np.int64)
        s = np.zeros((NPAM, nl))
        el = np.zeros((3, nl))
        fl = np.zeros((3, nl))
        tel = np.zeros((3, nl))
        tfl = np.zeros((3, nl))
        rh, rl, rk = (np.zeros((NPAM, nl)) for _ in range(3))
        trh, trl, trk = (np.zeros((NPAM, nl)) for _ in range(3))
        for _ in range(self.norder):
            deg, nk = rd.take(2)
            l = int(deg)
            nk = int(nk)
            nmod[l] = nk
            s[:nk, l] = rd.floats(nk)
            v = rd.floats(5)
            el[:, l] = (v[0], v[1], v[4])
            v = rd.floats(5)
            fl[:, l] = (v[0], v[1], v[4])
            rh[:nk, l] = rd.floats(nk)
            rl[:nk, l] = rd.floats(nk)
            rk[:nk, l] = rd.floats(nk)
            if float(deg) < 1.5:
                continue
            v = rd.floats(5)
            tel[:, l] = (v[0], v[1], v[4])
            v = rd.floats(5)
            tfl[:, l] = (v[0], v[1], v[4])
            trh[:nk, l] = rd.floats(nk)
            trl[:nk, l] = rd.floats(nk)
            trk[:nk, l] = rd.floats(nk)
        ell = np.arange(1, nl, dtype=np.float64)
        for a in (rl, rk, trl, trk):
            a[:, 1:] /= ell
        self.nmod = nmod
        self.s = s
        self.he = np.zeros(nl)
        self.ke = np.zeros(nl)
        self.hTE = np.zeros(nl)
        self.kTE = np.zeros(nl)
        self.he[1:] = el[0, 1:]
        self.ke[1:] = el[2, 1:] / ell
        self.hTE[1:] = tel[0, 1:]
        self.kTE[1:] = tel[2, 1:] / ell
        self.r = rh
        self.rprime = rk
        self.rT = trh
        self.rprimeT = trk
        # tangential-displacement (l) numbers of the optional horizontal read-out, scaled as k
        self.le = np.zeros(nl)
        self.lTE = np.zeros(nl)
        self.le[1:] = el[1, 1:] / ell
        self.lTE[1:] = tel[1, 1:] / ell
        self.rl = rl
        self.rlT = trl
        self.max_modes = int(nmod.max())


class SyntheticEarth:
    """Seeded synthetic Earth of the benchmark configurations.

    Per degree l >= 1: elastic h_e = -6 l/(l+30) - 0.3, k_e = -0.3*30/(l+30), l_e = 0.1*30/(l+30);
    K viscous modes with inverse relaxation times log-uniform in [1e-5, 1e-1] /yr, i.e.
    [1e-2, 1e2] /kyr (the unit the solver's decay exp(-s dt / 1000) expects); residues
    r_k = s_k w_k (2 X_E) / sum(w) with positive weights w_k ~ U(0, 1] from the seed, so that
    the fluid limit X_E + sum_k r_k / s_k equals 3 X_E for X in (h, k, l).  Degree-2 tidal numbers:
    the load numbers of degree 2 with the sign flipped (h_T = 0.675, k_T = 0.28125), residues
    built the same way.  ``relax_scale`` multiplies every relaxation time (s -> s / relax_scale).
    """

    def __init__(self, lmax, nmodes=8, seed=20261203, relax_scale=1.0):
        nl = int(lmax) + 1
        rng = np.random.default_rng(seed)
        self.norder = int(lmax)
        self.nmod = np.zeros(nl, dtype=np.int64)
        self.nmod[1:] = nmodes
        self.s = np.zeros((NPAM, nl))
        self.r = np.zeros((NPAM, nl))
        self.rprime = np.zeros((NPAM, nl))
        self.rT = np.zeros((NPAM, nl))
        self.rprimeT = np.zeros((NPAM, nl))
        self.he = np.zeros(nl)
        self.ke = np.zeros(nl)
        self.le = np.zeros(nl)
        self.hTE = np.zeros(nl)
        self.kTE = np.zeros(nl)
        l = np.arange(1, nl, dtype=np.float64)
        self.he[1:] = -6.0 * l / (l + 30.0) - 0.3
        self.ke[1:] = -0.3 * 30.0 / (l + 30.0)
        self.le[1:] = 0.1 * 30.0 / (l + 30.0)
        for ll in range(1, nl):
            s = 10.0 ** rng.uniform(-2.0, 2.0, nmodes) / float(relax_scale)
            w = 1.0 - rng.uniform(0.0, 1.0, nmodes)           # (0, 1]
            self.s[:nmodes, ll] = s
            self.r[:nmodes, ll] = s * w * (2.0 * self.he[ll]) / w.sum()
            self.rprime[:nmodes, ll] = s * w * (2.0 * self.ke[ll]) / w.sum()
            if ll == 2:
                self.hTE[2] = -self.he[2]
                self.kTE[2] = -self.ke[2]
                wt = 1.0 - rng.uniform(0.0, 1.0, nmodes)
                self.rT[:nmodes, 2] = s * wt * (2.0 * self.hTE[2]) / wt.sum()
                self.rprimeT[:nmodes, 2] = s * wt * (2.0 * self.kTE[2]) / wt.sum()
        self.max_modes = int(nmodes)


def mode_arrays(love, lmax):
    """Dense per-(mode, degree) arrays the device path uploads.

    Returns ``s[K, L+1]`` (1/kyr, 0 where the mode does not exist), ``a_sl = (r' - r)/s``,
    ``a_rr = r/s`` (solver.py:261-282) and the degree-2 rotational weights ``a_il, a_m, a_tsl,
    a_trr`` (length K), plus ``nmod[L+1]``.
    """
    nl = int(lmax) + 1
    K = int(love.max_modes)
    s = np.zeros((K, nl))
    a_sl = np.zeros((K, nl))
    a_rr = np.zeros((K, nl))
    a_il = np.zeros(K)
    a_m = np.zeros(K)
    a_tsl = np.zeros(K)
    a_trr = np.zeros(K)
    nmod = np.zeros(nl, dtype=np.int32)
    for l in range(1, nl):
        nk = int(love.nmod[l])
        nmod[l] = nk
        sl = love.s[:nk, l]
        s[:nk, l] = sl
        a_sl[:nk, l] = (love.rprime[:nk, l] - love.r[:nk, l]) / sl
        a_rr[:nk, l] = love.r[:nk, l] / sl
        if l == 2:
            a_il[:nk] = love.rprime[:nk, l] / sl
            a_m[:nk] = love.rprimeT[:nk, l] / sl
            a_tsl[:nk] = (love.rprimeT[:nk, l] - love.rT[:nk, l]) / sl
            a_trr[:nk] = love.rT[:nk, l] / sl
    return {"s": s, "a_sl": a_sl, "a_rr": a_rr, "a_il": a_il, "a_m": a_m, "a_tsl": a_tsl,
            "a_trr": a_trr, "nmod": nmod, "K": K}
