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


# The Love-number text file (the format SLEvolve's Fortran and Python readers share): a header
# line, then one block per degree l = 1, 2, ...  A block is a sequence of fields; a field starts on
# a new line and runs over as many lines as its count of numbers needs (numbers past the count on
# its last line are ignored, as Fortran list-directed input ignores them).  "K" stands for the
# block's mode count, the second number of its first field.  Lines of five numbers hold
# (h, l*l, -, -, l*k): the tangential (l) and potential (k) numbers are stored times the degree.
BLOCK_FIELDS = (("head", 2), ("relax", "K"), ("elastic", 5), ("fluid", 5),
                ("res_h", "K"), ("res_l", "K"), ("res_k", "K"))
TIDAL_FIELDS = (("t_elastic", 5), ("t_fluid", 5), ("t_res_h", "K"), ("t_res_l", "K"), ("t_res_k", "K"))


class _FieldCursor:
    """Walks the lines of a Love-number file one field at a time."""

    def __init__(self, text):
        self._lines = text.splitlines()
        self._at = 1   # the header line carries no numbers the solver uses

    def field(self, count, where):
        vals = []
        while len(vals) < count:
            if self._at >= len(self._lines):
                raise ValueError(f"Love-number file ends inside {where}")
            vals += self._lines[self._at].split()
            self._at += 1
        return np.array(vals[:count], dtype=np.float64)


def read_love_blocks(path, lmax):
    """{degree: {field name: values}} of the first ``lmax`` degree blocks of a Love-number file."""
    with open(path, "r") as fh:
        cur = _FieldCursor(fh.read())
    blocks = {}
    for _ in range(int(lmax)):
        blk = {}
        for name, count in BLOCK_FIELDS + TIDAL_FIELDS:
            if name.startswith("t_") and blk["degree"] < 2:
                break   # degree 1 has no tidal numbers
            n = blk["K"] if count == "K" else count
            v = cur.field(n, f"field {name!r} of block {len(blocks) + 1}")
            if name == "head":
                blk["degree"], blk["K"] = int(v[0]), int(v[1])
                if not 1 <= blk["degree"] <= lmax:
                    raise ValueError(f"degree {blk['degree']} outside 1..{lmax} in the Love-number file")
            else:
                blk[name] = v
        blocks[blk["degree"]] = blk
    return blocks


class LoveNumbers:
    """Earth model read from a Love-number text file, truncated at degree ``norder``, with the
    attributes of the reference's reader (SLEvolve python/slevolve/solver.py:114-225): elastic
    ``he, ke, le`` and tidal ``hTE, kTE, lTE`` per degree (k and l divided by the degree), mode
    count ``nmod``, inverse relaxation times ``s[k, l]`` (1/kyr) and residues ``r`` (h),
    ``rprime`` (k), ``rl`` (l) with their tidal counterparts ``rT, rprimeT, rlT`` (k and l
    residues divided by the degree)."""

    # attribute <- (field, position in its five-number line); residue attribute <- field
    _ELASTIC = {"he": ("elastic", 0), "le": ("elastic", 1), "ke": ("elastic", 4),
                "hTE": ("t_elastic", 0), "lTE": ("t_elastic", 1), "kTE": ("t_elastic", 4)}
    _RESIDUES = {"r": "res_h", "rl": "res_l", "rprime": "res_k",
                 "rT": "t_res_h", "rlT": "t_res_l", "rprimeT": "t_res_k"}
    _PER_DEGREE = ("le", "ke", "lTE", "kTE", "rl", "rprime", "rlT", "rprimeT")   # stored times l

    def __init__(self, path, norder):
        self.norder = int(norder)
        nl = self.norder + 1
        blocks = read_love_blocks(path, self.norder)
        self.nmod = np.zeros(nl, dtype=np.int64)
        self.s = np.zeros((NPAM, nl))
        for name in self._ELASTIC:
            setattr(self, name, np.zeros(nl))
        for name in self._RESIDUES:
            setattr(self, name, np.zeros((NPAM, nl)))
        for l, blk in blocks.items():
            K = blk["K"]
            self.nmod[l] = K
            self.s[:K, l] = blk["relax"]
            for name, (fld, pos) in self._ELASTIC.items():
                if fld in blk:
                    getattr(self, name)[l] = blk[fld][pos]
            for name, fld in self._RESIDUES.items():
                if fld in blk:
                    getattr(self, name)[:K, l] = blk[fld]
        for name in self._PER_DEGREE:
            a = getattr(self, name)
            a[..., 1:] /= np.arange(1, nl, dtype=np.float64)
        self.max_modes = int(self.nmod.max())


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
