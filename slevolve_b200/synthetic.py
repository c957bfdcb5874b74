"""Seeded synthetic inputs of the benchmark configurations (topography, ice histories, Earth).

Every generator is deterministic given its seed.  Grids follow the SLEvolve layout: ``[nlat, nlon]``
float64, Gauss-Legendre rows north -> south, longitude i * 360 / nlon, values rounded to whole
millimetres.  The topography needs one spectral synthesis; the caller passes the transform object
to use (``slevolve_b200.make_sht("cuda", ...)`` on a GPU host), so the same generator serves every
grid size.

Configurations (sizes and schedules of the benchmark definition):

``c0``  64 x 128, L = 63, 100 steps of 1 yr: random topography (70 % ocean, mean ocean depth
        -4000 m, highest land +3000 m), two Vialov caps (radius 15 deg, 3 km) at the south pole
        and 56 N 132 E on bed above -500 m, melting linearly to zero.
``c1``  256 x 512, L = 255, 550 steps of 1 yr: the same topography generator with the south polar
        continent's bed lowered to -500 ... -1500 m; a 3.5 km dome thinned by a seeded, band-limited
        rate of 1-20 m/yr, which ungrounds its margin and moves the grounding line.
``c2``  512 x 1024, L = 511, 1200 steps of 200 yr: three northern-hemisphere caps on a 100-kyr
        sawtooth (90 kyr growth, 10 kyr collapse), peak 3.5 km.
"""

from __future__ import annotations

import math

import numpy as np

from .love import SyntheticEarth

D2R = math.pi / 180.0
BASE_SEED = 20261203


def round_mm(f):
    return np.round(f * 1000.0) / 1000.0


def grid_latlon(gaulats, nlon):
    lat = np.degrees(np.arcsin(np.asarray(gaulats)))
    lon = np.arange(nlon) * 360.0 / nlon
    LON, LAT = np.meshgrid(lon, lat)
    return LAT, LON


def angular_distance(LAT, LON, lat0, lon0):
    p, p0, dl = LAT * D2R, lat0 * D2R, (LON - lon0) * D2R
    c = np.sin(p) * np.sin(p0) + np.cos(p) * np.cos(p0) * np.cos(dl)
    return np.arccos(np.clip(c, -1.0, 1.0)) / D2R


def vialov(d, R):
    """(1 - (d/R)^(4/3))^(3/8) inside d < R, 0 outside."""
    return np.clip(1.0 - (np.minimum(d, R) / R) ** (4.0 / 3.0), 0.0, None) ** 0.375


def area_weights(sht, nlon):
    return np.asarray(sht.weights)[:, None] * np.ones((1, nlon))


def band_limited_field(sht, seed, lmin, lmax_field, power):
    """Unit-variance random field: coefficients ~ N(0, l^-power) for lmin <= l <= lmax_field."""
    nl = sht.lmax + 1
    rng = np.random.default_rng(seed)
    l = np.arange(nl)[:, None]
    m = np.arange(nl)[None, :]
    amp = np.where((l >= lmin) & (l <= lmax_field) & (m <= l), np.maximum(l, 1.0) ** (-power / 2.0), 0.0)
    c = (rng.standard_normal((nl, nl)) + 1j * rng.standard_normal((nl, nl))) * amp / math.sqrt(2.0)
    c[:, 0] = c[:, 0].real * math.sqrt(2.0)
    g = np.asarray(sht.synthesis(c), dtype=np.float64)
    W = area_weights(sht, g.shape[1])
    g = g - (W * g).sum() / W.sum()
    return g / math.sqrt((W * g * g).sum() / W.sum())


def random_topography(sht, seed, ocean_frac=0.70, mean_depth=-4000.0, max_land=3000.0):
    """Band-limited field (degree power ~ l^-2) shifted to ``ocean_frac`` ocean by area, ocean
    scaled to the area-mean depth, land scaled to the maximum height; rounded to mm."""
    g = band_limited_field(sht, seed, 2, sht.lmax, 3.0)
    W = area_weights(sht, g.shape[1])
    order = np.argsort(g, axis=None, kind="stable")
    cw = np.cumsum(W.ravel()[order]) / W.sum()
    thr = g.ravel()[order][int(np.searchsorted(cw, ocean_frac))]
    g = g - thr
    oc = g < 0
    a = mean_depth / ((W * g)[oc].sum() / W[oc].sum())
    b = max_land / g[~oc].max()
    return round_mm(np.where(oc, a * g, b * g))


class Case:
    """One synthetic run: ``topo`` grid, ``love`` Earth, ``ice(k)`` for k = 0..nsteps, ``dt`` (yr)."""

    def __init__(self, name, nlat, lmax, nsteps, dt, topo, love, ice_fn, seed):
        self.name, self.nlat, self.nlon, self.lmax = name, nlat, 2 * nlat, lmax
        self.nsteps, self.dt, self.topo, self.love, self._ice, self.seed = nsteps, dt, topo, love, ice_fn, seed

    def ice(self, k):
        return self._ice(int(k))

    def describe(self):
        return {"case": self.name, "grid": [self.nlat, self.nlon], "lmax": self.lmax,
                "steps": self.nsteps, "dt_years": self.dt, "seed": self.seed,
                "modes": int(self.love.max_modes)}


def case_c0(sht, nsteps=100, seed=BASE_SEED):
    nlat, nlon, L = sht.nlat, sht.nlon, sht.lmax
    topo = random_topography(sht, seed)
    love = SyntheticEarth(L, 8, seed)
    LAT, LON = grid_latlon(sht.gaulats, nlon)
    shape = (vialov(angular_distance(LAT, LON, -90.0, 0.0), 15.0)
             + vialov(angular_distance(LAT, LON, 56.0, 132.0), 15.0)) * (topo > -500.0)

    def ice(k):
        return round_mm(3000.0 * (1.0 - k / nsteps) * shape)

    return Case("c0", nlat, L, nsteps, 1.0, topo, love, ice, seed)


def case_c1(sht, nsteps=550, seed=BASE_SEED + 1):
    nlat, nlon, L = sht.nlat, sht.nlon, sht.lmax
    topo = random_topography(sht, seed)
    love = SyntheticEarth(L, 8, seed)
    LAT, LON = grid_latlon(sht.gaulats, nlon)
    d = angular_distance(LAT, LON, -90.0, 0.0)
    R = 22.0
    cont = d < R
    topo = np.where(cont, round_mm(-500.0 - 1000.0 * (1.0 - d / R)), topo)
    dome = 3500.0 * vialov(d, R)
    rate = band_limited_field(sht, seed + 100, 1, min(L, 32), 2.0)
    rate = 1.0 + 19.0 * (rate - rate.min()) / (rate.max() - rate.min())  # 1..20 m/yr

    def ice(k):
        return round_mm(np.maximum(0.0, dome - rate * (k * 1.0)) * cont)

    return Case("c1", nlat, L, nsteps, 1.0, topo, love, ice, seed)


SHEETS_C2 = ((60.0, 265.0, 20.0), (63.0, 15.0, 12.0), (75.0, 60.0, 10.0))


def sawtooth(t_kyr, period=100.0, grow=90.0):
    ph = np.mod(t_kyr, period)
    return np.where(ph < grow, ph / grow, 1.0 - (ph - grow) / (period - grow))


def case_c2(sht, nsteps=1200, seed=BASE_SEED + 2, dt=200.0, amp=1.0, relax_scale=1.0):
    nlat, nlon, L = sht.nlat, sht.nlon, sht.lmax
    topo = random_topography(sht, seed)
    love = SyntheticEarth(L, 8, seed, relax_scale=relax_scale)
    LAT, LON = grid_latlon(sht.gaulats, nlon)
    shape = np.zeros_like(topo)
    for la, lo, R in SHEETS_C2:
        shape = np.maximum(shape, vialov(angular_distance(LAT, LON, la, lo), R))

    def ice(k):
        return round_mm(amp * 3500.0 * float(sawtooth(k * dt / 1000.0)) * shape)

    return Case("c2", nlat, L, nsteps, dt, topo, love, ice, seed)


CASES = {"c0": (64, case_c0), "c1": (256, case_c1), "c2": (512, case_c2)}


def case_glacial(sht, nstates=13, seed=BASE_SEED + 5):
    """Ice states 0..nstates-1 of two glacial cycles (growth, retreat, regrowth, present) on the
    c0-style topography of this grid: three caps (south pole, 62 N 100 W, 56 N 132 E) scaled by
    0.35 + 0.65 |sin(2.2 pi t)| (1 - 0.4 t), t in [0, 1]; the input of the segmented T0 guess.
    Returns (topography, list of ice grids, Earth model)."""
    nlon, L = sht.nlon, sht.lmax
    topo = random_topography(sht, seed)
    LAT, LON = grid_latlon(sht.gaulats, nlon)
    shape = (1.2 * vialov(angular_distance(LAT, LON, -90.0, 0.0), 15.0)
             + vialov(angular_distance(LAT, LON, 62.0, -100.0), 20.0)
             + vialov(angular_distance(LAT, LON, 56.0, 132.0), 15.0)) * (topo > -500.0)
    t = np.linspace(0.0, 1.0, nstates)
    amp = 0.35 + 0.65 * np.abs(np.sin(2.2 * np.pi * t)) * (1.0 - 0.4 * t)
    return topo, [round_mm(3000.0 * a * shape) for a in amp], SyntheticEarth(L, 8, seed)
