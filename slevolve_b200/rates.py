"""Analytic rates read-out of the FP64 GPU solver: dSL/dt and dR/dt at the end of a step and the
rotational rates, as the reference's ``SeaLevelSolver.step(..., rates=True)`` returns them
(SLEvolve python/slevolve/solver.py:229-240, 464-484, 722-806, 1086-1117).

The rate spectra (the viscous part read from the modal states and the elastic part of the step's
load increment taken to accrue linearly over the step) are formed on the device before the
commit (``k_rate_spec``, weights from ``RateTables``); the degree-2 rotational rates are a few
3 x 3 complex products formed here on the host from the step's rotational totals and the
degree-2 modal states; the rate grids come from the FP64 CUDA transforms on the end-of-step
ocean function.  Every expression keeps the reference's order of operations.
"""

from __future__ import annotations

import math

import numpy as np

from .love import mode_arrays


def ramp_factor(x):
    """phi(x) = (1 - e^-x) / x and 1 - phi(x), with their Taylor series below |x| = 1e-4
    (phi(0) = 1): the share of a linearly accruing load's response still held as memory at the
    end of the step, and the share reached (solver.py:229-240)."""
    x = np.asarray(x, dtype=np.float64)
    small = np.abs(x) < 1.0e-4
    xs = np.where(small, 1.0, x)
    phi = np.where(small, 1.0 - x / 2.0 + x * x / 6.0 - x ** 3 / 24.0, -np.expm1(-xs) / xs)
    omp = np.where(small, x / 2.0 - x * x / 6.0 + x ** 3 / 24.0, (xs + np.expm1(-xs)) / xs)
    return phi, omp


def ramp_table(ma, love, lmax, ttl, dt):
    """Host table of the ramp placement for steps of length ``dt`` years, in the layout
    ``sle_solver_set_ramp`` takes: omphi = 1 - phi per mode and degree (K x (lmax+1), zero where a
    degree has fewer modes), ttl c_sl and ttl c_rr per degree with c = sum_k a_k omphi_k, then the
    degree-2 c_il, c_m, c_tsl, c_trr (solver.py:348-368).  ``ma`` is ``mode_arrays(love, lmax)``."""
    s = ma["s"]
    phi, omp = ramp_factor(s * (float(dt) / 1000.0))
    omphi = np.where(s > 0, omp, 0.0)
    c_sl = (ma["a_sl"] * omphi).sum(0)
    c_rr = (ma["a_rr"] * omphi).sum(0)
    n2 = int(love.nmod[2]) if lmax >= 2 else 0
    c2 = omphi[:n2, 2] if lmax >= 2 else np.zeros(0)
    c4 = [float(c2 @ ma["a_il"][:n2]), float(c2 @ ma["a_m"][:n2]), float(c2 @ ma["a_tsl"][:n2]),
          float(c2 @ ma["a_trr"][:n2])]
    ttl = np.asarray(ttl, dtype=np.float64)
    return np.ascontiguousarray(np.concatenate([omphi.ravel(), ttl * c_sl, ttl * c_rr, c4]), dtype=np.float64)


class RateTables:
    """Per-step-length weights of the read-out: w = a s / 1000 per mode and degree (per year),
    ws = sum_k w, wsphi = sum_k w phi_k (solver.py:293-294, 347-362), and 1 - phi at degree 2."""

    def __init__(self, love, lmax):
        ma = mode_arrays(love, lmax)
        self.K = int(ma["K"])
        self.s = ma["s"]
        self.w_sl = ma["a_sl"] * self.s / 1000.0
        self.w_rr = ma["a_rr"] * self.s / 1000.0
        self.a_il, self.a_m, self.a_tsl, self.a_trr = ma["a_il"], ma["a_m"], ma["a_tsl"], ma["a_trr"]
        self.nmod2 = int(love.nmod[2]) if lmax >= 2 else 0
        self.dt = None

    def for_dt(self, dt):
        if dt != self.dt:
            phi, omp = ramp_factor(self.s * (dt / 1000.0))
            exists = self.s > 0
            self.phi = np.where(exists, phi, 1.0)
            self.omphi = np.where(exists, omp, 0.0)
            tab = [self.w_sl.ravel(), self.w_rr.ravel(), self.w_sl.sum(0), self.w_rr.sum(0),
                   (self.w_sl * self.phi).sum(0), (self.w_rr * self.phi).sum(0)]
            self.table = np.ascontiguousarray(np.concatenate(tab), dtype=np.float64)
            self.dt = dt
        return self.table


def rotation_rate(tabs, love, planet, h, il, mm, lam, oldil, oldm, dlam_prev2, r_il, r_m, r_la):
    """Left derivatives (per year) at the end of the step of the degree-2 rotational sea-level and
    radial terms (solver.py:722-764): the m equation differentiated with the step's converged
    il, m, Lambda; returns (rate_sl, rate_rr) 3 x 3 complex (U convention) and the rates dict."""
    p = planet
    n2 = tabs.nmod2
    dil = il - oldil
    dm = mm - oldm
    tot = lam[2, 0:3].copy()
    c = tabs.omphi[:n2, 2]
    r_il = r_il[:n2] + c[:, None, None] * dil[None]
    r_m = r_m[:n2] + c[:, None] * dm[None]
    r_la = r_la[:n2] + c[:, None] * (tot - dlam_prev2)[None]
    sk = tabs.s[:n2, 2] / 1000.0
    kTE2, hTE2, kE2 = love.kTE[2], love.hTE[2], love.ke[2]
    ild = dil / h
    sild = np.einsum("k,kij->ij", tabs.a_il[:n2] * sk, il[None] - r_il)
    smd = np.einsum("k,ki->i", tabs.a_m[:n2] * sk, mm[None] - r_m)
    alpha = 1 / (1 - kTE2 / p.kf)
    md = np.zeros(3)
    for i in (0, 1):
        md[i] = alpha * ((1 / (p.moiC - p.moiA)) * ((1 + kE2) * ild[i, 2] + sild[i, 2]) + smd[i] / p.kf)
    md[2] = -(1.0 / p.moiC) * ((1 + kE2) * ild[2, 2] + sild[2, 2])
    m1, m2, m3 = mm
    d1, d2, d3 = md
    r2w2 = p.radius ** 2 * p.omega ** 2
    II = 1j
    lad = np.zeros((3, 3), dtype=np.complex128)
    lad[0, 0] = (r2w2 / 3.0) * (2 * m1 * d1 + 2 * m2 * d2 + 2 * m3 * d3 + 2.0 * d3)
    lad[2, 0] = (r2w2 / (6.0 * math.sqrt(5.0))) * (2 * m1 * d1 + 2 * m2 * d2 - 4 * m3 * d3 - 4 * d3)
    lad[2, 1] = -(r2w2 / math.sqrt(30.0)) * ((d1 - II * d2) * (1.0 + m3) + (m1 - II * m2) * d3)
    lad[2, 2] = (r2w2 / math.sqrt(5.0 * 24.0)) * (2 * m2 * d2 - 2 * m1 * d1 + 2.0 * II * (d1 * m2 + m1 * d2))
    tsld = np.einsum("k,ki->i", tabs.a_tsl[:n2] * sk, tot[None] - r_la)
    trrd = np.einsum("k,ki->i", tabs.a_trr[:n2] * sk, tot[None] - r_la)
    rate_sl = np.zeros((3, 3), dtype=np.complex128)
    rate_rr = np.zeros((3, 3), dtype=np.complex128)
    rate_sl[2, 0:3] = ((1 + kTE2 - hTE2) * lad[2, 0:3] + tsld) / p.gacc
    rate_rr[2, 0:3] = (hTE2 * lad[2, 0:3] + trrd) / p.gacc
    return rate_sl, rate_rr, {"ildot": ild, "mdot": md, "lambdadot": lad}


def rate_grids(sht, dsl, drr, dice00, dt, cst, planet):
    """dSL/dt and dR/dt grids (solver.py:788-806): the degree-0 rate of sea level is the rate of
    the conservation constant on the end-of-step C*: (-(rho_i / rho_w) dI*_00 / dt
    - mean(C* dSL/dt|l>=1)) / mean(C*)."""
    p = planet
    g = np.array(sht.synthesis(dsl), copy=True)
    a = sht.analysis(g * cst)[0, 0].real
    c00 = sht.analysis(cst)[0, 0].real
    dsl[0, 0] = (-(p.rhoi / p.rhow) * dice00.real / float(dt) - a) / c00
    g = np.array(sht.synthesis(dsl), copy=True)
    gr = np.array(sht.synthesis(drr), copy=True)
    return {"dSLdt": g, "dRdt": gr, "dSLdt_lm": dsl, "dRdt_lm": drr}
