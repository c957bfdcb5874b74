"""Oracle (test infrastructure only): NumPy restatement of the reference solver's optional
read-outs, the analytic rates and the horizontal-displacement potential (SLEvolve
python/slevolve/solver.py), on the oracle's ``ModalState`` and step.

* ``ramp_factor``        solver.py:229-240
* ``RateWeights``        solver.py:293-294, 347-362 (w = a s / 1000, their sums, phi per step length)
* ``rate_spectra``       solver.py:454-474, 766-785 (modal read before the commit)
* ``rotation_rate``      solver.py:476-484, 722-764
* ``rate_grids``         solver.py:788-806
* ``horizontal_psi``     solver.py:424-448, 687-720 (ramp terms 706-715)
"""

from __future__ import annotations

import math

import numpy as np


def ramp_factor(x):
    x = np.asarray(x, dtype=np.float64)
    small = np.abs(x) < 1.0e-4
    xs = np.where(small, 1.0, x)
    phi = np.where(small, 1.0 - x / 2.0 + x * x / 6.0 - x ** 3 / 24.0, -np.expm1(-xs) / xs)
    omp = np.where(small, x / 2.0 - x * x / 6.0 + x ** 3 / 24.0, (xs + np.expm1(-xs)) / xs)
    return phi, omp


class RateWeights:
    def __init__(self, st):
        self.w_sl = st.a_sl * st.s / 1000.0
        self.w_rr = st.a_rr * st.s / 1000.0
        self.dt = None

    def set_dt(self, st, dt):
        if dt == self.dt:
            return
        phi, omp = ramp_factor(st.s * (dt / 1000.0))
        exists = st.s > 0
        self.phi = np.where(exists, phi, 1.0)
        self.omphi = np.where(exists, omp, 0.0)
        self.ws_sl = self.w_sl.sum(0)
        self.ws_rr = self.w_rr.sum(0)
        self.wsphi_sl = (self.w_sl * self.phi).sum(0)
        self.wsphi_rr = (self.w_rr * self.phi).sum(0)
        self.dt = dt


def rate_spectra(st, wt, cur, h, ttl, ttlekhl, ttlhe):
    """Rate spectra of sea level and radial displacement (no rotation), per year."""
    nl = st.lmax + 1
    q_sl = np.zeros((nl, nl), dtype=np.complex128)
    q_rr = np.zeros((nl, nl), dtype=np.complex128)
    for k in range(st.kmax):
        q_sl += wt.w_sl[k][:, None] * st.R[k]
        q_rr += wt.w_rr[k][:, None] * st.R[k]
    rs = wt.ws_sl[:, None] * st.p_load - q_sl + wt.wsphi_sl[:, None] * cur
    rr = wt.ws_rr[:, None] * st.p_load - q_rr + wt.wsphi_rr[:, None] * cur
    dsl = ttlekhl * cur / h + ttl * rs
    drr = ttlhe * cur / h + ttl * rr
    dsl[0, :] = 0.0
    drr[0, :] = 0.0
    return dsl, drr


def rotation_rate(st, wt, love, p, h, il, mm, lam, oldil, oldm, dlam_prev2):
    n2 = st.nmod2
    dil = il - oldil
    dm = mm - oldm
    tot = lam[2, 0:3].copy()
    c = wt.omphi[:n2, 2]
    r_il = st.r_il[:n2] + c[:, None, None] * dil[None]
    r_m = st.r_m[:n2] + c[:, None] * dm[None]
    r_la = st.r_lambda[:n2] + c[:, None] * (tot - dlam_prev2)[None]
    sk = st.s[:n2, 2] / 1000.0
    kTE2, hTE2, kE2 = love.kTE[2], love.hTE[2], love.ke[2]
    ild = dil / h
    sild = np.einsum("k,kij->ij", st.a_il[:n2] * sk, il[None] - r_il)
    smd = np.einsum("k,ki->i", st.a_m[:n2] * sk, mm[None] - r_m)
    alpha = 1 / (1 - kTE2 / p.kf)
    md = np.zeros(3)
    for i in (0, 1):
        md[i] = alpha * ((1 / (p.moiC - p.moiA)) * ((1 + kE2) * ild[i, 2] + sild[i, 2]) + smd[i] / p.kf)
    md[2] = -(1.0 / p.moiC) * ((1 + kE2) * ild[2, 2] + sild[2, 2])
    m1, m2, m3 = mm
    d1, d2, d3 = md
    r2w2 = p.radius ** 2 * p.omega ** 2
    lad = np.zeros((3, 3), dtype=np.complex128)
    lad[0, 0] = (r2w2 / 3.0) * (2 * m1 * d1 + 2 * m2 * d2 + 2 * m3 * d3 + 2.0 * d3)
    lad[2, 0] = (r2w2 / (6.0 * math.sqrt(5.0))) * (2 * m1 * d1 + 2 * m2 * d2 - 4 * m3 * d3 - 4 * d3)
    lad[2, 1] = -(r2w2 / math.sqrt(30.0)) * ((d1 - 1j * d2) * (1.0 + m3) + (m1 - 1j * m2) * d3)
    lad[2, 2] = (r2w2 / math.sqrt(5.0 * 24.0)) * (2 * m2 * d2 - 2 * m1 * d1 + 2.0 * 1j * (d1 * m2 + m1 * d2))
    tsld = np.einsum("k,ki->i", st.a_tsl[:n2] * sk, tot[None] - r_la)
    trrd = np.einsum("k,ki->i", st.a_trr[:n2] * sk, tot[None] - r_la)
    rate_sl = np.zeros((3, 3), dtype=np.complex128)
    rate_rr = np.zeros((3, 3), dtype=np.complex128)
    rate_sl[2, 0:3] = ((1 + kTE2 - hTE2) * lad[2, 0:3] + tsld) / p.gacc
    rate_rr[2, 0:3] = (hTE2 * lad[2, 0:3] + trrd) / p.gacc
    return rate_sl, rate_rr, {"ildot": ild, "mdot": md, "lambdadot": lad}


def rate_grids(sht, dsl, drr, dice00, dt, cxy, beta, p):
    nl = dsl.shape[0]
    g = sht.synthesis(dsl).copy()
    cst = cxy * beta
    a = sht.analysis(g * cst, out=np.zeros((nl, nl), complex))[0, 0].real
    c00 = sht.analysis(cst, out=np.zeros((nl, nl), complex))[0, 0].real
    dsl[0, 0] = (-(p.rhoi / p.rhow) * dice00.real / float(dt) - a) / c00
    g = sht.synthesis(dsl).copy()
    gr = sht.synthesis(drr).copy()
    return {"dSLdt": g, "dRdt": gr, "dSLdt_lm": dsl, "dRdt_lm": drr}


def horizontal_psi(st, love, p, ttl, dI, dS_prev, load_inc, rot_tot, tpw, ramp_inc=None):
    """Psi_lm of the horizontal displacement, U convention.  With the ramp placement
    (``ramp_inc`` = rho_i dI*_step + rho_w load_inc) the same-step viscous weights
    c_hl = sum_k a_hl (1 - phi_k) and the degree-2 tidal c_thl = sum_k a_thl (1 - phi_k) add
    their terms (solver.py:706-715)."""
    nl = st.lmax + 1
    a_hl = np.zeros((st.kmax, nl))
    a_thl = np.zeros(st.kmax)
    for l in range(1, nl):
        nm = int(love.nmod[l])
        a_hl[:nm, l] = love.rl[:nm, l] / love.s[:nm, l]
        if l == 2:
            a_thl[:nm] = love.rlT[:nm, l] / love.s[:nm, l]
    le = np.concatenate(([0.0], np.asarray(love.le[1:nl], float)))
    ttlle = ttl * le[:, None]
    visc_h = np.zeros((nl, nl), dtype=np.complex128)
    for k in range(st.kmax):
        visc_h += a_hl[k][:, None] * st.R[k]
    thl = np.zeros(3, dtype=np.complex128)
    if st.lmax >= 2:
        for k in range(st.nmod2):
            thl += a_thl[k] * st.r_lambda[k]
    A = p.rhoi * dI + p.rhow * dS_prev
    A += p.rhow * load_inc
    hz = ttlle * A + ttl * visc_h
    if ramp_inc is not None:
        c_hl = (a_hl * st.omphi).sum(0)
        hz += (ttl[:, 0] * c_hl)[:, None] * ramp_inc
    hz[0, :] = 0.0
    if tpw and rot_tot is not None and st.lmax >= 2:
        if ramp_inc is not None:
            n2 = st.nmod2
            c_thl = float(st.omphi[:n2, 2] @ a_thl[:n2])
            thl = thl + c_thl * (rot_tot - st.p_lambda)
        hz[2, 0:3] += (love.lTE[2] * rot_tot + thl) / p.gacc
    return hz
