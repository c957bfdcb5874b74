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


def _lambda_jacobian(m, r2w2):
    """d Lambda_2j / d m_i (3 x 3 complex, rows j = 0, 1, 2) of the centrifugal potential's degree-2
    terms as functions of the rotation vector perturbation m (U convention):
    Lambda_20 = r2w2 / (6 sqrt5) (m1^2 + m2^2 - 2 m3^2 - 4 m3),
    Lambda_21 = -r2w2 / sqrt30 (m1 - i m2)(1 + m3),
    Lambda_22 = r2w2 / sqrt120 (m2^2 - m1^2 + 2 i m1 m2)."""
    m1, m2, m3 = m
    c20, c21, c22 = r2w2 / (6.0 * math.sqrt(5.0)), -r2w2 / math.sqrt(30.0), r2w2 / math.sqrt(120.0)
    return np.array([[c20 * 2 * m1, c20 * 2 * m2, c20 * (-4 * m3 - 4)],
                     [c21 * (1 + m3), c21 * (-1j) * (1 + m3), c21 * (m1 - 1j * m2)],
                     [c22 * (-2 * m1 + 2j * m2), c22 * (2 * m2 + 2j * m1), 0.0]], dtype=np.complex128)


def rotation_rate(tabs, love, planet, h, il, mm, lam, oldil, oldm, dlam_prev2, r_il, r_m, r_la):
    """Left derivatives (per year) at the end of the step of the degree-2 rotational terms
    (the reference's _rotation_rate, solver.py:722-764), from the step's converged inertia
    perturbation ``il``, rotation vector ``mm`` and centrifugal potential ``lam``.

    Each degree-2 modal state is first advanced by the commit of this step (its share 1 - phi of
    the step's increment); a state's rate is then s_k (total - state_k) per mode.  The rotation
    rate dm/dt follows from the time derivative of the linearised Liouville equation, the potential
    rate from dLambda/dt = (dLambda/dm) dm/dt.  Returns (rate_sl, rate_rr) as 3 x 3 complex spectra
    (U convention, rows l = 0..2) and the dict of rotational rates."""
    p = planet
    n2 = tabs.nmod2
    share = tabs.omphi[:n2, 2]
    rate_k = tabs.s[:n2, 2] / 1000.0                       # 1/yr per mode
    tot = lam[2, 0:3]
    # states after this step's commit
    st_il = r_il[:n2] + share[:, None, None] * (il - oldil)
    st_m = r_m[:n2] + share[:, None] * (mm - oldm)
    st_la = r_la[:n2] + share[:, None] * (tot - dlam_prev2)
    # viscous parts of the rates: sum_k a_k s_k (total - state_k)
    visc_il = np.tensordot(tabs.a_il[:n2] * rate_k, il - st_il, axes=1)
    visc_m = (tabs.a_m[:n2] * rate_k) @ (mm - st_m)
    visc_tsl = (tabs.a_tsl[:n2] * rate_k) @ (tot - st_la)
    visc_trr = (tabs.a_trr[:n2] * rate_k) @ (tot - st_la)
    ildot = (il - oldil) / h
    # inertia forcing of the third column, elastic (1 + k_E) plus viscous
    forcing = (1 + love.ke[2]) * ildot[:, 2] + visc_il[:, 2]
    mdot = np.empty(3)
    mdot[:2] = (forcing[:2] / (p.moiC - p.moiA) + visc_m[:2] / p.kf) / (1 - love.kTE[2] / p.kf)
    mdot[2] = -forcing[2] / p.moiC
    r2w2 = p.radius ** 2 * p.omega ** 2
    lamdot = np.zeros((3, 3), dtype=np.complex128)
    m1, m2, m3 = mm
    lamdot[0, 0] = (r2w2 / 3.0) * (2 * (m1 * mdot[0] + m2 * mdot[1] + m3 * mdot[2]) + 2.0 * mdot[2])
    lamdot[2, 0:3] = _lambda_jacobian(mm, r2w2) @ mdot
    rate_sl = np.zeros((3, 3), dtype=np.complex128)
    rate_rr = np.zeros((3, 3), dtype=np.complex128)
    rate_sl[2, 0:3] = ((1 + love.kTE[2] - love.hTE[2]) * lamdot[2, 0:3] + visc_tsl) / p.gacc
    rate_rr[2, 0:3] = (love.hTE[2] * lamdot[2, 0:3] + visc_trr) / p.gacc
    return rate_sl, rate_rr, {"ildot": ildot, "mdot": mdot, "lambdadot": lamdot}


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
