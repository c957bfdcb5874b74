"""Oracle recursive modal state (test infrastructure only; see ``oracle/__init__``).

Restates ``ExactMemory`` of the reference (``python/slevolve/solver.py:244-506``), the
default (step-placement) path:

* weights (solver.py:261-282): a_sl = (r' - r)/s, a_rr = r/s per (mode k, degree l);
  at degree 2 a_il = r'/s, a_m = r'_T/s, a_tsl = (r'_T - r_T)/s, a_trr = r_T/s;
* decay (solver.py:331-346): d = exp(-s dt / 1000) (s in 1/kyr, dt in yr), 1 - d;
* ``advance_and_read`` (solver.py:386-422): R_k <- d R_k + (1 - d) P, then
  visc = sum_k a_sl R_k and rad = sum_k a_rr R_k with k ascending; the degree-2
  rotational states r_il, r_m, r_lambda follow the same update and are summed;
* ``commit`` (solver.py:486-506): P += load, p_il/p_m/p_lambda += increments.

The NumPy statement order of the reference is kept (multiply the state by d, add
(1 - d) P, accumulate), so sums match the reference bit for bit.
"""

from __future__ import annotations

import numpy as np


class ModalState:
    def __init__(self, love, lmax: int, dt_years: float):
        self.lmax = int(lmax)
        nl = self.lmax + 1
        kmax = int(love.max_modes)
        self.kmax = kmax
        s = np.zeros((kmax, nl))
        a_sl = np.zeros((kmax, nl))
        a_rr = np.zeros((kmax, nl))
        a_il = np.zeros(kmax)
        a_m = np.zeros(kmax)
        a_tsl = np.zeros(kmax)
        a_trr = np.zeros(kmax)
        for l in range(1, nl):
            nk = int(love.nmod[l])
            sl = love.s[:nk, l]
            s[:nk, l] = sl
            a_sl[:nk, l] = (love.rprime[:nk, l] - love.r[:nk, l]) / sl
            a_rr[:nk, l] = love.r[:nk, l] / sl
            if l == 2:
                a_il[:nk] = love.rprime[:nk, l] / sl
                a_m[:nk] = love.rprimeT[:nk, l] / sl
                a_tsl[:nk] = (love.rprimeT[:nk, l] - love.rT[:nk, l]) / sl
                a_trr[:nk] = love.rT[:nk, l] / sl
        self.s = s
        self.nmod = [int(love.nmod[l]) for l in range(nl)]
        self.nmod2 = int(love.nmod[2]) if nl > 2 else 0
        self.a_sl, self.a_rr = a_sl, a_rr
        self.a_il, self.a_m, self.a_tsl, self.a_trr = a_il, a_m, a_tsl, a_trr
        self.dt_years = None
        self.decay = np.zeros((kmax, nl))
        self.omd = np.ones((kmax, nl))
        # second-order load placement (solver.py:287-294, 348-368): off unless the solver sets it
        self.ramp = False
        self.phi = np.ones((kmax, nl))
        self.omphi = np.zeros((kmax, nl))
        self.set_dt(dt_years)

        self.R = np.zeros((kmax, nl, nl), dtype=np.complex128)
        self.p_load = np.zeros((nl, nl), dtype=np.complex128)
        self.p_ice = np.zeros((nl, nl), dtype=np.complex128)
        self.p_ocean = np.zeros((nl, nl), dtype=np.complex128)
        self.prev_ice = np.zeros((nl, nl), dtype=np.complex128)
        self.r_il = np.zeros((kmax, 3, 3))
        self.r_m = np.zeros((kmax, 3))
        self.r_lambda = np.zeros((kmax, 3), dtype=np.complex128)
        self.p_il = np.zeros((3, 3))
        self.p_m = np.zeros(3)
        self.p_lambda = np.zeros(3, dtype=np.complex128)

    def set_dt(self, dt_years: float):
        dt_years = float(dt_years)
        if dt_years == self.dt_years:
            return
        d = np.zeros_like(self.decay)
        for l in range(1, self.lmax + 1):
            nk = self.nmod[l]
            d[:nk, l] = np.exp(-self.s[:nk, l] * dt_years / 1000.0)
        self.decay[...] = d
        self.omd[...] = 1.0 - d
        self.dt_years = dt_years
        self._ramp_coeffs(dt_years)

    def _ramp_coeffs(self, dt_years):
        """phi and 1 - phi of every mode for the step length and the same-step viscous weights
        c = sum_k a_k (1 - phi_k) (solver.py:348-368)."""
        from .readouts import ramp_factor

        phi, omp = ramp_factor(self.s * (dt_years / 1000.0))
        exists = self.s > 0
        self.phi[...] = np.where(exists, phi, 1.0)
        self.omphi[...] = np.where(exists, omp, 0.0)
        self.c_sl = (self.a_sl * self.omphi).sum(0)
        self.c_rr = (self.a_rr * self.omphi).sum(0)
        n2 = self.nmod2
        c2 = self.omphi[:n2, 2] if self.lmax >= 2 else np.zeros(0)
        self.c_il = float(c2 @ self.a_il[:n2])
        self.c_m = float(c2 @ self.a_m[:n2])
        self.c_tsl = float(c2 @ self.a_tsl[:n2])
        self.c_trr = float(c2 @ self.a_trr[:n2])

    def advance_and_read(self):
        nl = self.lmax + 1
        visc = np.zeros((nl, nl), dtype=np.complex128)
        rad = np.zeros((nl, nl), dtype=np.complex128)
        P = self.p_load
        for k in range(self.kmax):
            Rk = self.R[k]
            Rk *= self.decay[k][:, None]
            Rk += P * self.omd[k][:, None]
            visc += Rk * self.a_sl[k][:, None]
            rad += Rk * self.a_rr[k][:, None]
        s_il = np.zeros((3, 3))
        s_m = np.zeros(3)
        s_tsl = np.zeros(3, dtype=np.complex128)
        s_trr = np.zeros(3, dtype=np.complex128)
        if self.lmax >= 2:
            for k in range(self.nmod2):
                d = self.decay[k, 2]
                o = 1.0 - d
                self.r_il[k] = d * self.r_il[k] + o * self.p_il
                self.r_m[k] = d * self.r_m[k] + o * self.p_m
                self.r_lambda[k] = d * self.r_lambda[k] + o * self.p_lambda
                s_il += self.a_il[k] * self.r_il[k]
                s_m += self.a_m[k] * self.r_m[k]
                s_tsl += self.a_tsl[k] * self.r_lambda[k]
                s_trr += self.a_trr[k] * self.r_lambda[k]
        return visc, rad, s_il, s_m, s_tsl, s_trr

    def commit(self, load, dil=None, dm=None, dlam=None):
        if self.ramp:
            # the step's increment already carries 1 - phi_k of its response in every mode
            # (solver.py:450-452, 486-499)
            for k in range(self.kmax):
                self.R[k] += self.omphi[k][:, None] * load
            if self.lmax >= 2:
                n2 = self.nmod2
                c = self.omphi[:n2, 2]
                if dil is not None:
                    self.r_il[:n2] += c[:, None, None] * dil[None]
                if dm is not None:
                    self.r_m[:n2] += c[:, None] * dm[None]
                if dlam is not None:
                    self.r_lambda[:n2] += c[:, None] * dlam[None]
        self.p_load += load
        if dil is not None:
            self.p_il += dil
        if dm is not None:
            self.p_m += dm
        if dlam is not None:
            self.p_lambda += dlam
