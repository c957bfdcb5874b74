"""Oracle sea-level time step (test infrastructure only; see ``oracle/__init__``).

Restates the reference solver's default path:

* ``SeaLevelSolver.__init__`` (solver.py:521-644): step-0 ocean function, grounded-ice mask
  beta0 (flotation test against the initial topography, solver.py:647-653), the three step-0
  analyses for areas and volume, and the degree weights T_l = 4 pi a^3 / (M (2l+1)),
  T_l (1 + k_l - h_l), T_l h_l.
* ``SeaLevelSolver.step`` (solver.py:814-1144): modal advance; grounded ice I* on the previous
  topography and its analysis; beta = (I* < EPS0), C* = C beta, tO = T0 (C* - C*_0) and their
  analyses; eustatic first guess; the inner fixed-point loop (rotation block solver.py:910-975,
  eq. B18 solver.py:977-991, synthesis, rO analysis, conservation constant, load update,
  convergence ratio xi solver.py:1023-1030, ocean-function / grounded re-guess
  solver.py:1032-1045 and 655-684); radial displacement; commit; post-step topography and the
  degree-0 diagnostics.
* options of ``OptSeaLevelSolver`` that keep the fixed point (solver_opt.py): ``"dsl"``
  (deltasl = dsl + conserv * synth(e00)[0,0], solver_opt.py:320-325, 669-676), ``"diag"``
  (degree-0 diagnostics by row-sum quadrature, solver_opt.py:893-916), ``inner="extrap"``
  (first guess 2 dS_{n-1} - dS_{n-2}, variable-step form solver_opt.py:148-165, applied at
  504-513 and stored at 817-822), and ``reuse="warm"`` (warm start from the converged increment
  and ocean mask of the same step of the previous outer pass, solver_opt.py:400-403, 514-528,
  932-947).

The ramp placement, axial rotation, Anderson mixing, rates and horizontal read-out are
default-off branches of the reference and are not restated (the GPU path rejects them).
"""

from __future__ import annotations

import math
import time

import numpy as np

from .memory import ModalState

PI = 3.1415926535898                       # truncated literal (solver.py:31)
EPS0 = float(np.finfo(np.float64).eps)     # solver.py:33
GR_MAXACC = 3                              # solver.py:38
II = 1j


class Planet:
    """Constants of ``planets_mod::earth_init`` (solver.py:98-110)."""

    def __init__(self):
        self.radius = 6.371e6
        self.mass = 5.976e24
        self.rhoi = 920.0
        self.rhow = 1000.0
        self.gacc = 9.80665
        self.omega = 7.292e-5
        self.moiA = 0.3296145 * self.mass * self.radius ** 2
        self.moiC = 0.3307007 * self.mass * self.radius ** 2
        self.kf = 0.9342 + 0.008


def extrap_guess(h1, h2, dt0, dt1, dt2):
    """dS_j guess from dS_{j-1}=h1, dS_{j-2}=h2 (solver_opt.py:148-165)."""
    if dt0 == dt1 == dt2:
        out = h1 * 2.0
        out -= h2
        return out
    w = (dt0 + dt1) / (dt1 + dt2)
    out = h1 * (dt0 / dt1 * (1.0 + w))
    out -= (dt0 / dt2 * w) * h2
    return out


class OracleSolver:
    def __init__(self, sht, love, topo0, ice0, *, norder, dt=1.0, tpw=True, checkmarine=True,
                 calcRG=True, epsilon1=1.0e-5, planet=None, opt=(), inner="off",
                 reuse="off", reuse_store=None, ramp=False):
        if inner not in ("off", "extrap"):
            raise ValueError(f"inner must be off|extrap, got {inner!r}")
        if reuse not in ("off", "warm"):
            raise ValueError(f"reuse must be off|warm, got {reuse!r}")
        self.sht = sht
        self.love = love
        self.norder = int(norder)
        self.nl = self.norder + 1
        self.dt = float(dt)
        self.tpw = bool(tpw)
        self.checkmarine = bool(checkmarine)
        self.calcRG = bool(calcRG)
        self.epsilon1 = float(epsilon1)
        self.p = planet or Planet()
        self.opt = set(opt)
        self.inner = inner
        self.reuse = reuse
        self.reuse_store = reuse_store if reuse_store is not None else {}
        p = self.p
        nl = self.nl
        self.nlat, self.nlon = topo0.shape

        self.tinit = np.ascontiguousarray(topo0, dtype=np.float64)
        self.tinit_0 = self.tinit
        self.cxy0 = (self.tinit < 0).astype(np.float64)
        self._marine_pos = self.tinit > 0
        self._marine_thr = np.abs(self.tinit) * p.rhow / p.rhoi
        g0 = self._icestar(ice0) if self.checkmarine else ice0
        self.beta0 = (g0 < EPS0).astype(np.float64)
        self.cstar0 = self.cxy0 * self.beta0
        self.cxy = self.cxy0.copy()
        self.topo_prev = self.tinit.copy()

        c = sht.analysis(self.cxy0, out=np.zeros((nl, nl), complex))
        self.ocean_area0 = c[0, 0].real * 4 * PI * p.radius ** 2
        c = sht.analysis(self.cstar0, out=np.zeros((nl, nl), complex))
        self.oceanBeta_area0 = c[0, 0].real * 4 * PI * p.radius ** 2
        ic0 = self._icestar(ice0) if self.checkmarine else ice0
        c = sht.analysis(ic0, out=np.zeros((nl, nl), complex))
        self.ice_volume0 = c[0, 0].real * 4 * PI * p.radius ** 2

        self.state = ModalState(love, self.norder, self.dt)
        self.ramp = bool(ramp)           # second-order load placement (solver.py:584-586)
        self.state.ramp = self.ramp
        self.il = np.zeros((3, 3))
        self.mm = np.zeros(3)
        self.lam = np.zeros((3, 3), dtype=np.complex128)

        l = np.arange(nl, dtype=np.float64)
        ttl = np.zeros(nl)
        ttl[1:] = (4.0 * PI * (p.radius ** 3)) / (p.mass * (2 * l[1:] + 1.0))
        ekhl = np.zeros(nl)
        ekhl[1:] = 1 + love.ke[1:nl] - love.he[1:nl]
        he = np.zeros(nl)
        he[1:] = love.he[1:nl]
        self.ttl = ttl[:, None]
        self.ttlekhl = (ttl * ekhl)[:, None]
        self.ttlhe = (ttl * he)[:, None]

        if "dsl" in self.opt:
            e00 = np.zeros((nl, nl), dtype=np.complex128)
            e00[0, 0] = 1.0
            self.K00 = float(sht.synthesis(e00)[0, 0])
        self.icexy_prev = np.ascontiguousarray(ice0, dtype=np.float64)
        self.iter = 0
        self.gr_counts = {"reguess": 0, "ice_analyses": 0}
        self.p_deltaS_hist = []   # converged load increments dS_{n-1}, dS_{n-2}
        self.dt_hist = [self.dt, self.dt]

    # ------------------------------------------------------------------ masks
    def _icestar(self, ice):
        keep = self._marine_pos | (ice > self._marine_thr)
        return ice * keep

    def _icestar_on(self, ice, topo):
        keep = (topo > 0) | (ice > np.abs(topo) * self.p.rhow / self.p.rhoi)
        return ice * keep

    def set_step_dt(self, dt):
        if dt is not None:
            self.dt = float(dt)
            self.state.set_dt(self.dt)

    # ------------------------------------------------------------------- step
    def step(self, icexy_cur, dt=None, rates=False):
        self.set_step_dt(dt)
        p, sht, nl = self.p, self.sht, self.nl
        self.iter += 1
        it = self.iter
        t_all = time.perf_counter()
        st = self.state
        visc, radial, sum_il, sum_m, exact_tsl, exact_trr = st.advance_and_read()
        dS_prev = st.p_ocean
        oldil = st.p_il.copy()
        oldm = st.p_m.copy()
        dlam_prev2 = st.p_lambda.copy()

        rs = self.reuse_store.get(it) if self.reuse != "off" else None
        if rs is not None:
            self.cxy[:] = rs["cxy"]

        ice = np.ascontiguousarray(icexy_cur, dtype=np.float64)
        cm = self.checkmarine
        gr_nacc = 0
        if cm:
            icestar = self._icestar_on(ice, self.topo_prev)
        else:
            icestar = ice.copy()
        icestarlm = sht.analysis(icestar, out=np.zeros((nl, nl), complex))
        if it == 1:
            src = self._icestar(self.icexy_prev) if cm else self.icexy_prev
            oldice = sht.analysis(src, out=np.zeros((nl, nl), complex))
        else:
            oldice = st.prev_ice.copy()
        dice = icestarlm - oldice
        dI = st.p_ice + dice

        beta = (icestar < EPS0).astype(np.float64)
        cstar = self.cxy * beta
        cstarlm = sht.analysis(cstar, out=np.zeros((nl, nl), complex))
        tO = self.tinit * (cstar - self.cstar0)
        tOlm = sht.analysis(tO, out=np.zeros((nl, nl), complex))

        load_inc = cstarlm / cstarlm[0, 0]
        load_inc *= (-p.rhoi / p.rhow) * dice[0, 0]
        dS_cur = np.zeros((nl, nl), dtype=np.complex128)
        if self.inner == "extrap" and len(self.p_deltaS_hist) >= 2:
            h1, h2 = self.p_deltaS_hist
            load_inc = extrap_guess(h1, h2, self.dt, self.dt_hist[0], self.dt_hist[1])
            dS_cur = dS_prev + load_inc
        if rs is not None:
            load_inc = rs["dS"].copy()
            dS_cur = dS_prev + load_inc

        dsl_rot = np.zeros((3, 3), dtype=np.complex128)
        rr_rot = np.zeros((3, 3), dtype=np.complex128)
        dil_cur = np.zeros((3, 3))
        dm_cur = np.zeros(3)
        dlam_cur2 = np.zeros(3, dtype=np.complex128)
        kTE2, hTE2, kE2 = self.love.kTE[2], self.love.hTE[2], self.love.ke[2]
        r2w2 = p.radius ** 2 * p.omega ** 2
        topo = self.topo_prev.copy()
        xi_trace = []

        ninner = 1
        while True:
            if self.tpw:
                z20 = p.rhow * dS_cur[2, 0] + p.rhoi * dI[2, 0]
                z21 = p.rhow * dS_cur[2, 1] + p.rhoi * dI[2, 1]
                self.il[2, 2] = (-8 * PI * p.radius ** 4 / (3 * math.sqrt(5.0))) * z20.real
                self.il[0, 2] = (-8 * PI * p.radius ** 4 / (math.sqrt(30.0))) * z21.real
                self.il[1, 2] = (8 * PI * p.radius ** 4 / (math.sqrt(30.0))) * (-1.0 * II * z21).real
                dil_cur = self.il - oldil
                if self.ramp:
                    # the current increments carry 1 - phi of their viscous response, implicit in m
                    # (solver.py:922-935)
                    sil_r = sum_il + st.c_il * dil_cur
                    al_ = 1 / (1 - kTE2 / p.kf)
                    for i in (0, 1):
                        self.mm[i] = al_ * (
                            (1 / (p.moiC - p.moiA)) * ((1 + kE2) * self.il[i, 2] + sil_r[i, 2])
                            + (1 / p.kf) * (sum_m[i] - st.c_m * oldm[i])
                        ) / (1 - al_ * st.c_m / p.kf)
                    self.mm[2] = -(1.0 / p.moiC) * ((1 + kE2) * self.il[2, 2] + sil_r[2, 2])
                else:
                    for i in (0, 1):
                        self.mm[i] = (1 / (1 - kTE2 / p.kf)) * (
                            (1 / (p.moiC - p.moiA)) * ((1 + kE2) * self.il[i, 2] + sum_il[i, 2])
                            + (1 / p.kf) * sum_m[i])
                    self.mm[2] = -(1.0 / p.moiC) * ((1 + kE2) * self.il[2, 2] + sum_il[2, 2])
                dm_cur = self.mm - oldm
                m1, m2, m3 = self.mm[0], self.mm[1], self.mm[2]
                self.lam[0, 0] = (r2w2 / 3.0) * ((m1 ** 2 + m2 ** 2 + m3 ** 2) + 2.0 * m3)
                self.lam[2, 0] = (r2w2 / (6.0 * math.sqrt(5.0))) * (m1 ** 2 + m2 ** 2 - 2.0 * m3 ** 2 - 4.0 * m3)
                self.lam[2, 1] = -(r2w2 / math.sqrt(30.0)) * ((m1 - II * m2) * (1.0 + m3))
                self.lam[2, 2] = (r2w2 / math.sqrt(5.0 * 24.0)) * (m2 ** 2 - m1 ** 2 + 2.0 * II * m1 * m2)
                dlam_cur2 = self.lam[2, 0:3] - dlam_prev2
                ekhTE = 1 + kTE2 - hTE2
                tot = dlam_prev2 + dlam_cur2
                tsl_v, trr_v = exact_tsl, exact_trr
                if self.ramp:
                    tsl_v = exact_tsl + st.c_tsl * dlam_cur2
                    trr_v = exact_trr + st.c_trr * dlam_cur2
                dsl_rot[:] = 0.0
                dsl_rot[2, 0:3] = (ekhTE * tot + tsl_v) / p.gacc
                if self.calcRG:
                    rr_rot[:] = 0.0
                    rr_rot[2, 0:3] = (hTE2 * tot + trr_v) / p.gacc

            # eq. B18 in the reference's statement order (solver.py:977-991)
            A = dI * p.rhoi
            A += dS_prev * p.rhow
            A += load_inc * p.rhow
            sl_inc = A * self.ttlekhl
            sl_inc += visc * self.ttl
            if self.ramp:   # same-step viscous weight of the current increment (solver.py:988-989)
                sl_inc += (self.ttl[:, 0] * st.c_sl)[:, None] * (p.rhoi * dice + p.rhow * load_inc)
            sl_inc[0:3, 0:3] += dsl_rot

            dslxy = sht.synthesis(sl_inc)
            rOxy = dslxy * cstar
            rOlm = sht.analysis(rOxy, out=np.zeros((nl, nl), complex))
            conserv = ((1 / cstarlm[0, 0])
                       * (-1.0 * (p.rhoi / p.rhow) * dI[0, 0] - rOlm[0, 0] + tOlm[0, 0])).real
            old = load_inc
            new = dS_prev * -1.0
            new += rOlm
            new += cstarlm * conserv
            new -= tOlm
            dS_cur = dS_prev + new
            load_inc = new

            if "dsl" in self.opt:
                deltasl = dslxy + conserv * self.K00
            else:
                sl_tot = sl_inc.copy()
                sl_tot[0, 0] += conserv
                deltasl = sht.synthesis(sl_tot)

            sa = np.abs(new).sum()
            so = np.abs(old).sum()
            if abs(sa - so) < EPS0 and abs(so) < EPS0:
                xi = 0.0
            elif abs(so) < EPS0:
                xi = abs((sa - so) / (EPS0 * 10))
            else:
                xi = abs((sa - so) / so)
            xi_trace.append(float(xi))

            if xi > self.epsilon1:
                topo = self.tinit - deltasl
                self.cxy = (topo < 0.0).astype(np.float64)
                if cm and gr_nacc < GR_MAXACC:
                    gnew = self._icestar_on(ice, topo)
                    bnew = gnew < EPS0
                    nd = int(np.count_nonzero(bnew != (beta != 0.0)))
                    self.gr_counts["reguess"] += 1
                    if nd:
                        icestar = gnew
                        beta = bnew.astype(np.float64)
                        icestarlm = sht.analysis(icestar, out=np.zeros((nl, nl), complex))
                        dice = icestarlm - oldice
                        dI = st.p_ice + dice
                        self.gr_counts["ice_analyses"] += 1
                        gr_nacc += 1
                cstar = self.cxy * beta
                cstarlm = sht.analysis(cstar, out=np.zeros((nl, nl), complex))
                tO = self.tinit * (cstar - self.cstar0)
                tOlm = sht.analysis(tO, out=np.zeros((nl, nl), complex))
            else:
                break
            if ninner == 9999:
                raise RuntimeError(f"inner loop failed to converge, xi={xi}")
            ninner += 1

        if self.inner == "extrap":
            self.p_deltaS_hist = [load_inc.copy()] + self.p_deltaS_hist[:1]
            self.dt_hist = [self.dt, self.dt_hist[0]]

        rrxy = None
        if self.calcRG:
            A = dI * p.rhoi
            A += dS_prev * p.rhow
            A += load_inc * p.rhow
            rrlm = A * self.ttlhe
            rrlm += radial * self.ttl
            if self.ramp:   # solver.py:1065-1067
                rrlm += (self.ttl[:, 0] * st.c_rr)[:, None] * (p.rhoi * dice + p.rhow * load_inc)
            rrlm[0:3, 0:3] += rr_rot
            rrxy = sht.synthesis(rrlm)

        cur = dice * p.rhoi
        cur += load_inc * p.rhow
        cur[0, :] = 0.0
        # optional read-outs, before the commit (solver.py:1075-1088)
        rate_sp = None
        if rates:
            from .readouts import RateWeights, rate_spectra, rotation_rate

            if getattr(self, "_rate_w", None) is None:
                self._rate_w = RateWeights(st)
            self._rate_w.set_dt(st, self.dt)
            dsl_r, drr_r = rate_spectra(st, self._rate_w, cur, float(self.dt), self.ttl, self.ttlekhl, self.ttlhe)
            rot_r = None
            if self.tpw and nl >= 3:
                rs_, rr_, rot_r = rotation_rate(st, self._rate_w, self.love, p, float(self.dt), self.il, self.mm,
                                                self.lam, oldil, oldm, dlam_prev2)
                dsl_r[0:3, 0:3] += rs_
                drr_r[0:3, 0:3] += rr_
            rate_sp = (dsl_r, drr_r, complex(dice[0, 0]), rot_r)
        hz = None
        if getattr(self, "horizontal", False):
            from .readouts import horizontal_psi

            ramp_inc = None
            if self.ramp:
                ramp_inc = p.rhoi * dice + p.rhow * load_inc
            hz = horizontal_psi(st, self.love, p, self.ttl, dI, dS_prev, load_inc,
                                dlam_prev2 + dlam_cur2 if self.tpw else None, self.tpw, ramp_inc=ramp_inc)
        if self.tpw:
            st.commit(cur, dil_cur, dm_cur, dlam_cur2)
        else:
            st.commit(cur)
        st.p_ice[:] = dI
        st.p_ocean[:] = dS_cur
        st.prev_ice[:] = icestarlm

        topo = self.tinit - deltasl
        self.cxy = (topo < 0.0).astype(np.float64)
        self.topo_prev = topo.copy()

        if "diag" in self.opt:
            slc = deltasl * self.cxy
            slc_ocn00 = sht.degree0(slc)
            c00 = sht.degree0(self.cxy)
            slc_b00 = sht.degree0(slc * beta)
            cst00 = sht.degree0(self.cxy * beta)
        else:
            slc = deltasl * self.cxy
            slc_ocn00 = sht.analysis(slc, out=np.zeros((nl, nl), complex))[0, 0]
            c00 = sht.analysis(self.cxy, out=np.zeros((nl, nl), complex))[0, 0]
            slc_b00 = sht.analysis(slc * beta, out=np.zeros((nl, nl), complex))[0, 0]
            cst00 = sht.analysis(self.cxy * beta, out=np.zeros((nl, nl), complex))[0, 0]
        gmslc_ocn = (slc_ocn00 / c00).real
        gmslc_ocnBeta = (slc_b00 / cst00).real

        if self.reuse != "off":
            ent = self.reuse_store.setdefault(it, {})
            ent["dS"] = load_inc.copy()
            ent["cxy"] = self.cxy != 0.0

        self.icexy_prev = ice
        self.beta = beta
        self.load_inc_lm = load_inc
        rate_out = None
        if rate_sp is not None:
            from .readouts import rate_grids

            rate_out = rate_grids(sht, rate_sp[0], rate_sp[1], rate_sp[2], self.dt, self.cxy, beta, p)
            if rate_sp[3] is not None:
                rate_out.update(rate_sp[3])
        return {
            "rates": rate_out,
            "horiz": hz,
            "iter": it,
            "numiter": ninner,
            "tgrid": topo,
            "ocean": self.cxy,
            "beta": beta,
            "R": rrxy,
            "G": (deltasl + rrxy) if rrxy is not None else None,
            "deltasl": deltasl,
            "dS_converged": dS_cur,
            "ocean_area": np.real(c00) * 4 * PI * p.radius ** 2,
            "oceanBeta_area": np.real(cst00) * 4 * PI * p.radius ** 2,
            "gmslc_ocn": gmslc_ocn,
            "gmslc_ocnBeta": gmslc_ocnBeta,
            "ice_volume": icestarlm[0, 0].real * 4 * PI * p.radius ** 2,
            "il": self.il.copy(),
            "mm": self.mm.copy(),
            "lambda": self.lam.copy(),
            "xi": xi_trace,
            "wall": time.perf_counter() - t_all,
        }
