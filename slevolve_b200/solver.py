"""GPU sea-level solver behind the reference's solver interface.

``SeaLevelSolver`` mirrors SLEvolve ``python/slevolve/solver.py:518-1144`` (constructor
arguments, ``step(icexy_cur, profile=False, dt=None, rates=False) -> dict``, step-0 attributes)
and ``OptSeaLevelSolver`` mirrors ``solver_opt.py:267-979`` (``opt`` set, ``inner``), so that the
forward driver (run_ais.py:322) and the outer driver (run_outer.py:216) can construct them in
place of the reference classes.  The whole step runs on the device (``libslevolve_b200.so``);
grids in the returned dict are copied to host memory on first access and alias per-solver host
buffers that the next step overwrites, as the reference's do (tests/test_small_case.py:110 of the
reference copies them for that reason).

Branches of the reference that this build does not provide raise ``NotImplementedError``: the
axial-rotation options, Anderson mixing, the reuse variants other than ``"warm"``, analytic rates
of a mixed-precision solve, ramp placement of a mixed-precision solve and the horizontal read-out
together with ramp placement.  Provided: ``ramp=True`` (second-order load placement, FP64),
``step(..., rates=True)`` and ``solver.horizontal = True``.  The ``raw`` option needs a raw-mode
backend (``make_sht("cuda", ..., raw=True)``) and raises ``ValueError`` otherwise, as in the reference
(solver_opt.py:299-301); with it, the spectra the step hands out (``dS_converged``, ``load_inc``,
``horiz``) are in the sign-free convention V[l, m] = (-1)^m U[l, m] of that backend.
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib
from .love import mode_arrays

PI = 3.1415926535898   # truncated legacy literal (solver.py:31)
EPS0 = float(np.finfo(np.float64).eps)


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


def degree_weights(love, norder, planet):
    """T_l, T_l (1 + k_l - h_l), T_l h_l with the reference's expressions (solver.py:596-603)."""
    nl = norder + 1
    l = np.arange(nl, dtype=np.float64)
    ttl = np.zeros(nl)
    ttl[1:] = (4.0 * PI * (planet.radius ** 3)) / (planet.mass * (2 * l[1:] + 1.0))
    ekhl = np.zeros(nl)
    ekhl[1:] = 1 + np.asarray(love.ke)[1:nl] - np.asarray(love.he)[1:nl]
    he = np.zeros(nl)
    he[1:] = np.asarray(love.he)[1:nl]
    return ttl, ttl * ekhl, ttl * he


def earth_struct(love, norder, planet):
    """The C ABI's Earth record for `love` truncated at `norder` (solver.py:252-368, 596-603).

    Returns (SleEarth, keep): `keep` owns the arrays the record points to and must outlive every
    call that reads the record."""
    ma = mode_arrays(love, norder)
    ttl, ttlekhl, ttlhe = degree_weights(love, norder, planet)
    keep = {
        "nmod": np.ascontiguousarray(ma["nmod"], dtype=np.int32),
        "s": np.ascontiguousarray(ma["s"]), "a_sl": np.ascontiguousarray(ma["a_sl"]),
        "a_rr": np.ascontiguousarray(ma["a_rr"]), "ttl": ttl, "ttlekhl": ttlekhl,
        "ttlhe": ttlhe, "a_il": np.ascontiguousarray(ma["a_il"]), "a_m": np.ascontiguousarray(ma["a_m"]),
        "a_tsl": np.ascontiguousarray(ma["a_tsl"]), "a_trr": np.ascontiguousarray(ma["a_trr"])}

    def dp(a):
        return a.ctypes.data_as(C.POINTER(C.c_double))

    nl = norder + 1
    kTE2 = float(love.kTE[2]) if nl > 2 else 0.0
    hTE2 = float(love.hTE[2]) if nl > 2 else 0.0
    kE2 = float(love.ke[2]) if nl > 2 else 0.0
    earth = _lib.SleEarth(nmodes=int(ma["K"]),
                          nmod=keep["nmod"].ctypes.data_as(C.POINTER(C.c_int)),
                          s=dp(keep["s"]), a_sl=dp(keep["a_sl"]), a_rr=dp(keep["a_rr"]),
                          ttl=dp(ttl), ttlekhl=dp(ttlekhl), ttlhe=dp(ttlhe),
                          a_il=dp(keep["a_il"]), a_m=dp(keep["a_m"]), a_tsl=dp(keep["a_tsl"]),
                          a_trr=dp(keep["a_trr"]), kTE2=kTE2, hTE2=hTE2, kE2=kE2)
    return earth, keep


class _StepResult(dict):
    """Step outputs; grid and spectrum entries are fetched from the device on first access."""

    _GRIDS = {"tgrid": _lib.F_TGRID, "ocean": _lib.F_OCEAN, "beta": _lib.F_BETA, "R": _lib.F_R,
              "G": _lib.F_G, "deltasl": _lib.F_DELTASL, "icestar": _lib.F_ICESTAR}
    _SPECS = {"dS_converged": _lib.F_DS_CONVERGED, "load_inc": _lib.F_LOAD_INC}

    def __init__(self, solver, scalars):
        super().__init__(scalars)
        self._solver = solver

    def __missing__(self, key):
        if key in self._GRIDS:
            if key in ("R", "G") and not self._solver.calcRG:
                return None
            v = self._solver._fetch(key, self._GRIDS[key])
        elif key in self._SPECS:
            v = self._solver._fetch(key, self._SPECS[key], spectral=True)
            if self._solver._raw:
                v[:, 1::2] *= -1.0
        else:
            raise KeyError(key)
        self[key] = v
        return v

    def get(self, key, default=None):
        try:
            return self[key]
        except KeyError:
            return default

    def __contains__(self, key):
        return dict.__contains__(self, key) or key in self._GRIDS or key in self._SPECS


class SeaLevelSolver:
    """Exact-memory sea-level solver on the GPU (the reference's plain path, FP64)."""

    _opt_default = ()
    _inner_default = "off"

    def __init__(self, sht, love, topo0, ice0, *, norder=512, dt=1, tpw=True, checkmarine=True,
                 calcRG=True, epsilon1=1.0e-5, planet=None, mem_threads=1, ramp=False,
                 axial_rotation="off", axial_tau_c=None, opt=None, inner=None, reuse="off",
                 reuse_store=None, anderson_depth=3, max_mask_refresh=3, anderson_freeze=2,
                 anderson_keep=False, precision="fp64"):
        opt = set(self._opt_default if opt is None else opt)
        prec = _lib.precision_code(precision)
        inner = self._inner_default if inner is None else inner
        if axial_rotation != "off":
            raise NotImplementedError("axial_rotation options are not provided by the GPU solver")
        if ramp and prec != _lib.PREC_FP64:
            raise NotImplementedError("ramp placement is provided for precision='fp64' solves")
        if inner not in ("off", "extrap", "anderson"):
            raise ValueError(f"inner must be one of ('off', 'extrap', 'anderson'), got {inner!r}")
        if inner == "anderson":
            raise NotImplementedError("Anderson mixing is not provided by the GPU solver")
        if reuse not in ("off", "warm", "warm+ice", "warm+corr", "warm+corr2"):
            raise ValueError(f"reuse must be off|warm|warm+ice|warm+corr|warm+corr2, got {reuse!r}")
        if reuse not in ("off", "warm"):
            raise NotImplementedError(f"reuse={reuse!r} is not provided by the GPU solver (off, warm are)")
        unknown = opt - {"raw", "diag", "dsl", "numba", "sums"}
        if unknown:
            raise ValueError(f"unknown opt {sorted(unknown)}")
        raw_backend = bool(getattr(sht, "raw", False))
        if ("raw" in opt) != raw_backend:
            raise ValueError("--opt raw must be used with a raw-mode SHT backend")
        # spectra handed out are in the backend's convention: V[l, m] = (-1)^m U[l, m] in raw mode
        self._raw = raw_backend
        topo0 = np.ascontiguousarray(topo0, dtype=np.float64)
        nlat, nlon = topo0.shape
        norder = int(norder)
        if sht is not None:
            for attr, val in (("nlat", nlat), ("nlon", nlon), ("lmax", norder)):
                got = getattr(sht, attr, val)
                if got != val:
                    raise ValueError(f"sht.{attr}={got} does not match the solver ({val})")
        self.sht = sht
        self.love = love
        self.norder = norder
        self.nl = norder + 1
        self.dt = float(dt)
        self.tpw = bool(tpw)
        self.checkmarine = bool(checkmarine)
        self.calcRG = bool(calcRG)
        self.horizontal = False
        self.ramp = bool(ramp)   # second-order load placement (solver.py:584-586)
        self.epsilon1 = float(epsilon1)
        self.p = planet or Planet()
        self.nlat, self.nlon = nlat, nlon
        self.opt = opt
        self.inner = inner
        self.reuse = reuse
        self.reuse_store = reuse_store if reuse_store is not None else {}
        self.reuse_stats = {"warm_steps": 0, "ice_reused": 0, "ice_recomputed": 0}
        self.inner_stats = {"mixed": 0, "plain": 0, "fallback": 0, "singular": 0,
                            "mask_refresh": 0, "frozen_iters": 0}
        self.gr_counts = {"reguess": 0, "ice_analyses": 0}
        self.prof = {}
        self.iter = 0

        L = _lib.lib()
        self._L = L
        p = self.p
        cfg = _lib.SleConfig(nlat=nlat, nlon=nlon, lmax=norder, dt_years=self.dt,
                             epsilon1=self.epsilon1, tpw=int(self.tpw),
                             checkmarine=int(self.checkmarine), calcRG=int(self.calcRG),
                             opt_dsl=int("dsl" in opt), opt_diag=int("diag" in opt),
                             inner_extrap=int(inner == "extrap"), radius=p.radius, mass=p.mass,
                             rhoi=p.rhoi, rhow=p.rhow, gacc=p.gacc, omega=p.omega, moiA=p.moiA,
                             moiC=p.moiC, kf=p.kf, precision=prec)
        self.precision = "mixed" if prec == _lib.PREC_MIXED else "fp64"
        earth, self._earth_arrays = earth_struct(love, norder, p)
        h = C.c_void_p()
        _lib.check(L.sle_solver_create(C.byref(cfg), C.byref(earth), C.byref(h)), "sle_solver_create")
        self._h = h
        self._host = {}
        self.tinit_0 = topo0
        self.tinit = topo0
        ice0 = np.ascontiguousarray(ice0, dtype=np.float64)
        if ice0.shape != topo0.shape:
            raise ValueError(f"ice0 shape {ice0.shape} != topography shape {topo0.shape}")
        a0, b0, v0 = C.c_double(), C.c_double(), C.c_double()
        _lib.check(L.sle_solver_init(h, topo0.ctypes.data, ice0.ctypes.data, 0, C.byref(a0),
                                     C.byref(b0), C.byref(v0)), "sle_solver_init")
        self.ocean_area0 = a0.value
        self.oceanBeta_area0 = b0.value
        self.ice_volume0 = v0.value
        self.cxy0 = self._fetch("_ocean0", _lib.F_OCEAN0).copy()
        self.beta0 = self._fetch("_beta0", _lib.F_BETA0).copy()
        self.cstar0 = self.cxy0 * self.beta0
        self._info = _lib.SleStepInfo()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.sle_solver_destroy(h)
            except Exception:
                pass
            self._h = None

    # ---------------------------------------------------------------- helpers
    def _host_buffer(self, key, shape, dtype):
        buf = self._host.get(key)
        if buf is None:
            try:
                import torch

                t = torch.empty(shape, dtype=torch.float64 if dtype == np.float64 else torch.complex128)
                t = t.pin_memory()
                buf = (t, t.numpy())
            except Exception:
                arr = np.empty(shape, dtype=dtype)
                buf = (None, arr)
            self._host[key] = buf
        return buf[1]

    def _fetch(self, key, field, spectral=False):
        if spectral:
            arr = self._host_buffer(key, (self.nl, self.nl), np.complex128)
        else:
            arr = self._host_buffer(key, (self.nlat, self.nlon), np.float64)
        _lib.check(self._L.sle_solver_get(self._h, int(field), arr.ctypes.data, 0), "sle_solver_get")
        return arr

    def stream_handle(self):
        s = C.c_void_p()
        _lib.check(self._L.sle_solver_stream(self._h, C.byref(s)), "sle_solver_stream")
        return s.value

    # ------------------------------------------------------------ snapshots
    _SNAP_KEYS = ("iter", "dt", "gr_counts", "reuse_stats", "inner_stats")

    def snapshot(self):
        """The solve's state after its last step, on the host: ``{"image": uint8 array, ...}``
        with the device image (modal state, load history, topography, masks, rotational state,
        step lengths; ``sle_solver_snapshot``) and the solver's own counters.  The dict can be
        saved with ``numpy.savez``.  The counterpart of the reference's modal-state checkpoint
        (fortran/src/modal_state_mod.f90:445-477) and of swapping the Python solver's ``state``
        object (tests/test_small_case.py:106)."""
        n = C.c_longlong()
        _lib.check(self._L.sle_solver_snapshot_bytes(self._h, C.byref(n)), "sle_solver_snapshot_bytes")
        img = np.empty(int(n.value), dtype=np.uint8)
        _lib.check(self._L.sle_solver_snapshot(self._h, C.c_void_p(img.ctypes.data), n.value),
                   "sle_solver_snapshot")
        snap = {"image": img, "ramp": self.ramp, "precision": self.precision,
                "tinit_0": np.array(self.tinit_0, copy=True), "ocean_area0": self.ocean_area0,
                "oceanBeta_area0": self.oceanBeta_area0, "ice_volume0": self.ice_volume0}
        for k in self._SNAP_KEYS:
            v = getattr(self, k)
            snap[k] = dict(v) if isinstance(v, dict) else v
        return snap

    def restore(self, snap):
        """Continue from ``snapshot()`` of this or another solver of the same grid, degree, mode
        capacity, precision and options: the next ``step`` gives bit for bit what the
        snapshotted solver's next step would have given."""
        if bool(snap.get("ramp", False)) != self.ramp or snap.get("precision", self.precision) != self.precision:
            raise ValueError("snapshot of a solve with other ramp or precision settings")
        img = np.ascontiguousarray(snap["image"], dtype=np.uint8)
        _lib.check(self._L.sle_solver_restore(self._h, C.c_void_p(img.ctypes.data), img.size),
                   "sle_solver_restore")
        for k in self._SNAP_KEYS:
            if k in snap:
                v = snap[k]
                setattr(self, k, dict(v) if isinstance(v, dict) else v)
        self.iter = int(self.iter)
        self.dt = float(self.dt)
        self._ramp_dt = None      # ramp table uploaded again for the next step's length
        # step-0 attributes of the restored solve (run_ais.py:360-367 reads them)
        if "tinit_0" in snap:
            self.tinit_0 = self.tinit = np.array(snap["tinit_0"], copy=True)
        for k in ("ocean_area0", "oceanBeta_area0", "ice_volume0"):
            if k in snap:
                setattr(self, k, float(snap[k]))
        self.cxy0 = self._fetch("_ocean0", _lib.F_OCEAN0).copy()
        self.beta0 = self._fetch("_beta0", _lib.F_BETA0).copy()
        self.cstar0 = self.cxy0 * self.beta0

    def set_step_dt(self, dt):
        """Length of the next steps (yr), as the reference's ``set_step_dt``; the device keeps the
        previous length for a non-positive value, so zero and negative lengths are refused."""
        if dt is not None:
            dt = float(dt)
            if not dt > 0.0:
                raise ValueError(f"step length must be positive (got dt={dt!r})")
            self.dt = dt

    # ------------------------------------------------------------------ step
    def _reuse_register(self, k):
        """Device reuse store for step k (reuse="warm"): kept in ``reuse_store`` across the
        solvers of successive outer passes."""
        from .reuse import ReuseStore

        st = self.reuse_store.get("_device_store")
        if st is None:
            nc = (self.nl * (self.nl + 1)) // 2
            st = self.reuse_store["_device_store"] = ReuseStore(nc, self.nlat * self.nlon)
        if k == 1:
            self._reuse_valid = st.recorded   # entries of the previous pass
        st.ensure(k)
        ds, mask = st.pointers()
        _lib.check(self._L.sle_solver_set_reuse(self._h, ds, mask, st.capacity, self._reuse_valid),
                   "sle_solver_set_reuse")
        return st

    def step_device(self, ice_ptr, on_device, dt=None):
        """One step from a raw pointer (host or device); returns the step info record.  The ramp
        coefficients follow the step length here, so a ramp solve stepped through this call gets
        the same placement as through ``step``."""
        self.set_step_dt(dt)
        self._ramp_setup(self.dt)
        st = self._reuse_register(self.iter + 1) if self.reuse == "warm" else None
        rc = self._L.sle_solver_step(self._h, C.c_void_p(ice_ptr), int(on_device),
                                     float(self.dt), C.byref(self._info))
        _lib.check(rc, "sle_solver_step")
        if st is not None:
            if self._info.iter <= self._reuse_valid:
                self.reuse_stats["warm_steps"] += 1
            st.recorded = max(st.recorded, self._info.iter)
        self.iter = self._info.iter
        self.gr_counts["reguess"] += self._info.gr_reguess
        self.gr_counts["ice_analyses"] += self._info.gr_ice_analyses
        return self._info

    def _rates_setup(self, rates, dt):
        """Turn the device rate read-out on (with this step's weights) or off."""
        if rates:
            if self.precision != "fp64":
                raise NotImplementedError("analytic rates are provided for precision='fp64' solves")
            from .rates import RateTables

            if getattr(self, "_rate_tabs", None) is None:
                self._rate_tabs = RateTables(self.love, self.norder)
            h = float(dt) if dt is not None else float(self.dt)
            tab = self._rate_tabs.for_dt(h)
            if getattr(self, "_rates_dt", None) != h:
                _lib.check(self._L.sle_solver_set_rate_tables(self._h, tab.ctypes.data), "sle_solver_set_rate_tables")
                self._rates_dt = h
            return h
        if getattr(self, "_rates_dt", None) is not None:
            _lib.check(self._L.sle_solver_set_rate_tables(self._h, None), "sle_solver_set_rate_tables")
            self._rates_dt = None
        return None

    def _ramp_setup(self, dt):
        """Coefficients of the ramp placement for this step's length, uploaded when the length
        changes (solver.py:348-368: omphi = 1 - phi, c_sl, c_rr per degree scaled by ttl, and the
        degree-2 c_il, c_m, c_tsl, c_trr)."""
        if not self.ramp:
            return
        h = float(dt) if dt is not None else float(self.dt)
        if getattr(self, "_ramp_dt", None) == h:
            return
        from .love import mode_arrays
        from .rates import ramp_table

        if getattr(self, "_ramp_ma", None) is None:
            self._ramp_ma = mode_arrays(self.love, self.norder)
        tab = ramp_table(self._ramp_ma, self.love, self.norder, self._earth_arrays["ttl"], h)
        _lib.check(self._L.sle_solver_set_ramp(self._h, tab.ctypes.data), "sle_solver_set_ramp")
        self._ramp_dt = h

    def _horizontal_setup(self):
        """Weights of the horizontal read-out (a_hl = l_k / s_k, ttl l^E; solver.py:424-434,
        697-700), uploaded once; off again when ``horizontal`` is cleared."""
        on = bool(getattr(self, "horizontal", False))
        if on and not getattr(self, "_horiz_set", False):
            love, L = self.love, self.norder
            K = int(love.max_modes)   # the solver's mode capacity (mode_arrays)
            nl = L + 1
            a_hl = np.zeros((K, nl))
            a_thl = np.zeros(K)
            for l in range(1, nl):
                nm = int(love.nmod[l])
                a_hl[:nm, l] = love.rl[:nm, l] / love.s[:nm, l]
                if l == 2:
                    a_thl[:nm] = love.rlT[:nm, l] / love.s[:nm, l]
            le = np.concatenate(([0.0], np.asarray(love.le[1:nl], float)))
            ttl = np.asarray(self._earth_arrays["ttl"], float)
            tab = np.ascontiguousarray(np.concatenate([a_hl.ravel(), ttl * le]), dtype=np.float64)
            _lib.check(self._L.sle_solver_set_horizontal(self._h, tab.ctypes.data), "sle_solver_set_horizontal")
            self._horiz_set, self._horiz_K, self._a_thl = True, K, a_thl
        elif not on and getattr(self, "_horiz_set", False):
            _lib.check(self._L.sle_solver_set_horizontal(self._h, None), "sle_solver_set_horizontal")
            self._horiz_set = False
        return on

    def _horizontal_read(self):
        """Psi_lm of the step in the U convention (solver.py:687-720): the device potential plus
        the degree-2 rotational term (l^T_E Lambda_tot + sum_k a_thl r_Lambda,k) / g."""
        K = self._horiz_K
        hz = np.empty((self.nl, self.nl), dtype=np.complex128)
        r_lam = np.empty(6 * K)
        lam12 = np.empty(12)
        _lib.check(self._L.sle_solver_get_horizontal(self._h, hz.ctypes.data, r_lam.ctypes.data, lam12.ctypes.data),
                   "sle_solver_get_horizontal")
        if self.tpw and self.norder >= 2:
            r_la = r_lam.reshape(K, 3, 2) @ np.array([1.0, 1j])
            thl = np.zeros(3, dtype=np.complex128)
            for k in range(int(self.love.nmod[2])):
                thl += self._a_thl[k] * r_la[k]
            prev = lam12[:6].reshape(3, 2) @ np.array([1.0, 1j])
            cur = lam12[6:].reshape(3, 2) @ np.array([1.0, 1j])
            rot = (self.love.lTE[2] * (prev + cur) + thl) / self.p.gacc
            hz[2, 0:3] += rot
        if self._raw:
            hz[:, 1::2] *= -1.0
        return hz

    def _rates_read(self, info, h):
        """The reference's rates dict of the step just taken (solver.py:766-806)."""
        from .rates import rate_grids, rotation_rate
        from .sht import make_sht

        tabs = self._rate_tabs
        K = tabs.K
        dsl = np.empty((self.nl, self.nl), dtype=np.complex128)
        drr = np.empty_like(dsl)
        rec = np.empty(20)
        rot = np.empty(18 * K)
        _lib.check(self._L.sle_solver_get_rates(self._h, dsl.ctypes.data, drr.ctypes.data, rec.ctypes.data,
                                                rot.ctypes.data), "sle_solver_get_rates")
        out_rot = None
        if self.tpw and self.norder >= 2:
            lam = np.array(info.lam[:]).reshape(3, 3, 2)
            rs, rr, out_rot = rotation_rate(
                tabs, self.love, self.p, h, np.array(info.il[:]).reshape(3, 3), np.array(info.mm[:]),
                lam[..., 0] + 1j * lam[..., 1], rec[2:11].reshape(3, 3), rec[11:14].copy(),
                rec[14:20].reshape(3, 2) @ np.array([1.0, 1j]), rot[:9 * K].reshape(K, 3, 3),
                rot[9 * K:12 * K].reshape(K, 3), rot[12 * K:].reshape(K, 3, 2) @ np.array([1.0, 1j]))
            dsl[0:3, 0:3] += rs
            drr[0:3, 0:3] += rr
        if getattr(self, "_rate_sht", None) is None:
            self._rate_sht = make_sht("cuda", self.nlat, self.nlon, self.norder)
        cst = self._fetch("_rate_ocean", _lib.F_OCEAN) * self._fetch("_rate_beta", _lib.F_BETA)
        out = rate_grids(self._rate_sht, dsl, drr, complex(rec[0], rec[1]), h, cst, self.p)
        if out_rot is not None:
            out.update(out_rot)
        return out

    def step(self, icexy_cur, profile=False, dt=None, rates=False):
        if dt is not None and not float(dt) > 0.0:
            raise ValueError(f"step length must be positive (got dt={dt!r})")
        h_rates = self._rates_setup(rates, dt)
        horiz = self._horizontal_setup()
        if horiz and self.ramp:
            raise NotImplementedError("the horizontal read-out is not provided together with ramp placement")
        t0 = time.perf_counter()
        try:
            import torch

            is_dev = isinstance(icexy_cur, torch.Tensor) and icexy_cur.is_cuda
        except ImportError:  # pragma: no cover
            is_dev = False
        if is_dev:
            ice = icexy_cur.to(torch.float64).contiguous()
            if tuple(ice.shape) != (self.nlat, self.nlon):
                raise ValueError(f"ice shape {tuple(ice.shape)} != {(self.nlat, self.nlon)}")
            torch.cuda.current_stream().synchronize()
            info = self.step_device(ice.data_ptr(), 1, dt)
        else:
            ice = np.ascontiguousarray(icexy_cur, dtype=np.float64)
            if ice.shape != (self.nlat, self.nlon):
                raise ValueError(f"ice shape {ice.shape} != {(self.nlat, self.nlon)}")
            info = self.step_device(ice.ctypes.data, 0, dt)
        wall = time.perf_counter() - t0
        lam = np.array(info.lam[:]).reshape(3, 3, 2)
        scal = {
            "iter": info.iter,
            "numiter": info.numiter,
            "horiz": self._horizontal_read() if horiz else None,
            "ocean_area": info.ocean_area,
            "oceanBeta_area": info.oceanBeta_area,
            "gmslc_ocn": info.gmslc_ocn,
            "gmslc_ocnBeta": info.gmslc_ocnBeta,
            "ice_volume": info.ice_volume,
            "il": np.array(info.il[:]).reshape(3, 3),
            "mm": np.array(info.mm[:]),
            "lambda": lam[..., 0] + 1j * lam[..., 1],
            "rates": self._rates_read(info, h_rates) if rates else None,
            "wall": wall,
            "xi": info.xi,
            "prof": {"total": wall} if profile else None,
        }
        if isinstance(self, OptSeaLevelSolver):
            scal["inner_stats"] = dict(self.inner_stats)
        if profile:
            self.prof = scal["prof"]
        return _StepResult(self, scal)


class OptSeaLevelSolver(SeaLevelSolver):
    """GPU counterpart of the reference's ``OptSeaLevelSolver`` (solver_opt.py:267-360):
    the ``opt`` set (``dsl``, ``diag`` change the work; ``numba``, ``sums`` are accepted) and
    ``inner`` in {"off", "extrap"}."""

    _opt_default = ()
    _inner_default = "off"


GpuSeaLevelSolver = SeaLevelSolver
