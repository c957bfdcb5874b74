"""Batches of independent sea-level solves on one GPU (``sle_batch_*`` in the C ABI).

``SolverBatch(nlat, nlon, lmax, nslots, ...)`` holds ``nslots`` solves ("slots") of one grid size
and one configuration (rotation, marine check, options, precision).  Each slot has its own Earth
model, step length, topography, ice history and modal state, all resident on the device.  One
``step`` advances every slot that is given ice by one time step of ``SeaLevelSolver.step``
(SLEvolve python/slevolve/solver.py:814-1144) with the kernel launches of a single solve; slots
converge independently and a converged slot drops out of the remaining inner iterations.  Slots
are loaded, stepped and released between steps in any order, which is what the serving loop
(``slevolve_b200.serving``) builds continuous batching on.

A slot's results do not depend on which other slots share the batch: every reduction is per slot
and in a fixed order, and the tensor-core contraction treats each field as its own columns.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .solver import PI, Planet, earth_struct

FIELDS = {"tgrid": _lib.F_TGRID, "ocean": _lib.F_OCEAN, "beta": _lib.F_BETA, "R": _lib.F_R,
          "G": _lib.F_G, "deltasl": _lib.F_DELTASL, "icestar": _lib.F_ICESTAR}


def _is_cuda_tensor(x):
    try:
        import torch
    except ImportError:  # pragma: no cover
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


class SolverBatch:
    """``nslots`` independent solves of one grid size stepped together on the GPU."""

    def __init__(self, nlat, nlon, lmax, nslots, *, max_modes=8, precision="mixed", tpw=True,
                 checkmarine=True, calcRG=True, epsilon1=1.0e-5, planet=None, opt=("dsl", "diag"),
                 inner="extrap"):
        opt = set(opt)
        unknown = opt - {"diag", "dsl", "numba", "sums"}
        if unknown:
            raise ValueError(f"unknown opt {sorted(unknown)}")
        if inner not in ("off", "extrap"):
            raise ValueError(f"inner must be 'off' or 'extrap' for a batch, got {inner!r}")
        self.nlat, self.nlon, self.lmax = int(nlat), int(nlon), int(lmax)
        self.nslots = int(nslots)
        self.p = planet or Planet()
        self.precision = "mixed" if _lib.precision_code(precision) == _lib.PREC_MIXED else "fp64"
        p = self.p
        cfg = _lib.SleConfig(nlat=self.nlat, nlon=self.nlon, lmax=self.lmax, dt_years=1.0,
                             epsilon1=float(epsilon1), tpw=int(bool(tpw)),
                             checkmarine=int(bool(checkmarine)), calcRG=int(bool(calcRG)),
                             opt_dsl=int("dsl" in opt), opt_diag=int("diag" in opt),
                             inner_extrap=int(inner == "extrap"), radius=p.radius, mass=p.mass,
                             rhoi=p.rhoi, rhow=p.rhow, gacc=p.gacc, omega=p.omega, moiA=p.moiA,
                             moiC=p.moiC, kf=p.kf, precision=_lib.precision_code(precision))
        L = _lib.lib()
        self._L = L
        h = C.c_void_p()
        _lib.check(L.sle_batch_create(C.byref(cfg), self.nslots, int(max_modes), C.byref(h)),
                   "sle_batch_create")
        self._h = h
        self.loaded = [False] * self.nslots
        self.area0 = [None] * self.nslots
        self._ice_ptrs = (C.c_void_p * self.nslots)()
        self._dts = (C.c_double * self.nslots)()
        self._infos = (_lib.SleStepInfo * self.nslots)()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._L.sle_batch_destroy(h)
            except Exception:
                pass
            self._h = None

    # ------------------------------------------------------------------ slots
    @property
    def device_bytes(self) -> int:
        n = C.c_longlong()
        _lib.check(self._L.sle_batch_info(self._h, None, None, C.byref(n)), "sle_batch_info")
        return int(n.value)

    def free_slots(self):
        return [i for i, x in enumerate(self.loaded) if not x]

    def load(self, slot, love, topo0, ice0, dt):
        """Give `slot` an Earth model, a step length (yr) and run step 0 on topo0 / ice0;
        returns (ocean_area0, oceanBeta_area0, ice_volume0)."""
        earth, keep = earth_struct(love, self.lmax, self.p)
        a, b, v = C.c_double(), C.c_double(), C.c_double()
        if _is_cuda_tensor(topo0) or _is_cuda_tensor(ice0):
            import torch

            t0 = torch.as_tensor(topo0, dtype=torch.float64, device="cuda").contiguous()
            i0 = torch.as_tensor(ice0, dtype=torch.float64, device="cuda").contiguous()
            if tuple(t0.shape) != (self.nlat, self.nlon) or tuple(i0.shape) != tuple(t0.shape):
                raise ValueError(f"grids must be {(self.nlat, self.nlon)}")
            torch.cuda.current_stream().synchronize()
            ptrs, on_dev = (t0.data_ptr(), i0.data_ptr()), 1
        else:
            t0 = np.ascontiguousarray(topo0, dtype=np.float64)
            i0 = np.ascontiguousarray(ice0, dtype=np.float64)
            if t0.shape != (self.nlat, self.nlon) or i0.shape != t0.shape:
                raise ValueError(f"grids must be {(self.nlat, self.nlon)}")
            ptrs, on_dev = (t0.ctypes.data, i0.ctypes.data), 0
        _lib.check(self._L.sle_batch_load(self._h, int(slot), C.byref(earth), float(dt), C.c_void_p(ptrs[0]),
                                          C.c_void_p(ptrs[1]), on_dev, C.byref(a), C.byref(b), C.byref(v)),
                   "sle_batch_load")
        del keep
        self.loaded[slot] = True
        self.area0[slot] = (a.value, b.value, v.value)
        return self.area0[slot]

    def set_reuse(self, slot, store, valid=None):
        """Attach a ``ReuseStore`` (warm start across passes, reuse="warm") to `slot`; entries
        0 .. valid-1 (default: all recorded ones) hold an earlier pass.  None detaches."""
        if store is None:
            _lib.check(self._L.sle_batch_set_reuse(self._h, int(slot), None, None, 0, 0), "sle_batch_set_reuse")
            return
        ds, mask = store.pointers()
        v = store.recorded if valid is None else int(valid)
        _lib.check(self._L.sle_batch_set_reuse(self._h, int(slot), ds, mask, store.capacity, min(v, store.capacity)),
                   "sle_batch_set_reuse")

    def release(self, slot):
        _lib.check(self._L.sle_batch_release(self._h, int(slot)), "sle_batch_release")
        self.loaded[slot] = False

    def autotune(self, nfields=None):
        """Time the launch shapes of the mixed-precision transforms for lists of ``nfields`` fields
        (default: one per slot, the width of the inner loop's synthesis and rO analysis) and use
        the fastest (``slevolve_b200.tuning``).  Returns (shape, timings); FP64 batches: no-op."""
        if self.precision != "mixed":
            return None, []
        from .tuning import apply, autotune

        best, timings = autotune(self.lmax, nfields or self.nslots)
        apply(self, best)
        self.tuning = best
        return best, timings

    # ------------------------------------------------------------- snapshots
    def snapshot_bytes(self) -> int:
        n = C.c_longlong()
        _lib.check(self._L.sle_batch_snapshot_bytes(self._h, C.byref(n)), "sle_batch_snapshot_bytes")
        return int(n.value)

    def snapshot(self, slot, out=None):
        """The slot's whole solve state as a host byte image (NumPy uint8; ``out``: a buffer of
        ``snapshot_bytes()`` bytes to fill, e.g. a pinned CPU tensor's NumPy view).  It restores
        into any slot of a batch of the same configuration, or into a solver (``restore``)."""
        n = self.snapshot_bytes()
        img = np.empty(n, dtype=np.uint8) if out is None else out
        if not (isinstance(img, np.ndarray) and img.dtype == np.uint8 and img.flags.c_contiguous
                and img.size >= n):
            raise ValueError(f"out must be a contiguous uint8 array of at least {n} bytes")
        _lib.check(self._L.sle_batch_snapshot(self._h, int(slot), C.c_void_p(img.ctypes.data), n),
                   "sle_batch_snapshot")
        return img

    def restore(self, slot, image):
        """Make `slot` continue the solve a snapshot image holds (its reuse store, if any, is
        attached again with ``set_reuse``)."""
        img = np.ascontiguousarray(image, dtype=np.uint8)
        _lib.check(self._L.sle_batch_restore(self._h, int(slot), C.c_void_p(img.ctypes.data), img.size),
                   "sle_batch_restore")
        self.loaded[slot] = True

    # ------------------------------------------------------------------- step
    def step_ptrs(self, ptrs, on_device, dts=None):
        """One step from raw grid pointers: {slot: pointer}; returns {slot: SleStepInfo}.
        Raises like the single solver when a slot fails (its record has the status)."""
        for i in range(self.nslots):
            self._ice_ptrs[i] = None
            self._dts[i] = 0.0
        for slot, ptr in ptrs.items():
            self._ice_ptrs[slot] = ptr
            if dts and slot in dts and dts[slot]:
                self._dts[slot] = float(dts[slot])
        rc = self._L.sle_batch_step(self._h, self._ice_ptrs, int(on_device), self._dts, self._infos)
        out = {slot: self._infos[slot] for slot in ptrs}
        _lib.check(rc, "sle_batch_step")
        return out

    def step_begin(self, ptrs, on_device, dts=None):
        """Enqueue one step from raw grid pointers ({slot: pointer}) and return at once; the
        grids must stay valid and unchanged until ``step_end``."""
        for i in range(self.nslots):
            self._ice_ptrs[i] = None
            self._dts[i] = 0.0
        for slot, ptr in ptrs.items():
            self._ice_ptrs[slot] = ptr
            if dts and slot in dts and dts[slot]:
                self._dts[slot] = float(dts[slot])
        self._pending = list(ptrs)
        _lib.check(self._L.sle_batch_step_begin(self._h, self._ice_ptrs, int(on_device), self._dts),
                   "sle_batch_step_begin")

    def step_end(self):
        """Wait for the step enqueued by ``step_begin``; returns {slot: SleStepInfo} and raises
        like ``step_ptrs`` when a slot failed."""
        rc = self._L.sle_batch_step_end(self._h, self._infos)
        # copies: the record buffer is reused by the next step
        out = {slot: _lib.SleStepInfo.from_buffer_copy(self._infos[slot]) for slot in getattr(self, "_pending", [])}
        self._pending = []
        _lib.check(rc, "sle_batch_step_end")
        return out

    def step_host_stream(self, host_steps, dts=None):
        """Step once per element of ``host_steps`` (a sequence of {slot: host grid}, NumPy arrays or
        CPU tensors, ideally in pinned memory), uploading step k + 1's ice on a copy stream while
        step k runs (two device staging grids per slot, kept for later calls with the same slots).
        Returns the list of {slot: SleStepInfo}.  The results are those of calling ``step`` once
        per element."""
        import torch

        n = len(host_steps)
        if n == 0:
            return []
        slots = sorted(host_steps[0])
        # staging grids, copy stream and events are kept for the next call (same slots)
        hs = getattr(self, "_host_stream", None)
        if hs is None or hs[0] != slots:
            stage = [{s: torch.empty((self.nlat, self.nlon), dtype=torch.float64, device="cuda") for s in slots}
                     for _ in range(2)]
            hs = (slots, stage, torch.cuda.Stream(), [torch.cuda.Event(), torch.cuda.Event()])
            self._host_stream = hs
        _, stage, copy, landed = hs
        batch_stream = torch.cuda.ExternalStream(self.stream_handle())
        copy.wait_stream(torch.cuda.current_stream())
        copy.wait_stream(batch_stream)

        def upload(k):
            if sorted(host_steps[k]) != slots:
                raise ValueError("every step of host_steps must give ice for the same slots")
            with torch.cuda.stream(copy):
                for s, h in host_steps[k].items():
                    src = h if isinstance(h, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(h, np.float64))
                    if tuple(src.shape) != (self.nlat, self.nlon):
                        raise ValueError(f"ice shape {tuple(src.shape)} != {(self.nlat, self.nlon)}")
                    stage[k % 2][s].copy_(src, non_blocking=True)
                landed[k % 2].record(copy)

        upload(0)
        out = []
        for k in range(n):
            batch_stream.wait_event(landed[k % 2])
            self.step_begin({s: stage[k % 2][s].data_ptr() for s in slots}, 1, dts)
            if k + 1 < n:
                upload(k + 1)   # into the grids step k - 1 read (it has ended)
            out.append(self.step_end())
        copy.synchronize()
        return out

    def step(self, ices, dts=None):
        """ices: {slot: grid (NumPy array or CUDA tensor)}; returns {slot: info dict}."""
        if not ices:
            return {}
        dev = [_is_cuda_tensor(x) for x in ices.values()]
        if any(dev) and not all(dev):
            raise ValueError("all ice grids of one step must be on the same side (host or device)")
        keep = {}
        if all(dev):
            import torch

            for slot, x in ices.items():
                if tuple(x.shape) != (self.nlat, self.nlon):
                    raise ValueError(f"ice shape {tuple(x.shape)} != {(self.nlat, self.nlon)}")
                keep[slot] = x.to(torch.float64).contiguous()
            torch.cuda.current_stream().synchronize()
            ptrs = {slot: t.data_ptr() for slot, t in keep.items()}
            infos = self.step_ptrs(ptrs, 1, dts)
        else:
            for slot, x in ices.items():
                a = np.ascontiguousarray(x, dtype=np.float64)
                if a.shape != (self.nlat, self.nlon):
                    raise ValueError(f"ice shape {a.shape} != {(self.nlat, self.nlon)}")
                keep[slot] = a
            ptrs = {slot: a.ctypes.data for slot, a in keep.items()}
            infos = self.step_ptrs(ptrs, 0, dts)
        return {slot: _info_dict(i) for slot, i in infos.items()}

    def get(self, slot, field, out=None):
        """A grid of the slot's last step ('tgrid', 'ocean', 'beta', 'R', 'G', 'deltasl',
        'icestar') as NumPy, or into `out` (a CUDA tensor or a NumPy array)."""
        code = FIELDS[field]
        if out is None:
            out = np.empty((self.nlat, self.nlon))
        _check_grid_out(out, self.nlat, self.nlon)
        if _is_cuda_tensor(out):
            _lib.check(self._L.sle_batch_get(self._h, int(slot), code, C.c_void_p(out.data_ptr()), 1),
                       "sle_batch_get")
        else:
            _lib.check(self._L.sle_batch_get(self._h, int(slot), code, C.c_void_p(out.ctypes.data), 0),
                       "sle_batch_get")
        return out

    def stream_handle(self):
        s = C.c_void_p()
        _lib.check(self._L.sle_batch_stream(self._h, C.byref(s)), "sle_batch_stream")
        return s.value


def _check_grid_out(out, nlat, nlon):
    """``out`` of ``get``: a C-contiguous float64 (nlat, nlon) NumPy array or CUDA tensor (the
    library writes nlat * nlon doubles through its pointer)."""
    shape = tuple(out.shape)
    if _is_cuda_tensor(out):
        import torch

        ok = out.dtype == torch.float64 and out.is_contiguous()
    else:
        ok = isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
    if not ok or shape != (nlat, nlon):
        raise ValueError(f"out must be a C-contiguous float64 grid of shape {(nlat, nlon)}")


def _info_dict(info):
    lam = np.array(info.lam[:]).reshape(3, 3, 2)
    return {"iter": info.iter, "numiter": info.numiter, "status": info.status, "xi": info.xi,
            "ocean_area": info.ocean_area, "oceanBeta_area": info.oceanBeta_area,
            "gmslc_ocn": info.gmslc_ocn, "gmslc_ocnBeta": info.gmslc_ocnBeta,
            "ice_volume": info.ice_volume, "il": np.array(info.il[:]).reshape(3, 3),
            "mm": np.array(info.mm[:]), "lambda": lam[..., 0] + 1j * lam[..., 1],
            "gr_reguess": info.gr_reguess, "gr_ice_analyses": info.gr_ice_analyses}


def slot_bytes(nlat, nlon, lmax, max_modes=8):
    """Device bytes one slot's solver state takes (the admission unit of the serving loop)."""
    ng = nlat * nlon
    nc = (lmax + 1) * (lmax + 2) // 2
    nl = lmax + 1
    return int(11 * ng * 8 + 8 * ng + 24 * nc * 16 + max_modes * nc * 16 + 5 * max_modes * nl * 8 + 3 * nl * 8
               + 1024 + (nc // 256 + ng // 512 + 128) * 8 + 4 * nlat * 8)


__all__ = ["SolverBatch", "slot_bytes", "PI"]
