"""Ice history of the outer driver, formed on the device.

The reference's ice-age driver (SLEvolve python/slevolve/run_outer.py) reads its ice states from
a memory-mapped stack of cached ice files and, with ``--ice-seq``, builds a custom history from
it (run_outer.py:156-174): a comma (or newline) separated list of entries ``i`` (ice file i) or
``i:j:w`` (the blend ``(1 - w) I_i + w I_j``), or ``@FILE`` holding that list.  With ``--times``
(run_outer.py:176-183, npyio.py:180-193) a file of one time per ice state gives every step its
own length, ``t_k - t_(k-1)``.

Here the snapshots are uploaded to the device once (a small cache of device grids) and each
step's grid is formed there: a plain entry is a device copy of its snapshot, a blended entry is
``sle_ice_blend`` (the reference's NumPy arithmetic, bit for bit).  The resulting CUDA tensors go
straight to ``SolverBatch.step`` / ``OptSeaLevelSolver.step``.
"""

from __future__ import annotations

import ctypes as C
from collections import OrderedDict

import numpy as np

from . import _lib


def parse_ice_seq(spec, read_file=None):
    """Entries of an ``--ice-seq`` value: a list of ``(i,)`` or ``(i, j, w)``.

    ``spec`` is the option's text; ``@PATH`` reads the list from PATH (``read_file(path)`` if
    given, else the file's text).  Entries are separated by commas or newlines; blank entries
    are skipped.  An entry that is neither ``i`` nor ``i:j:w`` raises ``ValueError`` (the
    reference fails with ``ValueError`` when it reaches such an entry)."""
    if spec.startswith("@"):
        path = spec[1:]
        if read_file is not None:
            spec = read_file(path)
        else:
            with open(path) as fh:
                spec = fh.read()
    items = []
    for raw in spec.replace("\n", ",").split(","):
        x = raw.strip()
        if not x:
            continue
        p = x.split(":")
        if len(p) == 1:
            items.append((int(p[0]),))
        elif len(p) == 3:
            items.append((int(p[0]), int(p[1]), float(p[2])))
        else:
            raise ValueError(f"--ice-seq entry {x!r}: expected i or i:j:w")
    return items


def read_times(times, nsteps=None, name="times"):
    """One time (years) per ice state, as ``npyio.read_times`` (npyio.py:180-193): at least two
    values, finite and strictly increasing; with ``nsteps`` at least ``nsteps + 1`` values, of
    which the first ``nsteps + 1`` are kept.  ``times`` is a path or an array."""
    if isinstance(times, (str, bytes)):
        t = np.loadtxt(times, dtype=np.float64, ndmin=1)
        name = times
    else:
        t = np.asarray(times, dtype=np.float64)
    if t.ndim != 1 or t.size < 2:
        raise ValueError(f"{name}: need one time per line, at least 2 values")
    if nsteps is not None:
        if t.size < nsteps + 1:
            raise ValueError(f"{name}: {t.size} times, need {nsteps + 1} (files 0..{nsteps})")
        t = t[: nsteps + 1]
    if not np.all(np.isfinite(t)) or not np.all(np.diff(t) > 0):
        raise ValueError(f"{name}: times must be finite and strictly increasing")
    return t


def step_lengths(times, nstates):
    """Step lengths (years) for a history of ``nstates`` ice states: ``diff(times)``; exactly
    ``nstates`` times are required (run_outer.py:178-181)."""
    t = np.asarray(times, dtype=np.float64)
    if t.size != nstates:
        raise ValueError(f"{t.size} times for {nstates} ice states")
    return np.diff(t)


class IceHistory:
    """Step k's ice grid on the device for a stack of ice states (``stack[i]``, e.g. a
    ``np.load(..., mmap_mode="r")`` array of shape (nfiles, nlat, nlon)) and an optional custom
    sequence (``parse_ice_seq`` entries; default: the stack's states in order).

    ``len(h)`` is the number of ice states, ``h.nsteps = len(h) - 1`` the number of steps after
    the initial state.  ``h.device(k)`` returns a new CUDA float64 tensor (or fills ``out``).
    Snapshots are uploaded on first use and kept in a cache of ``cache`` device grids (least
    recently used out first)."""

    def __init__(self, stack, items=None, cache=4):
        self.stack = stack
        n = len(stack)
        self.items = [(i,) for i in range(n)] if items is None else list(items)
        for it in self.items:
            for i in it[:2] if len(it) == 3 else it:
                if not -n <= i < n:
                    raise IndexError(f"ice state {i} outside the stack of {n}")
        self.shape = tuple(np.shape(stack[0]))
        self.cache = max(2, int(cache))
        self._dev = OrderedDict()

    def __len__(self):
        return len(self.items)

    @property
    def nsteps(self):
        return len(self.items) - 1

    def _snapshot(self, i):
        import torch

        i = i % len(self.stack)
        t = self._dev.pop(i, None)
        if t is None:
            host = np.ascontiguousarray(self.stack[i], dtype=np.float64)
            t = torch.from_numpy(host).to("cuda")
            while len(self._dev) >= self.cache:
                self._dev.popitem(last=False)
        self._dev[i] = t
        return t

    def device(self, k, out=None):
        import torch

        it = self.items[k]
        if len(it) == 1:
            src = self._snapshot(it[0])
            if out is None:
                return src.clone()
            out.copy_(src)
            return out
        i, j, w = it
        a = self._snapshot(i)
        b = self._snapshot(j)
        if out is None:
            out = torch.empty_like(a)
        if out.shape != a.shape or out.dtype != torch.float64 or not out.is_cuda or not out.is_contiguous():
            raise ValueError("out must be a contiguous CUDA float64 grid of the stack's shape")
        stream = torch.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().sle_ice_blend(C.c_void_p(out.data_ptr()), C.c_void_p(a.data_ptr()),
                                            C.c_void_p(b.data_ptr()), float(w), int(a.numel()),
                                            C.c_void_p(stream)), "sle_ice_blend")
        return out
