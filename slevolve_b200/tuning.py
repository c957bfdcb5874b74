"""Launch-shape autotuner of the mixed-precision transforms.

The split-TF32 transforms have three launch-time choices that change their speed and not their
results: how many fields one tensor-core launch carries (a transform list is cut into launches
of at most ``fields_per_launch`` fields, each launch streaming the whole Legendre table once), the
pipeline depth of the tensor-core kernel (``stages``: 2 or 4 shared-memory stages of 48 KB) and the
rows per block of the row-FFT fold (``fold_rows``: 4 or 8).  The best choice depends on the degree,
on the number of fields a step transforms at once and on the device, so it is measured: for each
candidate the tuner times, with CUDA events on the device, the analysis and the synthesis of
``nfields`` random fields on a plan of the degree, keeps the fastest and caches the result per
(device, degree, fields) for the life of the process.  The reference's precedent is the Fortran
transform's switch between its on-the-fly and table-GEMM Legendre paths, chosen by field count
(otf_kernels.inc:463-516).

``autotune(lmax, nfields)`` returns the winner and the timings; ``apply(target, tuning)`` sets it
on a ``CudaSHT`` or a ``SolverBatch``; ``SolverBatch.autotune()`` does both for a batch.
"""

from __future__ import annotations

import ctypes as C
import itertools

from . import _lib

FIELDS_PER_LAUNCH = (16, 32)
STAGES = (2, 4)
FOLD_ROWS = (4, 8)
DEFAULT = {"fields_per_launch": 32, "stages": 4, "fold_rows": 8}

_cache = {}


def candidates(nfields):
    """Every launch shape worth timing for a list of ``nfields`` fields (launches wider than the
    list are the same as the list's own width)."""
    fpls = sorted({min(f, max(1, nfields)) for f in FIELDS_PER_LAUNCH})
    return [{"fields_per_launch": f, "stages": s, "fold_rows": r}
            for f, s, r in itertools.product(fpls, STAGES, FOLD_ROWS)]


def _struct(t):
    return _lib.SleMxTuning(fields_per_launch=int(t["fields_per_launch"]), stages=int(t["stages"]),
                            fold_rows=int(t["fold_rows"]))


def apply(target, tuning):
    """Set a launch shape on a ``CudaSHT`` (its plan) or a ``SolverBatch`` (its plan; the batch
    captures its inner-loop graph again at the next step)."""
    L = _lib.lib()
    t = _struct(tuning)
    if hasattr(target, "nslots"):
        _lib.check(L.sle_batch_set_tuning(target._h, C.byref(t)), "sle_batch_set_tuning")
    else:
        _lib.check(L.sle_sht_set_tuning(target._h, C.byref(t)), "sle_sht_set_tuning")


def current(sht):
    """The launch shape set on a ``CudaSHT``."""
    L = _lib.lib()
    t = _lib.SleMxTuning()
    _lib.check(L.sle_sht_get_tuning(sht._h, C.byref(t)), "sle_sht_get_tuning")
    return {"fields_per_launch": t.fields_per_launch, "stages": t.stages, "fold_rows": t.fold_rows}


def autotune(lmax, nfields, reps=3, warmup=1, seed=7, use_cache=True):
    """Fastest launch shape for transforming ``nfields`` fields at degree ``lmax`` on the current
    device: returns (best shape, [(shape, ms per analysis + synthesis of the fields), ...])."""
    import torch

    from .sht import make_sht

    dev = torch.cuda.current_device()
    key = (torch.cuda.get_device_name(dev), dev, int(lmax), int(nfields))
    if use_cache and key in _cache:
        return _cache[key]
    n = int(lmax) + 1
    sht = make_sht("cuda", n, 2 * n, int(lmax), precision="mixed")
    g = torch.Generator(device="cuda").manual_seed(seed)
    grids = [torch.randn((n, 2 * n), dtype=torch.float64, device="cuda", generator=g) for _ in range(nfields)]
    specs = [torch.empty(sht.ncoef, dtype=torch.complex128, device="cuda") for _ in range(nfields)]
    outs = [torch.empty((n, 2 * n), dtype=torch.float64, device="cuda") for _ in range(nfields)]
    stream = torch.cuda.current_stream()
    timings = []
    for cand in candidates(nfields):
        apply(sht, cand)
        for _ in range(warmup):
            sht.analysis_device(grids, specs, layout=_lib.LAYOUT_PACKED)
            sht.synthesis_device(specs, outs, layout=_lib.LAYOUT_PACKED)
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sht.analysis_device(grids, specs, layout=_lib.LAYOUT_PACKED)
            sht.synthesis_device(specs, outs, layout=_lib.LAYOUT_PACKED)
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        timings.append((dict(cand), best))
    winner = min(timings, key=lambda x: x[1])[0]
    del sht
    _cache[key] = (winner, timings)
    return winner, timings
