"""ctypes binding of ``libslevolve_b200.so`` (declarations: include/slevolve_b200.h).

The library is built in-tree by ``python -m slevolve_b200.build``.  There is no fallback: if the
library is missing or fails to load, every entry point of the package raises ImportError.
"""

from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libslevolve_b200.so")

SLE_OK = 0
SLE_ERR_BAD_SHAPE = 1
SLE_ERR_BAD_ARG = 2
SLE_ERR_OOM = 3
SLE_ERR_CUDA = 4
SLE_ERR_NONCONVERGED = 5
SLE_ERR_NONFINITE = 6
SLE_ERR_UNSUPPORTED = 7
SLE_ERR_STATE = 8
SLE_ERR_TIMEOUT = 9

LAYOUT_DENSE = 0
LAYOUT_PACKED = 1

F_TGRID, F_OCEAN, F_BETA, F_R, F_G, F_DELTASL, F_DS_CONVERGED, F_LOAD_INC, F_ICESTAR = range(9)
F_OCEAN0, F_BETA0 = 9, 10


class SleConfig(C.Structure):
    _fields_ = [("nlat", C.c_int), ("nlon", C.c_int), ("lmax", C.c_int),
                ("dt_years", C.c_double), ("epsilon1", C.c_double),
                ("tpw", C.c_int), ("checkmarine", C.c_int), ("calcRG", C.c_int),
                ("opt_dsl", C.c_int), ("opt_diag", C.c_int), ("inner_extrap", C.c_int),
                ("radius", C.c_double), ("mass", C.c_double), ("rhoi", C.c_double),
                ("rhow", C.c_double), ("gacc", C.c_double), ("omega", C.c_double),
                ("moiA", C.c_double), ("moiC", C.c_double), ("kf", C.c_double),
                ("precision", C.c_int)]


_DP = C.POINTER(C.c_double)


class SleEarth(C.Structure):
    _fields_ = [("nmodes", C.c_int), ("nmod", C.POINTER(C.c_int)), ("s", _DP), ("a_sl", _DP),
                ("a_rr", _DP), ("ttl", _DP), ("ttlekhl", _DP), ("ttlhe", _DP), ("a_il", _DP),
                ("a_m", _DP), ("a_tsl", _DP), ("a_trr", _DP),
                ("kTE2", C.c_double), ("hTE2", C.c_double), ("kE2", C.c_double)]


class SleMxTuning(C.Structure):
    _fields_ = [("fields_per_launch", C.c_int), ("stages", C.c_int), ("fold_rows", C.c_int)]


class SleStepInfo(C.Structure):
    _fields_ = [("iter", C.c_int), ("numiter", C.c_int), ("status", C.c_int),
                ("gr_reguess", C.c_int), ("gr_ice_analyses", C.c_int), ("xi", C.c_double),
                ("ocean_area", C.c_double), ("oceanBeta_area", C.c_double),
                ("gmslc_ocn", C.c_double), ("gmslc_ocnBeta", C.c_double),
                ("ice_volume", C.c_double), ("il", C.c_double * 9), ("mm", C.c_double * 3),
                ("lam", C.c_double * 18)]


# name -> (restype, argtypes)
_SIGS = {
    "sle_abi_version": (C.c_int, []),
    "sle_last_error": (C.c_char_p, []),
    "sle_sht_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sle_sht_destroy": (C.c_int, [C.c_void_p]),
    "sle_sht_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_int), C.POINTER(C.c_longlong)]),
    "sle_sht_work_fraction": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "sle_sht_gauss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "sle_sht_analysis": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_void_p]),
    "sle_sht_synthesis": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_void_p]),
    "sle_sht_analysis_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sle_sht_set_precision": (C.c_int, [C.c_void_p, C.c_int]),
    "sle_sht_pack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sle_sht_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(SleMxTuning)]),
    "sle_sht_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(SleMxTuning)]),
    "sle_batch_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(SleMxTuning)]),
    "sle_sht_unpack": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sle_solver_create": (C.c_int, [C.POINTER(SleConfig), C.POINTER(SleEarth),
                                    C.POINTER(C.c_void_p)]),
    "sle_solver_destroy": (C.c_int, [C.c_void_p]),
    "sle_solver_init": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, _DP, _DP, _DP]),
    "sle_solver_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                  C.POINTER(SleStepInfo)]),
    "sle_solver_get": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int]),
    "sle_solver_set_rate_tables": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sle_solver_get_rates": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sle_solver_set_ramp": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sle_solver_set_horizontal": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sle_solver_get_horizontal": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "sle_solver_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "sle_solver_snapshot_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "sle_solver_snapshot": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    "sle_solver_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    "sle_batch_snapshot_bytes": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "sle_batch_snapshot": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]),
    "sle_batch_restore": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong]),
    "sle_batch_create": (C.c_int, [C.POINTER(SleConfig), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sle_batch_destroy": (C.c_int, [C.c_void_p]),
    "sle_batch_load": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(SleEarth), C.c_double, C.c_void_p,
                                 C.c_void_p, C.c_int, _DP, _DP, _DP]),
    "sle_batch_release": (C.c_int, [C.c_void_p, C.c_int]),
    "sle_batch_set_reuse": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "sle_solver_set_reuse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]),
    "sle_batch_step": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "sle_batch_step_begin": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "sle_batch_step_end": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sle_ice_blend": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_longlong, C.c_void_p]),
    "sle_topo_residual": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p,
                                  C.c_void_p, C.c_void_p]),
    "sle_topo_scratch_bytes": (C.c_longlong, []),
    "sle_batch_get": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]),
    "sle_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "sle_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_longlong)]),
    "sle_prof_enable": (C.c_int, [C.c_int]),
    "sle_prof_collect": (C.c_int, []),
    "sle_prof_reset": (C.c_int, []),
    "sle_prof_read": (C.c_int, [C.c_int, _DP, C.POINTER(C.c_longlong), _DP]),
    "sle_launch_count": (C.c_longlong, []),
    "sle_set_programmatic_launch": (C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    "sle_probe_fp64_tflops": (C.c_int, [_DP]),
}

(PROF_FFT, PROF_LEG_ANA, PROF_LEG_SYN, PROF_IFFT, PROF_ADVANCE, PROF_ANA_STEP, PROF_B18, PROF_UPDATE,
 PROF_REFRESH1, PROF_REFRESH2, PROF_DICE) = range(11)
PREC_FP64, PREC_MIXED = 0, 1
PRECISIONS = {"fp64": PREC_FP64, "mixed": PREC_MIXED}


def precision_code(precision) -> int:
    """'fp64' / 'mixed' (or the integer code) -> sle_precision; ValueError otherwise."""
    if isinstance(precision, str) and precision.lower() in PRECISIONS:
        return PRECISIONS[precision.lower()]
    if precision in (PREC_FP64, PREC_MIXED):
        return int(precision)
    raise ValueError(f"unknown precision {precision!r} (expected 'fp64' or 'mixed')")

_lib = None


def exported_symbols():
    return sorted(_SIGS)


def lib():
    """Load the library once; raise ImportError when it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m slevolve_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def set_programmatic_launch(on: bool) -> bool:
    """Programmatic dependent launches of the inner loop on / off (sle_set_programmatic_launch)
    for batches and transforms created afterwards; returns the previous setting."""
    prev = C.c_int(0)
    check(lib().sle_set_programmatic_launch(1 if on else 0, C.byref(prev)), "sle_set_programmatic_launch")
    return bool(prev.value)


def check(rc: int, what: str = ""):
    if rc == SLE_OK:
        return
    msg = lib().sle_last_error()
    msg = msg.decode(errors="replace") if msg else ""
    text = f"{what}: {msg}" if what else msg
    if rc in (SLE_ERR_BAD_SHAPE, SLE_ERR_BAD_ARG):
        raise ValueError(text)
    if rc == SLE_ERR_OOM:
        raise MemoryError(text)
    if rc == SLE_ERR_UNSUPPORTED:
        raise NotImplementedError(text)
    raise RuntimeError(text)
