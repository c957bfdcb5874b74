"""slevolve_b200 -- the SLEvolve per-time-step sea-level path on NVIDIA B200 (sm_100a).

Drop-in surface (mirrors the reference package ``slevolve``):

* ``make_sht("cuda", nlat, nlon, lmax)`` -> ``CudaSHT`` with ``analysis`` / ``synthesis``
  (reference sht.py:43-46, sht_ducc.py:206-217);
* ``SeaLevelSolver`` / ``OptSeaLevelSolver`` with the reference constructors and
  ``step(icexy_cur, profile=False, dt=None, rates=False) -> dict`` (solver.py:518-1144,
  solver_opt.py:267-979), computing the whole step on the GPU in FP64;
* ``LoveNumbers`` (the reference's Love-number text format) and ``SyntheticEarth``;
* ``horiz.gradient(U, nlat, nlon)``: grid components of the horizontal displacement from the
  step dict's ``horiz`` (horiz.py:39-60), on the CUDA transform.

The compute lives in ``_lib/libslevolve_b200.so`` (C ABI: include/slevolve_b200.h); importing
this package does not load it, constructing a transform or solver does, and raises ImportError
when it is missing.
"""

from .love import LoveNumbers, SyntheticEarth, mode_arrays  # noqa: F401
from .sht import CudaSHT, make_sht  # noqa: F401
from .solver import GpuSeaLevelSolver, OptSeaLevelSolver, Planet, SeaLevelSolver  # noqa: F401

__version__ = "0.1.0"
