#!/usr/bin/env python3
"""Golden fixture of the c1 configuration at its full size and length, made by running the REFERENCE.

    python tests/golden/make_golden_c1.py --reference /path/to/slevolve-checkout

The reference's plain ``SeaLevelSolver`` with its NumPy transform ``sht.SHT`` (solver.py:521-1144,
sht.py:148-343) steps the c1 configuration: 256 x 512 Gauss grid, L = 255, 550 steps of 1 yr, the
seeded synthetic Earth, the south polar continent with its bed at -500 ... -1500 m under a 3.5 km
dome thinned by 1-20 m/yr (grounding-line retreat and floating shelves).  Writes ``step_c1.npz``
beside this script:

* per step (all 550): the inner-iteration count, the degree-0 diagnostics (GMSL change over both
  masks, ocean areas, ice volume) and the rotational quantities il, m, Lambda;
* at the steps in ``SAVED``: the ocean / grounded-ice masks (bit-packed); topography in full at the
  steps in ``FULL_TOPO`` and radial displacement in full at ``FULL_R``; at the other saved steps
  both grids on every fourth row and column plus their exact row and column sums (the fixture
  stays near 5 MB).

About 3 minutes on 8 cores.  The inputs are not stored: ``slevolve_b200.synthetic.case_c1``
regenerates them from the seed with the oracle transform, and the fixture keeps the topography in
whole millimetres and per-step sums of the ice so a test can confirm it rebuilt the same inputs.
"""

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
NSTEPS = 550
SAVED = (1, 55, 110, 165, 220, 275, 330, 385, 440, 495, 550)
FULL_TOPO = (1, 275, 550)
FULL_R = (550,)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="SLEvolve checkout whose python/slevolve package is imported read-only")
    a = ap.parse_args()
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
    sys.dont_write_bytecode = True
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(a.reference, "python"))
    from slevolve.sht import SHT
    from slevolve.solver import SeaLevelSolver
    from oracle.sht import OracleSHT
    from slevolve_b200.synthetic import case_c1

    n, L = 256, 255
    case = case_c1(OracleSHT(n, 2 * n, L), nsteps=NSTEPS)
    topo_mm = np.round(case.topo * 1000.0).astype(np.int64)
    assert np.array_equal(topo_mm / 1000.0, case.topo)
    sht = SHT(n, 2 * n, L)
    t0 = time.time()
    slv = SeaLevelSolver(sht, case.love, case.topo, case.ice(0), norder=L, dt=1.0)
    fx = {"topo_mm": topo_mm.astype(np.int32),
          "step0_scalars": np.array([slv.ocean_area0, slv.oceanBeta_area0, slv.ice_volume0])}
    per_step = {k: [] for k in ("numiter", "gmslc_ocn", "gmslc_ocnBeta", "ocean_area",
                                "oceanBeta_area", "ice_volume", "mm", "il", "lambda", "ice_abs_sum")}
    for k in range(1, NSTEPS + 1):
        ice = np.ascontiguousarray(case.ice(k))
        r = slv.step(ice)
        per_step["ice_abs_sum"].append(float(np.abs(ice).sum()))
        for key in ("numiter", "gmslc_ocn", "gmslc_ocnBeta", "ocean_area", "oceanBeta_area",
                    "ice_volume"):
            per_step[key].append(r[key])
        for key in ("mm", "il", "lambda"):
            per_step[key].append(np.array(r[key], copy=True))
        if k in SAVED:
            for key, full in (("tgrid", FULL_TOPO), ("R", FULL_R)):
                g = np.array(r[key], copy=True)
                if k in full:
                    fx[f"{key}_{k}"] = g
                else:
                    fx[f"{key}_sub4_{k}"] = g[::4, ::4].copy()
                    fx[f"{key}_rowsum_{k}"] = g.sum(axis=1)
                    fx[f"{key}_colsum_{k}"] = g.sum(axis=0)
            fx[f"ocean_{k}"] = np.packbits(r["ocean"].astype(bool))
            fx[f"beta_{k}"] = np.packbits(r["beta"].astype(bool))
        if k % 50 == 0:
            print(f"step {k}  numiter {r['numiter']}  {time.time() - t0:.0f} s", flush=True)
    fx.update({k: np.asarray(v) for k, v in per_step.items()})
    fx["saved_steps"] = np.array(SAVED)
    np.savez_compressed(os.path.join(HERE, "step_c1.npz"), **fx)
    summary = {"seconds": time.time() - t0, "numiter_total": int(np.sum(per_step["numiter"])),
               "numiter_max": int(np.max(per_step["numiter"])),
               "gr_counts": {k: int(v) for k, v in getattr(slv, "gr_counts", {}).items()}}
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
