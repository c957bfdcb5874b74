#!/usr/bin/env python3
"""Golden fixture of the second-order load placement (``ramp``), made by running the REFERENCE.

    python tests/golden/make_golden_ramp.py --reference /path/to/slevolve-checkout

The reference's ``SeaLevelSolver(..., ramp=True)`` (solver.py:229-240, 348-368, 450-499,
904-991, 1065-1067) steps the c0 configuration (64 x 128, L = 63, the case's seeded Earth and ice
caps, rotation on) through 10 steps of varying length, the last four with ``rates=True``.
Writes ``ramp.npz`` beside this script: iteration counts and rotational totals of every step,
topography and radial displacement at four steps, the rate grids of the last step.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DTS = [1.0, 2.0, 0.5, 1.0, 3.0, 1.0, 1.5, 0.75, 1.0, 2.0]
SAVED = (2, 5, 8, 10)
RATES_FROM = 7


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="SLEvolve checkout whose python/slevolve package is imported read-only")
    a = ap.parse_args()
    sys.dont_write_bytecode = True
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(a.reference, "python"))
    from slevolve.sht import SHT
    from slevolve.solver import SeaLevelSolver
    from oracle.sht import OracleSHT
    from slevolve_b200.synthetic import case_c0

    n, L = 64, 63
    case = case_c0(OracleSHT(n, 2 * n, L), nsteps=len(DTS) + 8)
    slv = SeaLevelSolver(SHT(n, 2 * n, L), case.love, case.topo, case.ice(0), norder=L, dt=1.0, ramp=True)
    fx = {"dts": np.array(DTS), "rates_from": np.array(RATES_FROM)}
    out = {"numiter": [], "mm": [], "il": [], "lambda": []}
    for k, dt in enumerate(DTS, start=1):
        r = slv.step(np.ascontiguousarray(case.ice(k)), dt=dt, rates=k >= RATES_FROM)
        out["numiter"].append(r["numiter"])
        out["mm"].append(np.asarray(r["mm"]).copy())
        out["il"].append(np.asarray(r["il"]).copy())
        out["lambda"].append(np.asarray(r["lambda"]).copy())
        if k in SAVED:
            fx[f"tgrid_{k}"] = r["tgrid"].copy()
            fx[f"R_{k}"] = r["R"].copy()
        if k == len(DTS):
            for key in ("dSLdt", "dRdt", "ildot", "mdot", "lambdadot"):
                fx[f"rates_{key}"] = np.asarray(r["rates"][key]).copy()
        print(k, r["numiter"], flush=True)
    fx.update({key: np.array(v) for key, v in out.items()})
    np.savez_compressed(os.path.join(HERE, "ramp.npz"), **fx)


if __name__ == "__main__":
    main()
