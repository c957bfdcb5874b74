#!/usr/bin/env python3
"""Golden fixture of the analytic rates read-out, made by running the REFERENCE.

    python tests/golden/make_golden_rates.py --reference /path/to/slevolve-checkout

The reference's ``SeaLevelSolver`` steps the c0 configuration (64 x 128, L = 63, the case's seeded
Earth and ice caps, rotation on) with ``step(ice, dt=..., rates=True)`` (solver.py:722-806,
1086-1117): the rate spectra read from the modal states before the commit, the rotational rates
(il-dot, m-dot, Lambda-dot) and the rate grids dSL/dt, dR/dt synthesised on the end-of-step ocean
function.  Steps of varying length.  Writes ``rates.npz`` beside this script.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DTS = [1.0, 1.0, 2.0, 0.5, 1.0, 3.0, 1.0, 1.0]
SAVED = (1, 3, 4, 6, 8)   # steps whose rate grids are stored (spectra: steps 1 and 6)


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
    slv = SeaLevelSolver(SHT(n, 2 * n, L), case.love, case.topo, case.ice(0), norder=L, dt=1.0)
    fx = {"dts": np.array(DTS)}
    for k, dt in enumerate(DTS, start=1):
        r = slv.step(np.ascontiguousarray(case.ice(k)), dt=dt, rates=True)
        rt = r["rates"]
        fx[f"numiter_{k}"] = np.array(r["numiter"])
        if k in SAVED:
            fx[f"dSLdt_{k}"] = rt["dSLdt"].copy()
            fx[f"dRdt_{k}"] = rt["dRdt"].copy()
        if k in (1, 6):
            fx[f"dSLdt_lm_{k}"] = rt["dSLdt_lm"].copy()
            fx[f"dRdt_lm_{k}"] = rt["dRdt_lm"].copy()
        for key in ("ildot", "mdot", "lambdadot"):
            if key in rt:
                fx[f"{key}_{k}"] = np.asarray(rt[key]).copy()
        print(k, r["numiter"], float(np.abs(rt["dSLdt"]).max()), float(np.abs(rt["dRdt"]).max()), flush=True)
    np.savez_compressed(os.path.join(HERE, "rates.npz"), **fx)


if __name__ == "__main__":
    main()
