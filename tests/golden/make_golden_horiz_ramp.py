#!/usr/bin/env python3
"""Golden fixture of the horizontal read-out under the ramp placement, made by running the
REFERENCE.

    python tests/golden/make_golden_horiz_ramp.py --reference /path/to/slevolve-checkout

The reference's ``SeaLevelSolver(..., ramp=True)`` with ``horizontal = True`` (solver.py:687-720,
the ramp terms at 706-715) steps the c0 geometry (64 x 128, L = 63, the case's seeded topography
and ice caps, rotation on) with the reference's own Love-number file
``lovenum/prem_512.l96C.ump3.lm1`` through 8 steps of varying length.  Writes
``horiz_ramp.npz`` beside this script: the step lengths, Psi_lm at three steps and the
iteration counts (the Love arrays are those of ``horiz.npz``).
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DTS = [1.0, 2.0, 0.5, 1.0, 1.5, 1.0, 3.0, 1.0]
SAVED = (2, 5, 8)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="SLEvolve checkout whose python/slevolve package is imported read-only")
    a = ap.parse_args()
    sys.dont_write_bytecode = True
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(a.reference, "python"))
    from slevolve.sht import SHT
    from slevolve.solver import LoveNumbers, SeaLevelSolver
    from oracle.sht import OracleSHT
    from slevolve_b200.synthetic import case_c0

    n, L = 64, 63
    case = case_c0(OracleSHT(n, 2 * n, L), nsteps=len(DTS) + 8)
    love = LoveNumbers(os.path.join(a.reference, "lovenum", "prem_512.l96C.ump3.lm1"), L)
    slv = SeaLevelSolver(SHT(n, 2 * n, L), love, case.topo, case.ice(0), norder=L, dt=1.0, ramp=True)
    slv.horizontal = True
    fx = {"dts": np.array(DTS)}
    numiter = []
    for k, dt in enumerate(DTS, start=1):
        r = slv.step(np.ascontiguousarray(case.ice(k)), dt=dt)
        numiter.append(r["numiter"])
        if k in SAVED:
            fx[f"horiz_{k}"] = np.asarray(r["horiz"]).copy()
        print(k, r["numiter"], float(np.abs(r["horiz"]).max()), flush=True)
    fx["numiter"] = np.array(numiter)
    np.savez_compressed(os.path.join(HERE, "horiz_ramp.npz"), **fx)


if __name__ == "__main__":
    main()
