#!/usr/bin/env python3
"""Golden fixture of variable step lengths, made by running the REFERENCE.

    python tests/golden/make_golden_vardt.py --reference /path/to/slevolve-checkout

The reference's ``SeaLevelSolver`` (plain) and ``OptSeaLevelSolver(opt={numba, sums, dsl},
inner="extrap")`` step the c0 configuration (64 x 128, L = 63, the case's seeded Earth and ice
caps) through 24 steps whose lengths vary (``step(ice, dt=...)``, solver.py:814-830): the decay
factors are recomputed per distinct length (solver.py:330-345) and the extrapolated start uses the
non-uniform formula (solver_opt.py:148-165).  Writes ``step_vardt.npz`` beside this script:
the step lengths, the inner-iteration counts of every step, and topography, radial displacement
and masks at five of them.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
DTS = [1.0, 2.0, 0.5, 0.5, 1.5, 3.0, 1.0, 1.0, 1.0, 2.5, 0.75, 1.25,
       4.0, 0.25, 0.25, 0.5, 2.0, 2.0, 1.0, 6.0, 0.5, 1.0, 1.0, 1.0]
SAVED = (3, 6, 14, 20, 24)   # steps whose grids are stored (iteration counts: every step)


def run(cls, sht, case, L, **kw):
    slv = cls(sht, case.love, case.topo, case.ice(0), norder=L, dt=1.0, **kw)
    out = {"numiter": []}
    for k, dt in enumerate(DTS, start=1):
        r = slv.step(np.ascontiguousarray(case.ice(k)), dt=dt)
        out["numiter"].append(r["numiter"])
        if k not in SAVED:
            continue
        out[f"tgrid_{k}"] = r["tgrid"].copy()
        out[f"R_{k}"] = r["R"].copy()
        out[f"ocean_{k}"] = np.packbits(r["ocean"].astype(bool))
        out[f"beta_{k}"] = np.packbits(r["beta"].astype(bool))
    out["numiter"] = np.array(out["numiter"])
    return out


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
    from slevolve.solver_opt import OptSeaLevelSolver
    from oracle.sht import OracleSHT
    from slevolve_b200.synthetic import case_c0

    n, L = 64, 63
    case = case_c0(OracleSHT(n, 2 * n, L), nsteps=len(DTS) + 8)
    sht = SHT(n, 2 * n, L)
    fx = {"dts": np.array(DTS)}
    fx.update({f"plain_{k}": v for k, v in run(SeaLevelSolver, sht, case, L).items()})
    fx.update({f"extrap_{k}": v for k, v in run(OptSeaLevelSolver, sht, case, L, opt={"numba", "sums", "dsl"},
                                                 inner="extrap").items()})
    print("plain", fx["plain_numiter"].tolist())
    print("extrap", fx["extrap_numiter"].tolist())
    np.savez_compressed(os.path.join(HERE, "step_vardt.npz"), **fx)


if __name__ == "__main__":
    main()
