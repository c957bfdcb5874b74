"""Second-order load placement (``ramp=True``) of the GPU solver against the reference's own ramp
run (``tests/golden/ramp.npz``, made by ``make_golden_ramp.py``): c0 with rotation, 10 steps of
varying length, the last four with the rates read-out.  Bar: topography and radial displacement
within 1e-9 m, identical iteration counts, rotational totals within 1e-9 and the last step's rates
within 1e-8 of their largest values."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_ramp_against_reference():
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    fx = load_golden("ramp.npz")
    dts = fx["dts"]
    case = case_c0(OracleSHT(64, 128, 63), nsteps=len(dts) + 8)
    slv = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=63, dt=1.0, ramp=True)
    numiter = []
    for k, dt in enumerate(dts, start=1):
        r = slv.step(case.ice(k), dt=float(dt), rates=k >= int(fx["rates_from"]))
        numiter.append(r["numiter"])
        for key in ("mm", "il", "lambda"):
            ref = fx[key]
            assert np.abs(np.asarray(r[key]) - ref[k - 1]).max() <= 1e-9 * float(np.abs(ref).max()), (k, key)
        if f"tgrid_{k}" in fx:
            assert np.abs(r["tgrid"] - fx[f"tgrid_{k}"]).max() <= 1e-9, k
            assert np.abs(r["R"] - fx[f"R_{k}"]).max() <= 1e-9, k
        if k == len(dts):
            for key in ("dSLdt", "dRdt", "ildot", "mdot", "lambdadot"):
                ref = fx[f"rates_{key}"]
                assert np.abs(np.asarray(r["rates"][key]) - ref).max() <= 1e-8 * np.abs(ref).max(), key
    assert numiter == list(fx["numiter"])
