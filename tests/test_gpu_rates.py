"""Analytic rates read-out of the FP64 GPU solver against the reference's own output
(``tests/golden/rates.npz``, made by ``make_golden_rates.py``): c0 with rotation, steps of
varying length, ``step(ice, dt=..., rates=True)``.  Bar: the rate grids, spectra and rotational
rates within 1e-8 of the largest value of their kind (the solver's state agrees with the
reference to ~1e-12 relative; the rates are linear in it), identical iteration counts."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu
REL = 1e-8


def _close(got, ref, what):
    got, ref = np.asarray(got), np.asarray(ref)
    scale = float(np.abs(ref).max())
    assert np.abs(got - ref).max() <= REL * scale, (what, float(np.abs(got - ref).max()), scale)


def test_rates_against_reference():
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    fx = load_golden("rates.npz")
    dts = fx["dts"]
    case = case_c0(OracleSHT(64, 128, 63), nsteps=len(dts) + 8)
    slv = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=63, dt=1.0)
    for k, dt in enumerate(dts, start=1):
        r = slv.step(case.ice(k), dt=float(dt), rates=True)
        assert r["numiter"] == int(fx[f"numiter_{k}"]), k
        rt = r["rates"]
        for key in ("dSLdt", "dRdt", "dSLdt_lm", "dRdt_lm"):
            if f"{key}_{k}" in fx:
                _close(rt[key], fx[f"{key}_{k}"], (key, k))
        for key in ("ildot", "mdot", "lambdadot"):
            _close(rt[key], fx[f"{key}_{k}"], (key, k))
    # read-out off again: a plain step
    r = slv.step(case.ice(len(dts) + 1), dt=1.0)
    assert r["rates"] is None


def test_rates_need_the_fp64_form():
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    case = case_c0(OracleSHT(64, 128, 63), nsteps=4)
    slv = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=63, dt=1.0, precision="mixed")
    with pytest.raises(NotImplementedError):
        slv.step(case.ice(1), rates=True)
