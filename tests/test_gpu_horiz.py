"""Horizontal read-out (``solver.horizontal = True``, the step dict's ``horiz``: the potential
Psi_lm of the horizontal displacement in the U convention) against the reference's own output
(``tests/golden/horiz.npz``, made by ``make_golden_horiz.py`` with the reference's PREM Love file):
within 1e-9 of the largest coefficient at every stored step, identical iteration counts, and the
step itself unchanged by the read-out."""

import numpy as np
import pytest

from conftest import FixtureLove, load_golden

pytestmark = pytest.mark.gpu


def test_horizontal_potential_against_reference():
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    fx = load_golden("horiz.npz")
    dts = fx["dts"]
    love = FixtureLove(fx)
    case = case_c0(OracleSHT(64, 128, 63), nsteps=len(dts) + 8)
    slv = SeaLevelSolver(None, love, case.topo, case.ice(0), norder=63, dt=1.0)
    plain = SeaLevelSolver(None, love, case.topo, case.ice(0), norder=63, dt=1.0)
    slv.horizontal = True
    numiter = []
    for k, dt in enumerate(dts, start=1):
        r = slv.step(case.ice(k), dt=float(dt))
        q = plain.step(case.ice(k), dt=float(dt))
        numiter.append(r["numiter"])
        assert q["horiz"] is None
        assert np.array_equal(r["tgrid"], q["tgrid"]), k
        if f"horiz_{k}" in fx:
            ref = fx[f"horiz_{k}"]
            err = float(np.abs(r["horiz"] - ref).max())
            assert err <= 1e-9 * float(np.abs(ref).max()), (k, err)
    assert numiter == list(fx["numiter"])
    slv.horizontal = False
    assert slv.step(case.ice(len(dts) + 1), dt=1.0)["horiz"] is None
