"""The CPU oracle against the reference's own outputs (fixtures made by tests/golden/make_golden.py).

Tolerances: the SHT and the modal state agree with the reference to round-off (1e-13 relative);
solver steps to 1e-9 m in topography and radial displacement with identical iteration counts and
identical ocean / grounded-ice masks, the bar the reference sets for its own implementations
(tests/test_fortran_python.sh:37-47 of the reference).
"""

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, FixtureLove, load_golden
from oracle.memory import ModalState
from oracle.sht import OracleSHT, gauss_nodes
from oracle.solver import OracleSolver

TOL_M = 1e-9


@pytest.mark.parametrize("n,L", [(16, 15), (32, 31), (32, 20), (64, 63)])
def test_sht_against_reference(n, L):
    fx = load_golden("sht.npz")
    tag = f"n{n}_l{L}"
    z, w = gauss_nodes(n)
    assert np.array_equal(z, fx[f"{tag}_nodes"])
    assert np.array_equal(w, fx[f"{tag}_weights"])
    s = OracleSHT(n, 2 * n, L)
    a = s.analysis(fx[f"{tag}_grid"])
    ref = fx[f"{tag}_ana"]
    assert np.abs(a - ref).max() <= 1e-13 * np.abs(ref).max()
    g = s.synthesis(fx[f"{tag}_coef"])
    ref = fx[f"{tag}_syn"]
    assert np.abs(g - ref).max() <= 1e-13 * np.abs(ref).max()


def test_modal_state_against_reference():
    fx = load_golden("memory.npz")
    love = FixtureLove(fx)
    love.he = love.ke = love.hTE = love.kTE = np.zeros(int(fx["lmax"]) + 1)
    st = ModalState(love, int(fx["lmax"]), 1.0)
    worst = 0.0
    for n, dt in enumerate(fx["dts"]):
        st.set_dt(dt)
        out = st.advance_and_read()
        for got, key in zip(out, ("visc", "rad", "sum_il", "sum_m", "sum_tsl", "sum_trr")):
            ref = fx[key][n]
            sc = max(np.abs(ref).max(), 1e-300)
            worst = max(worst, np.abs(got - ref).max() / sc)
        st.commit(fx["load"][n], fx["dil"][n], fx["dm"][n], fx["dlam"][n])
    assert worst <= 1e-13, worst


def _love_and_topo(fx):
    love = FixtureLove(fx)
    topo = fx["topo_mm"] / 1000.0 if "topo_mm" in fx else fx["topo"]
    return love, topo


def _check_run(slv, fx, prefix, ice_fn, nsteps, saved):
    numiter = []
    for k in range(1, nsteps + 1):
        r = slv.step(ice_fn(k))
        numiter.append(r["numiter"])
        if f"{prefix}tgrid_{k}" in fx:
            assert np.abs(r["tgrid"] - fx[f"{prefix}tgrid_{k}"]).max() <= TOL_M, k
            assert np.abs(r["R"] - fx[f"{prefix}R_{k}"]).max() <= TOL_M, k
            oc = np.unpackbits(fx[f"{prefix}ocean_{k}"])[: r["ocean"].size].reshape(r["ocean"].shape)
            be = np.unpackbits(fx[f"{prefix}beta_{k}"])[: r["beta"].size].reshape(r["beta"].shape)
            assert np.array_equal(r["ocean"] != 0, oc != 0), k
            assert np.array_equal(r["beta"] != 0, be != 0), k
        for key in ("gmslc_ocn", "gmslc_ocnBeta", "ocean_area", "oceanBeta_area", "ice_volume"):
            ref = fx[f"{prefix}{key}"][k - 1]
            assert abs(r[key] - ref) <= 1e-9 * max(1.0, abs(ref)), (k, key)
        for key in ("mm", "il", "lambda"):   # rotational feedback: signs and magnitudes
            if f"{prefix}{key}" in fx:
                ref = fx[f"{prefix}{key}"]
                assert np.abs(np.asarray(r[key]) - ref[k - 1]).max() <= 1e-9 * float(np.abs(ref).max()), (k, key)
    assert numiter == list(fx[f"{prefix}numiter"])


def test_step_c0_plain_against_reference():
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("step_c0.npz")
    love, topo = _love_and_topo(fx)
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht)
    assert np.array_equal(case.topo, topo), "c0 topography generator drifted from the fixture"
    slv = OracleSolver(sht, love, topo, case.ice(0), norder=63, dt=1.0)
    _check_run(slv, fx, "plain_", case.ice, 100, None)


def test_step_c0_extrap_against_reference():
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("step_c0.npz")
    love, topo = _love_and_topo(fx)
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht)
    slv = OracleSolver(sht, love, topo, case.ice(0), norder=63, dt=1.0, opt={"dsl"}, inner="extrap")
    numiter = []
    for k in range(1, 101):
        r = slv.step(case.ice(k))
        numiter.append(r["numiter"])
        if f"extrap_tgrid_{k}" in fx:
            assert np.abs(r["tgrid"] - fx[f"extrap_tgrid_{k}"]).max() <= TOL_M
    assert numiter == list(fx["extrap_numiter"])


def test_step_marine_against_reference():
    from tests_helpers import marine_ice
    fx = load_golden("step_marine.npz")
    love, topo = _love_and_topo(fx)
    sht = OracleSHT(64, 128, 63)
    ice = marine_ice(sht.gaulats, 128, fx["ice_heights"])
    slv = OracleSolver(sht, love, topo, ice[0], norder=63, dt=1000.0)
    _check_run(slv, fx, "plain_", lambda k: ice[k], 8, None)
    assert slv.gr_counts["reguess"] > 0


def test_step_c1_small_against_reference():
    from slevolve_b200.synthetic import case_c1
    fx = load_golden("step_c1s.npz")
    love, topo = _love_and_topo(fx)
    sht = OracleSHT(64, 128, 63)
    case = case_c1(sht, nsteps=60)
    assert np.array_equal(case.topo, topo)
    probe = np.array([float(np.abs(case.ice(k)).sum()) for k in range(61)])
    assert np.array_equal(probe, fx["ice_probe"])
    slv = OracleSolver(sht, love, topo, case.ice(0), norder=63, dt=1.0)
    _check_run(slv, fx, "plain_", case.ice, 60, None)
    assert slv.gr_counts["ice_analyses"] > 0   # the grounded re-guess changed the mask


def test_synthetic512_oracle_record():
    """The oracle reproduced the reference's shipped L=511 golden grid when the fixtures were made."""
    with open(os.path.join(GOLDEN, "golden_meta.json")) as fh:
        meta = json.load(fh)
    rec = meta["synthetic512_oracle"]
    assert rec["max_abs_vs_tgrid8_m"] <= TOL_M
    assert rec["numiter"] == [5, 5, 6, 6, 5, 5, 5, 5]


@pytest.mark.parametrize("kind", ["plain", "extrap"])
def test_variable_step_lengths_against_reference(kind):
    """24 steps of varying length (step(ice, dt=...)): per-length decay factors and, with
    inner="extrap", the non-uniform extrapolated start (golden: make_golden_vardt.py)."""
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("step_vardt.npz")
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht, nsteps=len(fx["dts"]) + 8)
    kw = {} if kind == "plain" else {"opt": {"dsl"}, "inner": "extrap"}
    slv = OracleSolver(sht, case.love, case.topo, case.ice(0), norder=63, dt=1.0, **kw)
    numiter = []
    for k, dt in enumerate(fx["dts"], start=1):
        r = slv.step(case.ice(k), dt=float(dt))
        numiter.append(r["numiter"])
        if f"{kind}_tgrid_{k}" in fx:
            assert np.abs(r["tgrid"] - fx[f"{kind}_tgrid_{k}"]).max() <= TOL_M, k
            assert np.abs(r["R"] - fx[f"{kind}_R_{k}"]).max() <= TOL_M, k
    assert numiter == list(fx[f"{kind}_numiter"])


def test_rates_readout_against_reference():
    """The oracle's analytic rates (step(..., rates=True)) against the reference's own output
    (golden: make_golden_rates.py): 1e-8 of the largest value of each kind."""
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("rates.npz")
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht, nsteps=len(fx["dts"]) + 8)
    slv = OracleSolver(sht, case.love, case.topo, case.ice(0), norder=63, dt=1.0)
    for k, dt in enumerate(fx["dts"], start=1):
        r = slv.step(case.ice(k), dt=float(dt), rates=True)
        assert r["numiter"] == int(fx[f"numiter_{k}"])
        for key in ("dSLdt", "dRdt", "dSLdt_lm", "dRdt_lm", "ildot", "mdot", "lambdadot"):
            name = f"{key}_{k}"
            if name in fx:
                ref = fx[name]
                assert np.abs(np.asarray(r["rates"][key]) - ref).max() <= 1e-8 * np.abs(ref).max(), name


def test_horizontal_readout_against_reference():
    """The oracle's horizontal potential (horizontal = True) against the reference's own output
    with its PREM Love file (golden: make_golden_horiz.py): 1e-9 of the largest coefficient."""
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("horiz.npz")
    love = FixtureLove(fx)
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht, nsteps=len(fx["dts"]) + 8)
    slv = OracleSolver(sht, love, case.topo, case.ice(0), norder=63, dt=1.0)
    slv.horizontal = True
    numiter = []
    for k, dt in enumerate(fx["dts"], start=1):
        r = slv.step(case.ice(k), dt=float(dt))
        numiter.append(r["numiter"])
        if f"horiz_{k}" in fx:
            ref = fx[f"horiz_{k}"]
            assert np.abs(r["horiz"] - ref).max() <= 1e-9 * np.abs(ref).max(), k
    assert numiter == list(fx["numiter"])


def test_horizontal_readout_under_ramp_against_reference():
    """The oracle's horizontal potential with the ramp placement (its same-step c_hl and tidal
    c_thl terms) against the reference's own run (golden: make_golden_horiz_ramp.py, the PREM
    Love arrays of horiz.npz): 1e-9 of the largest coefficient, identical iteration counts.  The
    run without the ramp terms misses by far more than that."""
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("horiz_ramp.npz")
    love = FixtureLove(load_golden("horiz.npz"))
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht, nsteps=len(fx["dts"]) + 8)
    runs = {}
    for ramp in (True, False):
        slv = OracleSolver(sht, love, case.topo, case.ice(0), norder=63, dt=1.0, ramp=ramp)
        slv.horizontal = True
        numiter, psi = [], {}
        for k, dt in enumerate(fx["dts"], start=1):
            r = slv.step(case.ice(k), dt=float(dt))
            numiter.append(r["numiter"])
            if f"horiz_{k}" in fx:
                psi[k] = r["horiz"].copy()
        runs[ramp] = (numiter, psi)
    numiter, psi = runs[True]
    assert numiter == list(fx["numiter"])
    for k, got in psi.items():
        ref = fx[f"horiz_{k}"]
        assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max(), k
        assert np.abs(runs[False][1][k] - ref).max() > 1e-6 * np.abs(ref).max(), k


def test_ramp_placement_against_reference():
    """The oracle with the second-order load placement (ramp=True) against the reference's own
    run (golden: make_golden_ramp.py): 1e-9 m, identical iteration counts, rotational totals and,
    for the last step, the rates read-out under the ramp-consistent state."""
    from slevolve_b200.synthetic import case_c0
    fx = load_golden("ramp.npz")
    sht = OracleSHT(64, 128, 63)
    case = case_c0(sht, nsteps=len(fx["dts"]) + 8)
    slv = OracleSolver(sht, case.love, case.topo, case.ice(0), norder=63, dt=1.0, ramp=True)
    numiter = []
    for k, dt in enumerate(fx["dts"], start=1):
        r = slv.step(case.ice(k), dt=float(dt), rates=k >= int(fx["rates_from"]))
        numiter.append(r["numiter"])
        for key in ("mm", "il", "lambda"):
            ref = fx[key]
            assert np.abs(np.asarray(r[key]) - ref[k - 1]).max() <= 1e-9 * float(np.abs(ref).max()), (k, key)
        if f"tgrid_{k}" in fx:
            assert np.abs(r["tgrid"] - fx[f"tgrid_{k}"]).max() <= TOL_M, k
            assert np.abs(r["R"] - fx[f"R_{k}"]).max() <= TOL_M, k
        if k == len(fx["dts"]):
            for key in ("dSLdt", "dRdt", "ildot", "mdot", "lambdadot"):
                ref = fx[f"rates_{key}"]
                assert np.abs(np.asarray(r["rates"][key]) - ref).max() <= 1e-8 * np.abs(ref).max(), key
    assert numiter == list(fx["numiter"])


def test_c1_full_size_oracle_first_steps():
    """The oracle on c1 at its benchmark size (256 x 512, L = 255) against the reference's 550-step
    run (make_golden_c1.py): its inputs, step-0 areas and the first three steps (iteration counts,
    degree-0 diagnostics, the full topography and masks of step 1); the GPU test covers all 550."""
    from slevolve_b200.synthetic import case_c1

    fx = load_golden("step_c1.npz")
    osht = OracleSHT(256, 512, 255, workers=os.cpu_count() or 1)
    case = case_c1(osht, nsteps=550)
    assert np.array_equal(np.round(case.topo * 1000.0).astype(np.int64), fx["topo_mm"])
    orc = OracleSolver(osht, case.love, case.topo, case.ice(0), norder=255, dt=1.0)
    a0, b0, v0 = fx["step0_scalars"]
    assert abs(orc.ocean_area0 - a0) <= 1e-9 * abs(a0)
    assert abs(orc.ice_volume0 - v0) <= 1e-9 * abs(v0)
    for k in (1, 2, 3):
        ice = case.ice(k)
        assert float(np.abs(ice).sum()) == fx["ice_abs_sum"][k - 1]
        r = orc.step(ice)
        assert r["numiter"] == fx["numiter"][k - 1], k
        for key in ("gmslc_ocn", "ocean_area", "ice_volume"):
            assert abs(r[key] - fx[key][k - 1]) <= 1e-9 * max(1.0, abs(fx[key][k - 1])), (k, key)
        if k == 1:
            assert np.abs(r["tgrid"] - fx["tgrid_1"]).max() <= TOL_M
            shape = r["ocean"].shape
            ocean = np.unpackbits(fx["ocean_1"])[: shape[0] * shape[1]].reshape(shape) != 0
            assert np.array_equal(np.asarray(r["ocean"]) != 0, ocean)
