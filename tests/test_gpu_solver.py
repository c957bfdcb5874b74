"""The CUDA time step against the reference's own outputs and the CPU oracle.

Bar (the reference's own, tests/test_fortran_python.sh:37-47): topography and radial displacement
within 1e-9 m at every compared step, identical inner-iteration counts, identical ocean and
grounded-ice masks; degree-0 diagnostics within 1e-9 relative.
"""

import numpy as np
import pytest

from conftest import FixtureLove, load_golden

pytestmark = pytest.mark.gpu
TOL_M = 1e-9


def _unpack(bits, shape):
    return np.unpackbits(bits)[: int(np.prod(shape))].reshape(shape) != 0


def _check_against_fixture(slv, fx, prefix, ice_fn, nsteps):
    numiter = []
    for k in range(1, nsteps + 1):
        r = slv.step(ice_fn(k))
        numiter.append(r["numiter"])
        for key in ("tgrid", "R"):
            if f"{prefix}{key}_{k}" in fx:
                d = np.abs(r[key] - fx[f"{prefix}{key}_{k}"]).max()
                assert d <= TOL_M, (k, key, d)
            if f"{prefix}{key}_sub4_{k}" in fx:
                # every fourth row and column, and the exact row and column sums of the grid
                g = np.asarray(r[key])
                d = np.abs(g[::4, ::4] - fx[f"{prefix}{key}_sub4_{k}"]).max()
                assert d <= TOL_M, (k, key, d)
                assert np.abs(g.sum(axis=1) - fx[f"{prefix}{key}_rowsum_{k}"]).max() <= g.shape[1] * TOL_M, (k, key)
                assert np.abs(g.sum(axis=0) - fx[f"{prefix}{key}_colsum_{k}"]).max() <= g.shape[0] * TOL_M, (k, key)
        if f"{prefix}ocean_{k}" in fx:
            assert np.array_equal(r["ocean"] != 0, _unpack(fx[f"{prefix}ocean_{k}"], r["ocean"].shape)), k
            assert np.array_equal(r["beta"] != 0, _unpack(fx[f"{prefix}beta_{k}"], r["beta"].shape)), k
        if f"{prefix}gmslc_ocn" in fx:
            for key in ("gmslc_ocn", "gmslc_ocnBeta", "ocean_area", "oceanBeta_area", "ice_volume"):
                ref = fx[f"{prefix}{key}"][k - 1]
                assert abs(r[key] - ref) <= 1e-9 * max(1.0, abs(ref)), (k, key, r[key], ref)
        # rotational feedback (TPW direction, inertia perturbation, centrifugal potential):
        # the reference's signs and magnitudes, 1e-9 of the largest entry of the run
        for key in ("mm", "il", "lambda"):
            if f"{prefix}{key}" in fx:
                ref = fx[f"{prefix}{key}"]
                scale = float(np.abs(ref).max())
                assert np.abs(np.asarray(r[key]) - ref[k - 1]).max() <= 1e-9 * scale, (k, key)
    assert numiter == list(fx[f"{prefix}numiter"]), numiter


def test_c0_plain_100_steps():
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    fx = load_golden("step_c0.npz")
    love = FixtureLove(fx)
    topo = fx["topo_mm"] / 1000.0
    case = case_c0(OracleSHT(64, 128, 63))
    assert np.array_equal(case.topo, topo)
    slv = SeaLevelSolver(None, love, topo, case.ice(0), norder=63, dt=1.0)
    a0, b0, v0 = fx["plain_step0_scalars"]
    assert abs(slv.ocean_area0 - a0) <= 1e-9 * abs(a0)
    assert abs(slv.ice_volume0 - v0) <= 1e-9 * abs(v0)
    _check_against_fixture(slv, fx, "plain_", case.ice, 100)


def test_c0_extrap_dsl_100_steps():
    from slevolve_b200 import OptSeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    fx = load_golden("step_c0.npz")
    love = FixtureLove(fx)
    topo = fx["topo_mm"] / 1000.0
    case = case_c0(OracleSHT(64, 128, 63))
    slv = OptSeaLevelSolver(None, love, topo, case.ice(0), norder=63, dt=1.0,
                            opt={"numba", "sums", "dsl"}, inner="extrap")
    _check_against_fixture(slv, fx, "extrap_", case.ice, 100)


def test_marine_cap():
    from slevolve_b200 import SeaLevelSolver
    from tests_helpers import marine_ice
    from oracle.sht import gauss_nodes

    fx = load_golden("step_marine.npz")
    love = FixtureLove(fx)
    mu, _ = gauss_nodes(64)
    ice = marine_ice(mu, 128, fx["ice_heights"])
    slv = SeaLevelSolver(None, love, fx["topo"], ice[0], norder=63, dt=1000.0)
    _check_against_fixture(slv, fx, "plain_", lambda k: ice[k], 8)


def test_c1_small_grounding_line():
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c1
    from oracle.sht import OracleSHT

    fx = load_golden("step_c1s.npz")
    love = FixtureLove(fx)
    case = case_c1(OracleSHT(64, 128, 63), nsteps=60)
    slv = SeaLevelSolver(None, love, case.topo, case.ice(0), norder=63, dt=1.0)
    _check_against_fixture(slv, fx, "plain_", case.ice, 60)
    assert slv.gr_counts["ice_analyses"] > 0


@pytest.mark.parametrize("opt,raw", [({"numba", "sums", "dsl"}, False), ({"raw", "diag", "dsl"}, True)])
def test_reference_synthetic_512_golden(opt, raw):
    """The reference's shipped L=511 golden grid (8 steps, --opt all --inner extrap), every cell;
    also through a raw-mode (sign-free) transform with the solver's --opt raw, as the golden run
    used it."""
    from slevolve_b200 import OptSeaLevelSolver, make_sht
    from tests_helpers import synthetic512_ice

    fx = load_golden("synthetic512.npz")
    tg8 = load_golden("tgrid8.npz")["tgrid8"]
    assert np.array_equal(tg8[::8, ::8], fx["tgrid8_sub"])
    love = FixtureLove(fx)
    topo = fx["topo_mm"].astype(np.float64) / 1000.0
    sht = make_sht("cuda", 512, 1024, 511, raw=raw)
    ice = synthetic512_ice(sht.gaulats, topo, 1024, fx["polar"], fx["midlat"])
    if "ice_abs_sums" in fx:
        assert np.array_equal(np.array([float(np.abs(x).sum()) for x in ice]), fx["ice_abs_sums"])
    slv = OptSeaLevelSolver(sht, love, topo, ice[0], norder=511, dt=1.0, opt=opt, inner="extrap")
    ni = []
    for k in range(1, 9):
        r = slv.step(ice[k])
        ni.append(r["numiter"])
    assert ni == list(fx["numiter_doc"])
    assert np.abs(r["tgrid"] - tg8).max() <= TOL_M


def test_c1_full_size_550_steps():
    """c1 at its benchmark size and length (256 x 512, L = 255, 550 steps of 1 yr: grounding-line
    retreat under 1-20 m/yr thinning) against the reference's own run (make_golden_c1.py): the
    iteration count, degree-0 diagnostics and rotational quantities of every step, topography,
    radial displacement and both masks at eleven steps spread over the run."""
    from slevolve_b200 import SeaLevelSolver
    from slevolve_b200.synthetic import case_c1
    from oracle.sht import OracleSHT

    fx = load_golden("step_c1.npz")
    case = case_c1(OracleSHT(256, 512, 255), nsteps=550)
    assert np.array_equal(np.round(case.topo * 1000.0).astype(np.int64), fx["topo_mm"])
    slv = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=255, dt=1.0)
    a0, b0, v0 = fx["step0_scalars"]
    assert abs(slv.ocean_area0 - a0) <= 1e-9 * abs(a0)
    assert abs(slv.oceanBeta_area0 - b0) <= 1e-9 * abs(b0)
    assert abs(slv.ice_volume0 - v0) <= 1e-9 * abs(v0)

    def ice(k):
        g = case.ice(k)
        assert float(np.abs(g).sum()) == fx["ice_abs_sum"][k - 1], k
        return g

    _check_against_fixture(slv, fx, "", ice, 550)
    assert slv.gr_counts["ice_analyses"] > 0


def test_nonfinite_ice_is_reported_not_faulted():
    from slevolve_b200 import SeaLevelSolver, SyntheticEarth

    love = SyntheticEarth(15, 3, 2)
    topo = np.where(np.arange(32)[None, :] < 16, -1000.0, 500.0) * np.ones((16, 1))
    slv = SeaLevelSolver(None, love, topo, np.zeros((16, 32)), norder=15)
    bad = np.zeros((16, 32))
    bad[3, 4] = np.nan
    with pytest.raises(RuntimeError, match="non-finite"):
        slv.step(bad)


def test_nonconvergence_cap():
    """epsilon1 < 0 can never be met: the device loop stops at 9999 iterations with an error."""
    from slevolve_b200 import SeaLevelSolver, SyntheticEarth

    love = SyntheticEarth(15, 3, 2)
    topo = np.where(np.arange(32)[None, :] < 16, -1000.0, 500.0) * np.ones((16, 1))
    ice = np.zeros((16, 32))
    slv = SeaLevelSolver(None, love, topo, ice, norder=15, epsilon1=-1.0)
    ice1 = ice.copy()
    ice1[2:5, 20:24] = 100.0
    with pytest.raises(RuntimeError, match="failed to converge"):
        slv.step(ice1)


def test_outer_passes_with_warm_reuse_against_oracle():
    """Three outer (ice-age) passes over the c0 shape with the reference's Picard update of the
    initial topography (run_outer.py) and reuse="warm": every step of every pass against the
    CPU oracle driven the same way (same iteration counts, topography within 1e-9 m)."""
    from slevolve_b200 import OptSeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT
    from oracle.solver import OracleSolver

    osht = OracleSHT(64, 128, 63)
    case = case_c0(osht, nsteps=12)
    obs = case.topo.copy()
    T_gpu, T_orc = case.topo.copy(), case.topo.copy()
    store_gpu, store_orc = {}, {}
    warm = 0
    for it in range(3):
        kw = dict(norder=63, dt=1.0, opt={"dsl"}, inner="extrap", reuse="warm")
        slv = OptSeaLevelSolver(None, case.love, T_gpu, case.ice(0), reuse_store=store_gpu, **kw)
        orc = OracleSolver(osht, case.love, T_orc, case.ice(0), reuse_store=store_orc, **kw)
        for k in range(1, 13):
            r = slv.step(case.ice(k))
            o = orc.step(case.ice(k))
            assert r["numiter"] == o["numiter"], (it, k)
            assert np.abs(r["tgrid"] - o["tgrid"]).max() <= TOL_M, (it, k)
        warm += slv.reuse_stats["warm_steps"]
        T_gpu = T_gpu - (np.array(r["tgrid"]) - obs)
        T_orc = T_orc - (o["tgrid"] - obs)
    assert warm == 24   # passes 2 and 3 start every step from the stored state


@pytest.mark.parametrize("kind", ["plain", "extrap"])
def test_variable_step_lengths(kind):
    """24 steps of varying length through step(ice, dt=...): decay factors per distinct length
    and the non-uniform extrapolated start, against the reference (make_golden_vardt.py)."""
    from slevolve_b200 import OptSeaLevelSolver, SeaLevelSolver
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    fx = load_golden("step_vardt.npz")
    case = case_c0(OracleSHT(64, 128, 63), nsteps=len(fx["dts"]) + 8)
    if kind == "plain":
        slv = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=63, dt=1.0)
    else:
        slv = OptSeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=63, dt=1.0,
                                opt={"dsl"}, inner="extrap")
    numiter = []
    for k, dt in enumerate(fx["dts"], start=1):
        r = slv.step(case.ice(k), dt=float(dt))
        numiter.append(r["numiter"])
        if f"{kind}_tgrid_{k}" in fx:
            assert np.abs(r["tgrid"] - fx[f"{kind}_tgrid_{k}"]).max() <= TOL_M, k
            assert np.abs(r["R"] - fx[f"{kind}_R_{k}"]).max() <= TOL_M, k
            assert np.array_equal(r["ocean"] != 0, _unpack(fx[f"{kind}_ocean_{k}"], r["ocean"].shape)), k
            assert np.array_equal(r["beta"] != 0, _unpack(fx[f"{kind}_beta_{k}"], r["beta"].shape)), k
    assert numiter == list(fx[f"{kind}_numiter"])
