"""CPU-side checks of the C ABI and the host wrappers (no GPU needed)."""

import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "slevolve_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char\*)\s+(sle_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    from slevolve_b200 import _lib

    lib = _lib.lib()
    assert lib.sle_abi_version() == 1
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    # the ctypes table binds exactly the declared entry points
    assert set(_lib.exported_symbols()) <= set(declared_symbols())


def test_programmatic_launch_switch():
    """sle_set_programmatic_launch reports the previous mode; the initial mode follows
    SLEVOLVE_B200_NO_PDL (host state only, no device call)."""
    import sys

    from slevolve_b200 import _lib

    prev = _lib.set_programmatic_launch(False)
    try:
        assert _lib.set_programmatic_launch(True) is False
        assert _lib.set_programmatic_launch(True) is True
        assert _lib.lib().sle_set_programmatic_launch(0, None) == 0   # status; previous may be NULL
        assert _lib.set_programmatic_launch(True) is False
    finally:
        _lib.set_programmatic_launch(prev)
    code = "from slevolve_b200 import _lib; print(int(_lib.set_programmatic_launch(True)))"
    for value, mode in (("1", 0), ("yes", 0), ("0", 1), ("", 1), (None, 1)):
        env = {k: v for k, v in os.environ.items() if k != "SLEVOLVE_B200_NO_PDL"}
        if value is not None:
            env["SLEVOLVE_B200_NO_PDL"] = value
        out = subprocess.run([sys.executable, "-c", code], cwd=REPO, env=env, capture_output=True,
                             text=True, check=True, timeout=300).stdout
        assert int(out.strip().splitlines()[-1]) == mode, (value, out)


def test_error_mapping():
    from slevolve_b200 import _lib

    lib = _lib.lib()
    # argument validation happens before any device call
    import ctypes as C

    h = C.c_void_p()
    with pytest.raises(ValueError, match="nlat must be even"):
        _lib.check(lib.sle_sht_create(15, 32, 15, C.byref(h)), "create")
    with pytest.raises(ValueError, match="lmax must be <= nlon/2"):
        _lib.check(lib.sle_sht_create(16, 32, 17, C.byref(h)), "create")
    with pytest.raises(ValueError, match="power of two"):
        _lib.check(lib.sle_sht_create(16, 48, 15, C.byref(h)), "create")
    # read-out and driver-helper entry points: NULL arguments are refused before any device call
    assert lib.sle_solver_set_rate_tables(None, None) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_solver_get_rates(None, None, None, None, None) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_solver_set_horizontal(None, None) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_solver_get_horizontal(None, None, None, None) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_solver_set_ramp(None, None) == _lib.SLE_ERR_BAD_ARG
    n = C.c_longlong()
    assert lib.sle_solver_snapshot_bytes(None, C.byref(n)) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_solver_snapshot(None, None, 0) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_solver_restore(None, None, 0) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_batch_snapshot_bytes(None, C.byref(n)) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_batch_snapshot(None, 0, None, 0) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_batch_restore(None, 0, None, 0) == _lib.SLE_ERR_BAD_ARG
    assert lib.sle_topo_scratch_bytes() >= 16
    buf = (C.c_double * 2)()
    assert lib.sle_topo_residual(None, None, 0.0, None, None, None, None, 4, 8, 920.0, 1000.0, None, buf,
                                 None) == _lib.SLE_ERR_BAD_ARG
    with pytest.raises(ValueError, match="NULL"):
        _lib.check(lib.sle_solver_get_rates(None, None, None, None, None), "sle_solver_get_rates")


def test_solver_rejects_unprovided_options():
    from slevolve_b200 import OptSeaLevelSolver, SeaLevelSolver, SyntheticEarth

    love = SyntheticEarth(15, 2, 1)
    topo = np.full((16, 32), -1000.0)
    ice = np.zeros((16, 32))
    with pytest.raises(NotImplementedError):
        SeaLevelSolver(None, love, topo, ice, norder=15, axial_rotation="deg2")
    with pytest.raises(NotImplementedError):
        OptSeaLevelSolver(None, love, topo, ice, norder=15, inner="anderson")
    with pytest.raises(NotImplementedError):
        OptSeaLevelSolver(None, love, topo, ice, norder=15, reuse="warm+corr")
    with pytest.raises(ValueError):
        OptSeaLevelSolver(None, love, topo, ice, norder=15, inner="bogus")
    with pytest.raises(ValueError):
        OptSeaLevelSolver(None, love, topo, ice, norder=15, opt={"raw"})
    with pytest.raises(ValueError):
        OptSeaLevelSolver(None, love, topo, ice, norder=15, opt={"fast"})


def test_make_sht_unknown_backend():
    from slevolve_b200 import make_sht

    with pytest.raises(ValueError, match="unknown SHT backend"):
        make_sht("numpy", 16, 32, 15)


def test_degree_weights_match_oracle():
    from oracle.solver import OracleSolver  # noqa: F401  (constants restated there)
    from slevolve_b200.solver import Planet, degree_weights
    from slevolve_b200 import SyntheticEarth

    love = SyntheticEarth(31, 3, 5)
    p = Planet()
    ttl, tek, the = degree_weights(love, 31, p)
    l = np.arange(32, dtype=np.float64)
    ref = np.zeros(32)
    ref[1:] = (4.0 * 3.1415926535898 * (p.radius ** 3)) / (p.mass * (2 * l[1:] + 1.0))
    assert np.array_equal(ttl, ref)
    assert np.array_equal(tek[1:], ref[1:] * (1 + love.ke[1:] - love.he[1:]))


def test_love_reader_roundtrip(tmp_path):
    """Write a small Love file in the reference's text format and read it back."""
    from slevolve_b200 import LoveNumbers

    lmax, K = 4, 3
    rng = np.random.default_rng(3)
    s = rng.uniform(0.1, 10, (K, lmax + 1))
    lines = ["header"]
    vals = {}
    for l in range(1, lmax + 1):
        lines.append(f"{l} {K}")
        lines.append(" ".join(f"{x:.8E}" for x in s[:, l]))
        el = rng.normal(size=5)
        fl = rng.normal(size=5)
        rh, rl, rk = (rng.normal(size=K) for _ in range(3))
        vals[l] = (el, rh, rk, rl)
        lines.append(" ".join(f"{x:.8E}" for x in el))
        lines.append(" ".join(f"{x:.8E}" for x in fl))
        for r in (rh, rl, rk):
            lines.append(" ".join(f"{x:.8E}" for x in r))
        if l >= 2:
            for _ in range(2):
                lines.append(" ".join(f"{x:.8E}" for x in rng.normal(size=5)))
            for _ in range(3):
                lines.append(" ".join(f"{x:.8E}" for x in rng.normal(size=K)))
    path = tmp_path / "love.txt"
    path.write_text("\n".join(lines) + "\n")
    L = LoveNumbers(str(path), lmax)
    for l in range(1, lmax + 1):
        el, rh, rk, rl = vals[l]
        assert np.allclose(L.s[:K, l], s[:, l], rtol=1e-8)
        assert np.isclose(L.he[l], el[0], rtol=1e-8)
        assert np.isclose(L.ke[l], el[4] / l, rtol=1e-8)
        assert np.isclose(L.le[l], el[1] / l, rtol=1e-8)     # tangential numbers, scaled as k
        assert np.allclose(L.r[:K, l], rh, rtol=1e-8)
        assert np.allclose(L.rprime[:K, l], rk / l, rtol=1e-8)
        assert np.allclose(L.rl[:K, l], rl / l, rtol=1e-8)
    assert L.max_modes == K


def test_ramp_factor_series_and_limits():
    from slevolve_b200.rates import ramp_factor

    x = np.array([0.0, 1e-9, 5e-5, 9.99e-5, 1.0001e-4, 0.3, 2.0, 50.0])
    phi, omp = ramp_factor(x)
    assert phi[0] == 1.0 and omp[0] == 0.0
    exact = np.where(x > 0, -np.expm1(-np.where(x > 0, x, 1.0)) / np.where(x > 0, x, 1.0), 1.0)
    assert np.allclose(phi, exact, rtol=1e-13, atol=0)
    assert np.allclose(phi + omp, 1.0, rtol=0, atol=2e-16)


@pytest.mark.parametrize("dt", [1.0, 0.37, 2.5e-6, 500.0])
def test_ramp_table_matches_oracle(dt):
    """The host table of the GPU ramp placement against the oracle's coefficients (pinned to the
    reference's ramp run): same values bit for bit, in the layout sle_solver_set_ramp reads."""
    from oracle.memory import ModalState
    from slevolve_b200 import SyntheticEarth, mode_arrays
    from slevolve_b200.rates import ramp_table
    from slevolve_b200.solver import Planet, degree_weights

    lmax = 31
    love = SyntheticEarth(lmax, 3, 5)
    ma = mode_arrays(love, lmax)
    ttl = degree_weights(love, lmax, Planet())[0]
    tab = ramp_table(ma, love, lmax, ttl, dt)
    st = ModalState(love, lmax, dt)
    K, nl = int(ma["K"]), lmax + 1
    assert tab.shape == (K * nl + 2 * nl + 4,)
    om = tab[:K * nl].reshape(K, nl)
    assert np.array_equal(om[:st.kmax], st.omphi) and not om[st.kmax:].any()
    assert np.array_equal(tab[K * nl:K * nl + nl], ttl * st.c_sl)
    assert np.array_equal(tab[K * nl + nl:K * nl + 2 * nl], ttl * st.c_rr)
    assert np.array_equal(tab[-4:], [st.c_il, st.c_m, st.c_tsl, st.c_trr])
    assert om.max() > 0.0


def test_batch_get_out_checks():
    """``SolverBatch.get(out=...)``: the library writes nlat * nlon doubles through the pointer, so
    anything but a C-contiguous float64 grid of that shape is refused on the host."""
    from slevolve_b200.batch import _check_grid_out

    _check_grid_out(np.empty((16, 32)), 16, 32)
    for bad in (np.empty((16, 16)), np.empty((16, 32), np.float32), np.empty((32, 16)).T,
                np.empty((16, 64))[:, ::2]):
        with pytest.raises(ValueError, match="out must be"):
            _check_grid_out(bad, 16, 32)


def test_ramp_refused_for_mixed_precision():
    """Ramp placement is provided for FP64 solves; a mixed-precision one is refused before any
    device call."""
    from slevolve_b200 import SeaLevelSolver, SyntheticEarth

    love = SyntheticEarth(15, 2, 1)
    with pytest.raises(NotImplementedError, match="ramp"):
        SeaLevelSolver(None, love, np.full((16, 32), -1000.0), np.zeros((16, 32)), norder=15, ramp=True,
                       precision="mixed")


def test_rotation_rate_matches_oracle():
    """The package's rotational-rate read-out (Jacobian form) against the oracle's restatement of
    the reference's expressions (pinned to its rates golden): 1e-12 of the largest entry."""
    from oracle.memory import ModalState
    from oracle.readouts import RateWeights, rotation_rate as oracle_rate
    from slevolve_b200 import SyntheticEarth
    from slevolve_b200.rates import RateTables, rotation_rate
    from slevolve_b200.solver import Planet

    lmax, dt = 15, 3.7
    love = SyntheticEarth(lmax, 5, 9)
    p = Planet()
    rng = np.random.default_rng(4)
    st = ModalState(love, lmax, dt)
    n2 = st.nmod2
    st.r_il = rng.normal(size=(st.kmax, 3, 3)) * 1e30
    st.r_m = rng.normal(size=(st.kmax, 3)) * 1e-9
    st.r_lambda = (rng.normal(size=(st.kmax, 3)) + 1j * rng.normal(size=(st.kmax, 3))) * 1e-3
    wt = RateWeights(st)
    wt.set_dt(st, dt)
    tabs = RateTables(love, lmax)
    tabs.for_dt(dt)
    il = rng.normal(size=(3, 3)) * 1e30
    oldil = il + rng.normal(size=(3, 3)) * 1e28
    mm = rng.normal(size=3) * 1e-8
    oldm = mm + rng.normal(size=3) * 1e-10
    lam = np.zeros((3, 3), dtype=np.complex128)
    lam[2, :] = (rng.normal(size=3) + 1j * rng.normal(size=3)) * 1e-2
    lam[0, 0] = 0.3
    dprev = (rng.normal(size=3) + 1j * rng.normal(size=3)) * 1e-3
    a_sl, a_rr, a_d = oracle_rate(st, wt, love, p, dt, il, mm, lam, oldil, oldm, dprev)
    b_sl, b_rr, b_d = rotation_rate(tabs, love, p, dt, il, mm, lam, oldil, oldm, dprev,
                                    st.r_il, st.r_m, st.r_lambda)
    for a, b in ((a_sl, b_sl), (a_rr, b_rr), (a_d["mdot"], b_d["mdot"]), (a_d["ildot"], b_d["ildot"]),
                 (a_d["lambdadot"], b_d["lambdadot"])):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
    assert n2 > 0
