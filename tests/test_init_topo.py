"""The segmented initial-topography guess: the oracle against the reference's own output
(``tests/golden/init_topo.npz``, made by ``make_golden_init_topo.py``), and the package's leg
detection against the oracle's on varied volume series (no GPU)."""

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle.init_topo import segmented_guess, segments as oracle_segments  # noqa: E402
from oracle.sht import OracleSHT  # noqa: E402
from slevolve_b200.init_topo import relaxed_love, segments  # noqa: E402
from slevolve_b200.synthetic import case_glacial  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "init_topo.npz"))


def test_golden_inputs_regenerate():
    topo, ice, _ = case_glacial(OracleSHT(64, 128, 63))
    assert np.array_equal(topo, GOLD["topo"])
    assert np.array_equal(np.stack(ice), GOLD["ice"])


@pytest.mark.parametrize("name", ["uniform", "times"])
def test_oracle_reproduces_the_reference(name):
    topo, ice, love = case_glacial(OracleSHT(64, 128, 63))
    kw = {"uniform": dict(dt=10.0, threshold=0.01, start=None),
          "times": dict(dt=GOLD["times"], threshold=0.05, start=GOLD["start"])}[name]
    T0, info = segmented_guess(topo, ice, love, 63, kw["dt"], threshold=kw["threshold"], start=kw["start"])
    assert info["iters"] == int(GOLD[f"{name}_iters"])
    assert [[s["a"], s["b"]] for s in info["segments"]] == GOLD[f"{name}_legs"].tolist()
    assert np.allclose([s["tau"] for s in info["segments"]], GOLD[f"{name}_tau"], rtol=1e-14, atol=0)
    assert abs(info["c"] - float(GOLD[f"{name}_c"])) <= 1e-9
    assert np.abs(T0 - GOLD[f"{name}_T0"]).max() <= 1e-8


def test_leg_detection_matches_the_oracle():
    rng = np.random.default_rng(7)
    for trial in range(200):
        n = int(rng.integers(2, 40))
        V = np.cumsum(rng.normal(0.0, 1.0, n)) * 10.0 ** rng.uniform(10, 16)
        dt = float(rng.uniform(0.5, 20.0)) if trial % 2 else np.cumsum(rng.uniform(0.1, 5.0, n))
        thr = float(rng.choice([0.0, 0.01, 0.05, 0.3]))
        a, b = segments(V, dt, thr), oracle_segments(V, dt, thr)
        assert [(x["a"], x["b"]) for x in a] == [(x["a"], x["b"]) for x in b]
        for x, y in zip(a, b):
            assert x["tau"] == y["tau"] and x["dV"] == y["dV"], (trial, x, y)
    with pytest.raises(ValueError):
        segments([1.0], 1.0)
    with pytest.raises(ValueError):
        segments([1.0, 2.0, 3.0], [0.0, 1.0])


def test_relaxed_love_limits():
    from slevolve_b200.love import SyntheticEarth

    love = SyntheticEarth(31, 8, 5)
    h0, k0 = relaxed_love(love, 31, 0.0)
    assert np.array_equal(h0, love.he[:32]) and np.array_equal(k0, love.ke[:32])
    hinf, kinf = relaxed_love(love, 31, 1e12)
    assert np.allclose(hinf[1:], 3.0 * love.he[1:32], rtol=1e-12)   # fluid limit 3 X_E
    assert np.allclose(kinf[1:], 3.0 * love.ke[1:32], rtol=1e-12)
