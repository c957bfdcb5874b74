"""Host-side arithmetic of bench.py's roofline split (no GPU): the transform share, the modal
advance share, the elementwise passes and their time-weighted combination from a per-class
device-time profile; the serving loop's occupancy record."""

import importlib.util
import math
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(HERE, "..", "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _prof(nprof=3):
    per_step = {"k_fold_mx": (1.39, 32.3, 1034.7), "k_leg_tc<analysis of rO>": (0.69, 7.3, 234.7),
                "k_leg_tc<other analyses>": (1.65, 25.0, 800.0),
                "k_bsyn_mx + k_leg_tc<synthesis>": (0.97, 8.3, 266.7), "k_unfold_mx": (0.51, 8.3, 266.7),
                "k_advance": (0.32, 1.0, 32.0), "k_update": (0.5, 7.0, 150.0), "k_dice": (0.2, 7.0, 150.0)}
    return {k: {"ms": v[0] * nprof, "launches": v[1] * nprof, "fields": v[2] * nprof} for k, v in per_step.items()}


def test_step_shares_arithmetic():
    b = _bench()
    peaks = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
    sh = b.step_shares(_prof(), 3, peaks)
    nh, ncoef = 256, 512 * 513 // 2
    per = 12.0 * nh * ncoef + 2.5 * 1024 * 10 * 512
    fields = 234.7 + 800.0 + 266.7
    t = (1.39 + 0.69 + 1.65 + 0.97 + 0.51) / 1000.0
    assert sh["transforms"]["achieved"] == pytest.approx(fields * per / t / 1e12, rel=1e-12)
    assert sh["transforms"]["frac"] == pytest.approx(sh["transforms"]["achieved"] / (1590.0 * b.TENSOR_RATE),
                                                     rel=1e-12)
    adv = 19 * 16.0 * ncoef * 32.0 / 0.32e-3 / 1e9
    assert sh["modal_advance"]["achieved"] == pytest.approx(adv, rel=1e-12)
    upd = sh["elementwise"]["k_update"]
    assert upd["achieved"] == pytest.approx(80.0 * ncoef * 150.0 / 0.5e-3 / 1e9, rel=1e-12)
    # dI works only after a grounded-mask change: time reported, no fraction, not in the combination
    assert sh["elementwise"]["k_dice"]["frac"] is None
    assert sh["elementwise"]["k_dice"]["ms_per_step"] == pytest.approx(0.2)
    fr = [sh["transforms"]["frac"], sh["modal_advance"]["frac"], upd["frac"]]
    lo, hi = min(fr), max(fr)
    assert lo <= sh["combined_frac"] <= hi
    assert sh["transforms"]["ms_per_step"] == pytest.approx(5.21, rel=1e-12)
    # per transform class: the contractions in TFLOP/s, the row FFTs in GB/s
    cl = sh["transforms"]["classes"]
    assert set(cl) == {"k_fold_mx", "k_leg_tc<analysis of rO>", "k_leg_tc<other analyses>",
                       "k_bsyn_mx + k_leg_tc<synthesis>", "k_unfold_mx"}
    ro = cl["k_leg_tc<analysis of rO>"]
    assert ro["achieved"] == pytest.approx(12.0 * nh * ncoef * 234.7 / 0.69e-3 / 1e12, rel=1e-12)
    assert ro["frac"] == pytest.approx(ro["achieved"] / (1590.0 * b.TENSOR_RATE), rel=1e-12)
    fold = cl["k_fold_mx"]
    assert fold["bytes_per_field"] == 8.0 * 512 * 1024 + 16.0 * 512 * 256
    assert fold["achieved"] == pytest.approx(fold["bytes_per_field"] * 1034.7 / 1.39e-3 / 1e9, rel=1e-12)
    assert fold["frac"] == pytest.approx(fold["achieved"] / 6650.0, rel=1e-12)
    assert cl["k_unfold_mx"]["unit"] == "GB/s" and cl["k_bsyn_mx + k_leg_tc<synthesis>"]["unit"] == "TFLOP/s"
    assert cl["k_unfold_mx"]["ms_per_step"] == pytest.approx(0.51, rel=1e-12)


def test_step_shares_empty_profile():
    b = _bench()
    prof = {k: {"ms": 0.0, "launches": 0, "fields": 0.0} for k in _prof()}
    sh = b.step_shares(prof, 1, {"hbm_gbs": 1.0, "bf16_tflops": 2.0})
    assert sh["combined_frac"] == 0.0 and not math.isnan(sh["transforms"]["frac"])
    assert sh["transforms"]["classes"] == {}


def test_serving_occupancy_record():
    """Time-weighted mean of the admitted footprint from the server's (time, bytes) record."""
    from slevolve_b200.serving import Server

    srv = object.__new__(Server)
    srv._occ = [(0.0, 100), (1.0, 300), (3.0, 0)]
    srv.wall = 4.0
    srv.peak_used = 300
    srv.device_bytes = 1000
    occ = srv.occupancy()
    assert occ["mean_bytes"] == pytest.approx((100 * 1.0 + 300 * 2.0) / 4.0)
    assert occ["hbm_occupancy_mean"] == pytest.approx(occ["mean_bytes"] / 1000)
    assert occ["hbm_occupancy_peak"] == pytest.approx(0.3)
    # with the device memory in use recorded beside the admitted footprint
    srv._occ = [(0.0, 100, 500), (1.0, 300, 900), (3.0, 0, 400)]
    occ = srv.occupancy()
    assert occ["hbm_held_mean"] == pytest.approx((500 * 1.0 + 900 * 2.0 + 400 * 1.0) / 4.0 / 1000)
    assert occ["hbm_held_peak"] == pytest.approx(0.9)
