#!/usr/bin/env python3
"""Throughput of the SLEvolve sea-level time step on B200 at L = 511 (512 x 1024 grid): the
mixed-precision batched form against the FP64 form, with serving latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]

Workload: c2-shape members (512 x 1024 Gauss grid, L = 511, 8 viscous modes per degree, 200-yr
steps, three northern-hemisphere ice sheets on a 100-kyr sawtooth, shoreline migration,
grounded-ice test and rotational feedback on), options ``opt={"dsl", "diag"}``,
``inner="extrap"``.  A step is one full time step of a member, inner fixed-point loop included.

* ``value``  member-steps/s of a batch of B = 32 members stepped together in mixed precision
  (split-TF32 tensor-core Legendre contractions, FP32 accumulation; everything else FP64).  The members differ in
  Earth model (relaxation times scaled by a seeded factor log-uniform in [0.3, 3]) and ice
  amplitude (seeded, U[0.5, 1.5]) as in the uneven ensembles.  Ice resident in HBM, CUDA events
  on the batch's stream, L2 flushed (256 MiB write) between steps outside the timed intervals,
  W untimed warm-up steps first.
* ``fp64``   the same member-steps as single FP64 solves (the plain GPU form, bit-compatible with
  the reference): steps/s, and ``speedup`` = value / fp64 steps/s.
* ``accuracy`` member 0 of the batch against the FP64 solve of the same inputs over the timed
  steps: max and RMS error per output field, ocean / grounded-mask cells that differ, steps whose
  inner-iteration count differs.
* ``e2e``    the same member-steps as ``value`` (a fresh batch of the same members, its W warm-up
  steps through the same call, then steps W + 1 .. W + 20 with each member's own ice) through the
  public API ``SolverBatch.step_host_stream`` with host ice grids (pinned), copied to the device
  inside the timed region (each step's upload overlapping the previous step's compute), each
  member's step record read back after every step.
* ``latency`` a short serving run (``slevolve_b200.serving``): seeded members of L = 127 / 255 / 511
  arriving in a Poisson stream, p50 / p99 solve latency and member-steps/s (sample stated).
* ``ensemble`` the uneven ensemble (64 seeded members, L in {127, 255, 511}, 50-1200 steps each)
  run to completion in mixed precision with one continuously batched slot group per degree, the
  slot count of each group autotuned by a short timed probe: wall time and member-steps/s.
* ``roofline`` the dominant kernel by device time (a profiling pass with CUDA events around every
  transform launch and inner-loop pass, host-driven inner loop): algorithmic FLOPs of the split
  Legendre contraction (3 MMAs per product, 12 nh ncoef per field) over the measured time, against
  the dense tensor rate of the split's operand type (from the measured BF16 GEMM rate);
  ``traffic`` from the committed ncu summary; ``step_shares`` the same profile split by bound: all
  executed transforms (contraction + row FFT work over the transform kernels' time, against that
  tensor rate), the modal advance and each elementwise pass of the inner loop (algorithmic bytes
  over its time, against the copy bandwidth), and their time-weighted combination;
  ``gated_analyses`` the C* / tO / I* re-analyses separately.
* ``fp64.roofline`` the FP64 form's Legendre contractions (4 nh ncoef flops per field) against the
  FP64 FMA rate measured in the same run.
* ``cpu_baseline`` the CPU oracle (NumPy restatement of the reference solver, FP64) on this
  host's cores, 5 timed steps of the c2 run.

With N > 1 (torchrun) every rank runs an independent batch on its own GPU (members shard across
GPUs, no collective on the data path); ``value`` is the sum of member-steps over the
max-over-ranks time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "steps/sec at L=511, FP64 vs mixed+batched (≤1 mm err); p50/p99 latency"
WORKLOAD = ("c2-shape members, mixed precision, batched: 512x1024 Gauss grid, L=511, 8 modes/degree, "
            "200-yr steps, 3 NH ice sheets on a 100-kyr sawtooth, opt dsl+diag, inner extrap")
WORKLOAD_FP64 = "the same c2 member as a single FP64 solve (the plain GPU form)"
OPTS = ("dsl", "diag")
STEP_RECORD_BYTES = 1080   # per-slot step record the library reads back after every batched step
INNER = "extrap"
E2E_STEPS = 20   # batch steps of the e2e run (B x 4 MiB of pinned host ice each)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--batch", type=int, default=32, help="members per batch (mixed form)")
    ap.add_argument("--serve-requests", type=int, default=200, help="requests of the latency sample (0: skip)")
    ap.add_argument("--ensemble-members", type=int, default=64,
                    help="members of the uneven-ensemble run (L in {127, 255, 511}, 50-1200 steps; 0: skip)")
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--cpu-steps", type=int, default=5, help="timed oracle steps for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--init-topo", action="store_true",
                    help="instead: time the segmented initial-topography guess (GPU) against the CPU oracle")
    ap.add_argument("--kernel-case", action="store_true",
                    help="instead: only load a batch of --batch c2 members and run --steps batch steps "
                         "(the small case for ncu captures of single kernels)")
    ap.add_argument("--serve-load", action="store_true",
                    help="instead: the serving configuration at its load (budget 80 %% of HBM)")
    ap.add_argument("--load-requests", type=int, default=1200)
    ap.add_argument("--load-min-steps", type=int, default=50)
    ap.add_argument("--load-max-steps", type=int, default=1200)
    ap.add_argument("--load-arrival-s", type=float, default=2.0)
    ap.add_argument("--load-precision", default="mixed", choices=("mixed", "fp64"))
    return ap.parse_args()


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled every 20 ms through NVML while running
    (the data nvidia-smi's clocks query reports); falls back to ``nvidia-smi -lms 200``."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.rows = []   # (sm_mhz, sm_max_mhz, set of active reason names)
        self.proc = None
        self.stop = threading.Event()
        self.thread = None

    def _nvml_loop(self, nvml, h):
        mx = nvml.nvmlDeviceGetMaxClockInfo(h, nvml.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = nvml.nvmlDeviceGetClockInfo(h, nvml.NVML_CLOCK_SM)
                bits = nvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((float(sm), float(mx), {n for n, b in self.REASONS if bits & b}))
            except Exception:
                pass
            time.sleep(0.02)

    def _smi_loop(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        for line in self.proc.stdout:
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 6 and p[0].replace(".", "", 1).isdigit():
                names = {n for (n, _), v in zip(self.REASONS, p[2:6]) if v.lower() == "active"}
                self.rows.append((float(p[0]), float(p[1]), names))

    def __enter__(self):
        try:
            import pynvml as nvml
            import torch

            nvml.nvmlInit()
            props = torch.cuda.get_device_properties(torch.cuda.current_device())
            uuid = str(getattr(props, "uuid", "") or "")
            if uuid:
                # the NVML handle of the CUDA device in use (NVML indexes every GPU of the node)
                h = nvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            else:
                h = nvml.nvmlDeviceGetHandleByIndex(self.index)
            self.thread = threading.Thread(target=self._nvml_loop, args=(nvml, h), daemon=True)
        except Exception:
            self.thread = threading.Thread(target=self._smi_loop, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [r[0] for r in self.rows]
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(set().union(*[r[2] for r in self.rows])), "samples": len(self.rows)}


def build_case(sht_factory):
    from slevolve_b200.synthetic import case_c2

    return case_c2(sht_factory())


def cpu_oracle_run(case, nwarm, ntimed, workers):
    """Oracle steps/s on the host (NumPy/SciPy, all host threads for FFT and BLAS)."""
    from oracle.sht import OracleSHT
    from oracle.solver import OracleSolver

    t0 = time.perf_counter()
    osht = OracleSHT(case.nlat, case.nlon, case.lmax, workers=workers)
    slv = OracleSolver(osht, case.love, case.topo, case.ice(0), norder=case.lmax, dt=case.dt,
                       opt=set(OPTS), inner=INNER)
    setup = time.perf_counter() - t0
    for k in range(1, nwarm + 1):
        slv.step(case.ice(k))
    t0 = time.perf_counter()
    nit = 0
    for k in range(nwarm + 1, nwarm + ntimed + 1):
        nit += slv.step(case.ice(k))["numiter"]
    dt = time.perf_counter() - t0
    return {"steps_per_s": ntimed / dt, "seconds": dt, "setup_s": setup, "numiter_per_step": nit / ntimed}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle.sht import OracleSHT

    workers = os.cpu_count() or 1
    case = build_case(lambda: OracleSHT(512, 1024, 511, workers=workers))
    r = cpu_oracle_run(case, a.warmup, a.steps, workers)
    sample = f"{a.steps} timed steps after {a.warmup} warm-up steps of the same c2 run"
    # one member per step: steps/s of the single solve = member-steps/s, the unit of our arm
    line = {"impl": "reference", "metric": METRIC, "value": r["steps_per_s"], "unit": "member-steps/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000.0 / r["steps_per_s"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [512, 1024], "lmax": 511, "modes": 8,
                       "precision": "fp64", "numiter_per_step": r["numiter_per_step"],
                       "solver": "CPU oracle (NumPy restatement of the reference SeaLevelSolver)"},
            "cpu_baseline": {"value": r["steps_per_s"], "unit": "member-steps/s", "cores": workers,
                             "kind": "port", "sample": sample},
            "e2e": {"value": r["steps_per_s"], "unit": "member-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def load_peaks():
    """Roofline denominators: the measured copy bandwidth and BF16 GEMM rate of this GPU pool
    (MEASURED_PEAKS.json beside this file), else an earlier measurement on the same pool
    (6.65 TB/s, 1.59 PFLOP/s BF16 burst)."""
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return {"hbm_gbs": float(p["hbm_gbs"]), "bf16_tflops": float(p["bf16_tflops"])}, "of measured"
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


# Algorithmic bytes per iterating slot of the inner loop's elementwise passes (one read of each
# input, one write of each output; ng cells, nc packed coefficients): eq. B18 reads dI, the
# previous load increment, the current increment and the viscous term and writes the sea-level
# spectrum; the update reads dS_prev, rO, C*, tO and writes the increment (dS_cur only at its two
# degree-2 entries); the refresh of an iteration that does not converge reads dsl, T0 and ice plus
# the beta mask and writes the ocean function and the candidate grounded mask (marine test on;
# deltasl is written by the converged iteration only); the C* refresh reads the ocean, beta and
# C* masks and writes C*.
ELEMENTWISE = {"k_b18": ("nc", 80.0), "k_update": ("nc", 80.0), "k_refresh1": ("ng", 27.0),
               "k_refresh2_x8": ("ng", 4.0)}
# Passes whose work depends on the iteration's outcome: dI (k_dice) reads I*_lm, the old I*_lm
# and p_ice and writes dice and dI only after a grounded-mask change, and returns at once
# otherwise, so no byte count per launch applies; its time is reported without a fraction.
GATED_PASSES = ("k_dice",)
# MMAs per product of the split contraction and the dense tensor rate they run at, as a fraction of
# the measured BF16 GEMM rate
TENSOR_RATE = 0.5
TENSOR_NAME = "split-TF32 (TF32 hi + lo, three products)"
TENSOR_PEAK = "half the BF16 GEMM rate (the dense TF32 rate)"


def step_shares(prof, nprof, peaks, nlat=512, lmax=511, modes=8):
    """Roofline of the whole step split by bound, from the profiling pass's per-class device time
    over `nprof` batch steps (`prof[name] = {"ms", "launches", "fields"}`).

    * transforms: algorithmic work of every executed transform, the split contraction counted as
      three MMAs per product (12 nh ncoef per field) plus the row FFT (2.5 nlon log2(nlon) N),
      over the time of the fold, Legendre and unfold kernels, against the dense tensor rate of the
      split's operand type (TENSOR_RATE x the measured BF16 GEMM rate);
    * modal advance: (2K + 3) 16 ncoef bytes per member over its time, against the copy bandwidth;
    * elementwise: each inner-loop pass with its algorithmic bytes per iterating slot
      (ELEMENTWISE) over its time, against the copy bandwidth;
    * combined: the fractions weighted by their times.

    `transforms["classes"]` gives each transform kernel class its own figure: the Legendre
    contractions 12 nh ncoef FLOPs per field against the dense tensor rate, the fold and the unfold
    8 ng + 16 nm nh bytes per field (the FP64 grid one way, the FP32 S / D planes or E / O sums,
    16 bytes per latitude and order, the other) against the copy bandwidth.  The classes count
    every field of a launch; for the fold and the gated analyses that includes fields gated off
    (and mask sources, one byte per cell), so their figures are upper bounds."""
    nh, nlon = nlat // 2, 2 * nlat
    nm = lmax + 1
    ncoef = (lmax + 1) * (lmax + 2) // 2
    ng = nlat * nlon
    tpk = peaks["bf16_tflops"] * TENSOR_RATE
    tr_names = ("k_fold_mx", "k_leg_tc<analysis of rO>", "k_leg_tc<other analyses>",
                "k_bsyn_mx + k_leg_tc<synthesis>", "k_unfold_mx")
    fields = (prof["k_leg_tc<analysis of rO>"]["fields"] + prof["k_leg_tc<other analyses>"]["fields"]
              + prof["k_bsyn_mx + k_leg_tc<synthesis>"]["fields"])
    per_transform = 12.0 * nh * ncoef + 2.5 * nlon * np.log2(nlon) * nlat
    t_tr = sum(prof[n]["ms"] for n in tr_names) / 1000.0
    tr_ach = fields * per_transform / t_tr / 1e12 if t_tr > 0 else 0.0
    adv = prof["k_advance"]
    t_m = adv["ms"] / 1000.0
    m_ach = (2 * modes + 3) * 16.0 * ncoef * adv["fields"] / t_m / 1e9 if t_m > 0 else 0.0
    tr_frac, m_frac = tr_ach / tpk, m_ach / peaks["hbm_gbs"]
    out = {
        "transforms": {"transforms_per_step": fields / nprof, "flops_per_transform": per_transform,
                       "ms_per_step": 1000.0 * t_tr / nprof, "achieved": tr_ach, "unit": "TFLOP/s",
                       "peak": tpk, "frac": tr_frac},
        "modal_advance": {"bytes_per_step": (2 * modes + 3) * 16.0 * ncoef * adv["fields"] / nprof,
                          "ms_per_step": 1000.0 * t_m / nprof, "achieved": m_ach, "unit": "GB/s",
                          "peak": peaks["hbm_gbs"], "frac": m_frac},
    }
    classes = {}
    for name in tr_names:
        c = prof[name]
        t = c["ms"] / 1000.0
        if t <= 0:
            continue
        if name in ("k_fold_mx", "k_unfold_mx"):
            per = 8.0 * ng + 16.0 * nm * nh
            ach = per * c["fields"] / t / 1e9
            classes[name] = {"bound": "hbm", "bytes_per_field": per, "achieved": ach, "unit": "GB/s",
                             "peak": peaks["hbm_gbs"], "frac": ach / peaks["hbm_gbs"]}
        else:
            per = 12.0 * nh * ncoef
            ach = per * c["fields"] / t / 1e12
            classes[name] = {"bound": "tensor", "flops_per_field": per, "achieved": ach, "unit": "TFLOP/s",
                             "peak": tpk, "frac": ach / tpk}
        classes[name]["ms_per_step"] = 1000.0 * t / nprof
        classes[name]["fields_per_step"] = c["fields"] / nprof
    out["transforms"]["classes"] = classes
    weighted, tot = tr_frac * t_tr + m_frac * t_m, t_tr + t_m
    elem = {}
    for name, (kind, per) in ELEMENTWISE.items():
        c = prof.get(name)
        if not c or c["ms"] <= 0:
            continue
        t = c["ms"] / 1000.0
        per_slot = per * (ncoef if kind == "nc" else ng)
        ach = per_slot * c["fields"] / t / 1e9
        elem[name] = {"ms_per_step": 1000.0 * t / nprof, "launches_per_step": c["launches"] / nprof,
                      "slot_passes_per_step": c["fields"] / nprof, "bytes_per_slot": per_slot,
                      "achieved": ach, "unit": "GB/s", "peak": peaks["hbm_gbs"], "frac": ach / peaks["hbm_gbs"]}
        weighted += ach / peaks["hbm_gbs"] * t
        tot += t
    for name in GATED_PASSES:
        c = prof.get(name)
        if c and c["ms"] > 0:
            elem[name] = {"ms_per_step": c["ms"] / nprof, "launches_per_step": c["launches"] / nprof,
                          "slot_passes_per_step": c["fields"] / nprof, "frac": None,
                          "note": "works only after a grounded-mask change; no byte count per launch"}
    out["elementwise"] = elem
    out["combined_frac"] = weighted / tot if tot > 0 else 0.0
    return out


def traffic_per_launch(kernel):
    path = os.path.join(HERE, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(kernel)
    except Exception:
        return None


MIXED_CLASSES = (("PROF_FFT", "k_fold_mx"), ("PROF_ANA_STEP", "k_leg_tc<analysis of rO>"),
                 ("PROF_LEG_ANA", "k_leg_tc<other analyses>"), ("PROF_LEG_SYN", "k_bsyn_mx + k_leg_tc<synthesis>"),
                 ("PROF_IFFT", "k_unfold_mx"), ("PROF_ADVANCE", "k_advance"), ("PROF_B18", "k_b18"),
                 ("PROF_UPDATE", "k_update"), ("PROF_REFRESH1", "k_refresh1"),
                 ("PROF_REFRESH2", "k_refresh2_x8"), ("PROF_DICE", "k_dice"))
FP64_CLASSES = (("PROF_FFT", "k_fft_fold"), ("PROF_ANA_STEP", "k_leg_ana<rO>"), ("PROF_LEG_ANA", "k_leg_ana<other>"),
                ("PROF_LEG_SYN", "k_leg_syn"), ("PROF_IFFT", "k_ifft_unfold"), ("PROF_ADVANCE", "k_advance"))


def read_prof(L, lib, classes):
    """{name: {"ms", "launches", "fields"}} of the library's per-class event timing."""
    out = {}
    for cls, name in classes:
        ms, cnt, units = lib.C.c_double(), lib.C.c_longlong(), lib.C.c_double()
        L.sle_prof_read(getattr(lib, cls), lib.C.byref(ms), lib.C.byref(cnt), lib.C.byref(units))
        out[name] = {"ms": ms.value, "launches": cnt.value, "fields": units.value}
    return out


def fp64_roofline(L, lib, sht, case, ice_dev, W, nprof, torch, nh=256, ncoef=512 * 513 // 2):
    """Roofline of the FP64 form (the denominator of the mixed/FP64 speed-up): its Legendre
    contractions (k_leg_ana / k_leg_syn, 4 nh ncoef flops per field, the recurrence not counted)
    over their CUDA-event time in a host-driven profiling pass of the single FP64 solve, against
    the FP64 FMA rate measured in the same run (sle_probe_fp64_tflops)."""
    from slevolve_b200 import OptSeaLevelSolver

    peak = lib.C.c_double()
    lib.check(L.sle_probe_fp64_tflops(lib.C.byref(peak)), "sle_probe_fp64_tflops")
    slv = OptSeaLevelSolver(sht, case.love, case.topo, case.ice(0), norder=511, dt=case.dt,
                            opt=set(OPTS), inner=INNER)
    for k in range(1, W + 1):
        slv.step_device(ice_dev[k].data_ptr(), 1)
    torch.cuda.synchronize()
    L.sle_prof_reset()
    L.sle_prof_enable(1)
    for k in range(W + 1, W + 1 + nprof):
        slv.step_device(ice_dev[k].data_ptr(), 1)
    torch.cuda.synchronize()
    L.sle_prof_collect()
    L.sle_prof_enable(0)
    prof = read_prof(L, lib, FP64_CLASSES)
    del slv
    leg = ("k_leg_ana<rO>", "k_leg_ana<other>", "k_leg_syn")
    fields = sum(prof[n]["fields"] for n in leg)
    ms = sum(prof[n]["ms"] for n in leg)
    achieved = 4.0 * nh * ncoef * fields / (ms / 1000.0) / 1e12 if ms > 0 else 0.0
    launches = sum(prof[n]["launches"] for n in leg)
    return {"bound": "fp64", "kernel": "k_leg_ana + k_leg_syn (FP64 Legendre contractions)",
            "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s", "frac": achieved / peak.value,
            "per_launch_flops": 4.0 * nh * ncoef * fields / max(launches, 1),
            "avg_launch_us": 1000.0 * ms / max(launches, 1),
            "peak_source": "FP64 FMA rate measured in this run (sle_probe_fp64_tflops)",
            "kernels": {k: {"ms_per_step": v["ms"] / nprof, "launches_per_step": v["launches"] / nprof,
                            "fields_per_step": v["fields"] / nprof} for k, v in prof.items()}}


def members(case, B, seed=20261207):
    """Seeded batch members of the c2 run: Earth relaxation scale, ice amplitude (member 0 of the
    first rank is the c2 member itself)."""
    from slevolve_b200 import SyntheticEarth

    rng = np.random.default_rng(seed)
    out = []
    for b in range(B):
        first = b == 0 and seed == 20261207
        f = 1.0 if first else float(np.exp(rng.uniform(np.log(0.3), np.log(3.0))))
        amp = 1.0 if first else float(rng.uniform(0.5, 1.5))
        love = case.love if first else SyntheticEarth(511, 8, seed - 2 + b, relax_scale=f)
        out.append((love, amp, f))
    return out


def timed_steps(step_fn, stream, flush, ksteps, torch):
    """Device time (ms) of ksteps calls, CUDA events on `stream`, L2 flushed before each."""
    events = []
    for k in range(ksteps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        step_fn(k)
        with torch.cuda.stream(stream):
            e1.record(stream)
        events.append((e0, e1))
    torch.cuda.synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in events)


def serving_sample(n, precision, seed=20261208):
    """Poisson stream of n seeded members (L = 127 / 255 / 511, 20-120 steps, every tenth an
    outer-iteration request of 3 warm-started passes) at a rate that keeps about 80 % of the
    slots busy; returns the server statistics (device-memory budget 80 % of the GPU's memory;
    the admitted footprint is reported against the whole device)."""
    import torch

    from slevolve_b200.serving import MemberFactory, Server

    total = torch.cuda.mem_get_info()[1]
    groups = {127: 8, 255: 6, 511: 8}
    rng = np.random.default_rng(seed)
    mf = MemberFactory(seed)
    Ls = rng.choice(list(groups), size=n)
    steps = rng.integers(20, 121, size=n)
    # service-time estimate (member-steps/s per degree, measured order of magnitude) for the rate
    rate = {127: 9000.0, 255: 5000.0, 511: 1500.0} if precision == "mixed" else {127: 4000.0, 255: 1800.0, 511: 600.0}
    busy = sum(steps[i] * (3 if i % 10 == 9 else 1) / rate[L] * groups[L] for i, L in enumerate(Ls)) / n
    lam = 0.8 * sum(groups.values()) / max(busy * sum(groups.values()), 1e-6)
    t = np.cumsum(rng.exponential(1.0 / lam, size=n))
    reqs = [mf.make(i, int(L), int(steps[i]), arrival=float(t[i]), outer_passes=3 if i % 10 == 9 else 1)
            for i, L in enumerate(Ls)]
    srv = Server(groups, precision=precision, budget_bytes=0.8 * total, device_bytes=total)
    srv.run(reqs)
    st = srv.stats(reqs)
    st.update({"lambda_per_s": lam, "groups": {str(k): v for k, v in groups.items()},
               "sample": f"{n} requests, L in {{127, 255, 511}}, 20-120 steps, every tenth 3 warm-started "
                         "outer passes, Poisson arrivals"})
    return st


def serve_load(a):
    """The serving configuration at its load: c3-style members (L in {127, 255, 511}, 50-1200
    steps, relaxation scale log-uniform in [0.3, 3], ice amplitude U[0.5, 1.5]), every tenth an
    outer-iteration request of 3 warm-started passes, Poisson arrivals over --load-arrival-s
    seconds, a device-memory budget of 80 % of the GPU's memory and slot groups large enough for
    the budget to bind.  Prints one JSON line with p50 / p99 latency, admission waits,
    member-steps/s and the time-weighted HBM occupancy of the admitted requests."""
    import torch

    from slevolve_b200.serving import MemberFactory, Server, footprint

    total = torch.cuda.mem_get_info()[1]
    budget = 0.8 * total
    n = a.load_requests
    rng = np.random.default_rng(20261211)
    mf = MemberFactory(20261211)
    Ls = rng.choice([127, 255, 511], size=n)
    steps = rng.integers(a.load_min_steps, a.load_max_steps + 1, size=n)
    outer = np.arange(n) % 10 == 9
    reqs = [mf.make(i, int(L), int(steps[i]), outer_passes=3 if outer[i] else 1) for i, L in enumerate(Ls)]
    fp = np.array([footprint(r) for r in reqs], dtype=np.float64)
    # slots per degree: that degree's share of the budget in requests of its mean footprint
    groups = {}
    for L in (127, 255, 511):
        sel = Ls == L
        if sel.any():
            share = fp[sel].sum() / fp.sum()
            groups[L] = int(min(sel.sum(), max(8, np.ceil(share * budget / fp[sel].mean()))))
    lam = n / max(a.load_arrival_s, 1e-3)
    t = np.cumsum(rng.exponential(1.0 / lam, size=n))
    for r, ti in zip(reqs, t):
        r.arrival = float(ti)
    srv = Server(groups, precision=a.load_precision, budget_bytes=budget, device_bytes=total)
    srv.run(reqs)
    st = srv.stats(reqs)
    line = {"metric": "serving at load: p50/p99 solve latency, member-steps/s, HBM occupancy",
            "precision": a.load_precision, "groups": {str(k): v for k, v in groups.items()},
            "lambda_per_s": lam, "device_bytes": total, "budget_frac": 0.8,
            "sample": (f"{n} requests, L uniform in {{127, 255, 511}}, {a.load_min_steps}-{a.load_max_steps} steps, "
                       "every tenth 3 warm-started outer passes, Poisson arrivals over "
                       f"{a.load_arrival_s} s"), **st}
    print(json.dumps(line), flush=True)
    return 0


def run_kernel_case(a):
    """Load B c2 members (as the headline batch) and run K batch steps from step 400; no timing.
    The case the per-kernel ncu captures run (one kernel, a few launches)."""
    import torch

    from slevolve_b200 import make_sht
    from slevolve_b200.batch import SolverBatch

    case = build_case(lambda: make_sht("cuda", 512, 1024, 511))
    B = a.batch
    mem = members(case, B)
    bt = SolverBatch(512, 1024, 511, B, precision="mixed", opt=OPTS, inner=INNER)
    ice0 = np.ascontiguousarray(case.ice(400))
    for b, (love, amp, _) in enumerate(mem):
        bt.load(b, love, case.topo, np.round(amp * ice0 * 1000.0) / 1000.0, case.dt)
    for k in range(1, a.steps + 1):
        ice = torch.from_numpy(np.ascontiguousarray(case.ice(400 + k))).cuda()
        bt.step({b: torch.round(m[1] * ice * 1000.0) / 1000.0 for b, m in enumerate(mem)})
    torch.cuda.synchronize()
    print(json.dumps({"kernel_case": "ok", "batch": B, "steps": a.steps}), flush=True)
    return 0


def run_ours(a):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from slevolve_b200 import OptSeaLevelSolver, _lib, make_sht
    from slevolve_b200.batch import SolverBatch
    from slevolve_b200.serving import max_over_ranks

    L = _lib.lib()
    sht = make_sht("cuda", 512, 1024, 511)
    case = build_case(lambda: sht)
    B, K, W = a.batch, a.steps, a.warmup
    k0 = 400                           # mid-cycle start: ice sheets present
    nprof = 3                          # batch steps of the kernel timing pass (after 2 untimed)
    nsteps = max(W + K, 2 + nprof)
    ng = case.nlat * case.nlon
    ice_host = [np.ascontiguousarray(case.ice(k0 + k)) for k in range(nsteps + 1)]
    ice_dev = [torch.from_numpy(x).cuda() for x in ice_host]
    mem = members(case, B, seed=20261207 + 7919 * rank)   # each rank its own members
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")

    def new_batch():
        bt = SolverBatch(512, 1024, 511, B, precision="mixed", opt=OPTS, inner=INNER)
        for b, (love, amp, _) in enumerate(mem):
            bt.load(b, love, case.topo, np.round(amp * ice_host[0] * 1000.0) / 1000.0, case.dt)
        return bt

    amps = [torch.tensor(m[1], dtype=torch.float64, device="cuda") for m in mem]

    def member_ice(k):   # device ice of every member at step k (amplitude-scaled, rounded to mm)
        return {b: torch.round(amps[b] * ice_dev[k] * 1000.0) / 1000.0 for b in range(B)}

    # ------------------------------------------------ value: mixed batch, device-resident ice
    bt = new_batch()
    stream = torch.cuda.ExternalStream(bt.stream_handle())
    dev_ices = [member_ice(k) for k in range(nsteps + 1)]
    for k in range(1, W + 1):
        bt.step(dev_ices[k])
    numiter = []
    L.sle_prof_reset()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()

    def mixed_step(i):
        torch.cuda.nvtx.range_push("mixed_batch_step")   # profiler filter (ncu --nvtx-include)
        infos = bt.step_ptrs({b: t.data_ptr() for b, t in dev_ices[W + 1 + i].items()}, 1)
        torch.cuda.nvtx.range_pop()
        numiter.append(max(x.numiter for x in infos.values()))

    with ClockSampler(local) as clk:
        dev_ms = timed_steps(mixed_step, stream, flush, K, torch)
    launches = int(L.sle_launch_count())
    clocks = clk.summary()
    t_max = max_over_ranks(dev_ms, dist)
    value = B * K * world / (t_max / 1000.0)

    # -------------------------------------- accuracy: member 0 against its FP64 solve (same inputs)
    slv = OptSeaLevelSolver(sht, case.love, case.topo, ice_host[0], norder=511, dt=case.dt,
                            opt=set(OPTS), inner=INNER)
    bt0 = SolverBatch(512, 1024, 511, 1, precision="mixed", opt=OPTS, inner=INNER)
    bt0.load(0, case.love, case.topo, ice_host[0], case.dt)
    g64 = {f: torch.empty((512, 1024), dtype=torch.float64, device="cuda") for f in ("deltasl", "tgrid", "R")}
    gmx = {f: torch.empty_like(v) for f, v in g64.items()}
    acc = {f: {"max_m": 0.0, "rms_m": 0.0} for f in g64}
    mask_cells, iter_diff = 0, 0
    fcode = {"deltasl": _lib.F_DELTASL, "tgrid": _lib.F_TGRID, "R": _lib.F_R}
    for k in range(1, nsteps + 1):
        inf64 = slv.step_device(ice_dev[k].data_ptr(), 1)
        infmx = bt0.step_ptrs({0: ice_dev[k].data_ptr()}, 1)[0]
        iter_diff += int(inf64.numiter != infmx.numiter)
        for f in g64:
            _lib.check(L.sle_solver_get(slv._h, fcode[f], _lib.C.c_void_p(g64[f].data_ptr()), 1))
            bt0.get(0, f, out=gmx[f])
            d = (g64[f] - gmx[f]).abs()
            acc[f]["max_m"] = max(acc[f]["max_m"], float(d.max()))
            acc[f]["rms_m"] = max(acc[f]["rms_m"], float(torch.sqrt((d * d).mean())))
        o64 = torch.empty_like(g64["tgrid"])
        omx = torch.empty_like(o64)
        _lib.check(L.sle_solver_get(slv._h, _lib.F_OCEAN, _lib.C.c_void_p(o64.data_ptr()), 1))
        bt0.get(0, "ocean", out=omx)
        mask_cells = max(mask_cells, int((o64 != omx).sum()))
    accuracy = {"fields": acc, "steps": nsteps, "ocean_cells_differing_max": mask_cells,
                "steps_with_numiter_differing": iter_diff,
                "note": "rms_m = largest per-step RMS over the grid; the stop rule xi <= 1e-5 can end "
                        "the two runs after different iteration counts when xi is near the bound"}

    # ----------------------------------------- FP64 form: the same member-steps, one solve at a time
    fp_events = []
    slv2 = OptSeaLevelSolver(sht, case.love, case.topo, ice_host[0], norder=511, dt=case.dt,
                             opt=set(OPTS), inner=INNER)
    for k in range(1, W + 1):
        slv2.step_device(ice_dev[k].data_ptr(), 1)
    s2 = torch.cuda.ExternalStream(slv2.stream_handle())
    torch.cuda.synchronize()
    def fp64_step(i):
        torch.cuda.nvtx.range_push("fp64_step")
        slv2.step_device(ice_dev[W + 1 + i].data_ptr(), 1)
        torch.cuda.nvtx.range_pop()

    fp_ms = timed_steps(fp64_step, s2, flush, K, torch)
    fp64_sps = K / (fp_ms / 1000.0)
    del slv, slv2, bt0

    # ---------------------------------------------------- e2e: public API, host ice (pinned)
    # a fresh batch, warmed like the timed one, then the same member-steps as `value` (each
    # member's own ice, steps W + 1 .. W + Ke) from pinned host grids
    bte = new_batch()
    bte.step_host_stream([{b: t.cpu().pin_memory() for b, t in dev_ices[k].items()} for k in range(1, W + 1)])
    Ke = min(K, E2E_STEPS)
    host_steps = [{b: t.cpu().pin_memory() for b, t in dev_ices[W + 1 + i].items()} for i in range(Ke)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    # SolverBatch.step_host_stream: each step's ice upload (pinned host -> device) overlaps the
    # previous step's compute; the K steps are timed as one interval on the batch's stream (no L2
    # flush: every step uploads B x 4 MiB of ice and touches ~5 GB of solver state)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    bte.step_host_stream(host_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    e2e_value = B * Ke * world / (e2e_ms / 1000.0)
    del bte, host_steps

    # ------------------------------------ kernel timing pass (host-driven loop, event pairs)
    btp = new_batch()
    for k in range(1, 3):
        btp.step(dev_ices[k])
    torch.cuda.synchronize()
    L.sle_prof_reset()
    L.sle_prof_enable(1)
    for k in range(3, 3 + nprof):
        btp.step(dev_ices[k])
    torch.cuda.synchronize()
    L.sle_prof_collect()
    L.sle_prof_enable(0)
    del btp
    prof = {}
    prof.update(read_prof(L, _lib, MIXED_CLASSES))

    # ------------------------------ FP64 roofline: kernel timing pass of the single FP64 solve
    fp64_roof = fp64_roofline(L, _lib, sht, case, ice_dev, W, nprof, torch)

    # ------------------------------- uneven ensemble: members sharded over the ranks, max-over-ranks wall
    ensemble = None
    if a.ensemble_members > 0:
        from slevolve_b200.serving import run_ensemble, shard_requests, uneven_ensemble

        mine = shard_requests(uneven_ensemble(a.ensemble_members), rank, world)
        if dist is not None:
            dist.barrier()
        ensemble = run_ensemble(mine, "mixed")
        wall = max_over_ranks(ensemble["wall_s"], dist)
        steps = ensemble["member_steps"]
        if dist is not None:
            t = torch.tensor([float(steps)], device="cuda", dtype=torch.float64)
            dist.all_reduce(t)
            steps = int(t.item())
        ensemble.pop("budget_bytes", None)
        ensemble.update({"member_steps_all_ranks": steps, "wall_s_max_over_ranks": wall,
                         "member_steps_per_s_all_ranks": steps / wall,
                         "sample": (f"{a.ensemble_members} seeded members, L uniform in {{127, 255, 511}}, 50-1200 "
                                    "steps, relaxation scale log-uniform [0.3, 3], ice c0 caps / c2 sawtooth x "
                                    "U[0.5, 1.5], all at t = 0, sharded over the ranks by estimated work; slots "
                                    "per degree autotuned over {8, 16, 32}; per-rank figures are rank 0's")})

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    # ----------------------------------------------------------------------------- roofline
    nh, ncoef = 256, 512 * 513 // 2
    peaks, psrc = load_peaks()
    # Legendre analysis launches: class 5 (rO, every field active) and class 1 (gated ones)
    ana_ms = prof["k_leg_tc<analysis of rO>"]["ms"] + prof["k_leg_tc<other analyses>"]["ms"]
    shares = {k: v["ms"] for k, v in prof.items()}
    shares["k_leg_tc<analysis>"] = ana_ms
    dominant = max((k for k in shares if k not in ("k_leg_tc<analysis of rO>", "k_leg_tc<other analyses>")),
                   key=lambda k: shares[k])
    if dominant == "k_leg_tc<analysis>":
        dominant = "k_leg_tc<analysis of rO>"   # the launches whose columns are all active
    d = prof[dominant]
    if dominant.startswith("k_leg_tc") or dominant.startswith("k_bsyn"):
        tpk = peaks["bf16_tflops"] * TENSOR_RATE
        flops = 12.0 * nh * ncoef * d["fields"]
        achieved = flops / (d["ms"] / 1000.0) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": tpk, "unit": "TFLOP/s", "frac": achieved / tpk,
                "kernel": dominant, "per_launch_flops": flops / max(d["launches"], 1),
                "avg_launch_us": 1000.0 * d["ms"] / max(d["launches"], 1),
                "peak_source": f"{TENSOR_PEAK}, {psrc}"}
    elif dominant in ELEMENTWISE:
        e = step_shares(prof, nprof, peaks)["elementwise"][dominant]
        roof = {"bound": "hbm", "achieved": e["achieved"], "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": e["frac"], "kernel": dominant, "peak_source": f"copy bandwidth, {psrc}"}
    elif dominant == "k_advance":
        per_launch = (2 * 8 + 3) * 16.0 * ncoef * d["fields"] / max(d["launches"], 1)
        achieved = per_launch * d["launches"] / (d["ms"] / 1000.0) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "kernel": dominant, "peak_source": f"copy bandwidth, {psrc}"}
    else:
        # row FFT + fold: FP64 grid read + FP32 fold write per field
        per_field = 8.0 * ng + 16.0 * 512 * 256
        achieved = per_field * d["fields"] / (d["ms"] / 1000.0) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "kernel": dominant, "peak_source": f"copy bandwidth, {psrc}"}
    roof["traffic"] = traffic_per_launch(dominant)
    roof["kernels"] = {k: {"ms_per_batch_step": v["ms"] / nprof, "launches_per_batch_step": v["launches"] / nprof,
                           "fields_per_batch_step": v["fields"] / nprof} for k, v in prof.items()}
    roof["step_shares"] = step_shares(prof, nprof, peaks)
    ana = prof["k_leg_tc<other analyses>"]
    if ana["ms"] > 0:   # the gated analyses (C*, tO, I* refreshes): columns partly masked off
        tpk = peaks["bf16_tflops"] * TENSOR_RATE
        ach = 12.0 * nh * ncoef * ana["fields"] / (ana["ms"] / 1000.0) / 1e12
        roof["gated_analyses"] = {"achieved": ach, "peak": tpk, "frac": ach / tpk,
                                  "avg_launch_us": 1000.0 * ana["ms"] / max(ana["launches"], 1),
                                  "fields_counted": "every column of a launch, gated or not"}

    latency = None
    if a.serve_requests > 0:
        latency = {"mixed": serving_sample(a.serve_requests, "mixed"),
                   "fp64": serving_sample(a.serve_requests, "fp64")}

    cpu = None
    if not a.no_cpu_baseline:
        workers = os.cpu_count() or 1
        r = cpu_oracle_run(case, 2, a.cpu_steps, workers)
        cpu = {"value": r["steps_per_s"], "unit": "member-steps/s", "cores": workers, "kind": "port",
               "sample": f"{a.cpu_steps} timed FP64 steps (after 2 warm-up steps) of the c2 run, "
                         f"oracle numiter/step {r['numiter_per_step']:.2f}"}

    line = {"metric": METRIC, "value": value, "unit": "member-steps/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": t_max / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "tf32x3+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [512, 1024], "lmax": 511, "modes": 8,
                       "dt_years": 200.0, "precision": "mixed (split-TF32 Legendre contractions with FP32 accumulation, FP64 elsewhere)",
                       "batch_members": B, "first_step": k0, "opt": list(OPTS), "inner": INNER,
                       "max_numiter_per_batch_step": float(np.mean(numiter)),
                       "l2": ("value: flushed between steps (256 MiB write, outside the timed intervals); "
                              "e2e: not flushed, each step uploads B x 4 MiB of ice (more than L2) and "
                              "touches ~5 GB of solver state"),
                       "parallelism": f"members sharded x{world}"},
            "fp64": {"value": fp64_sps, "unit": "steps/s", "workload": WORKLOAD_FP64,
                     "ms_per_step": fp_ms / K, "speedup_mixed_batched": value / world / fp64_sps,
                     "roofline": fp64_roof},
            "accuracy": accuracy, "latency": latency, "ensemble": ensemble,
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "member-steps/s", "h2d_bytes_per_step": B * ng * 8,
                    "d2h_bytes_per_step": B * STEP_RECORD_BYTES, "steps": Ke, "ms_per_step": e2e_ms / Ke},
            "gpu_launches": launches, "clocks": clocks}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_init_topo(a):
    """The outer driver's segmented T0 guess on the seeded glacial-cycle case at 512 x 1024,
    L = 511 (13 ice states, 10-kyr steps): GPU wall time of one guess (after a short warm-up
    guess), and the CPU oracle (NumPy restatement) on the same inputs beside it."""
    import torch

    from slevolve_b200 import make_sht
    from slevolve_b200.init_topo import segmented_guess
    from slevolve_b200.synthetic import case_glacial

    L = 511
    topo, ice, love = case_glacial(make_sht("cuda", 512, 1024, L))
    segmented_guess(topo, ice[:4], love, L, 10.0, maxit=2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    T0, info = segmented_guess(topo, ice, love, L, 10.0)
    torch.cuda.synchronize()
    gpu_s = time.perf_counter() - t0
    line = {"metric": "segmented initial-topography guess, wall time", "value": gpu_s, "unit": "s",
            "higher_is_better": False, "n_gpus": 1, "data": "synthetic", "dtype": "f64",
            "config": {"workload": "segmented T0 guess of the outer driver: 512x1024, L=511, 13 ice states "
                                   "(two glacial cycles, three caps), 10-kyr steps, threshold 0.01, tol 1e-3 m"},
            "iters": info["iters"], "legs": [[s_["a"], s_["b"]] for s_ in info["segments"]], "c_m": info["c"],
            "cpu_baseline": None}
    if not a.no_cpu_baseline:
        from oracle.init_topo import segmented_guess as oracle_guess

        t0 = time.perf_counter()
        T0c, infoc = oracle_guess(topo, ice, love, L, 10.0)
        cpu_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": cpu_s, "unit": "s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": "the whole guess on the same inputs (NumPy oracle, threaded FFT/BLAS)"}
        line["speedup_vs_cpu"] = cpu_s / gpu_s
        line["max_diff_vs_cpu_m"] = float(np.abs(T0 - T0c).max())
        line["iters_cpu"] = infoc["iters"]
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.init_topo:
        return run_init_topo(a)
    if a.serve_load:
        return serve_load(a)
    if a.kernel_case:
        return run_kernel_case(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
