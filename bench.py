#!/usr/bin/env python3
"""Throughput of the SLEvolve sea-level time step on B200: steps/s at L = 511 (512 x 1024 grid).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the c2 benchmark shape (512 x 1024 Gauss grid, L = 511, 8 viscous modes per degree,
200-yr steps, three northern-hemisphere ice sheets on a 100-kyr sawtooth, shoreline migration,
grounded-ice test and rotational feedback on), FP64, with the reference's fastest exact options
(``opt={"dsl", "diag"}``, ``inner="extrap"``).  A step is one full ``step()`` of the solver,
inner fixed-point loop included.

* ``value``  steps/s with the ice history already resident in HBM (device pointers), timed with
  CUDA events on the solver's stream, L2 flushed (256 MiB write) between steps outside the timed
  intervals, W untimed warm-up steps first.
* ``e2e``    the same steps through the public API ``SeaLevelSolver.step(numpy ice)`` from pinned
  host memory, with the step's topography grid read back to the host, copies inside the timing.
* ``roofline`` the dominant kernel (by device time): a second pass over the same steps records a
  CUDA-event pair around every launch of each transform / modal-state kernel inside the library
  (the timed pass runs the inner loop as a CUDA graph, where per-node events are not available);
  algorithmic FLOPs 4 nh ncoef per transformed field over the kernel's measured time, against the
  FP64 FMA throughput measured on the same GPU; ``traffic`` from the committed ncu summary.
* ``cpu_baseline`` the CPU oracle (NumPy restatement of the reference solver) on this host's cores,
  5 timed steps of the same run.

With N > 1 (torchrun) every rank runs an independent replica on its own GPU (one solve per GPU,
no collective on the data path); ``value`` is the sum of steps over the max-over-ranks time.
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
WORKLOAD = ("c2-shape FP64 forward step: 512x1024 Gauss grid, L=511, 8 modes/degree, 200-yr steps, "
            "3 NH ice sheets on a 100-kyr sawtooth, opt dsl+diag, inner extrap")
OPTS = ("dsl", "diag")
INNER = "extrap"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--cpu-steps", type=int, default=5, help="timed oracle steps for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
            try:
                bus = torch.cuda.get_device_properties(torch.cuda.current_device()).pci_bus_id
                h = nvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
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
    line = {"impl": "reference", "metric": METRIC, "value": r["steps_per_s"], "unit": "steps/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1000.0 / r["steps_per_s"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [512, 1024], "lmax": 511, "modes": 8,
                       "precision": "fp64", "numiter_per_step": r["numiter_per_step"],
                       "solver": "CPU oracle (NumPy restatement of the reference SeaLevelSolver)"},
            "cpu_baseline": {"value": r["steps_per_s"], "unit": "steps/s", "cores": workers,
                             "kind": "port", "sample": sample},
            "e2e": {"value": r["steps_per_s"], "unit": "steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def traffic_per_launch(kernel):
    path = os.path.join(HERE, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh).get(kernel)
    except Exception:
        return None


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

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from slevolve_b200 import OptSeaLevelSolver, _lib, make_sht

    L = _lib.lib()
    sht = make_sht("cuda", 512, 1024, 511)
    case = build_case(lambda: sht)
    nsteps = a.warmup + a.steps
    ices = [np.ascontiguousarray(case.ice(k)) for k in range(nsteps + 1)]
    ng = case.nlat * case.nlon

    def new_solver():
        return OptSeaLevelSolver(sht, case.love, case.topo, ices[0], norder=511, dt=case.dt,
                                 opt=set(OPTS), inner=INNER)

    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")

    # ----------------------------------------------------------- value: device-resident inputs
    # (per-kernel timing off: the inner loop runs as a CUDA graph)
    slv = new_solver()
    stream = torch.cuda.ExternalStream(slv.stream_handle())
    ice_dev = [torch.from_numpy(x).cuda() for x in ices]
    torch.cuda.synchronize()
    for k in range(1, a.warmup + 1):
        slv.step_device(ice_dev[k].data_ptr(), 1)
    numiter = 0
    events = []
    L.sle_prof_reset()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(a.warmup + 1, nsteps + 1):
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            info = slv.step_device(ice_dev[k].data_ptr(), 1)
            with torch.cuda.stream(stream):
                e1.record(stream)
            numiter += info.numiter
            events.append((e0, e1))
        torch.cuda.synchronize()
        launches = int(L.sle_launch_count())
        # kernel timing pass: the same steps again on a fresh solver with a CUDA-event pair
        # around every launch of the transform and modal-state kernels (host-driven loop)
        slvp = new_solver()
        for k in range(1, a.warmup + 1):
            slvp.step_device(ice_dev[k].data_ptr(), 1)
        torch.cuda.synchronize()
        L.sle_prof_reset()
        L.sle_prof_enable(1)
        for k in range(a.warmup + 1, nsteps + 1):
            with torch.cuda.stream(torch.cuda.ExternalStream(slvp.stream_handle())):
                flush.zero_()
            slvp.step_device(ice_dev[k].data_ptr(), 1)
        torch.cuda.synchronize()
        L.sle_prof_collect()
        L.sle_prof_enable(0)
        del slvp
    dev_ms = sum(e0.elapsed_time(e1) for e0, e1 in events)
    prof = {}
    for cls, name in ((_lib.PROF_FFT, "k_fft_fold"), (_lib.PROF_LEG_ANA, "k_leg_ana"),
                      (_lib.PROF_LEG_SYN, "k_leg_syn"), (_lib.PROF_IFFT, "k_ifft_unfold"),
                      (_lib.PROF_ADVANCE, "k_advance")):
        ms, cnt, units = _lib.C.c_double(), _lib.C.c_longlong(), _lib.C.c_double()
        L.sle_prof_read(cls, _lib.C.byref(ms), _lib.C.byref(cnt), _lib.C.byref(units))
        prof[name] = {"ms": ms.value, "launches": cnt.value, "fields": units.value}
    clocks = clk.summary()
    t_max = dev_ms
    if dist is not None:
        t = torch.tensor([dev_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    total_steps = a.steps * world
    value = total_steps / (t_max / 1000.0)

    # ------------------------------------------------------------- e2e: public API, host buffers
    slv2 = new_solver()
    stream2 = torch.cuda.ExternalStream(slv2.stream_handle())
    pinned = [torch.from_numpy(x).pin_memory() for x in ices]
    for k in range(1, a.warmup + 1):
        r = slv2.step(pinned[k].numpy())
        _ = r["tgrid"]
    e2e_events = []
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    for k in range(a.warmup + 1, nsteps + 1):
        with torch.cuda.stream(stream2):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream2)
        r = slv2.step(pinned[k].numpy())
        tg = r["tgrid"]
        with torch.cuda.stream(stream2):
            e1.record(stream2)
        e2e_events.append((e0, e1))
    torch.cuda.synchronize()
    e2e_ms = sum(e0.elapsed_time(e1) for e0, e1 in e2e_events)
    if dist is not None:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = total_steps / (e2e_ms / 1000.0)
    assert np.isfinite(tg).all()

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    # ----------------------------------------------------------------------------- roofline
    nh, ncoef = 256, 512 * 513 // 2
    flops_leg = 4.0 * nh * ncoef                 # per transformed field (algorithmic)
    dominant = max(prof, key=lambda k: prof[k]["ms"])
    per_field_flops = {"k_leg_ana": flops_leg, "k_leg_syn": flops_leg,
                       "k_fft_fold": 2.5 * 1024 * 10 * 512, "k_ifft_unfold": 2.5 * 1024 * 10 * 512}
    peak = _lib.C.c_double()
    L.sle_probe_fp64_tflops(_lib.C.byref(peak))
    d = prof[dominant]
    if dominant == "k_advance":
        # HBM bytes per launch: (2K + 3) x 16 x ncoef; peak = measured copy bandwidth
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as fh:
            hbm = json.load(fh)["hbm_gbs"]
        per_launch = (2 * 8 + 3) * 16.0 * ncoef
        achieved = per_launch * d["launches"] / (d["ms"] / 1000.0) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "kernel": dominant, "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)"}
    else:
        flops = per_field_flops[dominant] * d["fields"]
        achieved = flops / (d["ms"] / 1000.0) / 1e12
        roof = {"bound": "fp64", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                "frac": achieved / peak.value, "kernel": dominant,
                "per_launch_flops": flops / max(d["launches"], 1),
                "avg_launch_us": 1000.0 * d["ms"] / max(d["launches"], 1),
                "peak_source": "FP64 FMA throughput measured on this GPU by sle_probe_fp64_tflops"}
    roof["traffic"] = traffic_per_launch(dominant)
    roof["kernels"] = {k: {"ms_per_step": v["ms"] / a.steps, "launches_per_step": v["launches"] / a.steps}
                       for k, v in prof.items()}

    cpu = None
    if not a.no_cpu_baseline:
        workers = os.cpu_count() or 1
        from oracle.sht import OracleSHT  # noqa: F401  (checker only: the CPU baseline leg)

        r = cpu_oracle_run(case, 2, a.cpu_steps, workers)
        cpu = {"value": r["steps_per_s"], "unit": "steps/s", "cores": workers, "kind": "port",
               "sample": f"{a.cpu_steps} timed steps (after 2 warm-up steps) of the same c2 run, "
                         f"oracle numiter/step {r['numiter_per_step']:.2f}"}

    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": [512, 1024], "lmax": 511, "modes": 8,
                       "dt_years": 200.0, "precision": "fp64", "opt": list(OPTS), "inner": INNER,
                       "numiter_per_step": numiter / a.steps,
                       "l2": "flushed between steps (256 MiB write, outside the timed intervals)",
                       "parallelism": f"replicas x{world}"},
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": ng * 8,
                    "d2h_bytes_per_step": ng * 8},
            "gpu_launches": launches, "clocks": clocks}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
