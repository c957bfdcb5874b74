"""Serving loop: continuous batching of sea-level solves on one GPU.

A request is one forward solve (an Earth model, a truncation degree L, a topography, an ice
history, a step count and a step length) or an ice-age outer-iteration request: several forward
passes over the same ice history, each starting from the initial topography updated by the
reference's Picard rule ``T0 <- T0 - (predicted present topography - observed)``
(SLEvolve python/slevolve/run_outer.py:243-273), warm-started from the previous pass's
converged state (``reuse="warm"``, solver_opt.py:400-403, 514-528, 932-947).

The server keeps one slot batch (``SolverBatch``) per truncation degree.  Each batch has its own
host thread: between two of its batch steps it retires finished solves, admits queued requests
while a slot is free and the device-memory budget holds their footprint (solver state of one
slot plus, for outer requests, the reuse store), and then advances every admitted solve by one
time step in one batched step.  Batches of different degrees run concurrently on their own CUDA
streams, so their kernels overlap on the device.  All solver state stays on the device from
admission to completion; the ice of each step is generated on the device.

A solve's result does not depend on what else is in its batch (per-slot reductions in a fixed
order, per-field tensor-core columns), so a request gives the same answer alone and in the mix.

Requests carry a priority.  With ``preempt=True``, a request that has arrived and finds every slot
of its degree taken by requests of lower priority preempts one of them between two batch steps:
the victim's whole solve state is copied to host memory (``SolverBatch.snapshot``), its slot goes
to the newcomer, and the victim waits in the queue until a slot frees, where it is restored
(``SolverBatch.restore``, possibly into another slot) and continues bit for bit where it stopped.
"""

from __future__ import annotations

import dataclasses
import math
import threading
import time
from typing import Callable, Optional

import numpy as np

from .batch import SolverBatch, slot_bytes
from .reuse import ReuseStore


@dataclasses.dataclass
class Request:
    """One solve.  ``ice(k)`` returns the ice grid of step k (a CUDA float64 tensor or NumPy
    array of the request's grid); ``outer_passes > 1`` makes it an outer-iteration request whose
    observed present topography is ``obs`` (default: ``topo``)."""

    rid: int
    lmax: int
    love: object
    topo: np.ndarray
    ice: Callable[[int], object]
    nsteps: int
    dt: float
    arrival: float = 0.0
    outer_passes: int = 1
    obs: Optional[np.ndarray] = None
    priority: int = 0
    # filled in by the server
    t_admit: float = math.nan
    t_done: float = math.nan
    numiter: int = 0
    passes_done: int = 0
    warm_steps: int = 0
    preemptions: int = 0
    result: dict = dataclasses.field(default_factory=dict)

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def store_bytes(req: Request) -> int:
    """Device bytes of an outer request's reuse store (0 for a forward solve)."""
    if req.outer_passes <= 1:
        return 0
    n = req.lmax + 1
    nc = n * (n + 1) // 2
    return req.nsteps * (16 * nc + n * 2 * n)


def footprint(req: Request, max_modes=8) -> int:
    """Device bytes a request holds while admitted (admission unit): one slot's solver state plus
    the reuse store of an outer request."""
    n = req.lmax + 1
    return slot_bytes(n, 2 * n, req.lmax, max_modes) + store_bytes(req)


class _Running:
    def __init__(self, req, slot):
        self.req = req
        self.slot = slot
        self.k = 0          # steps done in the current pass
        self.store = None   # ReuseStore of an outer request
        self.T0 = None      # current initial topography (device) of an outer request
        self.obs = None
        self.image = None   # host snapshot while preempted


def _room():
    """Free device memory.  Blocks that torch's caching allocator holds unused are not counted:
    they may be too fragmented for a store (the caller empties the cache before giving up)."""
    import torch

    return torch.cuda.mem_get_info()[0]


class Server:
    """groups: {lmax: slots}.  budget_bytes: device memory the admitted requests may hold (their
    slots' solver state plus the reuse stores of outer requests).  The slot batches are allocated
    when the server starts, so the device also holds the state of idle slots: a reuse store is
    allocated only while the device has room for it with ``store_margin`` bytes to spare, and a
    request that does not fit waits in the queue."""

    def __init__(self, groups, precision="mixed", budget_bytes=None, max_modes=8, opt=("dsl", "diag"),
                 inner="extrap", record=("deltasl", "tgrid"), preempt=False, device_bytes=None,
                 store_margin=4 << 30):
        self.precision = precision
        self.store_margin = int(store_margin)
        self.preempt = bool(preempt)
        self.preempted = 0
        # occupancy record: (time, admitted bytes, device bytes in use) at every change, against
        # device_bytes
        self.device_bytes = device_bytes
        self._occ = []
        self.max_modes = max_modes
        self.record = tuple(record)
        self.batches = {int(L): SolverBatch(L + 1, 2 * (L + 1), L, int(n), max_modes=max_modes,
                                            precision=precision, opt=opt, inner=inner)
                        for L, n in groups.items()}
        self.budget = budget_bytes if budget_bytes is not None else float("inf")
        self.used = 0
        self.peak_used = 0
        self.lock = threading.Lock()
        self.queue = {L: [] for L in self.batches}
        self.done = []
        self.steps = {L: 0 for L in self.batches}        # member-steps executed per group
        self.batch_steps = {L: 0 for L in self.batches}  # batched steps per group

    # ---------------------------------------------------------------- helpers
    def _note_used(self):
        """Record the admitted footprint and the device memory in use after a change (caller
        holds the lock)."""
        held = 0
        if self.device_bytes:
            import torch

            free, total = torch.cuda.mem_get_info()
            held = total - free
        self._occ.append((time.perf_counter() - getattr(self, "_t0", time.perf_counter()), self.used, held))

    def occupancy(self):
        """Time-weighted mean and peak of the admitted footprint over the run, in bytes and as a
        fraction of ``device_bytes`` (when given)."""
        ev = sorted(e if len(e) == 3 else (e[0], e[1], 0) for e in self._occ)
        wall = getattr(self, "wall", 0.0)
        if not ev or wall <= 0:
            return {"mean_bytes": 0.0, "peak_bytes": int(self.peak_used)}
        area, held_area, t_prev, u_prev, h_prev = 0.0, 0.0, 0.0, 0, 0
        for t, u, h in ev:
            area += u_prev * max(0.0, t - t_prev)
            held_area += h_prev * max(0.0, t - t_prev)
            t_prev, u_prev, h_prev = t, u, h
        area += u_prev * max(0.0, wall - t_prev)
        held_area += h_prev * max(0.0, wall - t_prev)
        out = {"mean_bytes": area / wall, "peak_bytes": int(self.peak_used)}
        if self.device_bytes:
            out["hbm_occupancy_mean"] = out["mean_bytes"] / self.device_bytes
            out["hbm_occupancy_peak"] = self.peak_used / self.device_bytes
            out["hbm_held_mean"] = held_area / wall / self.device_bytes
            out["hbm_held_peak"] = max(h for _, _, h in ev) / self.device_bytes
        return out

    @staticmethod
    def _next(q, now):
        """The arrived queued request to admit next: highest priority, then earliest arrival."""
        best = None
        for r in q:
            if r.arrival <= now and (best is None or (-r.priority, r.arrival, r.rid) <
                                     (-best.priority, best.arrival, best.rid)):
                best = r
        return best

    def _preempt_for(self, L, bt, running, req):
        """Free a slot for `req` by preempting the lowest-priority running request (the most
        recently admitted among equals) if its priority is below req's; returns the slot or None."""
        victims = [r for r in running.values() if r.req.priority < req.priority]
        if not victims:
            return None
        v = min(victims, key=lambda r: (r.req.priority, -r.req.t_admit))
        v.image = bt.snapshot(v.slot)
        bt.release(v.slot)
        del running[v.slot]
        v.req.preemptions += 1
        self.preempted += 1
        with self.lock:
            self.used -= footprint(v.req, self.max_modes) - store_bytes(v.req)   # the store stays
            self._note_used()
        self.queue[L].append(v.req)
        v.req._run = v
        return v.slot

    def _admit(self, L, running, now):
        bt = self.batches[L]
        free = [s for s in range(bt.nslots) if s not in running]
        q = self.queue[L]
        while q:
            req = self._next(q, now)
            if req is None:
                return
            resumed = getattr(req, "_run", None)
            fp = footprint(req, self.max_modes) - (store_bytes(req) if resumed is not None else 0)
            if not free and self.preempt:
                slot = self._preempt_for(L, bt, running, req)
                if slot is not None:
                    free.append(slot)
            if not free:
                return
            store = None
            with self.lock:
                if self.used + fp > self.budget:
                    return
                if resumed is None and req.outer_passes > 1:
                    # the store is allocated under the lock, once the device has room for it
                    # with store_margin to spare (the other groups' steps allocate their ice grids
                    # meanwhile)
                    import torch

                    need = store_bytes(req) + self.store_margin
                    if _room() < need:
                        torch.cuda.empty_cache()
                        if _room() < need:
                            return
                    n = req.lmax + 1
                    try:
                        store = ReuseStore(n * (n + 1) // 2, n * 2 * n, capacity=req.nsteps)
                    except torch.OutOfMemoryError:
                        # another group's step took the room meanwhile: try again later
                        torch.cuda.empty_cache()
                        return
                self.used += fp
                self.peak_used = max(self.peak_used, self.used)
                self._note_used()
            q.remove(req)
            slot = free.pop(0)
            if resumed is not None:
                # a preempted request: its state comes back from the host image
                run, req._run = resumed, None
                run.slot = slot
                bt.restore(slot, run.image)
                run.image = None
                if run.store is not None:
                    bt.set_reuse(slot, run.store, valid=run.store.recorded)   # as at the pass's load
                running[slot] = run
                continue
            run = _Running(req, slot)
            req.t_admit = time.perf_counter() - self._t0
            if req.outer_passes > 1:
                import torch

                run.store = store
                run.T0 = torch.as_tensor(np.ascontiguousarray(req.topo), dtype=torch.float64, device="cuda")
                obs = req.obs if req.obs is not None else req.topo
                run.obs = torch.as_tensor(np.ascontiguousarray(obs), dtype=torch.float64, device="cuda")
            self._load(bt, run)
            running[slot] = run

    def _load(self, bt, run):
        req = run.req
        topo = run.T0 if run.T0 is not None else req.topo
        bt.load(run.slot, req.love, topo, req.ice(0), req.dt)
        if run.store is not None:
            bt.set_reuse(run.slot, run.store, valid=run.store.recorded)
        run.k = 0

    def _finish_pass(self, L, bt, run, running):
        """End of a forward pass: next pass (outer request) or completion."""
        req = run.req
        req.passes_done += 1
        if run.store is not None:
            run.store.recorded = max(run.store.recorded, run.k)
        if req.passes_done < req.outer_passes:
            import torch

            pred = torch.empty_like(run.T0)
            bt.get(run.slot, "tgrid", out=pred)
            run.T0 = run.T0 - (pred - run.obs)   # Picard update of the initial topography
            self._load(bt, run)
            return
        for f in self.record:
            req.result[f] = bt.get(run.slot, f).copy()
        if run.T0 is not None:
            req.result["T0"] = run.T0.cpu().numpy()
        req.t_done = time.perf_counter() - self._t0
        bt.release(run.slot)
        del running[run.slot]
        with self.lock:
            self.used -= footprint(req, self.max_modes)
            self._note_used()
            self.done.append(req)

    def _group_loop(self, L):
        bt = self.batches[L]
        running = {}
        while True:
            now = time.perf_counter() - self._t0
            self._admit(L, running, now)
            if not running:
                q = self.queue[L]
                if not q:
                    return
                time.sleep(min(0.002, max(0.0, q[0].arrival - now)))
                continue
            ices = {s: r.req.ice(r.k + 1) for s, r in running.items()}
            infos = bt.step(ices)
            self.batch_steps[L] += 1
            self.steps[L] += len(ices)
            for s, info in infos.items():
                r = running[s]
                r.k += 1
                r.req.numiter += info["numiter"]
                if r.store is not None and r.req.passes_done > 0 and r.k <= r.store.recorded:
                    r.req.warm_steps += 1
            for s in list(running):
                r = running[s]
                if r.k >= r.req.nsteps:
                    self._finish_pass(L, bt, r, running)

    # -------------------------------------------------------------------- API
    def run(self, requests):
        """Serve `requests` (arrival times in seconds from now); returns them with their
        admission / completion times, iteration counts and recorded results."""
        for r in sorted(requests, key=lambda r: (r.arrival, r.rid)):
            if r.lmax not in self.batches:
                raise ValueError(f"no slot batch for lmax {r.lmax}")
            self.queue[r.lmax].append(r)
        self._t0 = time.perf_counter()
        threads = [threading.Thread(target=self._group_loop, args=(L,), daemon=True) for L in self.batches]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        self.wall = time.perf_counter() - self._t0
        return requests

    def stats(self, requests):
        lat = np.array([r.latency for r in requests])
        wait = np.array([r.t_admit - r.arrival for r in requests])
        steps = sum(self.steps.values())
        out = {"requests": len(requests), "wall_s": self.wall, "member_steps": steps,
               "member_steps_per_s": steps / self.wall,
               "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
               "admission_wait_p50_s": float(np.percentile(wait, 50)),
               "admission_wait_p99_s": float(np.percentile(wait, 99)),
               "peak_bytes": int(self.peak_used), "budget_bytes": self.budget,
               "batch_steps": dict(self.batch_steps), "preemptions": self.preempted}
        out.update({k: v for k, v in self.occupancy().items() if k != "peak_bytes"})
        return out


# ------------------------------------------------------------- synthetic members
class MemberFactory:
    """Seeded members of the uneven ensembles: L, Earth model (relaxation times scaled by a
    factor log-uniform in [0.3, 3]), topography from the seeded generator of the grid, ice from
    the two-cap melt history or the three-sheet 100-kyr sawtooth scaled by U[0.5, 1.5]."""

    def __init__(self, seed=20261206):
        self.rng = np.random.default_rng(seed)
        self._grid = {}

    def grid(self, L):
        if L not in self._grid:
            import torch

            from . import make_sht
            from .synthetic import (SHEETS_C2, angular_distance, grid_latlon, random_topography,
                                    vialov)

            n = L + 1
            sht = make_sht("cuda", n, 2 * n, L)
            topo = random_topography(sht, 20261203 + L)
            LAT, LON = grid_latlon(sht.gaulats, 2 * n)
            cap = (vialov(angular_distance(LAT, LON, -90.0, 0.0), 15.0)
                   + vialov(angular_distance(LAT, LON, 56.0, 132.0), 15.0)) * (topo > -500.0)
            nh = np.zeros_like(topo)
            for la, lo, R in SHEETS_C2:
                nh = np.maximum(nh, vialov(angular_distance(LAT, LON, la, lo), R))
            self._grid[L] = (topo, torch.as_tensor(cap, device="cuda"), torch.as_tensor(nh, device="cuda"))
        return self._grid[L]

    def make(self, rid, L, nsteps, arrival=0.0, outer_passes=1, kind=None):
        import torch

        from .love import SyntheticEarth
        from .synthetic import sawtooth

        topo, cap, nh = self.grid(L)
        f = float(np.exp(self.rng.uniform(np.log(0.3), np.log(3.0))))
        amp = float(self.rng.uniform(0.5, 1.5))
        kind = kind or ("melt" if self.rng.uniform() < 0.5 else "sawtooth")
        love = SyntheticEarth(L, 8, 20261203 + rid, relax_scale=f)
        if kind == "melt":
            dt = 1.0

            def ice(k, amp=amp, n=nsteps, shape=cap):
                return torch.round(amp * (3000.0 * (1.0 - k / n)) * shape * 1000.0) / 1000.0
        else:
            dt = 200.0

            def ice(k, amp=amp, shape=nh):
                return torch.round(amp * (3500.0 * float(sawtooth(k * 200.0 / 1000.0))) * shape * 1000.0) / 1000.0
        return Request(rid=rid, lmax=L, love=love, topo=topo, ice=ice, nsteps=nsteps, dt=dt, arrival=arrival,
                       outer_passes=outer_passes)


# ---------------------------------------------------------------- ensembles
def autotune_slots(lmax, candidates=(8, 16, 32), precision="mixed", probe_steps=2, seed=20261209):
    """Slot count of the highest member-steps/s for degree ``lmax``: each candidate batch is
    loaded with seeded members (sawtooth ice), stepped once untimed (plan tables, graph capture),
    then ``probe_steps`` times under CUDA events.  Returns (best, {candidate: member-steps/s})."""
    import torch

    mf = MemberFactory(seed)
    rates = {}
    for n in candidates:
        reqs = [mf.make(i, lmax, probe_steps + 1, kind="sawtooth") for i in range(n)]
        bt = SolverBatch(lmax + 1, 2 * (lmax + 1), lmax, n, precision=precision)
        for s, r in enumerate(reqs):
            bt.load(s, r.love, r.topo, r.ice(0), r.dt)
        bt.step({s: r.ice(1) for s, r in enumerate(reqs)})
        ices = [{s: r.ice(k) for s, r in enumerate(reqs)} for k in range(2, probe_steps + 2)]
        st = torch.cuda.ExternalStream(bt.stream_handle())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        for ice in ices:
            bt.step(ice)
        e1.record(st)
        torch.cuda.synchronize()
        rates[n] = n * probe_steps / (e0.elapsed_time(e1) / 1000.0)
        del bt
    return max(rates, key=rates.get), rates


def uneven_ensemble(n=64, degrees=(127, 255, 511), steps=(50, 1200), seed=20261210):
    """The uneven ensemble of seeded members: degree uniform over ``degrees``, step count uniform
    in ``steps``, Earth relaxation scale log-uniform in [0.3, 3], ice from the melting caps or the
    sawtooth sheets scaled by U[0.5, 1.5]; every member arrives at time 0."""
    rng = np.random.default_rng(seed)
    mf = MemberFactory(seed)
    Ls = rng.choice(list(degrees), size=n)
    ks = rng.integers(steps[0], steps[1] + 1, size=n)
    return [mf.make(i, int(L), int(k)) for i, (L, k) in enumerate(zip(Ls, ks))]


def run_ensemble(requests, precision="mixed", slots=None, autotune=True, candidates=(8, 16, 32),
                 tune_shapes=True):
    """Run a set of requests to completion with one slot batch per degree (continuous batching:
    a member that finishes frees its slot for the next one of its degree).  ``slots``: {lmax:
    slot count}; missing degrees are autotuned (or get min(32, members)).  With ``tune_shapes``,
    each mixed-precision batch also times the transforms' launch shapes for its slot count and
    uses the fastest (``SolverBatch.autotune``) before the run.  Returns the server statistics
    plus the slot choice, the launch shapes and the autotune measurements."""
    degrees = sorted({r.lmax for r in requests})
    slots = dict(slots or {})
    tuned = {}
    for L in degrees:
        if L in slots:
            continue
        count = sum(1 for r in requests if r.lmax == L)
        if autotune:
            cand = tuple(c for c in candidates if c <= max(count, min(candidates)))
            best, rates = autotune_slots(L, cand, precision)
            tuned[str(L)] = {str(k): v for k, v in rates.items()}
            slots[L] = best
        else:
            slots[L] = min(32, count)
    srv = Server(slots, precision=precision)
    shapes = {}
    if tune_shapes and precision == "mixed":
        for L, bt in srv.batches.items():
            shapes[str(L)] = bt.autotune()[0]
    srv.run(requests)
    st = srv.stats(requests)
    st.update({"slots": {str(k): v for k, v in slots.items()}, "launch_shapes": shapes,
               "autotune_member_steps_per_s": tuned,
               "members": {str(L): sum(1 for r in requests if r.lmax == L) for L in degrees}})
    return st


# ------------------------------------------------------------ several GPUs
def request_cost(r):
    """Estimated work of a request: (lmax + 1)^3 per step (the transforms' contraction) x steps x
    passes."""
    return (r.lmax + 1) ** 3 * r.nsteps * max(1, getattr(r, "outer_passes", 1))


def shard_requests(requests, rank, world):
    """The requests rank ``rank`` of ``world`` GPUs runs: sorted by estimated work (most first,
    ties by id) and dealt round robin, so that the shards are disjoint, cover every request and
    carry similar work.  Independent members: no data moves between ranks."""
    order = sorted(requests, key=lambda r: (-request_cost(r), r.rid))
    return [r for i, r in enumerate(order) if i % world == rank]


def max_over_ranks(x, dist=None, device="cuda"):
    """max of ``x`` over the ranks of the default process group (``x`` itself without one)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
