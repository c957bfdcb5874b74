"""Batches of solves (sle_batch_*): every slot's result is the one it gets alone.

FP64 slots are compared bit for bit with the single-solve path (the FP64 parity of which the
other GPU tests establish against the reference); mixed-precision slots bit for bit with the same
member alone in a one-slot mixed batch, and against the FP64 run within the mixed form's 1 mm
bar.  Members differ in Earth model (relaxation times scaled), ice amplitude and step length, as
the uneven ensembles do.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, L = 64, 63
OPT = {"dsl", "diag"}
FIELDS = ("deltasl", "tgrid", "R", "ocean", "beta")


def _members():
    from slevolve_b200 import SyntheticEarth, make_sht
    from slevolve_b200.synthetic import case_c0

    sht = make_sht("cuda", N, 2 * N, L)
    base = case_c0(sht, nsteps=40)
    out = []
    for i, (relax, amp, dt) in enumerate(((1.0, 1.0, 1.0), (0.4, 1.3, 2.0), (2.5, 0.6, 1.0), (1.0, 0.9, 1.5))):
        love = SyntheticEarth(L, 8, 20261203 + 3 + i, relax_scale=relax)
        out.append({"love": love, "topo": base.topo, "dt": dt,
                    "ice": (lambda k, a=amp: np.round(a * base.ice(k), 3))})
    return out


def _alone_fp64(m, nsteps):
    from slevolve_b200 import OptSeaLevelSolver

    s = OptSeaLevelSolver(None, m["love"], m["topo"], m["ice"](0), norder=L, dt=m["dt"], opt=OPT, inner="extrap")
    res = []
    for k in range(1, nsteps + 1):
        r = s.step(m["ice"](k))
        res.append({f: np.array(r[f]) for f in FIELDS} | {"numiter": r["numiter"]})
    return res


def _batch(precision, nslots):
    from slevolve_b200.batch import SolverBatch

    return SolverBatch(N, 2 * N, L, nslots, precision=precision, opt=OPT, inner="extrap")


def _snap(batch, slot, info):
    return {f: batch.get(slot, f).copy() for f in FIELDS} | {"numiter": info["numiter"]}


def _same(a, b, where):
    assert a["numiter"] == b["numiter"], (where, a["numiter"], b["numiter"])
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), (where, f, np.abs(a[f] - b[f]).max())


def test_fp64_batch_slots_match_single_solves():
    ms = _members()[:3]
    nsteps = 6
    alone = [_alone_fp64(m, nsteps) for m in ms]
    bt = _batch("fp64", 4)
    slots = [2, 0, 3]           # out of order, slot 1 left empty
    for m, s in zip(ms, slots):
        bt.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
    for k in range(1, nsteps + 1):
        infos = bt.step({s: m["ice"](k) for m, s in zip(ms, slots)})
        for i, (m, s) in enumerate(zip(ms, slots)):
            _same(_snap(bt, s, infos[s]), alone[i][k - 1], (i, k))


def test_programmatic_launches_do_not_change_results():
    """A mixed batch of four uneven members stepped with the inner loop's kernels launched as
    programmatic dependents and as plain launches (each mode in its own batch, whose loop graph is
    captured with it): bit-identical results."""
    from slevolve_b200 import _lib

    ms = _members()
    nsteps = 4
    runs = []
    prev = _lib.set_programmatic_launch(True)
    try:
        for mode in (True, False):
            _lib.set_programmatic_launch(mode)
            bt = _batch("mixed", len(ms))
            for s, m in enumerate(ms):
                bt.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
            res = []
            for k in range(1, nsteps + 1):
                infos = bt.step({s: m["ice"](k) for s, m in enumerate(ms)})
                res.append([_snap(bt, s, infos[s]) for s in range(len(ms))])
            runs.append(res)
            del bt
    finally:
        _lib.set_programmatic_launch(prev)
    for k in range(nsteps):
        for s in range(len(ms)):
            _same(runs[0][k][s], runs[1][k][s], (k + 1, s))


def test_continuous_batching_join_leave():
    """Slots join and leave between steps; each member still gets its solo result."""
    ms = _members()
    nsteps = 5
    alone = [_alone_fp64(m, nsteps) for m in ms]
    bt = _batch("fp64", 2)
    # schedule: member 0 at t=0 (slot 0), member 1 at t=2 (slot 1), member 2 takes slot 0 when
    # member 0 finishes, member 3 takes slot 1 when member 1 finishes
    queue = [(0, 0), (2, 1)]
    running = {}   # slot -> (member, steps done)
    nxt = 2
    t = 0
    done = set()
    while len(done) < len(ms):
        for start, mi in list(queue):
            if start <= t:
                free = [s for s in range(2) if s not in running]
                if free:
                    s = free[0]
                    m = ms[mi]
                    bt.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
                    running[s] = [mi, 0]
                    queue.remove((start, mi))
        if running:
            ices = {s: ms[mi]["ice"](k + 1) for s, (mi, k) in running.items()}
            infos = bt.step(ices)
            for s in list(running):
                mi, k = running[s]
                _same(_snap(bt, s, infos[s]), alone[mi][k], (mi, k + 1))
                running[s][1] = k + 1
                if k + 1 == nsteps:
                    bt.release(s)
                    del running[s]
                    done.add(mi)
                    if nxt < len(ms):
                        queue.append((t + 1, nxt))
                        nxt += 1
        t += 1
        assert t < 100


def test_mixed_slot_alone_equals_in_mix():
    ms = _members()
    nsteps = 5
    solo = []
    for m in ms:
        bt = _batch("mixed", 1)
        bt.load(0, m["love"], m["topo"], m["ice"](0), m["dt"])
        res = []
        for k in range(1, nsteps + 1):
            info = bt.step({0: m["ice"](k)})[0]
            res.append(_snap(bt, 0, info))
        solo.append(res)
    bt = _batch("mixed", 6)
    slots = [5, 1, 3, 0]
    for m, s in zip(ms, slots):
        bt.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
    for k in range(1, nsteps + 1):
        infos = bt.step({s: m["ice"](k) for m, s in zip(ms, slots)})
        for i, s in enumerate(slots):
            _same(_snap(bt, s, infos[s]), solo[i][k - 1], (i, k))


def test_host_stream_equals_step_by_step():
    """step_host_stream (uploads overlapping the previous step's compute, begin / end halves of
    the C step) gives bit for bit the results of one ``step`` call per step; slot calls are
    refused while a step is in flight."""
    import torch

    ms = _members()[:3]
    nsteps = 4
    host = [{s: torch.from_numpy(np.ascontiguousarray(m["ice"](k))).pin_memory() for s, m in enumerate(ms)}
            for k in range(1, nsteps + 1)]
    a = _batch("mixed", 3)
    b = _batch("mixed", 3)
    for s, m in enumerate(ms):
        a.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
        b.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
    ref = []
    for k in range(nsteps):
        infos = a.step({s: host[k][s].numpy() for s in range(3)})
        ref.append((infos, {s: {f: a.get(s, f).copy() for f in FIELDS} for s in range(3)}))
    recs = b.step_host_stream(host[:-1])
    infos = b.step_host_stream(host[-1:])
    recs += infos
    for s in range(3):
        assert recs[-1][s].numiter == ref[-1][0][s]["numiter"]
        for f in FIELDS:
            assert np.array_equal(b.get(s, f), ref[-1][1][s][f]), (s, f)
    assert [[r[s].numiter for s in range(3)] for r in recs] == [[x[0][s]["numiter"] for s in range(3)]
                                                               for x in ref]
    ptr = torch.zeros((N, 2 * N), dtype=torch.float64, device="cuda")
    b.step_begin({0: ptr.data_ptr()}, 1)
    with pytest.raises(RuntimeError, match="in flight"):
        b.release(0)
    b.step_end()


def test_mixed_batch_within_1mm_of_fp64():
    """Mixed-precision slots against the FP64 solve of the same member (the 1 mm bar)."""
    ms = _members()[:2]
    nsteps = 20
    bt = _batch("mixed", 2)
    for s, m in enumerate(ms):
        bt.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
    alone = [_alone_fp64(m, nsteps) for m in ms]
    worst = 0.0
    for k in range(1, nsteps + 1):
        infos = bt.step({s: m["ice"](k) for s, m in enumerate(ms)})
        for s in range(2):
            for f in ("deltasl", "tgrid", "R"):
                d = np.abs(bt.get(s, f) - alone[s][k - 1][f]).max()
                worst = max(worst, d)
    assert worst < 1e-3, worst


def test_full_width_batch_within_1mm_of_fp64():
    """32 mixed slots: every analysis of the inner loop carries 32 fields (64 B-operand columns),
    the width at which the hi*hi and hi*lo products run as one MMA of 128 columns.  Each slot
    stays within the mixed form's 1 mm bar of its FP64 solve."""
    from slevolve_b200 import SyntheticEarth, make_sht
    from slevolve_b200.synthetic import case_c0

    sht = make_sht("cuda", N, 2 * N, L)
    base = case_c0(sht, nsteps=40)
    nslot, nsteps = 32, 6
    ms = []
    for s in range(nslot):
        love = SyntheticEarth(L, 8, 20261203 + 40 + s, relax_scale=0.5 + 0.05 * s)
        ms.append({"love": love, "topo": base.topo, "dt": 1.0 + 0.02 * s,
                   "ice": (lambda k, a=0.6 + 0.03 * s: np.round(a * base.ice(k), 3))})
    bt = _batch("mixed", nslot)
    for s, m in enumerate(ms):
        bt.load(s, m["love"], m["topo"], m["ice"](0), m["dt"])
    alone = [_alone_fp64(m, nsteps) for m in ms]
    worst = 0.0
    for k in range(1, nsteps + 1):
        infos = bt.step({s: m["ice"](k) for s, m in enumerate(ms)})
        for s in range(nslot):
            for f in ("deltasl", "tgrid", "R"):
                worst = max(worst, float(np.abs(bt.get(s, f) - alone[s][k - 1][f]).max()))
    assert worst < 1e-3, worst
