"""The serving loop's host logic without a GPU: the queue order, admission against the HBM budget
and the free slots, preemption (snapshot, release, re-admission from the host image) and the
admitted-footprint accounting, with a stand-in for the slot batch that records what the server
asks of it; the launch-shape candidates the tuner times."""

import threading

import numpy as np

from slevolve_b200.batch import slot_bytes
from slevolve_b200.serving import Request, Server, footprint, store_bytes

L = 63


class FakeBatch:
    """The slot-batch calls the admission path makes, recorded in order."""

    def __init__(self, nslots):
        self.nslots = nslots
        self.loaded = {}
        self.log = []

    def load(self, slot, love, topo, ice0, dt):
        assert slot not in self.loaded, slot
        self.loaded[slot] = ice0
        self.log.append(("load", slot, ice0))

    def snapshot(self, slot):
        self.log.append(("snapshot", slot))
        return ("image", self.loaded[slot])

    def release(self, slot):
        self.log.append(("release", slot))
        del self.loaded[slot]

    def restore(self, slot, image):
        assert slot not in self.loaded, slot
        self.log.append(("restore", slot, image[1]))
        self.loaded[slot] = image[1]

    def set_reuse(self, *args, **kwargs):
        self.log.append(("set_reuse",))


def _server(nslots, budget=float("inf"), preempt=False):
    srv = object.__new__(Server)
    srv.precision = "mixed"
    srv.store_margin = 0
    srv.preempt = preempt
    srv.preempted = 0
    srv.device_bytes = None
    srv._occ = []
    srv.max_modes = 8
    srv.record = ()
    srv.batches = {L: FakeBatch(nslots)}
    srv.budget = budget
    srv.used = 0
    srv.peak_used = 0
    srv.lock = threading.Lock()
    srv.queue = {L: []}
    srv.done = []
    srv.steps = {L: 0}
    srv.batch_steps = {L: 0}
    srv._t0 = 0.0
    return srv


def _req(rid, arrival=0.0, priority=0, outer_passes=1):
    return Request(rid=rid, lmax=L, love=None, topo=np.zeros((L + 1, 2 * (L + 1))), ice=lambda k, r=rid: r,
                   nsteps=10, dt=1.0, arrival=arrival, priority=priority, outer_passes=outer_passes)


def test_footprint_arithmetic():
    fwd, outer = _req(0), _req(1, outer_passes=3)
    n = L + 1
    nc = n * (n + 1) // 2
    assert store_bytes(fwd) == 0
    assert store_bytes(outer) == 10 * (16 * nc + n * 2 * n)
    assert footprint(fwd) == slot_bytes(n, 2 * n, L, 8)
    assert footprint(outer) == footprint(fwd) + store_bytes(outer)


def test_queue_order():
    q = [_req(0, arrival=0.0), _req(1, arrival=0.5, priority=1), _req(2, arrival=2.0, priority=5),
         _req(3, arrival=0.4, priority=1)]
    assert Server._next(q, 0.2).rid == 0                 # only request 0 has arrived
    assert Server._next(q, 1.0).rid == 3                 # highest priority, then earliest arrival
    assert Server._next(q, 3.0).rid == 2
    assert Server._next(q[1:2], 0.1) is None             # nothing arrived yet


def test_admission_budget_and_slots():
    fp = footprint(_req(0))
    srv = _server(nslots=3, budget=2 * fp + fp // 2)
    reqs = [_req(i, arrival=0.1 * i) for i in range(4)]
    srv.queue[L].extend(reqs)
    running = {}
    srv._admit(L, running, now=1.0)
    # the budget admits two of the four, in arrival order, into the first free slots
    assert sorted(r.req.rid for r in running.values()) == [0, 1]
    assert srv.used == 2 * fp and srv.peak_used == 2 * fp
    assert [r.rid for r in srv.queue[L]] == [2, 3]
    assert srv.batches[L].log == [("load", 0, 0), ("load", 1, 1)]
    # a request that finishes gives its footprint and its slot back; the next one is admitted
    srv._finish_pass(L, srv.batches[L], running[0], running)
    assert srv.used == fp and [r.rid for r in srv.done] == [0]
    srv._admit(L, running, now=1.0)
    assert sorted(r.req.rid for r in running.values()) == [1, 2] and running[0].req.rid == 2
    assert srv.used == 2 * fp
    # without a budget the slots are the limit
    srv2 = _server(nslots=2)
    srv2.queue[L].extend(_req(i) for i in range(3))
    running2 = {}
    srv2._admit(L, running2, now=0.0)
    assert len(running2) == 2 and len(srv2.queue[L]) == 1


def test_preemption_and_resume():
    srv = _server(nslots=1, preempt=True)
    low, high = _req(0, priority=0), _req(1, arrival=0.5, priority=2)
    running = {}
    srv.queue[L].append(low)
    srv._admit(L, running, now=0.0)
    assert running[0].req is low
    # a higher-priority arrival takes the slot: the running request is snapshotted, released and
    # queued again with its host image
    srv.queue[L].append(high)
    srv._admit(L, running, now=1.0)
    bt = srv.batches[L]
    assert running[0].req is high
    assert bt.log == [("load", 0, 0), ("snapshot", 0), ("release", 0), ("load", 0, 1)]
    assert low.preemptions == 1 and srv.preempted == 1
    assert srv.queue[L] == [low] and low._run.image == ("image", 0)
    assert srv.used == footprint(high)
    # an equal or lower priority does not preempt
    srv.queue[L].append(_req(2, priority=2))
    srv._admit(L, running, now=1.0)
    assert running[0].req is high and len(srv.queue[L]) == 2
    srv.queue[L].pop()
    # when the slot frees, the preempted request comes back from its image, not from a fresh load
    srv._finish_pass(L, bt, running[0], running)
    srv._admit(L, running, now=2.0)
    assert running[0].req is low and bt.log[-1] == ("restore", 0, 0)
    assert low._run is None and running[0].image is None
    assert srv.used == footprint(low)


def test_tuning_candidates():
    from slevolve_b200 import tuning

    c32 = tuning.candidates(32)
    assert len(c32) == 8 and tuning.DEFAULT in c32
    assert {c["fields_per_launch"] for c in c32} == {16, 32}
    assert all(c["stages"] in tuning.STAGES and c["fold_rows"] in tuning.FOLD_ROWS for c in c32)
    # launches wider than the list are the list's own width
    assert {c["fields_per_launch"] for c in tuning.candidates(20)} == {16, 20}
    c8 = tuning.candidates(8)
    assert {c["fields_per_launch"] for c in c8} == {8} and len(c8) == 4
    assert {c["fields_per_launch"] for c in tuning.candidates(0)} == {1}
