"""The serving loop: continuous batching with admission by device-memory footprint.

Every request's result (sea-level change and topography after its last step, and the updated
initial topography of an outer-iteration request) must be the same when it is served alone and
when it shares its slot batch with others that arrive and leave around it: bit-identical, the
per-slot arithmetic not depending on the batch.  The tolerance stated for the mixed form against
FP64 (1 mm) is tested elsewhere; here the bar is identity."""

import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from slevolve_b200.serving import MemberFactory

    mf = MemberFactory(seed=11)
    # all arrive at once: the L=63 group has 2 slots for 4 requests, so requests join as others
    # leave (continuous batching) and share batched steps
    reqs = [mf.make(0, 63, 9),
            mf.make(1, 127, 7),
            mf.make(2, 63, 12),
            mf.make(3, 63, 6, outer_passes=2),
            mf.make(4, 127, 8),
            mf.make(5, 63, 5)]
    return reqs


def _fresh(r):
    return dataclasses.replace(r, arrival=0.0, result={}, passes_done=0, numiter=0, warm_steps=0, preemptions=0)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_each_result_same_alone_and_in_the_mix(precision):
    from slevolve_b200.serving import Server

    reqs = _requests()
    srv = Server({63: 2, 127: 2}, precision=precision)
    mix = srv.run([dataclasses.replace(r) for r in reqs])
    st = srv.stats(mix)
    assert st["requests"] == len(reqs)
    assert srv.batch_steps[63] < sum(r.nsteps * r.outer_passes for r in reqs if r.lmax == 63)  # slots shared steps
    by_id = {r.rid: r for r in mix}
    for r in reqs:
        alone = Server({r.lmax: 1}, precision=precision).run([_fresh(r)])[0]
        m = by_id[r.rid]
        assert m.numiter == alone.numiter, r.rid
        for key in alone.result:
            assert np.array_equal(m.result[key], alone.result[key]), (r.rid, key)
    outer = by_id[3]
    assert outer.passes_done == 2 and outer.warm_steps == outer.nsteps


def test_admission_respects_the_memory_budget():
    from slevolve_b200.serving import Server, footprint

    reqs = _requests()
    budget = max(footprint(r) for r in reqs) + min(footprint(r) for r in reqs)
    srv = Server({63: 3, 127: 2}, precision="mixed", budget_bytes=budget)
    out = srv.run(reqs)
    assert len(srv.done) == len(reqs)
    assert srv.peak_used <= budget
    assert all(r.t_done >= r.t_admit >= r.arrival for r in out)
