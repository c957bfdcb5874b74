"""Snapshot / restore of a solve (checkpoint, preemption, migration between slots).

The bar is identity: a solve restored from a snapshot taken after step k, into a fresh solver or
into another batch slot, must continue bit for bit as the uninterrupted solve (iteration counts,
topography, radial displacement, masks, converged load increment).  The reference checkpoints the
same state in its Fortran solver (fortran/src/modal_state_mod.f90:445-477)."""

import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case():
    from slevolve_b200.synthetic import case_c0
    from oracle.sht import OracleSHT

    return case_c0(OracleSHT(64, 128, 63), nsteps=12)


def _outputs(r):
    return {k: np.array(r[k], copy=True) for k in ("tgrid", "R", "ocean", "beta", "dS_converged")}


@pytest.mark.parametrize("precision,inner", [("fp64", "off"), ("fp64", "extrap"), ("mixed", "extrap")])
def test_solver_restored_into_a_fresh_solver_continues_bit_for_bit(precision, inner):
    from slevolve_b200 import OptSeaLevelSolver

    case = _case()
    kw = dict(norder=63, dt=1.0, opt={"dsl"}, inner=inner, precision=precision)
    ref = OptSeaLevelSolver(None, case.love, case.topo, case.ice(0), **kw)
    snap = None
    want = {}
    for k in range(1, 11):
        r = ref.step(case.ice(k), dt=1.0 if k < 7 else 2.0)   # the step length changes after the snapshot
        if k == 5:
            snap = ref.snapshot()
        if k > 5:
            want[k] = (r["numiter"], _outputs(r))
    other = OptSeaLevelSolver(None, case.love, case.topo, case.ice(3), **kw)
    other.step(case.ice(4))   # a solver with a history of its own, overwritten by the restore
    other.restore(snap)
    assert other.iter == 5
    for k in range(6, 11):
        r = other.step(case.ice(k), dt=1.0 if k < 7 else 2.0)
        ni, out = want[k]
        assert r["numiter"] == ni, k
        for key, v in out.items():
            assert np.array_equal(np.asarray(r[key]), v), (k, key)


def test_batch_slot_migrates_to_another_batch_and_slot():
    from slevolve_b200.batch import SolverBatch

    case = _case()
    a = SolverBatch(64, 128, 63, 2, precision="mixed")
    b = SolverBatch(64, 128, 63, 3, precision="mixed")
    a.load(0, case.love, case.topo, case.ice(0), 1.0)
    a.load(1, case.love, case.topo, case.ice(0) * 0.5, 1.0)
    for k in range(1, 4):
        a.step({0: case.ice(k), 1: case.ice(k) * 0.5})
    img = a.snapshot(0)
    want = []
    for k in range(4, 9):
        info = a.step({0: case.ice(k), 1: case.ice(k) * 0.5})
        want.append((info[0]["numiter"], a.get(0, "tgrid").copy(), a.get(0, "R").copy()))
    b.restore(2, img)
    for i, k in enumerate(range(4, 9)):
        info = b.step({2: case.ice(k)})
        ni, tg, rr = want[i]
        assert info[2]["numiter"] == ni, k
        assert np.array_equal(b.get(2, "tgrid"), tg), k
        assert np.array_equal(b.get(2, "R"), rr), k


def test_restore_refuses_an_image_of_another_configuration():
    from slevolve_b200 import SeaLevelSolver

    case = _case()
    s64 = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=63, dt=1.0)
    s64.step(case.ice(1))
    snap = s64.snapshot()
    s31 = SeaLevelSolver(None, case.love, case.topo, case.ice(0), norder=31, dt=1.0)
    with pytest.raises(ValueError, match="belongs to"):
        s31.restore(snap)
    bad = dict(snap)
    bad["image"] = snap["image"][:100]
    with pytest.raises(ValueError):
        s64.restore(bad)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_serving_preemption_gives_the_same_results(precision):
    """A high-priority request arriving while a long low-priority one holds the only slot
    preempts it (snapshot to the host, slot handed over, restore later): both results equal the
    requests served alone."""
    from slevolve_b200.serving import MemberFactory, Server

    mf = MemberFactory(seed=5)
    low = mf.make(0, 63, 1500, kind="melt")
    high = dataclasses.replace(mf.make(1, 63, 20, kind="sawtooth"), arrival=0.25, priority=1)
    srv = Server({63: 1}, precision=precision, preempt=True)
    out = {r.rid: r for r in srv.run([dataclasses.replace(low), dataclasses.replace(high)])}
    assert out[0].preemptions >= 1 and srv.stats(list(out.values()))["preemptions"] >= 1
    assert out[1].t_done < out[0].t_done
    for r in (low, high):
        alone = Server({63: 1}, precision=precision).run([dataclasses.replace(r, arrival=0.0, result={})])[0]
        assert out[r.rid].numiter == alone.numiter, r.rid
        for key in alone.result:
            assert np.array_equal(out[r.rid].result[key], alone.result[key]), (r.rid, key)
