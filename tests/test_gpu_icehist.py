"""Ice history formed on the device: a blended entry equals the reference's NumPy expression
``(1.0 - w) * I_i + w * I_j`` (run_outer.py:169-170) bit for bit; plain entries are the
snapshots; the device cache returns the right grids after evictions; a batch stepped with the
device history equals the same batch stepped with the NumPy-formed grids."""

import numpy as np
import pytest

from slevolve_b200.icehist import IceHistory, parse_ice_seq

pytestmark = pytest.mark.gpu


def _stack(n, shape, seed=20261211):
    rng = np.random.default_rng(seed)
    out = rng.normal(0.0, 800.0, (n,) + shape)
    out[out < 0] = 0.0          # ice thickness: zero over much of the grid
    out[0, 0, :4] = [1e-300, 3e300, -0.0, 5e-324]
    return out


@pytest.mark.parametrize("shape", [(64, 128), (512, 1024)])
def test_blend_is_the_numpy_expression(shape):
    import torch

    stack = _stack(5, shape)
    ws = [0.0, 1.0, 0.5, 0.1, 1.0 / 3.0, 0.75, 0.9999999, 2.5, -0.25]
    items = [(0,)] + [(i % 5, (3 * i + 1) % 5, w) for i, w in enumerate(ws)] + [(4,), (-1,)]
    h = IceHistory(stack, items, cache=2)
    for k, it in enumerate(items):
        got = h.device(k).cpu().numpy()
        if len(it) == 1:
            want = stack[it[0]]
        else:
            i, j, w = it
            want = (1.0 - w) * stack[i] + w * stack[j]
        assert np.array_equal(got.view(np.uint64), np.ascontiguousarray(want).view(np.uint64)), (k, it)
    out = torch.empty(shape, dtype=torch.float64, device="cuda")
    assert h.device(3, out=out) is out


def test_history_feeds_the_solver_like_host_grids():
    from slevolve_b200 import SyntheticEarth, make_sht
    from slevolve_b200.batch import SolverBatch
    from slevolve_b200.synthetic import case_c0

    N, L = 64, 63
    base = case_c0(make_sht("cuda", N, 2 * N, L), nsteps=40)
    stack = np.stack([base.ice(k) for k in range(0, 40, 8)])
    items = parse_ice_seq("0,0:1:0.25,0:1:0.5,1,1:2:0.3,2")
    h = IceHistory(stack, items)
    love = SyntheticEarth(L, 8, 20261203 + 77)
    a = SolverBatch(N, 2 * N, L, 1, precision="fp64", opt={"dsl", "diag"}, inner="extrap")
    b = SolverBatch(N, 2 * N, L, 1, precision="fp64", opt={"dsl", "diag"}, inner="extrap")
    a.load(0, love, base.topo, stack[0], 1.0)
    b.load(0, love, base.topo, stack[0], 1.0)
    for k in range(1, len(items)):
        it = items[k]
        host = stack[it[0]] if len(it) == 1 else (1.0 - it[2]) * stack[it[0]] + it[2] * stack[it[1]]
        ia = a.step({0: h.device(k)})[0]
        ib = b.step({0: np.ascontiguousarray(host)})[0]
        assert ia["numiter"] == ib["numiter"]
        for f in ("deltasl", "tgrid", "R"):
            assert np.array_equal(a.get(0, f), b.get(0, f)), (k, f)
