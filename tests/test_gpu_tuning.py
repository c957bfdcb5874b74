"""Launch-shape tuning of the mixed-precision transforms: every shape gives the same results
bit for bit (the shape changes how fields are grouped into launches and how the pipeline and the
row FFTs are blocked, not the arithmetic of a field: every launch computes all its columns with
the same accumulation structure), the tuner returns one of its candidates, and a batch stepped
after tuning equals one stepped with the default shape."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_every_launch_shape_gives_identical_transforms():
    import torch

    from slevolve_b200 import _lib, make_sht
    from slevolve_b200.tuning import apply, candidates

    n, L, nf = 64, 63, 40
    sht = make_sht("cuda", n, 2 * n, L, precision="mixed")
    g = torch.Generator(device="cuda").manual_seed(3)
    grids = [torch.randn((n, 2 * n), dtype=torch.float64, device="cuda", generator=g) * (i + 1) for i in range(nf)]
    ref = None
    for cand in candidates(nf):
        apply(sht, cand)
        spec = [torch.empty(sht.ncoef, dtype=torch.complex128, device="cuda") for _ in range(nf)]
        sht.analysis_device(grids, spec, layout=_lib.LAYOUT_PACKED)
        out = [torch.empty_like(x) for x in grids]
        sht.synthesis_device(spec, out, layout=_lib.LAYOUT_PACKED)
        got = (torch.stack(spec).cpu().numpy(), torch.stack(out).cpu().numpy())
        if ref is None:
            ref = got
        else:
            assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]), cand


def test_tuned_batch_matches_default_batch():
    from slevolve_b200.batch import SolverBatch
    from slevolve_b200.synthetic import case_c0
    from slevolve_b200.tuning import DEFAULT, candidates
    from oracle.sht import OracleSHT

    case = case_c0(OracleSHT(64, 128, 63), nsteps=6)
    a = SolverBatch(64, 128, 63, 3, precision="mixed")
    b = SolverBatch(64, 128, 63, 3, precision="mixed")
    best, timings = b.autotune()
    assert best in candidates(3) and len(timings) == len(candidates(3))
    assert set(DEFAULT) == set(best)
    for bt in (a, b):
        for s in range(3):
            bt.load(s, case.love, case.topo, case.ice(0) * (1.0 + 0.25 * s), 1.0)
    for k in range(1, 5):
        ia = a.step({s: case.ice(k) * (1.0 + 0.25 * s) for s in range(3)})
        ib = b.step({s: case.ice(k) * (1.0 + 0.25 * s) for s in range(3)})
        for s in range(3):
            assert ia[s]["numiter"] == ib[s]["numiter"]
            assert np.array_equal(a.get(s, "tgrid"), b.get(s, "tgrid")), (k, s)
