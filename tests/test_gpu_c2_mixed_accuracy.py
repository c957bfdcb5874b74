"""The mixed-precision step against the FP64 step over the whole c2 run (512 x 1024, L = 511,
1200 steps of 200 yr, three northern ice sheets on a 100-kyr sawtooth).

Bar (the mixed form's contract): topography, sea-level change and radial displacement within
1 mm of the FP64 solve of the same inputs at every step where both forms take the same number of
inner iterations.  The stop rule xi <= 1e-5 can end the two forms one iteration apart when xi
lands next to the threshold; the two iterates then differ by up to the size of one inner update
(the reference's own plain and extrapolated starts differ in the same way, 3e-4 m at L = 511).
Such steps must be rare (<= 1 % of the run), the FP64 xi at the stopping iteration must lie
within 10 % of the threshold, and the error must fall back below 1 mm within five steps.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
BAR_M = 1e-3


def test_c2_mixed_vs_fp64_1200_steps():
    import torch

    from slevolve_b200 import OptSeaLevelSolver, _lib, make_sht
    from slevolve_b200.synthetic import case_c2

    sht = make_sht("cuda", 512, 1024, 511)
    case = case_c2(sht)
    kw = dict(norder=511, dt=case.dt, opt={"dsl", "diag"}, inner="extrap")
    s64 = OptSeaLevelSolver(sht, case.love, case.topo, case.ice(0), precision="fp64", **kw)
    smx = OptSeaLevelSolver(sht, case.love, case.topo, case.ice(0), precision="mixed", **kw)
    L = _lib.lib()
    fields = {"deltasl": _lib.F_DELTASL, "tgrid": _lib.F_TGRID, "R": _lib.F_R}
    a = {f: torch.empty((512, 1024), dtype=torch.float64, device="cuda") for f in fields}
    b = {f: torch.empty_like(v) for f, v in a.items()}
    worst_same = 0.0
    flips = []
    errs = []
    for k in range(1, case.nsteps + 1):
        ice = torch.from_numpy(np.ascontiguousarray(case.ice(k))).cuda()
        i64 = s64.step_device(ice.data_ptr(), 1)
        imx = smx.step_device(ice.data_ptr(), 1)
        e = 0.0
        for f, code in fields.items():
            _lib.check(L.sle_solver_get(s64._h, code, _lib.C.c_void_p(a[f].data_ptr()), 1))
            _lib.check(L.sle_solver_get(smx._h, code, _lib.C.c_void_p(b[f].data_ptr()), 1))
            e = max(e, float((a[f] - b[f]).abs().max()))
        errs.append(e)
        if i64.numiter == imx.numiter:
            worst_same = max(worst_same, e)
        else:
            flips.append((k, i64.numiter, imx.numiter, i64.xi, imx.xi, e))
    print(f"c2 mixed vs FP64: max error at equal iteration counts {worst_same:.3e} m, "
          f"median step error {np.median(errs):.3e} m, {len(flips)} steps with different counts {flips}")
    assert worst_same <= BAR_M, worst_same
    assert len(flips) <= case.nsteps // 100, flips
    for k, n64, nmx, xi64, ximx, e in flips:
        near = [xi for xi in (xi64, ximx) if abs(xi - 1e-5) <= 0.1e-5]
        assert near, (k, xi64, ximx)
        assert min(errs[k - 1: k + 5]) <= BAR_M, (k, errs[k - 1: k + 5])
