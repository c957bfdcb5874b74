"""Mixed-precision transforms (split-TF32 tensor-core Legendre contraction) against the FP64 ones.

Bar: 1e-6 of the largest coefficient / grid value for the contraction (TF32 hi + lo operands,
three products, FP32 accumulation), and the FP64 degree-0 coefficient of the analysis and the
degree-0 term of the synthesis within 1e-13 relative (they bypass the tensor cores).  TF32 has
FP32's exponent range, so the relative error does not depend on the field's magnitude: fields
scaled by 1e-20 and 1e+20 meet the same bar (the FP32 row FFTs bound the range).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL_TC = 1e-6


def _pair(n, L):
    from slevolve_b200 import make_sht

    return make_sht("cuda", n, 2 * n, L), make_sht("cuda", n, 2 * n, L, precision="mixed")


@pytest.mark.parametrize("n,L", [(64, 63), (128, 127), (256, 255), (512, 511)])
def test_mixed_analysis_synthesis_against_fp64(n, L):
    from slevolve_b200.synthetic import band_limited_field

    f64, mx = _pair(n, L)
    g = band_limited_field(f64, 7, 1, L, 2.0) * 1000.0 + 300.0
    a64 = f64.analysis(g).copy()
    amx = mx.analysis(g).copy()
    ref = np.abs(a64).max()
    assert np.abs(amx - a64).max() <= REL_TC * ref
    assert abs(amx[0, 0].real - a64[0, 0].real) <= 1e-13 * abs(a64[0, 0].real)
    s64 = f64.synthesis(a64).copy()
    smx = mx.synthesis(a64).copy()
    assert np.abs(smx - s64).max() <= REL_TC * np.abs(s64).max()


def test_mixed_degree0_only_is_fp64():
    """A field with only the (0,0) coefficient: the mixed synthesis adds it in FP64, so the grid
    equals the FP64 one to rounding; the mixed analysis of a constant grid gives U_00 in FP64."""
    f64, mx = _pair(128, 127)
    c = np.zeros((128, 128), dtype=np.complex128)
    c[0, 0] = 123.456
    s64 = f64.synthesis(c).copy()
    smx = mx.synthesis(c).copy()
    assert np.abs(smx - s64).max() <= 1e-13 * np.abs(s64).max()
    g = np.full((128, 256), -3.25)
    a64 = f64.analysis(g).copy()
    amx = mx.analysis(g).copy()
    assert abs(amx[0, 0].real - a64[0, 0].real) <= 1e-13 * abs(a64[0, 0].real)
    assert np.abs(amx[1:, :]).max() <= 1e-6 * abs(a64[0, 0].real)


@pytest.mark.parametrize("scale", [1e-20, 1e-8, 1e8, 1e20])
def test_mixed_accuracy_independent_of_magnitude(scale):
    """The relative error of the contraction does not depend on the field's magnitude (TF32
    operands keep FP32's exponent range)."""
    from slevolve_b200.synthetic import band_limited_field

    f64, mx = _pair(128, 127)
    g = (band_limited_field(f64, 11, 1, 127, 2.0) + 0.5) * scale
    a64 = f64.analysis(g).copy()
    amx = mx.analysis(g).copy()
    assert np.abs(amx - a64).max() <= REL_TC * np.abs(a64).max()
    s64 = f64.synthesis(a64).copy()
    smx = mx.synthesis(a64).copy()
    assert np.abs(smx - s64).max() <= REL_TC * np.abs(s64).max()


def test_mixed_fields_of_different_magnitudes_in_one_launch():
    """Fields of one launch with magnitudes 1e-6 .. 1e6, each within the bar of its own largest
    coefficient."""
    import torch

    from slevolve_b200 import _lib
    from slevolve_b200.synthetic import band_limited_field

    f64, mx = _pair(64, 63)
    grids = [torch.tensor(band_limited_field(f64, 20 + i, 1, 63, 2.0) * 10.0 ** (3 * i - 6), device="cuda")
             for i in range(5)]
    out = {}
    for sh in (f64, mx):
        co = [torch.empty(sh.ncoef, dtype=torch.complex128, device="cuda") for _ in grids]
        for i in range(0, len(grids), 4):
            sh.analysis_device(grids[i:i + 4], co[i:i + 4], layout=_lib.LAYOUT_PACKED)
        out[sh.precision] = [c.cpu().numpy() for c in co]
    for a, b in zip(out["fp64"], out["mixed"]):
        assert np.abs(a - b).max() <= REL_TC * np.abs(a).max()
