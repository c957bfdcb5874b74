"""The allocation-free analysis entry point (sle_sht_analysis_noalloc) against sle_sht_analysis.

Some hosts keep all of the GPU's memory for their own allocator and do not allow a library to
call cudaMalloc while they run; this entry point takes its scratch from a fixed array built into
the library instead.  It is called here through the C ABI, twice in a row per grid size (the
scratch is shared by every call and keeps the previous call's contents), and its packed
coefficients must agree with the allocating entry point's to 1e-12 relative, the transform
tolerance of the other GPU tests.  The device's free memory must not change across a call.
This file is collected last on purpose.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL = 1e-12


def _noalloc(L, sht, g, out, stream):
    from slevolve_b200 import _lib

    _lib.check(L.sle_sht_analysis_noalloc(sht._h, C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr()), stream),
               "sle_sht_analysis_noalloc")


@pytest.mark.parametrize("n", [64, 512])
def test_noalloc_analysis_matches_allocating_entry_point(n):
    import torch

    from slevolve_b200 import _lib, make_sht

    L = _lib.lib()
    sht = make_sht("cuda", n, 2 * n, n - 1)
    rng = np.random.default_rng(2026 + n)
    for call in range(2):
        g = torch.tensor(rng.standard_normal((n, 2 * n)), device="cuda")
        ref = torch.empty(sht.ncoef, dtype=torch.complex128, device="cuda")
        got = torch.full((sht.ncoef,), float("nan"), dtype=torch.complex128, device="cuda")
        sht.analysis_device([g], [ref], layout=_lib.LAYOUT_PACKED)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        _noalloc(L, sht, g, got, stream)
        torch.cuda.synchronize()
        if call == 1:   # the first call on the device may load the library's module
            assert torch.cuda.mem_get_info()[0] == free0
        r = ref.cpu().numpy()
        o = got.cpu().numpy()
        assert np.isfinite(o).all()
        assert np.abs(o - r).max() <= REL * np.abs(r).max()


def test_noalloc_computes_fp64_on_a_mixed_plan():
    import torch

    from slevolve_b200 import _lib, make_sht

    L = _lib.lib()
    n = 64
    fp64 = make_sht("cuda", n, 2 * n, n - 1)
    mixed = make_sht("cuda", n, 2 * n, n - 1, precision="mixed")
    g = torch.tensor(np.random.default_rng(7).standard_normal((n, 2 * n)), device="cuda")
    ref = torch.empty(fp64.ncoef, dtype=torch.complex128, device="cuda")
    got = torch.empty(fp64.ncoef, dtype=torch.complex128, device="cuda")
    fp64.analysis_device([g], [ref], layout=_lib.LAYOUT_PACKED)
    _noalloc(L, mixed, g, got, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    r, o = ref.cpu().numpy(), got.cpu().numpy()
    assert np.abs(o - r).max() <= REL * np.abs(r).max()


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    from slevolve_b200 import _lib, make_sht

    L = _lib.lib()
    sht = make_sht("cuda", 1024, 2048, 1023)
    g = torch.zeros((1024, 2048), dtype=torch.float64, device="cuda")
    out = torch.empty(sht.ncoef, dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError, match="exceeds the fixed scratch"):
        _lib.check(L.sle_sht_analysis_noalloc(sht._h, C.c_void_p(g.data_ptr()),
                                              C.c_void_p(out.data_ptr()), None), "noalloc")
