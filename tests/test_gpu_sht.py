"""CUDA transform against the reference's golden vectors and the CPU oracle.

Tolerance: 1e-12 relative to the largest coefficient / grid value (the reference's own round-trip
bar is 1e-12, tests/test_sht_roundtrip.py:49 of the reference).  Gauss nodes agree to 1 ulp.
"""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu
REL = 1e-12


def _sht(n, L, nlon=None):
    from slevolve_b200 import make_sht

    return make_sht("cuda", n, nlon or 2 * n, L)


@pytest.mark.parametrize("n,L", [(16, 15), (32, 31), (32, 20), (64, 63)])
def test_against_reference_golden(n, L):
    fx = load_golden("sht.npz")
    tag = f"n{n}_l{L}"
    s = _sht(n, L)
    # nodes and weights come from the same Newton iteration; the initial cos() guess may
    # differ by an ulp, which can move the converged values by an ulp or two
    assert np.abs(s.gaulats - fx[f"{tag}_nodes"]).max() <= 4.5e-16
    assert np.allclose(s.weights, fx[f"{tag}_weights"], rtol=2e-15, atol=0)
    a = s.analysis(fx[f"{tag}_grid"]).copy()
    ref = fx[f"{tag}_ana"]
    assert np.abs(a - ref).max() <= REL * np.abs(ref).max()
    g = s.synthesis(fx[f"{tag}_coef"]).copy()
    ref = fx[f"{tag}_syn"]
    assert np.abs(g - ref).max() <= REL * np.abs(ref).max()


@pytest.mark.parametrize("n,L", [(128, 63), (256, 255), (512, 511)])
def test_against_oracle_random(n, L):
    from oracle.sht import OracleSHT

    rng = np.random.default_rng(n + L)
    s = _sht(n, L)
    o = OracleSHT(n, 2 * n, L)
    g = rng.standard_normal((n, 2 * n))
    a = s.analysis(g).copy()
    ref = o.analysis(g)
    assert np.abs(a - ref).max() <= REL * np.abs(ref).max()
    c = np.tril(rng.standard_normal((L + 1, L + 1)) + 1j * rng.standard_normal((L + 1, L + 1)))
    c[:, 0] = c[:, 0].real
    gg = s.synthesis(c).copy()
    ref = o.synthesis(c)
    assert np.abs(gg - ref).max() <= REL * np.abs(ref).max()


@pytest.mark.parametrize("n,L", [(64, 63), (512, 511)])
def test_roundtrip(n, L):
    """synthesis -> analysis -> synthesis (the reference's tests/test_sht_roundtrip.py)."""
    rng = np.random.default_rng(7)
    s = _sht(n, L)
    c = np.tril(rng.normal(size=(L + 1, L + 1)) + 1j * rng.normal(size=(L + 1, L + 1)))
    c[:, 0] = c[:, 0].real
    g = s.synthesis(c).copy()
    c2 = s.analysis(g).copy()
    g2 = s.synthesis(c2).copy()
    assert np.abs(c2 - c).max() / np.abs(c).max() < 1e-12
    assert np.abs(g2 - g).max() / np.abs(g).max() < 1e-12


def test_more_than_eight_latitude_groups():
    """640 latitudes = 10 groups of 32: the analysis runs in two passes per segment."""
    from oracle.sht import OracleSHT

    rng = np.random.default_rng(13)
    n, nlon, L = 640, 1024, 100
    s = _sht(n, L, nlon)
    o = OracleSHT(n, nlon, L)
    g = rng.standard_normal((n, nlon))
    ref = o.analysis(g)
    assert np.abs(s.analysis(g) - ref).max() <= REL * np.abs(ref).max()
    c = np.tril(rng.standard_normal((L + 1, L + 1)) + 1j * rng.standard_normal((L + 1, L + 1)))
    ref = o.synthesis(c)
    assert np.abs(s.synthesis(c) - ref).max() <= REL * np.abs(ref).max()


def test_nyquist_order_and_small_lmax():
    """lmax = nlon/2 (the Nyquist order kept by the reference numpy backend) and lmax < nlat-1."""
    from oracle.sht import OracleSHT

    rng = np.random.default_rng(11)
    for n, nlon, L in ((16, 32, 16), (64, 128, 20)):
        s = _sht(n, L, nlon)
        o = OracleSHT(n, nlon, L)
        g = rng.standard_normal((n, nlon))
        ref = o.analysis(g)
        assert np.abs(s.analysis(g) - ref).max() <= REL * np.abs(ref).max()
        c = np.tril(rng.standard_normal((L + 1, L + 1)) + 1j * rng.standard_normal((L + 1, L + 1)))
        ref = o.synthesis(c)
        assert np.abs(s.synthesis(c) - ref).max() <= REL * np.abs(ref).max()


def test_batched_and_device_paths():
    import torch

    n, L = 128, 127
    s = _sht(n, L)
    rng = np.random.default_rng(5)
    grids = [torch.tensor(rng.standard_normal((n, 2 * n)), device="cuda") for _ in range(4)]
    outs = [torch.empty((L + 1, L + 1), dtype=torch.complex128, device="cuda") for _ in range(4)]
    s.analysis_device(grids, outs)
    torch.cuda.synchronize()
    for g, o in zip(grids, outs):
        single = s.analysis(g.cpu().numpy()).copy()
        assert np.array_equal(o.cpu().numpy(), single)
    back = [torch.empty((n, 2 * n), dtype=torch.float64, device="cuda") for _ in range(4)]
    s.synthesis_device(outs, back)
    for g, b in zip(grids, back):
        single = s.synthesis(s.analysis(g)).cpu().numpy()
        assert np.array_equal(b.cpu().numpy(), single)
    # device tensors of the wrong shape or type are refused on the host, before any launch
    with pytest.raises(ValueError, match="coeffs shape"):
        s.synthesis(torch.zeros((L, L), dtype=torch.complex128, device="cuda"))
    with pytest.raises(ValueError, match="out must be"):
        s.synthesis(outs[0], out=torch.empty((n, n), dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError, match="out must be"):
        s.analysis(grids[0], out=torch.empty((L + 1, L + 1), dtype=torch.complex64, device="cuda"))


def test_work_fraction_reported():
    s = _sht(512, 511)
    assert 0.3 < s.work_fraction <= 1.0
