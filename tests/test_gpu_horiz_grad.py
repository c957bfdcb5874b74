"""``slevolve_b200.horiz.gradient`` (three FP64 CUDA syntheses and the row combine on the device)
against the oracle's gradient and against analytic fields, the check of the reference's own
self-test (python/slevolve/tools/horiz_grad.py:27-42: 64 x 128, L = 63, 1e-10)."""

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_gradient_analytic_and_reference_psi():
    from oracle.horiz import gradient as oracle_gradient
    from oracle.sht import OracleSHT
    from slevolve_b200.horiz import gradient

    nlat, nlon, L = 64, 128, 63
    o = OracleSHT(nlat, nlon, L)
    c = o.gaulats[:, None]
    s = np.sqrt(1.0 - c * c)
    ph = (2.0 * np.pi * np.arange(nlon) / nlon)[None, :]
    psi = c ** 2 + s * c * np.sin(ph) + s ** 3 * np.cos(3 * ph)
    dth = -2 * c * s + (c * c - s * s) * np.sin(ph) + 3 * s * s * c * np.cos(3 * ph)
    dph = c * np.cos(ph) - 3 * s * s * np.sin(3 * ph)
    ut, up = gradient(o.analysis(psi), nlat, nlon)
    assert np.abs(ut - dth).max() < 1e-10
    assert np.abs(up - dph).max() < 1e-10

    fx = load_golden("horiz.npz")
    for k in (1, 8):
        U = fx[f"horiz_{k}"]
        rt, rp = oracle_gradient(U, nlat, nlon)
        ut, up = gradient(U, nlat, nlon)
        assert np.abs(ut - rt).max() <= 1e-10 * np.abs(rt).max(), k
        assert np.abs(up - rp).max() <= 1e-10 * np.abs(rp).max(), k
