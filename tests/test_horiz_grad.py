"""Grid conversion of the horizontal-displacement potential (the reference's ``horiz.gradient``,
python/slevolve/horiz.py:39-60), on the CPU.

* The oracle (oracle/horiz.py: the derivative carried through the Legendre recursion) against
  analytic fields with known gradients, to 1e-10, the bar of the reference's own self-test
  (python/slevolve/tools/horiz_grad.py:27-42).
* The package's recurrence (``gradient_coeffs`` + ``combine_rows``, and the torch glue of
  ``_gradient_with``) over the oracle transform against the oracle, on random spectra and on the
  reference's own Psi_lm output (golden ``horiz.npz``), to 1e-12 of the largest value.
"""

import numpy as np
import pytest

from conftest import load_golden


def _analytic(x, nlon):
    """Psi = cos^2 + sin cos sin(phi) + sin^3 cos(3 phi) and its gradient (u_theta, u_phi)."""
    c = x[:, None]
    s = np.sqrt(1.0 - c * c)
    ph = (2.0 * np.pi * np.arange(nlon) / nlon)[None, :]
    psi = c ** 2 + s * c * np.sin(ph) + s ** 3 * np.cos(3 * ph)
    dth = -2 * c * s + (c * c - s * s) * np.sin(ph) + 3 * s * s * c * np.cos(3 * ph)
    dph = c * np.cos(ph) - 3 * s * s * np.sin(3 * ph)
    return psi, dth, dph


class _TorchOnOracle:
    """The oracle transform behind the torch-tensor interface of the CUDA transform (CPU tensors)."""

    def __init__(self, o):
        self.o = o
        self.gaulats = o.gaulats

    def synthesis(self, c):
        import torch

        return torch.from_numpy(np.array(self.o.synthesis(c.numpy())))


@pytest.mark.parametrize("nlat,nlon,L", [(64, 128, 63), (32, 64, 31), (96, 192, 60)])
def test_oracle_gradient_analytic(nlat, nlon, L):
    from oracle.horiz import gradient
    from oracle.sht import OracleSHT

    sh = OracleSHT(nlat, nlon, L)
    psi, dth, dph = _analytic(sh.gaulats, nlon)
    ut, up = gradient(sh.analysis(psi), nlat, nlon)
    assert np.abs(ut - dth).max() < 1e-10
    assert np.abs(up - dph).max() < 1e-10


def _recurrence(o, U):
    from slevolve_b200.horiz import combine_rows, gradient_coeffs

    A, B, C = gradient_coeffs(U)
    return combine_rows(o.synthesis(A), o.synthesis(B), o.synthesis(C), o.gaulats[:, None])


@pytest.mark.parametrize("nlat,nlon,L", [(64, 128, 63), (32, 64, 20), (128, 256, 127)])
def test_recurrence_matches_oracle(nlat, nlon, L):
    from oracle.horiz import gradient
    from oracle.sht import OracleSHT

    o = OracleSHT(nlat, nlon, L)
    rng = np.random.default_rng(nlat + L)
    U = (rng.normal(size=(L + 1, L + 1)) + 1j * rng.normal(size=(L + 1, L + 1)))
    U = np.tril(U) / (1.0 + np.arange(L + 1))[:, None] ** 2
    rt, rp = gradient(U, nlat, nlon)
    ut, up = _recurrence(o, U)
    assert np.abs(ut - rt).max() <= 1e-12 * np.abs(rt).max()
    assert np.abs(up - rp).max() <= 1e-12 * np.abs(rp).max()


def test_recurrence_on_reference_psi():
    """The reference's own Psi_lm (its horizontal read-out at 64 x 128, L = 63) through the torch
    glue of the package (CPU tensors over the oracle transform) and through the oracle."""
    import torch

    from oracle.horiz import gradient
    from oracle.sht import OracleSHT
    from slevolve_b200.horiz import _gradient_with

    fx = load_golden("horiz.npz")
    o = OracleSHT(64, 128, 63)
    for k in (1, 8):
        U = fx[f"horiz_{k}"]
        rt, rp = gradient(U, 64, 128)
        ut, up = _gradient_with(_TorchOnOracle(o), U, torch.device("cpu"))
        assert np.abs(rt).max() > 0
        assert np.abs(ut - rt).max() <= 1e-12 * np.abs(rt).max(), k
        assert np.abs(up - rp).max() <= 1e-12 * np.abs(rp).max(), k


def test_gradient_argument_checks():
    from slevolve_b200.horiz import gradient, gradient_coeffs

    with pytest.raises(ValueError, match="lmax"):
        gradient(np.zeros((64, 64), complex), 32, 64)
    with pytest.raises(ValueError, match="square"):
        gradient_coeffs(np.zeros((4, 5), complex))
    # the m = 0 imaginary part is dropped, the l = 0 row carries no gradient
    U = np.zeros((4, 4), complex)
    U[0, 0] = 1.0 + 2.0j
    U[2, 0] = 3.0j
    A, B, C = gradient_coeffs(U)
    assert not A.any() and not B.any() and not C.any()
