"""The segmented initial-topography guess on the GPU (FP64 CUDA transforms, device residual
reductions) against the reference's own output (``tests/golden/init_topo.npz``): same legs and
iteration count, the uniform term and T0 within 1e-9 m, the parity bar of the step itself (the device
sums and transforms round differently from NumPy's at the 1e-13 level)."""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", ["uniform", "times"])
def test_gpu_guess_matches_the_reference(name):
    from slevolve_b200.init_topo import segmented_guess
    from slevolve_b200.love import SyntheticEarth

    g = np.load(os.path.join(HERE, "golden", "init_topo.npz"))
    topo, ice = g["topo"], list(g["ice"])
    love = SyntheticEarth(63, 8, 20261203 + 5)
    kw = {"uniform": dict(dt=10.0, threshold=0.01, start=None),
          "times": dict(dt=g["times"], threshold=0.05, start=g["start"])}[name]
    T0, info = segmented_guess(topo, ice, love, 63, kw["dt"], threshold=kw["threshold"], start=kw["start"])
    assert info["iters"] == int(g[f"{name}_iters"])
    assert [[s["a"], s["b"]] for s in info["segments"]] == g[f"{name}_legs"].tolist()
    assert np.allclose([s["tau"] for s in info["segments"]], g[f"{name}_tau"], rtol=1e-12, atol=0)
    dc = abs(info["c"] - float(g[f"{name}_c"]))
    dT = float(np.abs(T0 - g[f"{name}_T0"]).max())
    assert dc <= 1e-9, dc
    assert dT <= 1e-9, dT


def test_device_residual_matches_numpy():
    """One residual evaluation against the reference's NumPy expression on the same grids."""
    import torch

    from slevolve_b200.init_topo import _Grids

    g = np.load(os.path.join(HERE, "golden", "init_topo.npz"))
    topo, I0, Ip = g["topo"], g["ice"][0], g["ice"][-1]
    rng = np.random.default_rng(3)
    S = rng.normal(0.0, 30.0, topo.shape)
    dev = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()   # noqa: E731
    gr = _Grids(dev(topo), dev(I0), dev(Ip), 920.0, 1000.0, 6.371e6, torch)
    _, gw = np.polynomial.legendre.leggauss(64)
    area = np.broadcast_to((gw[::-1] * 2 * np.pi / 128 * 6.371e6 ** 2)[:, None], topo.shape).copy()

    def grounded(I, T):
        return (I > 0) & ((T > 0) | (920.0 * I > 1000.0 * np.abs(T)))

    gp = grounded(Ip, topo)
    Cp = (topo < 0) & ~gp
    for c in (-40.0, -3.5, 0.0, 12.25, 70.0):
        T0 = topo + c + S
        g0 = grounded(I0, T0)
        C0 = (T0 < 0) & ~g0
        want = ((np.clip(-T0, 0, None) * C0 * area).sum() - (np.clip(-topo, 0, None) * Cp * area).sum()
                + 920.0 / 1000.0 * ((I0 * g0 - Ip * gp) * area).sum())
        got = gr.residual(dev(S), c)
        assert abs(got - want) <= 1e-12 * np.abs(area).sum() * 100.0, (c, got, want)
