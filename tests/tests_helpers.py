"""Input builders shared by the CPU and GPU tests (no reference checkout needed)."""

import numpy as np

from slevolve_b200.synthetic import angular_distance, grid_latlon, round_mm, vialov


def marine_topo(gaulats, nlon):
    """Polar marine continent of the reference's tests/test_small_case.py:86-92 (restated)."""
    colat = np.degrees(np.arccos(gaulats))[:, None] * np.ones((1, nlon))
    topo = np.where(colat <= 20.0, 300.0 - 1100.0 * colat / 20.0, -800.0)
    return np.where(colat > 25.0, -4000.0,
                    np.where(colat > 20.0, -800.0 - 640.0 * (colat - 20.0), topo))


def marine_ice(gaulats, nlon, heights):
    colat = np.degrees(np.arccos(gaulats))[:, None] * np.ones((1, nlon))
    shape = np.sqrt(np.clip(1.0 - (colat / 14.0) ** 2, 0.0, None))
    return [h * shape for h in heights]


def synthetic512_ice(gaulats, topo, nlon, polar, midlat):
    """Ice of the reference's synthetic case (tools/make_synthetic_case.py:66-79, 178-190)."""
    LAT, LON = grid_latlon(gaulats, nlon)
    p = vialov(90.0 + LAT, 17.0)
    m = vialov(angular_distance(LAT, LON, 56.0, 132.0), 12.0)
    grounded = topo > -500.0
    return [round_mm((hp * p + hm * m) * grounded) for hp, hm in zip(polar, midlat)]
