"""Oracle (test infrastructure only): NumPy restatement of the segmented initial-topography guess
of the reference's outer driver (SLEvolve python/slevolve/init_topo_segmented.py).

Only ``tests/`` and the CPU-baseline legs may use it.  It follows the reference's arithmetic
expression by expression (NumPy sums and orders of operations), so that with the reference's
own NumPy transform it reproduces the reference's output; with ``OracleSHT`` it agrees to the
transforms' 1e-13.

* ``grounded``            init_topo_segmented.py:39-40
* ``segments``            init_topo_segmented.py:43-66 (5-point running mean, extrema, pruning of
                          short legs, intensity-weighted age tau of each leg)
* ``ConservationCase``    init_topo_segmented.py:69-98 (areas, present masks, water-volume
                          residual, bisection for the uniform term)
* ``segmented_guess``     init_topo_segmented.py:101-146 (relaxed Love numbers per leg, the
                          G - R operators, the fixed point for dSL)
"""

from __future__ import annotations

import numpy as np

from .sht import OracleSHT

MASS = 5.976e24   # Planet().mass (solver.py:98-110)


def grounded(I, T, rhoi, rhow):
    return (I > 0) & ((T > 0) | (rhoi * I > rhow * np.abs(T)))


def segments(V, dt, threshold=0.01):
    V = np.asarray(V, float)
    n = V.size
    last = n - 1
    if np.ndim(dt) == 0:
        def age(i):
            return dt * (last - i)
    else:
        tk = np.asarray(dt, float)
        if tk.shape != (n,):
            raise ValueError("one time per ice state")

        def age(i):
            return float(tk[last] - tk[i]) if np.ndim(i) == 0 else tk[last] - tk[i]
    smooth = np.convolve(np.pad(V, 2, mode="edge"), np.ones(5) / 5, "valid")
    slope = np.sign(np.diff(smooth))
    ext = [0] + [i for i in range(1, n - 1) if slope[i - 1] * slope[i] < 0] + [n - 1]
    floor = threshold * (smooth.max() - smooth.min())
    while len(ext) > 2:
        legs = [abs(smooth[ext[i + 1]] - smooth[ext[i]]) for i in range(len(ext) - 1)]
        i = int(np.argmin(legs))
        if legs[i] >= floor:
            break
        if i == 0:
            del ext[1]
        elif i == len(ext) - 2:
            del ext[-2]
        else:
            del ext[i:i + 2]
    out = []
    for a, b in zip(ext[:-1], ext[1:]):
        st = np.arange(a + 1, b + 1)
        dv = np.abs(V[st] - V[st - 1])
        out.append({"a": int(a), "b": int(b), "t_a_ka": age(a), "t_b_ka": age(b),
                    "tau": float((dv * age(st)).sum() / dv.sum()), "dV": float(V[b] - V[a])})
    return out


class ConservationCase:
    def __init__(self, Tp, I0, Ip, rhoi=920.0, rhow=1000.0, radius=6.371e6):
        nl, no = Tp.shape
        self.Tp, self.I0, self.Ip, self.rhoi, self.rhow = Tp, I0, Ip, rhoi, rhow
        _, gw = np.polynomial.legendre.leggauss(nl)
        gw = gw[::-1]
        self.area = np.broadcast_to((gw * 2 * np.pi / no * radius ** 2)[:, None], (nl, no)).copy()
        self.gp = grounded(Ip, Tp, rhoi, rhow)
        self.Cp = (Tp < 0) & ~self.gp

    def rms(self, f):
        m = np.ones(f.shape, bool)   # the reference's global mask: boolean-indexed, flattened sums
        return float(np.sqrt((self.area[m] * f[m] ** 2).sum() / self.area[m].sum()))

    def residual(self, T0):
        g0 = grounded(self.I0, T0, self.rhoi, self.rhow)
        C0 = (T0 < 0) & ~g0
        V0 = (np.clip(-T0, 0, None) * C0 * self.area).sum()
        Vp = (np.clip(-self.Tp, 0, None) * self.Cp * self.area).sum()
        dI = self.I0 * g0 - self.Ip * self.gp
        return V0 - Vp + self.rhoi / self.rhow * (dI * self.area).sum(), g0, C0, dI

    def solve_c(self, S, c, half=80.0):
        lo, hi = c - half, c + half
        for _ in range(60):
            mid = 0.5 * (lo + hi)
            if self.residual(self.Tp + mid + S)[0] > 0:
                lo = mid
            else:
                hi = mid
        return 0.5 * (lo + hi)


def relaxed_love(love, lmax, tau):
    """Elastic (h, k) plus the viscous modes relaxed for tau kyr (init_topo_segmented.py:114-118)."""
    h, k = love.he.copy(), love.ke.copy()
    for ll in range(1, lmax + 1):
        nm = love.nmod[ll]
        s = love.s[:nm, ll]
        f = 1.0 - np.exp(-s * tau)
        h[ll] += (love.r[:nm, ll] / s * f).sum()
        k[ll] += (love.rprime[:nm, ll] / s * f).sum()
    return h, k


def segmented_guess(Tp, ice, love, lmax, dt, threshold=0.01, start=None, c0=62.0, rhoi=920.0,
                    rhow=1000.0, radius=6.371e6, c_half=80.0, tol=1e-3, maxit=40, sht=None):
    nl, no = Tp.shape
    N = len(ice) - 1
    cs = ConservationCase(Tp, np.asarray(ice[0]), np.asarray(ice[N]), rhoi, rhow, radius)
    V = np.array([(np.asarray(ice[n]) * cs.area).sum() for n in range(N + 1)])
    segs = segments(V, dt, threshold)
    l = np.arange(lmax + 1, dtype=float)
    ttl = np.zeros_like(l)
    ttl[1:] = 4 * np.pi * radius ** 3 / (MASS * (2 * l[1:] + 1))
    sht = sht if sht is not None else OracleSHT(nl, no, lmax)

    def operator(h, k):
        fac = ttl * (1 + k - h)

        def apply(load):
            r = sht.synthesis(sht.analysis(np.ascontiguousarray(load)).copy() * fac[:, None]).copy()
            return r - (r * cs.area).sum() / cs.area.sum()
        return apply

    hk = [relaxed_love(love, lmax, sg["tau"]) for sg in segs]
    ops = [operator(h, k) for h, k in hk]
    w = np.abs([sg["dV"] for sg in segs])
    w = w / w.sum()
    if len(segs) == 1:
        water = ops[0]
    else:
        water = operator(sum(wi * h for wi, (h, k) in zip(w, hk)), sum(wi * k for wi, (h, k) in zip(w, hk)))
    Ib = [np.asarray(ice[sg["a"]]) for sg in segs] + [cs.Ip]
    dSL = np.zeros_like(Tp) if start is None else np.asarray(start, float) - Tp
    c = c0
    for it in range(maxit):
        T0 = Tp + dSL
        _, g0, C0, dI = cs.residual(T0)
        dS = dSL * cs.Cp - T0 * (cs.Cp.astype(float) - C0)
        if len(segs) > 1:
            L = [cs.I0 * g0] + [I * grounded(I, T0, rhoi, rhow) for I in Ib[1:-1]] + [cs.Ip * cs.gp]
            Sx = -sum(op(rhoi * (L[j] - L[j + 1])) for j, op in enumerate(ops)) - water(-rhow * dS)
        else:
            Sx = -ops[0](rhoi * dI - rhow * dS)
        cn = cs.solve_c(Sx, c, c_half)
        new = cn + Sx
        ch = cs.rms(new - dSL)
        dSL = new
        c = cn
        if ch < tol:
            break
    return Tp + dSL, {"segments": segs, "c": c, "iters": it + 1, "last_change_m": ch}
