"""Segmented initial-topography guess T0 for the first outer pass, on the GPU.

The reference's outer driver starts its Picard iteration on the ice-age topography from a
partially relaxed guess (SLEvolve python/slevolve/init_topo_segmented.py): the ice-volume series
of the ice states is cut into monotonic legs (``segments``, init_topo_segmented.py:43-66); each
leg's load acts through a G - R operator whose Love numbers are relaxed for the leg's mean age;
the sea-level change dSL = c + S is iterated to a fixed point (area-weighted RMS change below
``tol``, at most ``maxit`` iterations), the uniform term c found by bisection on the
water-volume residual (init_topo_segmented.py:84-98, 101-146).

Here the grids stay on the device: every G - R operator is one analysis and one synthesis of the
FP64 CUDA transform (``make_sht("cuda")``), the bisection evaluates the residual with one fused
reduction kernel per step (``sle_topo_residual``), and the elementwise updates run on the device.
The leg detection works on the ice-volume series (N + 1 numbers) on the host, as do the relaxed
Love numbers (a few hundred numbers per leg).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

MASS = 5.976e24   # Planet().mass (solver.py:98-110)


def segments(V, dt, threshold=0.01):
    """Monotonic legs of the ice-volume series ``V`` (states 0..N).  ``dt``: kyr per step, or the
    states' times t_0..t_N in kyr.  Each leg: first and last state ``a``, ``b``, their ages, the
    |dV|-weighted mean age ``tau`` of its steps and its volume change ``dV``
    (init_topo_segmented.py:43-66: 5-point running mean with edge padding, interior extrema, the
    smallest leg below ``threshold`` x range pruned first, never an end point)."""
    V = np.asarray(V, float)
    n = V.size
    if n < 2:
        raise ValueError("need at least two ice states")
    last = n - 1
    if np.ndim(dt) == 0:
        ages = float(dt) * (last - np.arange(n))
    else:
        tk = np.asarray(dt, float)
        if tk.shape != (n,):
            raise ValueError("one time per ice state")
        ages = tk[last] - tk
    smooth = np.convolve(np.pad(V, 2, mode="edge"), np.ones(5) / 5, "valid")
    slope = np.sign(np.diff(smooth))
    cuts = [0] + [i for i in range(1, n - 1) if slope[i - 1] * slope[i] < 0] + [last]
    floor = threshold * (smooth.max() - smooth.min())
    while len(cuts) > 2:
        legs = [abs(smooth[cuts[i + 1]] - smooth[cuts[i]]) for i in range(len(cuts) - 1)]
        i = int(np.argmin(legs))
        if legs[i] >= floor:
            break
        if i == 0:
            del cuts[1]
        elif i == len(cuts) - 2:
            del cuts[-2]
        else:
            del cuts[i:i + 2]
    out = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        st = np.arange(a + 1, b + 1)
        dv = np.abs(V[st] - V[st - 1])
        out.append({"a": int(a), "b": int(b), "t_a_ka": float(ages[a]), "t_b_ka": float(ages[b]),
                    "tau": float((dv * ages[st]).sum() / dv.sum()), "dV": float(V[b] - V[a])})
    return out


def relaxed_love(love, lmax, tau):
    """Load Love numbers h, k of degrees 0..lmax relaxed for ``tau`` kyr: the elastic values plus
    sum_k r_k / s_k (1 - exp(-s_k tau)) over the degree's modes (init_topo_segmented.py:114-118)."""
    h, k = np.array(love.he[:lmax + 1], float), np.array(love.ke[:lmax + 1], float)
    for ll in range(1, lmax + 1):
        nm = int(love.nmod[ll])
        s = love.s[:nm, ll]
        f = 1.0 - np.exp(-s * tau)
        h[ll] += (love.r[:nm, ll] / s * f).sum()
        k[ll] += (love.rprime[:nm, ll] / s * f).sum()
    return h, k


class _Grids:
    """Present state, areas and the conservation residual on the device."""

    def __init__(self, Tp, I0, Ip, rhoi, rhow, radius, torch):
        self.t = torch
        self.Tp, self.I0, self.Ip = Tp, I0, Ip
        self.rhoi, self.rhow = float(rhoi), float(rhow)
        nl, no = Tp.shape
        _, gw = np.polynomial.legendre.leggauss(nl)
        wrow = gw[::-1] * 2 * np.pi / no * radius ** 2
        self.wrow = torch.from_numpy(np.ascontiguousarray(wrow)).cuda()
        self.area = self.wrow[:, None].expand(nl, no).contiguous()
        self.area_sum = self.area.sum()
        self.gp = self.grounded(Ip, Tp)
        self.gp_u8 = self.gp.to(torch.uint8).contiguous()
        self.Cp = (Tp < 0) & ~self.gp
        self.Cp_f = self.Cp.to(torch.float64)
        self.Vp = float(((-Tp).clamp(min=0) * self.Cp * self.area).sum())
        self.scratch = torch.zeros(int(_lib.lib().sle_topo_scratch_bytes()), dtype=torch.uint8, device="cuda")
        self.out2 = (C.c_double * 2)()

    def grounded(self, I, T):
        return (I > 0) & ((T > 0) | (self.rhoi * I > self.rhow * T.abs()))

    def state(self, T0):
        g0 = self.grounded(self.I0, T0)
        C0 = (T0 < 0) & ~g0
        dI = self.I0 * g0 - self.Ip * self.gp
        return g0, C0, dI

    def residual(self, S, c):
        """Water-volume residual of T0 = (Tp + c) + S (init_topo_segmented.py:84-90)."""
        nl, no = self.Tp.shape
        st = self.t.cuda.current_stream().cuda_stream
        _lib.check(_lib.lib().sle_topo_residual(
            C.c_void_p(self.Tp.data_ptr()), C.c_void_p(S.data_ptr()), float(c), C.c_void_p(self.I0.data_ptr()),
            C.c_void_p(self.Ip.data_ptr()), C.c_void_p(self.gp_u8.data_ptr()), C.c_void_p(self.wrow.data_ptr()),
            nl, no, self.rhoi, self.rhow, C.c_void_p(self.scratch.data_ptr()), self.out2, C.c_void_p(st)),
            "sle_topo_residual")
        return self.out2[0] - self.Vp + self.rhoi / self.rhow * self.out2[1]

    def solve_c(self, S, c, half):
        lo, hi = c - half, c + half
        for _ in range(60):
            mid = 0.5 * (lo + hi)
            if self.residual(S, mid) > 0:
                lo = mid
            else:
                hi = mid
        return 0.5 * (lo + hi)

    def rms(self, f):
        return float(self.t.sqrt((self.area * f * f).sum() / self.area_sum))


def segmented_guess(Tp, ice, love, lmax, dt, threshold=0.01, start=None, c0=62.0, rhoi=920.0, rhow=1000.0,
                    radius=6.371e6, c_half=80.0, tol=1e-3, maxit=40, sht=None):
    """Return (T0 as a NumPy grid, info).  ``Tp``: present topography [nlat, nlon]; ``ice``: the
    ice states 0..N (NumPy grids or CUDA tensors; the last is the present); ``love``: an Earth
    model with ``he, ke, nmod, s, r, rprime`` (``LoveNumbers`` / ``SyntheticEarth``); ``dt``: kyr
    per step or the states' times in kyr; ``start``: starting T0 (default Tp).  Arguments as in
    the reference's ``segmented_guess``."""
    import torch

    from .sht import make_sht

    def dev(x):
        if isinstance(x, torch.Tensor):
            return x.to(device="cuda", dtype=torch.float64).contiguous()
        return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()

    Tp_d = dev(Tp)
    nl, no = Tp_d.shape
    N = len(ice) - 1
    g = _Grids(Tp_d, dev(ice[0]), dev(ice[N]), rhoi, rhow, radius, torch)
    V = np.array([float((dev(ice[n]) * g.area).sum()) for n in range(N + 1)])
    segs = segments(V, dt, threshold)
    sht = sht if sht is not None else make_sht("cuda", nl, no, lmax)
    l = np.arange(lmax + 1, dtype=float)
    ttl = np.zeros_like(l)
    ttl[1:] = 4 * np.pi * radius ** 3 / (MASS * (2 * l[1:] + 1))

    def operator(h, k):
        fac = torch.from_numpy(ttl * (1 + k - h)).cuda()[:, None]

        def apply(load):
            r = sht.synthesis(sht.analysis(load.contiguous()) * fac)
            return r - (r * g.area).sum() / g.area_sum
        return apply

    hk = [relaxed_love(love, lmax, sg["tau"]) for sg in segs]
    ops = [operator(h, k) for h, k in hk]
    w = np.abs([sg["dV"] for sg in segs])
    w = w / w.sum()
    if len(segs) == 1:
        water = ops[0]
    else:
        water = operator(sum(wi * h for wi, (h, k) in zip(w, hk)), sum(wi * k for wi, (h, k) in zip(w, hk)))
    Ib = [dev(ice[sg["a"]]) for sg in segs[1:]]
    dSL = torch.zeros_like(Tp_d) if start is None else dev(start) - Tp_d
    c = float(c0)
    ch = float("inf")
    it = 0
    for it in range(maxit):
        T0 = Tp_d + dSL
        g0, C0, dI = g.state(T0)
        dS = dSL * g.Cp - T0 * (g.Cp_f - C0.to(torch.float64))
        if len(segs) > 1:
            L = [g.I0 * g0] + [I * g.grounded(I, T0) for I in Ib] + [g.Ip * g.gp]
            Sx = -sum(op(rhoi * (L[j] - L[j + 1])) for j, op in enumerate(ops)) - water(-rhow * dS)
        else:
            Sx = -ops[0](rhoi * dI - rhow * dS)
        Sx = Sx.contiguous()
        cn = g.solve_c(Sx, c, c_half)
        new = cn + Sx
        ch = g.rms(new - dSL)
        dSL = new
        c = cn
        if ch < tol:
            break
    T0 = (Tp_d + dSL).cpu().numpy()
    return T0, {"segments": segs, "c": c, "iters": it + 1, "last_change_m": ch, "threshold": threshold,
                "dt_kyr": dt if np.ndim(dt) == 0 else [float(x) for x in dt], "lmax": lmax}
