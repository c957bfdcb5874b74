#!/usr/bin/env python3
"""Generate the golden fixtures of this directory by running the REFERENCE SLEvolve Python code.

    python tests/golden/make_golden.py --reference /path/to/slevolve-checkout

The reference package (``<checkout>/python/slevolve``) is imported read-only; nothing of it is
copied.  Its outputs on seeded inputs are written as compressed ``.npz`` fixtures so that the
tests (here and on GPU hosts, which have no reference checkout) can pin both the CPU oracle
(``oracle/``) and the CUDA path against the reference itself.

Fixtures
--------
``sht.npz``          ``sht.SHT`` (sht.py:148-343) and ``gaulw`` on four grids: nodes, weights,
                     analysis of a random grid, synthesis of random coefficients.
``memory.npz``       ``ExactMemory`` (solver.py:244-506): 30 advance/commit cycles with
                     non-uniform steps on a random 8-mode Earth, lmax 12.
``step_c0.npz``      ``SeaLevelSolver`` (plain) on the c0 configuration (64 x 128, L = 63,
                     100 steps of 1 yr) and ``OptSeaLevelSolver(opt={numba,sums,dsl},
                     inner="extrap")`` on the same inputs.
``step_marine.npz``  ``SeaLevelSolver`` on a marine polar cap (64 x 128, L = 63, 8 steps of
                     1 kyr; the idealised geometry of the reference's tests/test_small_case.py:
                     floating ice, grounded re-guess, shoreline migration).
``step_c1s.npz``     ``SeaLevelSolver`` on the c1 generator at 64 x 128, L = 63, 60 steps
                     (marine dome thinned by 1-20 m/yr: grounding-line retreat).
``synthetic512.npz`` inputs of the reference's own synthetic case (topography seed, Love file
                     ``prem_512.l96C.ump3.lm1``) and a subsample plus row/column sums of the
                     reference's shipped golden grid ``reference/synthetic/tgrid8.npy``
                     (512 x 1024, L = 511, 8 steps, ``--opt all --inner extrap``).
``golden_meta.json`` provenance and the oracle-vs-reference summaries.
"""

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, REPO)

STEPS_SAVED_C0 = (1, 10, 50, 100)
STEPS_SAVED_C1S = (1, 30, 60)
SYNTH_POLAR = [3000.0, 2625.0, 2250.0, 1875.0, 1500.0, 1125.0, 750.0, 375.0, 0.0]
SYNTH_MIDLAT = [2500.0, 2400.0, 2150.0, 1800.0, 1350.0, 900.0, 500.0, 200.0, 0.0]


def love_arrays(love, lmax):
    K = int(love.max_modes)
    nl = lmax + 1
    return {"love_s": love.s[:K, :nl].copy(), "love_r": love.r[:K, :nl].copy(),
            "love_rprime": love.rprime[:K, :nl].copy(), "love_rT": love.rT[:K, :nl].copy(),
            "love_rprimeT": love.rprimeT[:K, :nl].copy(), "love_he": love.he[:nl].copy(),
            "love_ke": love.ke[:nl].copy(), "love_hTE": love.hTE[:nl].copy(),
            "love_kTE": love.kTE[:nl].copy(), "love_nmod": np.asarray(love.nmod[:nl], np.int64)}


def run_solver(cls, sht, love, topo, ice_fn, nsteps, lmax, dt, saved, **kw):
    slv = cls(sht, love, topo, ice_fn(0), norder=lmax, dt=dt, **kw)
    out = {"numiter": [], "gmslc_ocn": [], "gmslc_ocnBeta": [], "ocean_area": [],
           "oceanBeta_area": [], "ice_volume": [], "mm": [], "il": [], "lambda": []}
    fields = {}
    for k in range(1, nsteps + 1):
        r = slv.step(np.ascontiguousarray(ice_fn(k)))
        for key in ("numiter", "gmslc_ocn", "gmslc_ocnBeta", "ocean_area", "oceanBeta_area",
                    "ice_volume"):
            out[key].append(r[key])
        out["mm"].append(r["mm"].copy())
        out["il"].append(r["il"].copy())
        out["lambda"].append(r["lambda"].copy())
        if k in saved:
            fields[f"tgrid_{k}"] = r["tgrid"].copy()
            fields[f"R_{k}"] = r["R"].copy()
            fields[f"ocean_{k}"] = np.packbits(r["ocean"].astype(bool))
            fields[f"beta_{k}"] = np.packbits(r["beta"].astype(bool))
            if k == nsteps:
                fields[f"dS_{k}"] = r["dS_converged"].copy()
    res = {k: np.asarray(v) for k, v in out.items()}
    res.update(fields)
    res["step0_scalars"] = np.array([slv.ocean_area0, slv.oceanBeta_area0, slv.ice_volume0])
    return res


def marine_geometry(gaulats, nlon):
    """Idealised polar marine cap of the reference's tests/test_small_case.py:86-92 (restated)."""
    colat = np.degrees(np.arccos(gaulats))[:, None] * np.ones((1, nlon))
    topo = np.where(colat <= 20.0, 300.0 - 1100.0 * colat / 20.0, -800.0)
    topo = np.where(colat > 25.0, -4000.0,
                    np.where(colat > 20.0, -800.0 - 640.0 * (colat - 20.0), topo))
    shape = np.sqrt(np.clip(1.0 - (colat / 14.0) ** 2, 0.0, None))
    heights = [0.0, 300.0, 700.0, 1000.0, 1000.0, 800.0, 400.0, 150.0, 0.0]
    return topo, shape, heights


def synthetic512_ice(gaulats, topo, nlon):
    """Ice of the reference's synthetic case (tools/make_synthetic_case.py:66-79, 178-190):
    Vialov sheets at the south pole (R 17 deg) and 56 N 132 E (R 12 deg) on bed above -500 m."""
    from slevolve_b200.synthetic import angular_distance, grid_latlon, round_mm, vialov
    LAT, LON = grid_latlon(gaulats, nlon)
    polar = vialov(90.0 + LAT, 17.0)
    mid = vialov(angular_distance(LAT, LON, 56.0, 132.0), 12.0)
    grounded = topo > -500.0
    return [round_mm((hp * polar + hm * mid) * grounded) for hp, hm in zip(SYNTH_POLAR, SYNTH_MIDLAT)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="SLEvolve checkout whose python/slevolve package is imported read-only")
    ap.add_argument("--skip512", action="store_true", help="skip the L=511 oracle run")
    a = ap.parse_args()
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache_golden")
    sys.dont_write_bytecode = True
    sys.path.insert(0, os.path.join(a.reference, "python"))
    from slevolve.sht import SHT, gaulw
    from slevolve.solver import ExactMemory, LoveNumbers, NPAM, SeaLevelSolver
    from slevolve.solver_opt import OptSeaLevelSolver
    from slevolve_b200.synthetic import case_c0, case_c1
    from oracle.sht import OracleSHT
    from oracle.solver import OracleSolver
    meta = {"generated": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
            "numpy": np.__version__, "reference": "SLEvolve python/slevolve (imported read-only)"}

    # ---------------------------------------------------------------- SHT
    rng = np.random.default_rng(424242)
    sht_fx = {}
    for (n, L) in ((16, 15), (32, 31), (32, 20), (64, 63)):
        s = SHT(n, 2 * n, L)
        z, w = gaulw(n)
        g = rng.standard_normal((n, 2 * n))
        c = np.tril(rng.standard_normal((L + 1, L + 1)) + 1j * rng.standard_normal((L + 1, L + 1)))
        c[:, 0] = c[:, 0].real
        tag = f"n{n}_l{L}"
        sht_fx[f"{tag}_nodes"] = z
        sht_fx[f"{tag}_weights"] = w
        sht_fx[f"{tag}_grid"] = g
        sht_fx[f"{tag}_ana"] = s.analysis(g, out=np.zeros((L + 1, L + 1), complex)).copy()
        sht_fx[f"{tag}_coef"] = c
        sht_fx[f"{tag}_syn"] = s.synthesis(c, out=np.zeros((n, 2 * n))).copy()
    np.savez_compressed(os.path.join(HERE, "sht.npz"), **sht_fx)

    # ------------------------------------------------------------- memory
    rng = np.random.default_rng(12345)
    lmax, kmax, nsteps = 12, 8, 30
    nl = lmax + 1

    class _Love:
        pass

    love = _Love()
    love.nmod = np.zeros(nl, dtype=np.int64)
    love.s = np.zeros((NPAM, nl))
    love.r, love.rprime, love.rT, love.rprimeT = (np.zeros((NPAM, nl)) for _ in range(4))
    for l in range(1, nl):
        nm = kmax if l == 2 else int(rng.integers(1, kmax + 1))
        love.nmod[l] = nm
        love.s[:nm, l] = 10.0 ** rng.uniform(-2, 2, nm)
        for arr in (love.r, love.rprime, love.rT, love.rprimeT):
            arr[:nm, l] = rng.normal(size=nm)
    love.max_modes = int(love.nmod.max())
    love.he, love.ke, love.hTE, love.kTE = (np.zeros(nl) for _ in range(4))
    st = ExactMemory(love, lmax, 1.0, True)
    dts = rng.uniform(1.0, 2000.0, nsteps)
    mem = {"dts": dts, "lmax": lmax}
    mem.update({k: v for k, v in love_arrays(love, lmax).items() if "love_h" not in k and "love_k" not in k})
    loads, visc, rad, sil, sm, stsl, strr = [], [], [], [], [], [], []
    for n in range(nsteps):
        st.set_dt(dts[n])
        v, r_, a1, a2, a3, a4 = st.advance_and_read()
        visc.append(v.copy()); rad.append(r_.copy()); sil.append(a1.copy()); sm.append(a2.copy())
        stsl.append(a3.copy()); strr.append(a4.copy())
        Ld = np.tril(rng.normal(size=(nl, nl)) + 1j * rng.normal(size=(nl, nl)))
        Ld[0, :] = 0.0
        il = np.zeros((3, 3)); il[:, 2] = rng.normal(size=3)
        m = rng.normal(size=3)
        lam = rng.normal(size=3) + 1j * rng.normal(size=3)
        st.commit(Ld, il, m, lam)
        loads.append((Ld, il, m, lam))
    mem.update({"load": np.array([x[0] for x in loads]), "dil": np.array([x[1] for x in loads]),
                "dm": np.array([x[2] for x in loads]), "dlam": np.array([x[3] for x in loads]),
                "visc": np.array(visc), "rad": np.array(rad), "sum_il": np.array(sil),
                "sum_m": np.array(sm), "sum_tsl": np.array(stsl), "sum_trr": np.array(strr)})
    np.savez_compressed(os.path.join(HERE, "memory.npz"), **mem)

    # ------------------------------------------------------------- step c0
    t0 = time.time()
    n, L = 64, 63
    ref_sht = SHT(n, 2 * n, L)
    orc_sht = OracleSHT(n, 2 * n, L)
    case = case_c0(orc_sht)
    topo_mm = np.round(case.topo * 1000.0).astype(np.int64)
    assert np.array_equal(topo_mm / 1000.0, case.topo)
    fx = {"topo_mm": topo_mm}
    fx.update(love_arrays(case.love, L))
    plain = run_solver(SeaLevelSolver, ref_sht, case.love, case.topo, case.ice, 100, L, 1.0, STEPS_SAVED_C0)
    fx.update({f"plain_{k}": v for k, v in plain.items()})
    opt = run_solver(OptSeaLevelSolver, ref_sht, case.love, case.topo, case.ice, 100, L, 1.0,
                     (1, 100), opt={"numba", "sums", "dsl"}, inner="extrap")
    fx.update({f"extrap_{k}": v for k, v in opt.items()})
    np.savez_compressed(os.path.join(HERE, "step_c0.npz"), **fx)
    # oracle vs reference on the same inputs
    orc = OracleSolver(orc_sht, case.love, case.topo, case.ice(0), norder=L, dt=1.0)
    worst = 0.0
    ni = []
    for k in range(1, 101):
        r = orc.step(case.ice(k))
        ni.append(r["numiter"])
        if k in STEPS_SAVED_C0:
            worst = max(worst, float(np.abs(r["tgrid"] - plain[f"tgrid_{k}"]).max()))
    meta["c0_oracle_vs_reference_plain"] = {"max_abs_tgrid_m": worst,
                                            "numiter_equal": bool(np.array_equal(ni, plain["numiter"]))}
    meta["c0_seconds"] = time.time() - t0

    # ---------------------------------------------------------- marine cap
    topo, shape, heights = marine_geometry(ref_sht.gaulats, 2 * n)
    ice = [h * shape for h in heights]
    fx = {"topo": topo}
    love = LoveNumbers(os.path.join(a.reference, "lovenum", "prem_512.l96C.ump3.lm1"), L)
    fx.update(love_arrays(love, L))
    fx["ice_heights"] = np.array(heights)
    res = run_solver(SeaLevelSolver, ref_sht, love, topo, lambda k: ice[k], 8, L, 1000.0, (1, 2, 4, 8))
    fx.update({f"plain_{k}": v for k, v in res.items()})
    np.savez_compressed(os.path.join(HERE, "step_marine.npz"), **fx)

    # ---------------------------------------------------- c1 generator, small
    case = case_c1(orc_sht, nsteps=60)
    topo_mm = np.round(case.topo * 1000.0).astype(np.int64)
    assert np.array_equal(topo_mm / 1000.0, case.topo)
    fx = {"topo_mm": topo_mm}
    fx.update(love_arrays(case.love, L))
    rate_probe = case.ice(1) - case.ice(0)
    fx["ice_probe"] = np.array([float(np.abs(case.ice(k)).sum()) for k in range(61)])
    res = run_solver(SeaLevelSolver, ref_sht, case.love, case.topo, case.ice, 60, L, 1.0, STEPS_SAVED_C1S)
    fx.update({f"plain_{k}": v for k, v in res.items()})
    np.savez_compressed(os.path.join(HERE, "step_c1s.npz"), **fx)
    meta["c1s_numiter"] = [int(x) for x in res["numiter"]]
    meta["c1s_rate_probe"] = float(np.abs(rate_probe).max())

    # ------------------------------------------------- reference synthetic L=511
    seed = np.load(os.path.join(a.reference, "reference", "synthetic", "topography_seed.npy"))
    tg8 = np.load(os.path.join(a.reference, "reference", "synthetic", "tgrid8.npy"))
    topo_mm = np.round(seed * 1000.0).astype(np.int64)
    assert np.array_equal(topo_mm / 1000.0, seed)
    love = LoveNumbers(os.path.join(a.reference, "lovenum", "prem_512.l96C.ump3.lm1"), 511)
    fx = {"topo_mm": topo_mm.astype(np.int32), "polar": np.array(SYNTH_POLAR),
          "midlat": np.array(SYNTH_MIDLAT)}
    fx.update(love_arrays(love, 511))
    fx["tgrid8_sub"] = tg8[::8, ::8].copy()
    fx["tgrid8_rowsum"] = tg8.sum(axis=1)
    fx["tgrid8_colsum"] = tg8.sum(axis=0)
    fx["numiter_doc"] = np.array([5, 5, 6, 6, 5, 5, 5, 5])
    if not a.skip512:
        t1 = time.time()
        osht = OracleSHT(512, 1024, 511, workers=os.cpu_count() or 1)
        ice = synthetic512_ice(osht.gaulats, seed, 1024)
        fx["ice_abs_sums"] = np.array([float(np.abs(x).sum()) for x in ice])
        orc = OracleSolver(osht, love, seed, ice[0], norder=511, dt=1.0, opt={"dsl"}, inner="extrap")
        ni = []
        for k in range(1, 9):
            r = orc.step(ice[k])
            ni.append(r["numiter"])
        meta["synthetic512_oracle"] = {
            "max_abs_vs_tgrid8_m": float(np.abs(r["tgrid"] - tg8).max()),
            "numiter": ni, "seconds": time.time() - t1}
    np.savez_compressed(os.path.join(HERE, "synthetic512.npz"), **fx)
    with open(os.path.join(HERE, "golden_meta.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
