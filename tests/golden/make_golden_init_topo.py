#!/usr/bin/env python3
"""Golden fixture of the segmented initial-topography guess, made by running the REFERENCE.

    python tests/golden/make_golden_init_topo.py --reference /path/to/slevolve-checkout

The reference's ``slevolve.init_topo_segmented.segmented_guess`` (init_topo_segmented.py:101-146)
is imported read-only and run on the seeded glacial-cycle case of ``slevolve_b200.synthetic``
(64 x 128, L = 63, 13 ice states), generated with the oracle's transform.  Two substitutions, both
at the reference's own seams: its transform factory ``sht_ducc.make_sht`` (ducc0 is not installed
here) returns the reference's NumPy ``slevolve.sht.SHT``, which the reference holds to 1e-13 of
ducc (sht_ducc.py:34); and its ``LoveNumbers`` file reader returns the case's seeded synthetic
Earth.  Cases: uniform 10-kyr steps; non-uniform times with threshold 0.05 and a start T0.

Writes ``init_topo.npz`` (inputs, T0, c, iteration counts, legs) beside this script.
"""

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="SLEvolve checkout whose python/slevolve package is imported read-only")
    a = ap.parse_args()
    sys.dont_write_bytecode = True
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(a.reference, "python"))
    import slevolve.init_topo_segmented as its
    import slevolve.sht as rsht
    import slevolve.sht_ducc as sd
    from oracle.sht import OracleSHT
    from slevolve_b200.synthetic import case_glacial

    topo, ice, love = case_glacial(OracleSHT(64, 128, 63))
    sd.make_sht = lambda backend, nl, no, lmax, workers=1, chunk=16, raw=False: rsht.SHT(nl, no, lmax)
    its.LoveNumbers = lambda path, lmax: love
    out = {"topo": topo, "ice": np.stack(ice)}
    times = np.cumsum(np.r_[0.0, np.linspace(6.0, 14.0, len(ice) - 1)]) - 120.0
    start = topo + 0.001 * np.round(1000.0 * (5.0 * np.cos(np.arange(topo.size).reshape(topo.shape) * 1e-3)))
    cases = {"uniform": dict(dt=10.0, threshold=0.01, start=None),
             "times": dict(dt=times, threshold=0.05, start=start)}
    out["times"] = times
    out["start"] = start
    for name, kw in cases.items():
        T0, info = its.segmented_guess(topo, ice, "synthetic-earth", 63, kw["dt"], threshold=kw["threshold"],
                                       start=kw["start"])
        out[f"{name}_T0"] = T0
        out[f"{name}_c"] = np.array(info["c"])
        out[f"{name}_iters"] = np.array(info["iters"])
        out[f"{name}_last_change"] = np.array(info["last_change_m"])
        out[f"{name}_legs"] = np.array([[sg["a"], sg["b"]] for sg in info["segments"]])
        out[f"{name}_tau"] = np.array([sg["tau"] for sg in info["segments"]])
        out[f"{name}_dV"] = np.array([sg["dV"] for sg in info["segments"]])
        print(name, info["iters"], info["c"], [(sg["a"], sg["b"]) for sg in info["segments"]], flush=True)
    np.savez_compressed(os.path.join(HERE, "init_topo.npz"), **out)


if __name__ == "__main__":
    main()
