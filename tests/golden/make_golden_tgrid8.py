#!/usr/bin/env python3
"""Copy the reference's shipped L = 511 golden grid into a compressed fixture.

    python tests/golden/make_golden_tgrid8.py --reference /path/to/slevolve-checkout

``reference/synthetic/tgrid8.npy`` of the reference checkout is the topography after 8 steps of its
synthetic case (512 x 1024 Gauss grid, L = 511, ``--opt all --inner extrap``; its inputs are in
``synthetic512.npz``).  It is stored whole, so the tests compare every cell, as the reference's own
test does (tests/test_fortran_synthetic.sh, 1e-9 m).  Writes ``tgrid8.npz`` beside this script.
"""

import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="SLEvolve checkout (read-only)")
    a = ap.parse_args()
    tg = np.load(os.path.join(a.reference, "reference", "synthetic", "tgrid8.npy"))
    assert tg.shape == (512, 1024) and tg.dtype == np.float64
    np.savez_compressed(os.path.join(HERE, "tgrid8.npz"), tgrid8=tg)


if __name__ == "__main__":
    main()
