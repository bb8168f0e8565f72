"""Generate the golden fixtures of the parity tests from the CPU oracle.

The oracle is pinned by the reference's published known answers
(tests/test_oracle_kat.py); these fixtures freeze its outputs for a few small
cases so that a change in either implementation shows up as a diff.
Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.rcwa_oracle import OfdSetup, RcwaLayerSpec as L, RcwaPole, rcwa_run  # noqa: E402

CASES = {
    "grating_1d_16f": OfdSetup(nHx=5, period_x=3e-7, layers=[L(1, 1, .5, 0), L(4, 1, .5, 2e-7), L(2.25, 2.25, .5, 0)],
                               freqs=np.linspace(4.3e14, 7.5e14, 16)),
    "rect2d_conical": OfdSetup(nHx=3, period_x=5e-7, nHy=3, period_y=4e-7,
                               layers=[L(1, 1, .5, 0), L(2.25, 1, .6, 2e-7, 0, 0, .6), L(6.0, 1, .3, 1e-7, .2, 0, .8),
                                       L(2.25, 2.25, .5, 0)],
                               freqs=[3.5e14, 4.5e14], theta=35.0, phi=20.0),
    "drude_film": OfdSetup(nHx=2, period_x=5e-7, layers=[L(1, 1, .5, 0), L(1, 1, .5, 3e-8), L(2.25, 2.25, .5, 0)],
                           freqs=[4e14, 5.5e14, 7e14],
                           poles=[RcwaPole(1, 1, 1.0, 1.36e16, 3.0e13, 0.0), RcwaPole(1, 2, 1.0, 1.36e16, 3.0e13, 0.0)]),
}


def main():
    for name, s in CASES.items():
        out = rcwa_run(s)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), freqs=np.array([r["freq"] for r in out]),
                            R=np.array([r["R"] for r in out]), T=np.array([r["T"] for r in out]),
                            ordR=np.array([r["ordR"] for r in out]), ordT=np.array([r["ordT"] for r in out]))
        print(name)


if __name__ == "__main__":
    main()
