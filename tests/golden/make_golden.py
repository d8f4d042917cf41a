"""Generates tests/golden/bump_17x9x9.npz: the oracle's level-1 residual after
start-up and its first 10 cycle residual norms on the 17x9x9-node bump case;
and bump_17x9x9_ddadi.npz: the first 10 residual norms with the DDADI
implicit stage (LUSGS=0).

These are regression pins of the oracle itself (the reference ships no golden
vectors and cannot be compiled here).  Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from finflo_b200 import case  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402
from tests.util import interior  # noqa: E402


def main():
    blk, prm, fs = case.bump_case(17, 9, 9)
    o = Oracle(blk, prm)
    o.start()
    o.statim(); o.adjuin(); o.residu(1, 1)
    out = {"res_" + n: interior(blk, blk.arrays[n]).copy() for n in ("DRO", "DM", "DN", "DW", "DE")}
    out["hist10"] = np.array([o.cycle(i + 1)[0] for i in range(10)])
    here = os.path.dirname(os.path.abspath(__file__))
    np.savez_compressed(os.path.join(here, "bump_17x9x9.npz"), **out)
    blk, prm, fs = case.bump_case(17, 9, 9)
    prm.ddadi = 1
    o = Oracle(blk, prm)
    o.start()
    hist = np.array([o.cycle(i + 1)[0] for i in range(10)])
    np.savez_compressed(os.path.join(here, "bump_17x9x9_ddadi.npz"), hist10=hist)


if __name__ == "__main__":
    main()
