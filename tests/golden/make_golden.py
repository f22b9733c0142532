"""Regenerate the P_N golden fixtures from the reference's validation data.

Reads ``code/validationData/{AxPlus,AxMinus,AyPlus,AyMinus}.csv`` (64 x 64, the
nPN = 7 flux-matrix splittings A+- = (A +- |A|)/2 shipped with the reference)
and stores them as float64 in ``pn_golden.npz`` beside this script. The
argument is the root of a TITUS checkout (the directory holding ``code/``):

    python tests/golden/make_golden.py <path-to-TITUS-checkout>
"""
import os
import sys

import numpy as np


def main(ref_root: str) -> None:
    src = os.path.join(ref_root, "code", "validationData")
    out = {}
    for name in ("AxPlus", "AxMinus", "AyPlus", "AyMinus"):
        out[name] = np.loadtxt(os.path.join(src, name + ".csv"), delimiter=",")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pn_golden.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path-to-TITUS-checkout>")
    main(sys.argv[1])
