"""Regenerates the golden fixtures under tests/golden/.

setup_ref.npz: shape tables (normals, areas, Laplace basis, ellipsoid fit)
produced by the reference's OWN setup sources (trifac.c, areanorm.c,
sphfunc.c, ellfit.c, ludcmp.c, lubksb.c), compiled by oracle/Makefile into
oracle/_ref/libref_setup.so.  Needs the reference tree to rebuild that library.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

CASES = [(3, 3, 2), (4, 2, 3), (6, 6, 3)]


def main():
    out = {}
    for lm, mm, nrows in CASES:
        tabs = oracle.setup_shape(lm, mm, nrows, 1.2, 1.0, 0.85, reference=True)
        for name, arr in zip(("normal", "darea", "dsph", "cg"), tabs):
            out[f"case_{lm}_{mm}_{nrows}_{name}"] = arr
    np.savez_compressed(os.path.join(HERE, "setup_ref.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
