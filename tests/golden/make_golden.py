"""Regenerates tests/golden/k0_lkh8_nu045.txt from the reference's own fixture.

The reference ships tests/1.K: the 24x24 stiffness of a unit hex8 element with
E = 1, nu = 0.45 (tests/testMaterial.txt), in the node order of the closed-form
lk_H8 (matlab/homogenize.m:121-167): counter-clockwise bottom face, then top.
This script reads it as text (row, col, value triplets after two size lines)
and writes the dense matrix, one row per line.  It needs the reference tree
and is run by hand; the committed output is what the tests read.

usage: python tests/golden/make_golden.py <path-to-reference-tree>
       (or set FEMH_REFERENCE_TREE)
"""
import os
import sys

import numpy as np


def main(ref_root: str) -> None:
    toks = open(os.path.join(ref_root, "tests", "1.K")).read().split()
    n, m = int(toks[0]), int(toks[1])
    vals = np.array(toks[2:], dtype=float).reshape(-1, 3)
    K = np.zeros((n, m))
    for i, j, v in vals:
        K[int(i), int(j)] = v
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "k0_lkh8_nu045.txt")
    with open(out, "w") as f:
        f.write("# 24x24 hex8 stiffness, E=1 nu=0.45 h=1, lk_H8 node order; from the reference's tests/1.K\n")
        for row in K:
            f.write(" ".join(repr(float(x)) for x in row) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FEMH_REFERENCE_TREE")
    if not tree:
        sys.exit("usage: make_golden.py <path-to-reference-tree>  (or set FEMH_REFERENCE_TREE)")
    main(tree)
