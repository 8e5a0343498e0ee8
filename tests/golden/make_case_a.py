"""Generate tests/golden/case_a.npz from the reference's sample deck.

Golden case A is the reference's own input: Taylor_bar.k (1,950 nodes,
1,536 hexahedra, node sets BAR and WALL) with the Control.dat deck.  This
script runs where the reference tree is mounted (it is not needed, and not
run, on a GPU box) and restates the pre-processing that turns the mesh into
the arrays the hot path consumes:
  *NODE / *ELEMENT_SOLID / *SET_NODE_LIST fixed-width reads  PRE_MODEL.F90:149-231
                                                             (taylor_b200/kfile.py)
  raw nodal windows = max element extent per axis            PRE_MODEL_ADIAL.F90:64-153
  nodal volumes = 1/8 of each adjacent hex (GET_VOL2)         PRE_MODEL_VOLUMES.F90:70-117,
                                                             PRE_MODEL_VOL2.F90:36-52
  the deck values the hot path uses (window 2.75, QL, props, v0, fixity, dt)
                                                             Control.dat, READ.F90:354-511
Usage: python tests/golden/make_case_a.py <reference_dir>   (the directory holding Taylor_bar.k)
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from taylor_b200 import kfile  # noqa: E402  the product's reader of the deck

HERE = os.path.dirname(os.path.abspath(__file__))


def det_abs(a):
    return abs(a[0, 0] * (a[1, 1] * a[2, 2] - a[2, 1] * a[1, 2]) + a[0, 1] * (a[2, 0] * a[1, 2] - a[1, 0] * a[2, 2])
               + a[0, 2] * (a[1, 0] * a[2, 1] - a[2, 0] * a[1, 1]))


def windows_and_volumes(coo, elems):
    n = len(coo)
    adial = np.zeros((n, 3))
    vol = np.zeros(n)
    for el in elems:
        xe = coo[el]                      # (8,3)
        ext = xe.max(0) - xe.min(0)       # max |x_k - x_j| over the element's nodes
        for k in el:
            adial[k] = np.maximum(adial[k], ext)
        # GET_VOL2: columns X7-X1; X2-X1 | X5-X1 | X4-X1; X3-X6 | X6-X8 | X8-X3
        x = xe
        A = np.stack([x[6] - x[0], x[1] - x[0], x[2] - x[5]], axis=1)
        B = np.stack([x[6] - x[0], x[4] - x[0], x[5] - x[7]], axis=1)
        Cm = np.stack([x[6] - x[0], x[3] - x[0], x[7] - x[2]], axis=1)
        dvol = (det_abs(A) + det_abs(B) + det_abs(Cm)) / 6.0
        vol[el] += 0.125 * dvol
    return adial, vol


def main(ref):
    deck = kfile.read_k(os.path.join(ref, "Taylor_bar.k"))
    coo, elems, sets = deck["coo"], deck["elems"], deck["sets"]
    win_raw, vol = windows_and_volumes(coo, elems)
    out = os.path.join(HERE, "case_a.npz")
    np.savez_compressed(out, coo=coo, win_raw=win_raw, vol=vol, elems=elems, bar=sets[1], wall=sets[2],
                        norm_win=2.75, v0=373.0, dt=0.78363e-07, time_end=5.5e-05, ql_coef=0.001,
                        props=np.array([0.3, 78.2e9, 2700.0, 0.29e9, 125.0, 0.1]), mat_type=2)
    print("wrote", out, "nodes", len(coo), "elements", len(elems), "wall", len(sets[2]))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_case_a.py <reference_dir>")
    main(sys.argv[1])
