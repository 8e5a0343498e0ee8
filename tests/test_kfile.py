"""The keyword-deck reader (taylor_b200/kfile.py) with the reference's
fixed-width rules, and the pre-processing oracle on a tetrahedral block."""
import os

import numpy as np

from oracle import premodel as P
from taylor_b200 import kfile

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "case_a.npz")


def _deck(coo, blocks, sets):
    """A deck in the layout of the reference's Taylor_bar.k: *NODE records
    (I8, 3F16.0, 2I8), one *ELEMENT_SOLID card per block (10I8), node sets
    (8I10).  blocks: list of (E, 8) 1-based connectivity arrays."""
    out = ["*KEYWORD", "$ written by the test", "*NODE", "$    nid               x               y               z"]
    for i, x in enumerate(coo):
        out.append(f"{i + 1:8d}" + "".join(f"{repr(float(v)):>16s}" for v in x) + f"{0:8d}{0:8d}")
    eid = 0
    for b, el in enumerate(blocks):
        out.append("*ELEMENT_SOLID")
        for e in el:
            eid += 1
            out.append(f"{eid:8d}{b + 1:8d}" + "".join(f"{int(v):8d}" for v in e))
    for sid, ids in sets.items():
        out.append("*SET_NODE_LIST")
        out.append(f"{sid:10d}")
        for k in range(0, len(ids), 8):
            out.append("".join(f"{int(v):10d}" for v in ids[k:k + 8]))
    out.append("*END")
    return "\n".join(out) + "\n"


def test_reads_golden_case_a_arrays():
    z = np.load(GOLDEN)
    text = _deck(z["coo"], [z["elems"] + 1], {1: z["bar"], 2: z["wall"]})
    d = kfile.read_k(text)
    np.testing.assert_array_equal(d["coo"], z["coo"])
    np.testing.assert_array_equal(d["elems"], z["elems"])
    np.testing.assert_array_equal(d["sets"][2], z["wall"])
    assert list(d["block_type"]) == [2] and np.all(d["eltype"] == 2)


def test_tet_block_rule_and_oracle():
    # a unit cube as a hex block and, beside it, a tetrahedral block whose
    # elements repeat their fourth node (LS-DYNA's degenerate form)
    coo = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1],
                    [2, 0, 0], [2, 1, 0], [2, 0, 1]], float)
    hexes = np.array([[1, 2, 3, 4, 5, 6, 7, 8]])
    tets = np.array([[2, 9, 10, 11, 11, 11, 11, 11], [2, 3, 10, 11, 11, 11, 11, 11]])
    d = kfile.read_k(_deck(coo, [hexes, tets], {}))
    assert list(d["block_type"]) == [2, 1]
    assert list(d["eltype"]) == [2, 1, 1]
    w, v = P.windows_and_volumes(d["coo"], d["elems"], d["eltype"])
    # volumes: the cube splits 1/8 to each corner; each tetrahedron 1/4 of
    # its volume to each of its four nodes
    t1 = abs(np.linalg.det(np.array([coo[10] - coo[9], coo[1] - coo[9], coo[8] - coo[9]]))) / 6.0
    t2 = abs(np.linalg.det(np.array([coo[10] - coo[9], coo[1] - coo[9], coo[2] - coo[9]]))) / 6.0
    np.testing.assert_allclose(v[0], 0.125)
    np.testing.assert_allclose(v[8], 0.25 * t1)
    np.testing.assert_allclose(v[1], 0.125 + 0.25 * (t1 + t2))
    np.testing.assert_allclose(v.sum(), 1.0 + t1 + t2)
    np.testing.assert_array_equal(w[8], [1.0, 1.0, 1.0])   # extents of its tetrahedron's four nodes
    np.testing.assert_array_equal(w[4], [1.0, 1.0, 1.0])
