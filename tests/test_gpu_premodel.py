"""Device mesh pre-processing against the oracle's restatement: windows and
volumes bit for bit (the reference's element-order sums), smoothing cells,
second moments and DIST_MAX to the last few ulps (pow differs)."""
import os

import numpy as np
import pytest

from oracle import premodel as P
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _check(coo, elems, norm_win=2.0):
    got = mega.pre_model_hex(coo, elems, norm_win=norm_win)
    w, v = P.hex_windows_and_volumes(coo, elems)
    np.testing.assert_array_equal(got["win_raw"], w)
    np.testing.assert_array_equal(got["vol"], v)
    np.testing.assert_array_equal(got["win"], w * norm_win)
    sm, mom, dmax = P.smoothing_lengths(v, w)
    np.testing.assert_allclose(got["sm_len"], sm, rtol=1e-14)
    np.testing.assert_allclose(got["mom"], mom, rtol=1e-14)
    np.testing.assert_allclose(got["dist_max"], dmax, rtol=1e-14)
    assert got["min_raw_window"] == w.min()
    return got


def test_case_a_mesh():
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "case_a.npz"))
    got = _check(d["coo"], d["elems"], norm_win=float(d["norm_win"]))
    np.testing.assert_array_equal(got["win_raw"], d["win_raw"])
    np.testing.assert_array_equal(got["vol"], d["vol"])


def test_jittered_hex_box():
    coo, elems = cases.hex_box(30, 24, 20, 0.4e-3, jitter=0.1, seed=5)
    _check(coo, elems)


def test_bad_connectivity_is_reported():
    coo, elems = cases.hex_box(4, 4, 4, 1e-3)
    bad = elems.copy()
    bad[3, 5] = len(coo) + 7
    got = mega.pre_model_hex(coo, bad, allow_status=True)
    assert got["status"] & _lib.ST_BAD_MESH


def test_mixed_hex_and_tet_blocks():
    """A box of hexahedra beside a block of tetrahedra (each hex of a second
    box split in five, the fourth node repeated): windows and volumes bit
    for bit against the oracle's element-order loops."""
    coo, elems = cases.hex_box(6, 6, 6, 1.0e-3, jitter=0.05, seed=5)
    n0 = len(coo)
    coo2, el2 = cases.hex_box(5, 5, 5, 1.0e-3, jitter=0.05, seed=6)
    coo2 = coo2 + np.array([7.0e-3, 0.0, 0.0])
    five = ((0, 1, 3, 4), (1, 2, 3, 6), (1, 4, 5, 6), (3, 4, 6, 7), (1, 3, 4, 6))
    tets = np.array([[h[a], h[b], h[c], h[d]] + [h[d]] * 4 for h in el2 for (a, b, c, d) in five]) + n0
    allc = np.concatenate([coo, coo2])
    alle = np.concatenate([elems, tets])
    et = np.concatenate([np.full(len(elems), 2), np.full(len(tets), 1)]).astype(np.int32)
    got = mega.pre_model(allc, alle, et, norm_win=2.0)
    w, v = P.windows_and_volumes(allc, alle, et)
    np.testing.assert_array_equal(got["win_raw"], w)
    np.testing.assert_array_equal(got["vol"], v)
    np.testing.assert_allclose(v[n0:].sum(), np.prod(coo2.max(axis=0) - coo2.min(axis=0)), rtol=0.2)
    hex_only = mega.pre_model_hex(coo, elems)
    np.testing.assert_array_equal(hex_only["vol"], got["vol"][:n0])
