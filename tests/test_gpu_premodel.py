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
