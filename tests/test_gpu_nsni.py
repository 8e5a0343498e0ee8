"""Naturally stabilised nodal integration (ITYPE_INT = 2) on the GPU against
the oracle: the resident run in FP64 and mixed mode, the stress gradients
it carries, and the entry points that refuse it."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _run_both(c, steps, mode="fp64", **kw):
    p = cases.param_kwargs(c, itype_int=2, **kw)
    m = mega.Mega(c, _lib.params(**p))
    m.search_and_shapes()
    r = O.Run(c, O.params(**p), nthreads=8)
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    dt = cases.stable_dt(c, nb["gn"], nb["gstart"], nb["gstack"])
    m.step(steps, dt, mode=mode)
    r.step(steps, dt)
    return m, r


def test_nsni_resident_fp64_matches_oracle():
    c = cases.taylor_bar(h=0.8e-3)
    m, r = _run_both(c, 60)
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max()
    sg = m.download(_lib.F_NSNI_SGRAD)
    assert np.abs(r.sgrad).max() > 0.0
    assert np.abs(sg - r.sgrad).max() <= 1e-6 * np.abs(r.sgrad).max()
    eps = m.download(_lib.F_EPS)
    assert np.abs(eps - r.state[:, 2]).max() <= 1e-6 * r.state[:, 2].max()
    s = m.scalars()
    assert abs(s["int_energy"] - r.en[0]) <= 1e-6 * r.en[0]
    assert abs(s["kin_energy"] - r.en[1]) <= 1e-8 * r.en[1]
    m.close()


def test_nsni_differs_from_dni():
    """The stabilisation is really applied: the same bar without it ends
    elsewhere."""
    c = cases.taylor_bar(h=0.8e-3)
    m, r = _run_both(c, 60)
    d = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    d.search_and_shapes()
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    dt = cases.stable_dt(c, nb["gn"], nb["gstart"], nb["gstack"])
    d.step(60, dt)
    xn, xd = m.download(_lib.F_COO_CURRENT), d.download(_lib.F_COO_CURRENT)
    assert np.abs(xn - xd).max() > 1e-3 * np.abs(xd - c["coo"]).max()
    m.close()
    d.close()


def test_nsni_resident_mixed_close_to_oracle():
    c = cases.taylor_bar(h=0.8e-3)
    m, r = _run_both(c, 60, mode="mixed")
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-4 * np.abs(uo).max()
    sg = m.download(_lib.F_NSNI_SGRAD)
    assert np.linalg.norm(sg - r.sgrad) <= 1e-3 * np.linalg.norm(r.sgrad)
    m.close()


def test_nsni_refused_where_it_has_no_state():
    c = cases.taylor_bar(h=1.0e-3)
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], 2, 0)
    n = c["n"]
    z3 = np.zeros(3 * n)
    en = np.any(c["ebc"] == 1, axis=1).astype(np.int32)
    with pytest.raises(_lib.MegaError):  # the drop-in's argument list has no room for NSNI's arrays
        mega.construct_fint(_lib.params(**cases.param_kwargs(c, itype_int=2)), c["coo"], c["win"], c["vol"],
                            c["props"], c["mat_type"], en, np.zeros((n, 20)), np.zeros((n, 6)), np.zeros((n, 6)),
                            z3, z3, nb["gn"], nb["gstart"], nb["gstack"], np.zeros(nb["nnz"]),
                            np.zeros((nb["nnz"], 3)), True, 0.0)
    with pytest.raises(_lib.MegaError):  # SNNI is not built
        mega.Mega(c, _lib.params(**cases.param_kwargs(c, itype_int=1)))
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    with pytest.raises(_lib.MegaError):  # DNI context: no stress gradients
        m.download(_lib.F_NSNI_SGRAD)
    m.close()


def test_config1_bar_1000_steps_matches_oracle():
    """The 16,154-node bar (0.4 mm lattice, +-5 % jitter) with stabilised
    nodal integration for its full 1,000 steps from impact: the end-state
    length, mushroom radius and peak plastic strain of the GPU within 0.5 %
    of the oracle in FP64, and the mixed run within 1e-3 of the FP64 run on
    length and peak plastic strain."""
    import os
    c = cases.taylor_bar(h=0.4e-3)
    p = cases.param_kwargs(c, itype_int=2)
    r = O.Run(c, O.params(**p), nthreads=os.cpu_count() or 8)
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    dt = cases.stable_dt(c, nb["gn"], nb["gstart"], nb["gstack"])
    r.step(1000, dt)
    ref = cases.bar_metrics(c, r.coo_cur.reshape(-1, 3), r.state[:, 2])
    got = {}
    for mode in ("fp64", "mixed"):
        m = mega.Mega(c, _lib.params(**p))
        m.search_and_shapes()
        m.step(1000, dt, mode=mode)
        got[mode] = cases.bar_metrics(c, m.download(_lib.F_COO_CURRENT), m.download(_lib.F_EPS))
        m.close()
    for k in ("length", "radius", "peak_eps"):
        assert abs(got["fp64"][k] - ref[k]) <= 5e-3 * abs(ref[k]), (k, got["fp64"][k], ref[k])
    for k in ("length", "peak_eps"):
        assert abs(got["mixed"][k] - got["fp64"][k]) <= 1e-3 * abs(got["fp64"][k]), (k, got["mixed"][k])
    assert ref["length"] < 0.95 * c["L"] and ref["peak_eps"] > 0.5  # a real impact, not a rest state
