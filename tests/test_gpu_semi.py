"""Semi-Lagrangian stepping (LLAGRANGIAN = .FALSE.) on the GPU against the
oracle: lists re-searched on the current coordinates in the LINIT bins and
shapes rebuilt on them every step."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _pair(c, **kw):
    p = cases.param_kwargs(c, lagrangian=0, **kw)
    m = mega.Mega(c, _lib.params(**p))
    r = O.Run(c, O.params(**p), nthreads=8)
    return m, r, p


def test_semi_lagrangian_linit_lists_bit_exact():
    c = cases.taylor_bar(h=0.8e-3)
    m, r, _ = _pair(c)
    got = m.search_and_shapes(download=True)
    np.testing.assert_array_equal(got["gn"], r.nb["gn"])
    np.testing.assert_array_equal(got["gstack"], r.nb["gstack"])
    assert np.abs(got["shp"] - r.shp).max() <= 1e-12
    m.close()


def test_semi_lagrangian_matches_oracle():
    c = cases.taylor_bar(h=0.8e-3)
    m, r, _ = _pair(c)
    m.search_and_shapes()
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    nnz0 = r.nb["nnz"]
    m.step(60, dt)
    r.step(60, dt)
    assert r.nb["nnz"] != nnz0  # the lists really were rebuilt
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max()
    v = m.download(_lib.F_VEL).reshape(-1)
    assert np.abs(v - r.vel).max() <= 1e-6 * np.abs(r.vel).max()
    eps = m.download(_lib.F_EPS)
    assert r.state[:, 2].max() > 0.0
    assert np.abs(eps - r.state[:, 2]).max() <= 1e-6 * r.state[:, 2].max()
    s = m.scalars()
    assert abs(s["kin_energy"] - r.en[1]) <= 1e-8 * r.en[1]
    assert abs(s["int_energy"] - r.en[0]) <= 1e-6 * r.en[0]
    m.close()


def test_semi_lagrangian_differs_from_lagrangian():
    c = cases.taylor_bar(h=0.8e-3)
    m, r, _ = _pair(c)
    m.search_and_shapes()
    lag = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    lag.search_and_shapes()
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    m.step(60, dt)
    lag.step(60, dt)
    xs, xl = m.download(_lib.F_COO_CURRENT), lag.download(_lib.F_COO_CURRENT)
    assert np.abs(xs - xl).max() > 1e-3 * np.abs(xl - c["coo"]).max()
    m.close()
    lag.close()


def test_semi_lagrangian_refuses_what_it_does_not_build():
    c = cases.taylor_bar(h=1.0e-3)
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c, lagrangian=0)))
    m.search_and_shapes()
    with pytest.raises(_lib.MegaError):  # FP64 only
        m.step(1, 3e-8, mode="mixed")
    with pytest.raises(_lib.MegaError):  # no tiled gathers to tune
        m.autotune(3e-8)
    m.close()
    with pytest.raises(_lib.MegaError):  # DNI only
        mega.Mega(c, _lib.params(**cases.param_kwargs(c, lagrangian=0, itype_int=2)))
