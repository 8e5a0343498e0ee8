"""Resident runs against the oracle under the switches the Taylor bar's
defaults leave untouched: small-strain kinematics, the exact INV3, the
spherical support, gravity and nodal body forces, mass-proportional
damping, two bodies (the split reaction sums), QL off."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _variant(name):
    c = cases.taylor_bar(h=0.8e-3, seed=3)
    kw = {}
    if name == "small_strain":
        kw["finite_strain"] = 0
    elif name == "inv3_exact":
        kw["inv3_exact"] = 1
    elif name == "spherical_support":
        kw["shsup"] = 1
    elif name == "gravity_and_body_force":
        kw["gravity"] = (0.0, 2.0e5, -5.0e5)
        rng = np.random.default_rng(9)
        c["bodyforce"] = rng.normal(scale=1.0e5, size=(c["n"], 3))
    elif name == "damping":
        pr = c["props"].copy()
        pr[:, 20] = 2.0e5
        c["props"] = pr
    elif name == "two_bodies":
        c["body_id"] = np.where(c["coo"][:, 0] > 0.0, 2, 1).astype(np.int32)
    elif name == "ql_off":
        kw["ql"] = 0
    return c, cases.param_kwargs(c, **kw)


@pytest.mark.parametrize("name", ["small_strain", "inv3_exact", "spherical_support", "gravity_and_body_force",
                                  "damping", "two_bodies", "ql_off"])
def test_variant_matches_oracle(name):
    c, p = _variant(name)
    m = mega.Mega(c, _lib.params(**p))
    m.search_and_shapes()
    r = O.Run(c, O.params(**p), nthreads=8)
    dt = 0.8 * cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    m.step(40, dt)
    r.step(40, dt)
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max(), name
    v = m.download(_lib.F_VEL).reshape(-1)
    assert np.abs(v - r.vel).max() <= 1e-6 * np.abs(r.vel).max(), name
    if r.state[:, 2].max() > 0.0:
        assert np.abs(m.download(_lib.F_EPS) - r.state[:, 2]).max() <= 1e-6 * r.state[:, 2].max(), name
    fe = m.download(_lib.F_FEXT).reshape(-1)
    assert np.abs(fe - r.fext).max() <= 1e-7 * max(np.abs(r.fext).max(), 1e-30), name
    s = m.scalars()
    tf, tfo = np.array(s["total_force"]), np.asarray(r.total_force)
    assert np.abs(tf - tfo).max() <= 1e-6 * max(np.abs(tfo).max(), 1e-30), name
    if name == "two_bodies":
        assert np.abs(tfo[:3]).max() > 0.0 and np.abs(tfo[3:]).max() > 0.0
    assert abs(s["kin_energy"] - r.en[1]) <= 1e-8 * r.en[1], name
    assert abs(s["ext_energy"] - r.en[2]) <= 1e-6 * max(abs(r.en[2]), 1e-30) + 1e-12, name
    m.close()
