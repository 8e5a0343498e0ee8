"""The damaged constitutive models on the GPU against the oracle:
VON_MISES_DAM (material 6) and DRUCK_PRAG (material 3), resident in both
precisions and through the CONSTRUCT_FINT / CONSTRUCT_FINT_PD drop-ins
(GSTATE(1, 2, 4, 5) carried through the call)."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu

MODELS = {
    6: dict(k_i=1e-3, k_c=5e-2, dam_max=0.9),
    3: dict(k_i=1e-3, k_c=5e-2, dam_max=0.9, q_phi=0.3, k_phi=300e6, q_psi=0.1),
}
AUX = [0, 1, 3, 4]  # STATE(1, 2, 4, 5)


def _case(mat, h=0.8e-3):
    return cases.with_damage(cases.taylor_bar(h=h), mat, **MODELS[mat])


@pytest.mark.parametrize("mat", [6, 3])
def test_resident_fp64_matches_oracle(mat):
    c = _case(mat)
    p = cases.param_kwargs(c)
    m = mega.Mega(c, _lib.params(**p))
    m.search_and_shapes()
    r = O.Run(c, O.params(**p), nthreads=8)
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    m.step(60, dt)
    r.step(60, dt)
    aux = m.download(_lib.F_STATE_AUX)
    ref = r.state[:, AUX]
    assert ref[:, 2].max() > 0.1 and (ref[:, 2] > 0).sum() > 50   # damage grew
    np.testing.assert_allclose(aux, ref, rtol=1e-6, atol=1e-9 * np.abs(ref).max())
    eps = m.download(_lib.F_EPS)
    assert r.state[:, 2].max() > 0.0
    assert np.abs(eps - r.state[:, 2]).max() <= 1e-6 * r.state[:, 2].max()
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max()
    s = m.download(_lib.F_STRESS)
    assert np.abs(s - r.stress).max() <= 1e-6 * np.abs(r.stress).max()
    m.close()


@pytest.mark.parametrize("mat", [6, 3])
def test_resident_mixed_close_to_oracle(mat):
    c = _case(mat)
    p = cases.param_kwargs(c)
    m = mega.Mega(c, _lib.params(**p))
    m.search_and_shapes()
    r = O.Run(c, O.params(**p), nthreads=8)
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    m.step(60, dt, mode="mixed")
    r.step(60, dt)
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-3 * np.abs(uo).max()
    dam, dam_o = m.download(_lib.F_STATE_AUX)[:, 2], r.state[:, 3]
    assert abs(dam.mean() - dam_o.mean()) <= 1e-3 * dam_o.mean()
    assert abs(dam.max() - dam_o.max()) <= 1e-3 * dam_o.max()
    m.close()


def test_state_aux_round_trip_and_absent_without_damage():
    c = _case(6, h=1.0e-3)
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    m.search_and_shapes()
    a = np.random.default_rng(1).uniform(0.0, 1e-3, (c["n"], 4))
    m.upload(_lib.F_STATE_AUX, a)
    np.testing.assert_array_equal(m.download(_lib.F_STATE_AUX), a)   # through the node renumbering
    m.close()
    j2 = cases.taylor_bar(h=1.0e-3)
    m = mega.Mega(j2, _lib.params(**cases.param_kwargs(j2)))
    with pytest.raises(_lib.MegaError):
        m.download(_lib.F_STATE_AUX)
    m.close()


@pytest.mark.parametrize("mat", [6, 3])
def test_construct_fint_dropin_carries_damage_state(mat):
    c = _case(mat, h=1.0e-3)
    p = cases.param_kwargs(c)
    op = O.params(**p)
    r = O.Run(c, op, nthreads=8)
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    r.step(40, dt)
    dsp = dt * r.vel + dt * dt * 0.5 * r.acl
    dsp_tot = r.dsp_tot + dsp
    st0, sg0, se0 = r.state.copy(), r.stress.copy(), r.strain.copy()
    assert st0[:, 3].max() > 0.0
    ost, osg, ose = st0.copy(), sg0.copy(), se0.copy()  # updated in place by the oracle
    ref = O.construct_fint(op, c, ost, osg, ose, dsp, dsp_tot, r.nb, r.shp, r.dshp, False, dt)
    en = np.any(c["ebc"] == 1, axis=1).astype(np.int32)
    got = mega.construct_fint(_lib.params(**p), c["coo"], c["win"], c["vol"], c["props"], c["mat_type"], en, st0,
                              sg0, se0, dsp, dsp_tot, r.nb["gn"], r.nb["gstart"], r.nb["gstack"], r.shp,
                              r.dshp.reshape(-1, 3), False, dt)
    rel = np.linalg.norm(got["fint"] - ref["fint"]) / np.linalg.norm(ref["fint"])
    assert rel <= 1e-9, rel
    assert np.any(ost[:, 3] != st0[:, 3])       # damage moved in the call
    np.testing.assert_allclose(got["state"][:, AUX + [2]], ost[:, AUX + [2]], rtol=1e-9, atol=1e-14)
    np.testing.assert_allclose(got["stress"], osg, rtol=1e-9, atol=1e-6)
    np.testing.assert_allclose(got["gmax_wvel"], ref["gmax_wvel"], rtol=1e-8)


@pytest.mark.parametrize("mat", [6, 3])
def test_construct_fint_pd_dropin_damaged(mat):
    c = cases.taylor_bar(h=0.8, R=3.2, L=10.0, seed=4, norm_win=2.2)  # millimetre units
    c = cases.with_damage(c, mat, 1e-4, 5e-2, 0.9, q_phi=0.3, k_phi=3e8, q_psi=0.1)
    n = c["n"]
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], 0, 1)
    kw = cases.param_kwargs(c, shsup=1, peridynamics=1)
    op, gp = O.params(**kw), _lib.params(**kw)
    shp_o, ik_o, st = O.pd_shape(c, nb)
    assert st == 0
    rng = np.random.default_rng(3)
    u = (c["coo"] @ np.array([[0.01, 0.002, 0], [0, -0.004, 0], [0.003, 0, -0.02]]).T).ravel()
    u += rng.normal(scale=2e-7, size=3 * n)
    du = 0.05 * u
    cur = c["coo"].ravel() + u
    stress = rng.normal(scale=5e8, size=(n, 6))
    strain = rng.normal(scale=1e-3, size=(n, 6))
    state = np.zeros((n, 20))
    state[:, 2] = rng.uniform(0, 0.5, n)
    state[:, 3] = rng.uniform(0, 0.3, n)
    state[:, 4] = rng.uniform(0, 1e-3, n)
    so, eo, sto = stress.copy(), strain.copy(), state.copy()
    fo, wo, _ = O.construct_fint_pd(op, c, cur, sto, so, eo, du, nb, shp_o, ik_o, False, 1e-8)
    g = mega.construct_fint_pd(gp, c["coo"], cur, c["win"], c["vol"], c["props"], c["mat_type"], state, stress,
                               strain, du, nb["gn"], nb["gstart"], nb["gstack"], shp_o, ik_o, False, 1e-8)
    assert np.any(sto[:, 3] != state[:, 3])       # damage moved in the call
    assert np.linalg.norm(g["fint"] - fo) <= 1e-10 * np.linalg.norm(fo)
    np.testing.assert_allclose(g["stress"], so, rtol=1e-9, atol=1e-3)
    np.testing.assert_allclose(g["state"][:, AUX + [2]], sto[:, AUX + [2]], rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(g["gmax_wvel"], wo, rtol=1e-9)
