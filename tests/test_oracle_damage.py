"""The damaged constitutive models of the oracle: DRUCK_PRAG (material 3,
CONSTITUTE_DRUCKPRAG.F90) and VON_MISES_DAM (material 6,
CONSTITUTE_VONMISES_DAM.F90).

The reference ships no test vectors for them, so the C restatement is pinned
to a second, line-by-line restatement in plain Python below (each written
from the Fortran on its own) and to properties the Fortran implies: no
damage below K_I, irreversibility through DAM_SV, the DAM_MAX cap, the
undamaged J2 limit equal to material 2, and the Drucker-Prager return onto
the yield surface for Q_PSI = 0.
"""
import math

import numpy as np

from oracle import oracle as O
from taylor_b200 import cases

S23 = math.sqrt(2.0 / 3.0)


def _norm(v):
    return math.sqrt(v[0] ** 2 + v[1] ** 2 + v[2] ** 2 + 2.0 * (v[3] ** 2 + v[4] ** 2 + v[5] ** 2))


def _dev(v):
    kk = v[0] + v[1] + v[2]
    return [v[0] - kk / 3.0, v[1] - kk / 3.0, v[2] - kk / 3.0, v[3], v[4], v[5]]


def _cmat_dot(pr, inc):
    lam, mu, l2m = pr[27], pr[28], pr[29]
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    c[0, 0] = c[1, 1] = c[2, 2] = l2m
    c[3, 3] = c[4, 4] = c[5, 5] = mu
    out = []
    for r in range(6):
        v = 0.0
        for k in range(6):
            v += c[r, k] * inc[k]
        out.append(v)
    return out


def _damage(tot, pr, dam, dsv):
    k_i, k_c, dmax = pr[8], pr[9], pr[10]
    eta = _norm(tot)
    if eta < dsv + k_i:
        pass
    elif k_i < eta < k_c:
        dam = k_c * (eta - k_i) / (eta * (k_c - k_i))
        dsv = eta
        dsv = dsv - k_i
    if dam > dmax:
        dam = dmax
    return dam, dsv


def py_von_mises_dam(stress, tot, inc, st, pr, maxit=20):
    nu, E, sig0, B, ce = pr[0], pr[1], pr[3], pr[4], pr[5]
    mu = E / (2.0 * (1.0 + nu))
    eps, dam, dsv = st[2], st[3], st[4]
    ci = _cmat_dot(pr, inc)
    eff = [stress[k] / (1.0 - dam) + ci[k] for k in range(6)]
    dev = _dev(eff)
    dam, dsv = _damage(tot, pr, dam, dsv)
    kk = eff[0] + eff[1] + eff[2]
    sph = [-kk / 3.0] * 3 + [0.0] * 3
    tn = _norm(dev)
    sig23 = S23 * sig0
    xk = sig23 * (1.0 + B * eps) ** ce
    if tn - xk > 0.0:
        dg, epst = 0.0, eps
        for i in range(1, maxit + 1):
            xk = sig23 * (1.0 + B * eps) ** ce
            y = tn - xk - 2.0 * mu * dg
            if abs(y) > sig23 * float(np.float32(1e-5)):
                xkp = B * ce * sig0 * (1.0 + B * eps) ** (ce - 1.0)
                dg = dg - y / (-2.0 * mu * (1.0 + xkp / 3.0 / mu))
            else:
                eps = epst + S23 * dg
                break
            eps = epst + S23 * dg
        dev = [d - dg * 2.0 * mu * d / tn for d in dev]
    out = st.copy()
    out[2], out[3], out[4] = eps, dam, dsv
    return np.array([(-sph[k] + dev[k]) * (1.0 - dam) for k in range(6)]), out


def py_druck_prag(stress, tot, inc, st, pr):
    nu, E = pr[0], pr[1]
    q_phi, k_phi, q_psi = pr[24], pr[25], pr[26]
    es, ev, eps, dam, dsv = st[0], st[1], st[2], st[3], st[4]
    ci = _cmat_dot(pr, inc)
    eff = [stress[k] / (1.0 - dam) + ci[k] for k in range(6)]
    dam, dsv = _damage(tot, pr, dam, dsv)
    dev = _dev(eff)
    tau_pre = _norm(dev)
    sph_pre = (eff[0] + eff[1] + eff[2]) / 3.0
    f = tau_pre + q_phi * sph_pre - k_phi
    if f < 0.0:
        s = list(eff)
    else:
        tau = k_phi - q_phi * sph_pre
        bulk, shear = E / (3.0 * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))
        gamma = f / (2.0 * shear + bulk * q_phi * q_psi)
        sph = sph_pre - bulk * q_psi * gamma
        s = [d * tau / tau_pre for d in dev]
        for k in range(3):
            s[k] = s[k] + sph
        es = es + gamma * math.sqrt(2.0 / 3.0 + 2.0 / 9.0 * q_psi ** 2)
        eps = eps + es
    out = st.copy()
    out[0], out[1], out[2], out[3], out[4] = es, ev, eps, dam, dsv
    return np.array([v * (1.0 - dam) for v in s]), out


def _props(mat, k_i=2e-3, k_c=5e-2, dmax=0.8, q_phi=0.3, k_phi=250e6, q_psi=0.1):
    pv = cases.props_vector(mat, 117e9, 0.35, 8930.0, 400e6, 0.25, 1.0)
    pv[8], pv[9], pv[10] = k_i, k_c, dmax
    pv[24], pv[25], pv[26] = q_phi, k_phi, q_psi
    return pv


def _inputs(n, seed, scale=3e-3):
    rng = np.random.default_rng(seed)
    stress = rng.normal(0.0, 150e6, (n, 6))
    tot = rng.normal(0.0, scale, (n, 6))
    inc = rng.normal(0.0, 4e-4, (n, 6))
    state = np.zeros((n, 20))
    state[:, 2] = rng.uniform(0.0, 0.2, n)
    state[:, 3] = rng.uniform(0.0, 0.5, n) * (rng.uniform(size=n) < 0.5)
    state[:, 4] = rng.uniform(0.0, 4e-3, n)
    state[:, 0] = rng.uniform(0.0, 0.05, n)
    return stress, tot, inc, state


def test_c_restatement_matches_python_restatement():
    for mat, py in ((6, py_von_mises_dam), (3, py_druck_prag)):
        pv = _props(mat)
        n = 400
        stress, tot, inc, state = _inputs(n, 10 + mat)
        got, gst, it, st = O.damaged(stress, tot, inc, np.full(n, mat), np.tile(pv, (n, 1)), state)
        assert st == 0
        plastic = 0
        for i in range(n):
            ref, rst = py(stress[i], tot[i], inc[i], state[i], pv)
            np.testing.assert_allclose(got[i], ref, rtol=1e-13, atol=1e-6)
            np.testing.assert_allclose(gst[i], rst, rtol=1e-13, atol=1e-18)
            plastic += it[i] > 0
        # both branches of each model are exercised
        assert 0.1 * n < plastic < 0.95 * n, plastic
        dam_changed = np.sum(gst[:, 3] != state[:, 3])
        assert dam_changed > 0.1 * n


def test_no_damage_below_threshold_and_undamaged_limit_is_j2():
    n = 200
    stress, tot, inc, state = _inputs(n, 3, scale=1e-4)
    state[:, 3] = state[:, 4] = 0.0
    pv6 = _props(6, k_i=1.0, k_c=2.0)  # thresholds far above the strains
    got, gst, it6, _ = O.damaged(stress, tot, inc, np.full(n, 6), np.tile(pv6, (n, 1)), state)
    assert np.all(gst[:, 3] == 0.0) and np.all(gst[:, 4] == 0.0)
    # with DAM = 0 the effective predictor is the elastic predictor and
    # VON_MISES_DAM reduces to VON_MISES
    ci = np.array([_cmat_dot(pv6, inc[i]) for i in range(n)])
    spred = stress + ci
    j2, jst, it2, _ = O.constitution(spred, np.full(n, 2), np.tile(pv6, (n, 1)), 0.0, state)
    np.testing.assert_allclose(got, j2, rtol=1e-14, atol=1e-6)
    np.testing.assert_array_equal(gst[:, 2], jst[:, 2])
    np.testing.assert_array_equal(it6, it2)


def test_damage_is_irreversible_and_capped():
    pv = _props(6, k_i=1e-3, k_c=1e-1, dmax=0.5)
    one = np.zeros((1, 6))

    def walk(path):
        st = np.zeros((1, 20))
        dams = []
        for eta in path:
            tot = np.array([[eta, 0, 0, 0, 0, 0]])
            _, st, _, _ = O.damaged(one, tot, one, [6], pv[None, :], st)
            dams.append(st[0, 3])
        return np.array(dams)

    dams = walk([1.1e-3, 1.3e-3, 1.2e-3, 1.05e-3, 1.5e-3, 3e-3, 1e-3])
    assert np.all(np.diff(dams) >= 0.0)          # unloading never heals
    assert dams[1] == dams[2] == dams[3]          # below DAM_SV + K_I: frozen
    assert dams[4] > dams[3]                      # reloading past it: grows
    assert dams[5] == 0.5 and dams[6] == 0.5      # DAM_MAX cap, kept
    k_c, k_i, eta = 1e-1, 1e-3, 1.3e-3
    assert dams[1] == k_c * (eta - k_i) / (eta * (k_c - k_i))
    # eta above K_C takes no branch: the damage stays where it was, as written
    assert walk([2e-1])[0] == 0.0


def test_drucker_prager_return_lands_on_the_surface_without_dilatancy():
    pv = _props(3, k_i=1.0, k_c=2.0, q_phi=0.4, k_phi=150e6, q_psi=0.0)
    n = 300
    stress, tot, inc, state = _inputs(n, 7, scale=1e-4)
    state[:, 3] = 0.0
    got, gst, it, _ = O.damaged(stress, tot, inc, np.full(n, 3), np.tile(pv, (n, 1)), state)
    ci = np.array([_cmat_dot(pv, inc[i]) for i in range(n)])
    eff = stress + ci
    p_pre = eff[:, :3].sum(1) / 3.0
    for i in np.nonzero(it)[0]:
        d = _dev(got[i])
        p = got[i, :3].sum() / 3.0
        assert abs(p - p_pre[i]) <= 1e-9 * abs(p_pre[i]) + 1.0     # no dilatancy: pressure kept
        f = _norm(d) + pv[24] * p - pv[25]
        assert abs(f) <= 1e-9 * pv[25]
    elastic = it == 0
    np.testing.assert_allclose(got[elastic], eff[elastic], rtol=1e-15, atol=1e-6)
    assert 0 < elastic.sum() < n


def test_construct_fint_with_damaged_materials_runs_clean():
    for mat, kw in ((6, {}), (3, dict(q_phi=0.3, k_phi=300e6, q_psi=0.1))):
        c = cases.with_damage(cases.taylor_bar(h=1.0e-3), mat, 1e-3, 5e-2, 0.9, **kw)
        p = cases.param_kwargs(c)
        r = O.Run(c, O.params(**p), nthreads=4)
        dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
        r.step(30, dt)
        assert np.all(np.isfinite(r.coo_cur))
        assert r.state[:, 3].max() > 0.0       # damage grew at the impact face
        assert r.state[:, 2].max() > 0.0       # and plastic flow happened
