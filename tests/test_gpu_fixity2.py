"""Prescribed-velocity fixity (code 2, MAIN.F90:447-470) on the resident
path against the oracle: a bar whose wall layer is fixed in z (code 1) and
whose top layer is driven in z through three windows, and in x on one side,
then released.  The windows are crossed inside the run, so the window
selection (strict inequalities on the step's start time), the zero velocity
outside every window and the reaction -FINT are all exercised."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu

STEPS = 120


def _driven_bar(semi=False):
    c = cases.taylor_bar(h=0.8e-3, L=12e-3, seed=4, v0=0.0)
    top = c["layer"] == c["layer"].max()
    ebc = c["ebc"].copy()
    ebc[top, 2] = 2
    ebc[top & (c["coo"][:, 0] > 0.0), 0] = 2
    c["ebc"] = ebc
    vin = c["vinit"].copy()
    vin[top, 2] = -1.0         # a code-2 DOF keeps its initial velocity until the first corrector
    c["vinit"] = vin
    kw = dict(lagrangian=0) if semi else {}
    return c, cases.param_kwargs(c, **kw)


def _windows(dt):
    # (t1, t2) in units of dt, displacement per window: z down, z up, x out
    t = np.array([[-0.5, 40.5], [40.5, 70.5], [85.5, 100.5]]) * dt
    d = np.array([[2.0e-6, 0.0, -8.0e-5], [0.0, 0.0, 2.0e-5], [-1.0e-6, 0.0, -1.0e-5]])
    return t, d


def _run(semi, mode):
    c, kw = _driven_bar(semi)
    m = mega.Mega(c, _lib.params(**kw))
    m.search_and_shapes()
    r = O.Run(c, O.params(**kw), nthreads=8)
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    t, d = _windows(dt)
    m.set_fixity2(t, d)
    r.set_fixity2(t, d)
    m.step(STEPS // 2, dt, mode=mode)
    m.step(STEPS - STEPS // 2, dt, mode=mode)   # a split run: the device time carries over
    r.step(STEPS, dt)
    return c, m, r, dt


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_prescribed_velocity_matches_oracle(mode):
    c, m, r, dt = _run(False, mode)
    tol = 1e-7 if mode == "fp64" else 2e-4
    x = m.download(_lib.F_COO_CURRENT)
    u, uo = x - c["coo"], r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(u - uo).max() <= tol * np.abs(uo).max()
    v = m.download(_lib.F_VEL).reshape(-1)
    assert np.abs(v - r.vel).max() <= tol * np.abs(r.vel).max()
    # the code-2 DOFs move exactly at the window velocities: after the last
    # window (t > 100.5 dt) they are at rest, and their reaction is -FINT
    e2 = c["ebc"].reshape(-1) == 2
    assert np.all(v[e2] == 0.0)
    pr = m.download(_lib.F_PRFORCE).reshape(-1)
    fi = m.download(_lib.F_FINT).reshape(-1)
    np.testing.assert_array_equal(pr[e2], -fi[e2])
    s = m.scalars()
    np.testing.assert_allclose(s["total_force"][:3], r.total_force[:3], rtol=tol * 10, atol=1e-9)
    m.close()


def test_prescribed_velocity_path_of_a_node():
    """The driven top layer's z displacement is the integral of the window
    velocities, step by step as the corrector assigns them (the first
    corrector runs at TIME = 0, outside the first window's open interval)."""
    c, kw = _driven_bar()
    m = mega.Mega(c, _lib.params(**kw))
    m.search_and_shapes()
    dt = 4.0e-8
    t, d = _windows(dt)
    m.set_fixity2(t, d)
    top = np.flatnonzero(c["layer"] == c["layer"].max())
    z = 0.0
    time = 0.0
    vz = c["vinit"][top[0], 2]
    for k in range(STEPS):
        m.step(1, dt)
        z += dt * vz                        # predictor with zero acceleration on the driven DOF
        w = [i for i in range(len(t)) if t[i, 0] < time < t[i, 1]]
        vz = d[w[0], 2] / (t[w[0], 1] - t[w[0], 0]) if w else 0.0
        time = time + dt
    dtot = m.download(_lib.F_DSP_TOT)
    np.testing.assert_allclose(dtot[top, 2], z, rtol=1e-12, atol=1e-18)
    m.close()


def test_prescribed_velocity_semi_lagrangian():
    c, m, r, dt = _run(True, "fp64")
    x = m.download(_lib.F_COO_CURRENT)
    u, uo = x - c["coo"], r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(u - uo).max() <= 1e-7 * np.abs(uo).max()
    m.close()


def test_fixity2_arguments():
    c, kw = _driven_bar()
    m = mega.Mega(c, _lib.params(**kw))
    with pytest.raises(_lib.MegaError):
        m.set_fixity2([[2.0, 1.0]], [[0.0, 0.0, 1.0]])   # a window that ends before it starts (READ.F90:265)
    m.close()
    plain = cases.taylor_bar(h=0.8e-3, L=12e-3, seed=4)
    q = mega.Mega(plain, _lib.params(**cases.param_kwargs(plain)))
    with pytest.raises(_lib.MegaError):
        q.set_fixity2([[0.0, 1.0]], [[0.0, 0.0, 1.0]])    # no DOF has code 2
    q.close()
