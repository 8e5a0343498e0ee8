"""The C++ oracle against a second restatement of the same Fortran written
independently in numpy (oracle/second.py): the RK shapes of golden case A
(the reference's own deck), and a few explicit steps of the Lagrangian DNI
loop from impact (force, stress, plastic strain, displacement, velocity).
Agreement to rounding pins the oracle's transcription of RK1, INV3,
HUGHES_WINGET, ROTATE_TENSOR, VON_MISES, the FINT.F90 scatter and MAIN's
integrator independently of either restatement."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import second as S
from taylor_b200 import cases


@pytest.fixture(scope="module")
def runs(case_a):
    c = case_a
    p = O.params(**cases.param_kwargs(c))
    r = O.Run(c, p, nthreads=1)
    s = S.Step(c, r.nb, ql=True, ql_coef=0.001, ql_len=c["ql_len"])
    return c, r, s


def test_shapes_agree(runs):
    c, r, s = runs
    assert np.abs(s.shp - r.shp).max() <= 1e-13 * np.abs(r.shp).max()
    d = r.dshp.reshape(-1, 3)
    assert np.abs(s.dshp - d).max() <= 1e-13 * np.abs(d).max()


def test_steps_agree(runs):
    c, r, s = runs
    for k in range(6):
        r.step(1, c["dt"])
        s.step(c["dt"])
        f = r.fint
        assert np.abs(s.fint - f).max() <= 1e-11 * np.abs(f).max(), k
        assert np.abs(s.stress - r.stress).max() <= 1e-11 * np.abs(r.stress).max(), k
    assert np.abs(s.eps - r.state[:, 2]).max() <= 1e-11 * max(r.state[:, 2].max(), 1e-30)
    u, uo = s.coo_cur - c["coo"].reshape(-1), r.coo_cur - c["coo"].reshape(-1)
    assert np.abs(u - uo).max() <= 1e-13 * np.abs(uo).max()
    assert np.abs(s.vel - r.vel).max() <= 1e-12 * np.abs(r.vel).max()
    assert r.state[:, 2].max() > 0.0  # the impact is plastic after six steps


def test_second_restatement_kernels():
    """INV3 returns det^2 A^-1 as written; Hughes-Winget's rotation is
    orthogonal in exact arithmetic for the exact inverse (here, for small L,
    det ~ 1 so INV3 ~ the inverse)."""
    rng = np.random.default_rng(2)
    A = np.eye(3) + 0.1 * rng.normal(size=(50, 3, 3))
    inv = np.linalg.inv(A)
    det = np.linalg.det(A)
    np.testing.assert_allclose(S.inv3(A), inv * (det ** 2)[:, None, None], rtol=1e-12, atol=1e-14)
    L = 1e-4 * rng.normal(size=(50, 3, 3))
    R, _, _ = S.hughes_winget(L)
    RtR = np.einsum("nij,nik->njk", R, R)
    assert np.abs(RtR - np.eye(3)).max() < 1e-7
