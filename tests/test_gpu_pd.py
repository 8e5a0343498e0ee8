"""Peridynamics on the GPU against the oracle: the correspondence
CONSTRUCT_FINT_PD drop-in (FP64) and the bond-based PMB stepper (float force,
double positions)."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _pd_case():
    # millimetre units: INVERSE's absolute pivot test (D + 1 == 1,
    # INVERSE.F90:41) would call the SI-unit shape tensors (~1e-16) singular
    return cases.taylor_bar(h=0.8, R=3.2, L=10.0, seed=4, norm_win=2.2)


def test_construct_fint_pd_matches_oracle():
    c = _pd_case()
    n = c["n"]
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], 0, 1)
    op = O.params(**cases.param_kwargs(c, shsup=1, peridynamics=1))
    gp = _lib.params(**cases.param_kwargs(c, shsup=1, peridynamics=1))
    shp_o, ik_o, st = O.pd_shape(c, nb)
    assert st == 0
    z3 = np.zeros(3 * n)
    g0 = mega.construct_fint_pd(gp, c["coo"], c["coo"], c["win"], c["vol"], c["props"], c["mat_type"],
                                np.zeros((n, 20)), np.zeros((n, 6)), np.zeros((n, 6)), z3, nb["gn"], nb["gstart"],
                                nb["gstack"], np.zeros(nb["nnz"]), np.zeros((n, 3, 3)), True, 1e-8)
    np.testing.assert_allclose(g0["shp"], shp_o, rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(g0["ginvk"], ik_o, rtol=1e-10)
    # a deformed, plastic state: affine stretch plus noise
    rng = np.random.default_rng(3)
    u = (c["coo"] @ np.array([[0.01, 0.002, 0], [0, -0.004, 0], [0.003, 0, -0.02]]).T).ravel()
    u += rng.normal(scale=2e-7, size=3 * n)
    du = 0.05 * u
    cur = c["coo"].ravel() + u
    stress = rng.normal(scale=5e8, size=(n, 6))
    strain = rng.normal(scale=1e-3, size=(n, 6))
    state = np.zeros((n, 20))
    state[:, 2] = rng.uniform(0, 0.5, n)
    fo, wo, sto = O.construct_fint_pd(op, c, cur, sto_state := state.copy(), so := stress.copy(),
                                      eo := strain.copy(), du, nb, shp_o, ik_o, False, 1e-8)
    g = mega.construct_fint_pd(gp, c["coo"], cur, c["win"], c["vol"], c["props"], c["mat_type"], state, stress,
                               strain, du, nb["gn"], nb["gstart"], nb["gstack"], shp_o, ik_o, False, 1e-8)
    assert np.linalg.norm(g["fint"] - fo) <= 1e-10 * np.linalg.norm(fo)
    np.testing.assert_allclose(g["stress"], so, rtol=1e-9, atol=1e-3)
    np.testing.assert_allclose(g["state"][:, 2], sto_state[:, 2], rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(g["gmax_wvel"], wo, rtol=1e-9)


def _oracle_pmb(case, nb, broken, nsteps, dt):
    n = case["n"]
    u = np.zeros(3 * n)
    v = case["vinit"].ravel().copy()
    a = np.zeros(3 * n)
    for _ in range(nsteps):
        u = u + dt * v + 0.5 * dt * dt * a
        f, _ = O.pmb_force(case, nb, u, broken)
        an = f / case["rho"]
        v = v + 0.5 * dt * (a + an)
        a = an
    return u, v


def _plate_and_lists():
    # notch end between lattice bond midpoints, so the crossing test has no ties
    c = cases.pd_plate(h=0.5e-3, nx=40, ny=40, nz=4, notch=6.1e-3, v_edge=20.0)
    nb = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], 0, 1)
    got_nb = mega.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], 0, 1)
    np.testing.assert_array_equal(got_nb["gstack"], nb["gstack"])
    broken0 = cases.notch_broken(c, nb["gn"], nb["gstart"], nb["gstack"])
    assert broken0.sum() > 0
    dt = 0.5 * c["h"] / np.sqrt(72e9 / c["rho"])
    return c, nb, broken0, dt


def _pair_mismatch(nb, n, flags):
    rows = np.repeat(np.arange(n), nb["gn"])
    cols = nb["gstack"] - 1
    key = {(int(i), int(j)): k for k, (i, j) in enumerate(zip(rows, cols))}
    return sum(1 for k, (i, j) in enumerate(zip(rows, cols)) if flags[k] != flags[key[(int(j), int(i))]])


def test_pmb_device_cut_matches_host_notch():
    c, nb, broken0, dt = _plate_and_lists()
    p = mega.Pmb(c, None, mode="mixed")
    k = p.cut(*cases.notch_rect(c))
    flags, nbk = p.download(3)
    np.testing.assert_array_equal(flags.astype(np.uint8), broken0)
    assert k == int(broken0.sum())
    # a second cut over the same rectangle breaks nothing new
    assert p.cut(*cases.notch_rect(c)) == 0
    p.close()


def test_pmb_fp64_matches_oracle_exactly():
    c, nb, broken0, dt = _plate_and_lists()
    p = mega.Pmb(c, broken0, mode="fp64")
    assert p.nnz == nb["nnz"]
    nsteps = 300
    p.step(nsteps, dt)
    u, _ = p.download(0)
    flags, nbk = p.download(3)
    bo = broken0.copy()
    uo, vo = _oracle_pmb(c, nb, bo, nsteps, dt)
    assert bo.sum() > broken0.sum()  # bonds broke during the run
    np.testing.assert_array_equal(flags.astype(np.uint8), bo)
    assert np.abs(u - uo).max() <= 1e-9 * np.abs(uo).max()
    assert _pair_mismatch(nb, c["n"], flags) == 0  # both copies of a bond break together
    p.close()


def test_pmb_float_force_error_bound():
    """Float bond arithmetic: displacement within 1 % of the FP64 oracle and
    the broken-bond count within 3 % after 300 steps through fracture."""
    c, nb, broken0, dt = _plate_and_lists()
    p = mega.Pmb(c, broken0, mode="mixed")
    nsteps = 300
    p.step(nsteps, dt)
    u, _ = p.download(0)
    flags, nbk = p.download(3)
    bo = broken0.copy()
    uo, vo = _oracle_pmb(c, nb, bo, nsteps, dt)
    assert np.abs(u - uo).max() <= 1e-2 * np.abs(uo).max()
    newly_gpu = int(flags.sum() - broken0.sum())
    newly_orc = int(bo.sum() - broken0.sum())
    assert abs(newly_gpu - newly_orc) <= max(4, 0.03 * newly_orc)
    assert _pair_mismatch(nb, c["n"], flags) == 0
    p.close()
