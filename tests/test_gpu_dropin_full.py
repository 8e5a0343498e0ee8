"""The force subroutines with the reference's own argument lists
(construct_fint_gpu: FINT.F90:16-25, construct_fint_pd_gpu: FINT_PD.F90:
16-25), called as gfortran calls them (every argument by reference,
column-major arrays): equal to the short-list drop-ins where those apply,
and against the oracle on the paths only the full list reaches -- NSNI
(ITYPE_INT = 2, GSTACK_DDSHP and LOCAL_DX/DY/DZ_STRESS) and the
semi-Lagrangian call on GCOO_CUURENT."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _state_after(c, kw, steps=25):
    """A plastic mid-impact state from the oracle (its lists, shapes, state)."""
    r = O.Run(c, O.params(**kw), nthreads=8)
    dt = cases.stable_dt(c, r.nb["gn"], r.nb["gstart"], r.nb["gstack"])
    r.step(steps, dt)
    return r, dt


def test_full_list_equals_short_list():
    c = cases.taylor_bar(h=0.8e-3, L=16e-3)
    kw = cases.param_kwargs(c)
    r, dt = _state_after(c, kw)
    n = c["n"]
    en = np.any(c["ebc"] == 1, axis=1).astype(np.int32)
    st20 = r.state.copy()
    a = mega.construct_fint(_lib.params(**kw), c["coo"], c["win"], c["vol"], c["props"], c["mat_type"], en, st20,
                            r.stress, r.strain, r.dsp, r.dsp_tot, r.nb["gn"], r.nb["gstart"], r.nb["gstack"], r.shp,
                            r.dshp.reshape(-1, 3), False, dt)
    b = mega.construct_fint_full(_lib.params(**kw), c["coo"], c["win"], c["vol"], c["props"], c["mat_type"], en,
                                 st20, r.stress, r.strain, r.dsp, r.dsp_tot, r.nb["gn"], r.nb["gstart"],
                                 r.nb["gstack"], r.shp, r.dshp.reshape(-1, 3), False, dt, sm_len=c["sm_len"])
    for k in ("fint", "fext", "stress", "strain", "state", "gmax_wvel", "gstrain_eq"):
        np.testing.assert_array_equal(a[k], b[k])
    assert b["dlt_fint"] == -1.0  # untouched, as CONSTRUCT_FINT leaves it (FINT.F90:1250-1330 commented out)
    assert np.all(b["ddshp"] == 0.0) and n > 0


def test_full_list_nsni_matches_oracle():
    c = cases.taylor_bar(h=0.8e-3, L=16e-3)
    kw = cases.param_kwargs(c, itype_int=2)
    p = _lib.params(**kw)
    op = O.params(**kw)
    n = c["n"]
    en = np.any(c["ebc"] == 1, axis=1).astype(np.int32)
    # LINIT through the full list: shapes and second derivatives written
    nb = mega.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], itype_int=2)
    nnz = nb["nnz"]
    z = np.zeros(3 * n)
    got0 = mega.construct_fint_full(p, c["coo"], c["win"], c["vol"], c["props"], c["mat_type"], en,
                                    np.zeros((n, 20)), np.zeros((n, 6)), np.zeros((n, 6)), z, z, nb["gn"],
                                    nb["gstart"], nb["gstack"], np.zeros(nnz), np.zeros((nnz, 3)), True, 0.0,
                                    sm_len=c["sm_len"])
    r, dt = _state_after(c, kw)
    np.testing.assert_array_equal(nb["gstack"], r.nb["gstack"])
    assert np.abs(got0["ddshp"].ravel() - r.ddshp).max() <= 1e-9 * np.abs(r.ddshp).max()
    assert np.abs(got0["dshp"].ravel() - r.dshp).max() <= 1e-12 * np.abs(r.dshp).max()
    # one step's call from the oracle's mid-impact state, its own second derivatives
    sg = r.sgrad.copy()
    got = mega.construct_fint_full(p, c["coo"], c["win"], c["vol"], c["props"], c["mat_type"], en, r.state,
                                   r.stress, r.strain, r.dsp, r.dsp_tot, r.nb["gn"], r.nb["gstart"], r.nb["gstack"],
                                   r.shp, r.dshp.reshape(-1, 3), False, dt, sm_len=c["sm_len"],
                                   ddshp=r.ddshp.reshape(-1, 6), sgrad=sg)
    st, sx, sn = r.state.copy(), r.stress.copy(), r.strain.copy()
    sgo = r.sgrad.copy()
    ref = O.construct_fint(op, c, st, sx, sn, r.dsp, r.dsp_tot, r.nb, r.shp.copy(), r.dshp.copy(), False, dt,
                           nthreads=8, ddshp=r.ddshp.copy(), sgrad=sgo)
    rel = np.linalg.norm(got["fint"] - ref["fint"]) / np.linalg.norm(ref["fint"])
    assert rel <= 1e-9, rel
    assert np.abs(got["stress"] - sx).max() <= 1e-9 * np.abs(sx).max()
    assert np.abs(got["sgrad"] - sgo).max() <= 1e-8 * np.abs(sgo).max()


def test_full_list_semi_lagrangian_matches_oracle():
    c = cases.taylor_bar(h=0.8e-3, L=16e-3)
    kw = cases.param_kwargs(c, lagrangian=0)
    r, dt = _state_after(c, kw, steps=10)
    en = np.any(c["ebc"] == 1, axis=1).astype(np.int32)
    cur = r.coo_cur.reshape(-1, 3).copy()
    got = mega.construct_fint_full(_lib.params(**kw), c["coo"], c["win"], c["vol"], c["props"], c["mat_type"], en,
                                   r.state, r.stress, r.strain, r.dsp, r.dsp_tot, r.nb["gn"], r.nb["gstart"],
                                   r.nb["gstack"], np.zeros(r.nb["nnz"]), np.zeros((r.nb["nnz"], 3)), False, dt,
                                   coo_current=cur)
    st, sx, sn = r.state.copy(), r.stress.copy(), r.strain.copy()
    shp, dshp = np.zeros(r.nb["nnz"]), np.zeros(3 * r.nb["nnz"])
    ref = O.construct_fint(O.params(**kw), c, st, sx, sn, r.dsp, r.dsp_tot, r.nb, shp, dshp, False, dt, nthreads=8,
                           coo_current=cur)
    assert np.abs(got["shp"] - shp).max() <= 1e-12
    rel = np.linalg.norm(got["fint"] - ref["fint"]) / np.linalg.norm(ref["fint"])
    assert rel <= 1e-9, rel


def test_full_list_pd_equals_short_list_and_time_step():
    # millimetre units, as the short-list PD tests use (INVERSE's absolute
    # pivot test would call SI-unit shape tensors singular)
    c = cases.taylor_bar(h=0.8, R=3.2, L=10.0, seed=4, norm_win=2.2)
    n, coo = c["n"], c["coo"]
    kw = cases.param_kwargs(c, peridynamics=1, shsup=1, auto_ts=1, dlt_fac=0.7)
    p = _lib.params(**kw)
    nb = mega.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"], shsup=True)
    rng = np.random.default_rng(4)
    cur = coo + rng.normal(scale=2e-3, size=coo.shape)
    dinc = rng.normal(scale=1e-4, size=3 * n)
    z = dict(state=np.zeros((n, 20)), stress=np.zeros((n, 6)), strain=np.zeros((n, 6)))
    a = mega.construct_fint_pd(p, coo, cur, c["win"], c["vol"], c["props"], c["mat_type"], z["state"], z["stress"],
                               z["strain"], dinc, nb["gn"], nb["gstart"], nb["gstack"], np.zeros(nb["nnz"]),
                               np.zeros((n, 3, 3)), True, 1e-8)
    b = mega.construct_fint_pd_full(p, coo, cur, c["win"], c["vol"], c["props"], c["mat_type"], z["state"],
                                    z["stress"], z["strain"], dinc, nb["gn"], nb["gstart"], nb["gstack"],
                                    np.zeros(nb["nnz"]), np.zeros((n, 3, 3)), True, 1e-8)
    for k in ("fint", "stress", "strain", "gmax_wvel", "shp", "ginvk"):
        np.testing.assert_array_equal(a[k], b[k])
    # AUTO_TS: nearest current neighbour over the wave speed, smallest, times DLT_FAC
    rows = np.repeat(np.arange(n), nb["gn"])
    cols = nb["gstack"] - 1
    d = np.linalg.norm(cur[cols] - cur[rows], axis=1)
    d[cols == rows] = np.inf
    dmin = np.full(n, np.inf)
    np.minimum.at(dmin, rows, d)
    np.testing.assert_allclose(b["gchar_dist"], dmin, rtol=1e-15)
    np.testing.assert_allclose(b["dlt_fint"], 0.7 * np.min(dmin / b["gmax_wvel"]), rtol=1e-15)


def test_fortran_calling_convention_program(tmp_path):
    """A gcc-built C program that calls construct_fint_gpu as gfortran
    would (tests/fortran_abi_check.c) and checks it against the short-list
    drop-in bit for bit."""
    import subprocess
    from test_abi import _build_fortran_abi_check
    exe = _build_fortran_abi_check(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK")
