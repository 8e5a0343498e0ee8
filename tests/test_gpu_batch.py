"""Many bars in one context (instances searched apart, stepped together)
against the same bars in their own contexts."""
import numpy as np
import pytest

from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _batch(nbars=3):
    return cases.batch_bars(nbars, seed=3, h_range=(0.7e-3, 1.2e-3))


def _params(b, dist_max):
    return _lib.params(**cases.param_kwargs(b, dist_max=tuple(float(v) for v in dist_max), ql_len=b["ql_len"]))


def test_batch_lists_equal_single_searches():
    b = _batch()
    m = mega.Mega(b, _params(b, b["dist_max"].max(axis=0)))
    m.set_instances(b["counts"], b["dist_max"])
    got = m.search_and_shapes(download=True)
    off = np.concatenate([[0], np.cumsum(b["counts"])])
    for k, bar in enumerate(b["bars"]):
        ref = mega.bin_search(bar["coo"], bar["win"], bar["sm_len"], b["dist_max"][k])
        rows = slice(off[k], off[k + 1])
        np.testing.assert_array_equal(got["gn"][rows], ref["gn"])
        s0, s1 = got["gstart"][off[k]] - 1, got["gstart"][off[k + 1] - 1] - 1 + got["gn"][off[k + 1] - 1]
        np.testing.assert_array_equal(got["gstack"][s0:s1], ref["gstack"] + off[k])
    m.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_steps_equal_single_contexts(mode):
    b = _batch()
    dt = 3.0e-8
    m = mega.Mega(b, _params(b, b["dist_max"].max(axis=0)))
    m.set_instances(b["counts"], b["dist_max"])
    m.search_and_shapes()
    m.step(60, dt, mode=mode)
    xb = m.download(_lib.F_COO_CURRENT)
    eb = m.download(_lib.F_EPS)
    m.close()
    off = np.concatenate([[0], np.cumsum(b["counts"])])
    for k, bar in enumerate(b["bars"]):
        s = mega.Mega(bar, _params(b, b["dist_max"][k]))
        s.search_and_shapes()
        s.step(60, dt, mode=mode)
        x = s.download(_lib.F_COO_CURRENT)
        e = s.download(_lib.F_EPS)
        s.close()
        xs, es = xb[off[k]:off[k + 1]], eb[off[k]:off[k + 1]]
        if mode == "fp64":
            # same lists, same row and column orders: identical arithmetic
            np.testing.assert_array_equal(xs, x)
            np.testing.assert_array_equal(es, e)
        else:
            # the tile partition differs, and with it the float offsets of the
            # staged displacements
            u = x - bar["coo"]
            assert np.abs(xs - x).max() <= 1e-5 * np.abs(u).max()
            assert np.abs(es - e).max() <= 1e-4 * max(e.max(), 1e-12)


def test_precision_mask_refuses_unbuilt_mode():
    bar = cases.taylor_bar(h=1.0e-3)
    m = mega.Mega(bar, _lib.params(**cases.param_kwargs(bar)))
    m.set_precisions(fp64=False, mixed=True)
    m.search_and_shapes()
    m.step(2, 3e-8, mode="mixed")
    with pytest.raises(_lib.MegaError):
        m.step(1, 3e-8, mode="fp64")
    m.close()


def test_autotune_keeps_state_and_results():
    bar = cases.taylor_bar(h=0.8e-3)
    p = _lib.params(**cases.param_kwargs(bar))
    dt = 3.0e-8
    a = mega.Mega(bar, p)
    b = mega.Mega(bar, p)
    a.search_and_shapes()
    b.search_and_shapes()
    a.step(20, dt)
    b.step(20, dt)
    before = [a.download(f) for f in (_lib.F_DSP_TOT, _lib.F_VEL, _lib.F_STRESS, _lib.F_EPS)]
    for mode in ("fp64", "mixed"):
        choice, times = a.autotune(dt, mode=mode, reps=3)
        assert all(0 <= c < _lib.TUNE_VARIANTS for c in choice)
        assert np.all((times > 0) | (times == -1.0))  # -1: a streamed variant the tiles do not fit
    after = [a.download(f) for f in (_lib.F_DSP_TOT, _lib.F_VEL, _lib.F_STRESS, _lib.F_EPS)]
    for x, y in zip(before, after):
        np.testing.assert_array_equal(x, y)
    # another variant only regroups each row's partial sums
    a.step(20, dt)
    b.step(20, dt)
    xa, xb = a.download(_lib.F_COO_CURRENT), b.download(_lib.F_COO_CURRENT)
    assert np.abs(xa - xb).max() <= 1e-10 * np.abs(xb - bar["coo"]).max()
    a.close()
    b.close()


def test_instances_with_their_own_steps():
    """mega_set_instance_dt: each bar advances by its own stable step, and
    equals its own context stepped with that step (FP64, bit for bit)."""
    b = _batch()
    dts = [2.0e-8, 3.0e-8, 2.5e-8][:len(b["bars"])]
    m = mega.Mega(b, _params(b, b["dist_max"].max(axis=0)))
    m.set_instances(b["counts"], b["dist_max"])
    m.search_and_shapes()
    m.set_instance_dt(dts)
    m.step(40, 1.0e-8, mode="fp64")
    xb = m.download(_lib.F_COO_CURRENT)
    m.close()
    off = np.concatenate([[0], np.cumsum(b["counts"])])
    for k, bar in enumerate(b["bars"]):
        s = mega.Mega(bar, _params(b, b["dist_max"][k]))
        s.search_and_shapes()
        s.step(40, dts[k], mode="fp64")
        np.testing.assert_array_equal(xb[off[k]:off[k + 1]], s.download(_lib.F_COO_CURRENT))
        s.close()
    with pytest.raises(_lib.MegaError):
        single = mega.Mega(b["bars"][0], _params(b, b["dist_max"][0]))
        single.search_and_shapes()
        try:
            single.set_instance_dt([1e-8])   # no instances declared
        finally:
            single.close()
