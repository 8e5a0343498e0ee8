"""Edge cases of the CUDA path against the oracle: tiny models, isolated
nodes, ragged neighbour counts, neighbourhoods dense enough to shrink the
tiles, and a list buffer too small for the search."""
import numpy as np
import pytest

from oracle import oracle as O
from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _small_case(coo, win_scale=2.0, h=1e-3):
    """A free block of nodes (no wall, at rest) in the bar's material."""
    coo = np.asarray(coo, np.float64).reshape(-1, 3)
    n = len(coo)
    win_raw = np.full((n, 3), h)
    vol = np.full(n, h ** 3)
    sm_len, dist_max = cases.smoothing_lengths(vol, win_raw)
    pv = cases.props_vector(2, 117e9, 0.35, 8930.0, 400e6, 0.25, 1.0)
    return dict(n=n, coo=coo, win=win_raw * win_scale, win_raw=win_raw, vol=vol,
                mass=np.repeat((vol * 8930.0)[:, None], 3, axis=1).copy(), ebc=np.zeros((n, 3), np.int32),
                vinit=np.zeros((n, 3)), props=np.tile(pv, (n, 1)), mat_type=np.full(n, 2, np.int32),
                body_id=np.ones(n, np.int32), bodyforce=None, sm_len=sm_len, dist_max=dist_max,
                ql_len=0.1 * h, wall=np.zeros(n, bool))


def test_single_and_two_nodes():
    for coo in ([[0.0, 0.0, 0.0]], [[0.0, 0.0, 0.0], [0.5e-3, 0.0, 0.0]]):
        c = _small_case(coo)
        ref = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
        got = mega.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
        np.testing.assert_array_equal(got["gstack"], ref["gstack"])
        # one or two nodes cannot span a linear basis: the moment matrix is
        # singular, reported as the reference stops (no trap, no NaN run)
        # (QL off: its six shifted points would regularise the matrix)
        m = mega.Mega(c, _lib.params(**cases.param_kwargs(c, ql=0)))
        st = m.search_and_shapes(allow_status=True)["status"]
        assert st & _lib.ST_SINGULAR_MOMENT
        m.close()


def test_isolated_node_in_a_lattice_is_reported():
    c0 = cases.taylor_bar(h=1.0e-3)
    coo = np.vstack([c0["coo"], [[0.05, 0.05, 0.05]]])  # far from the bar
    c = _small_case(coo, h=1.0e-3)
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c, ql=0)))
    st = m.search_and_shapes(allow_status=True)["status"]
    assert st & _lib.ST_SINGULAR_MOMENT
    m.close()


def test_ragged_windows_match_oracle():
    """Windows drawn from 1.6 to 3.2 spacings: rows from a dozen to a few
    hundred entries, lists bit-exact and one resident run against the oracle."""
    c = cases.taylor_bar(h=0.8e-3, seed=11)
    rng = np.random.default_rng(5)
    scale = rng.uniform(1.6, 3.2, c["n"])
    c["win"] = c["win_raw"] * scale[:, None]
    c["sm_len"], c["dist_max"] = cases.smoothing_lengths(c["vol"], c["win_raw"])
    ref = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    assert ref["gn"].max() > 4 * ref["gn"].min()
    got = mega.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    np.testing.assert_array_equal(got["gn"], ref["gn"])
    np.testing.assert_array_equal(got["gstack"], ref["gstack"])
    p = cases.param_kwargs(c)
    m = mega.Mega(c, _lib.params(**p))
    m.search_and_shapes()
    r = O.Run(c, O.params(**p), nthreads=8)
    dt = 0.5 * cases.stable_dt(c, ref["gn"], ref["gstart"], ref["gstack"])
    m.step(40, dt)
    r.step(40, dt)
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max()
    m.close()


def test_dense_neighbourhoods_shrink_the_tiles():
    """Supports of 4.5 spacings (up to 729 neighbours a node) overflow a
    64-row tile's 1,024-entry set; the tiles halve until they fit and the
    result still matches the oracle."""
    c = cases.taylor_bar(h=1.0e-3, R=6.4e-3, L=8e-3, norm_win=4.5, seed=2)
    p = cases.param_kwargs(c)
    ref = O.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    assert ref["gn"].max() > 600
    m = mega.Mega(c, _lib.params(**p))
    m.search_and_shapes()
    r = O.Run(c, O.params(**p), nthreads=8)
    dt = cases.stable_dt(c, ref["gn"], ref["gstart"], ref["gstack"])
    m.step(30, dt)
    r.step(30, dt)
    x = m.download(_lib.F_COO_CURRENT)
    uo = r.coo_cur.reshape(-1, 3) - c["coo"]
    assert np.abs(x - c["coo"] - uo).max() <= 1e-7 * np.abs(uo).max()
    m.close()


def test_list_buffer_too_small_is_reported():
    c = cases.taylor_bar(h=1.0e-3)
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    import ctypes as C
    n = c["n"]
    gn = np.zeros(n, np.int32)
    gstart = np.zeros(n, np.int32)
    small = np.zeros(10, np.int32)
    nnz = C.c_int64(0)
    gmaxn = C.c_int32(0)
    st = _lib.lib().mega_search_and_shapes(m.h, _lib.ptr(gn), _lib.ptr(gstart), _lib.ptr(small), 10, None, None,
                                           C.byref(nnz), C.byref(gmaxn))
    assert st > 0 and st & _lib.ST_STACK_OVERFLOW
    assert nnz.value > 10 and gn.sum() == nnz.value
    m.close()


@pytest.mark.parametrize("itype", [0, 2])
def test_shapes_on_renumbered_lists_equal_the_downloaded_path(itype):
    """Without a list download the shapes (and NSNI's second derivatives) are
    computed directly on the renumbered lists; the steps that follow are the
    same to the bit as after the path that builds them in the caller's
    numbering first."""
    c = cases.taylor_bar(h=0.8e-3)
    p = _lib.params(**cases.param_kwargs(c, itype_int=itype))
    a, b = mega.Mega(c, p), mega.Mega(c, p)
    a.search_and_shapes(download=True)
    b.search_and_shapes(download=False)
    a.step(30, 3e-8)
    b.step(30, 3e-8)
    for f in (_lib.F_COO_CURRENT, _lib.F_STRESS, _lib.F_EPS):
        np.testing.assert_array_equal(a.download(f), b.download(f))
    a.close()
    b.close()


def test_mixed_only_context_steps_like_the_two_precision_one():
    """A context asked for mixed records alone writes them straight from the
    shape kernel (no double gradients kept); its mixed steps are the same to
    the bit as those of a context that built both precisions."""
    c = cases.taylor_bar(h=0.8e-3, seed=2)
    p = _lib.params(**cases.param_kwargs(c))
    a, b = mega.Mega(c, p), mega.Mega(c, p)
    b.set_precisions(fp64=False, mixed=True)
    a.search_and_shapes()
    b.search_and_shapes()
    a.step(30, 3e-8, mode="mixed")
    b.step(30, 3e-8, mode="mixed")
    for f in (_lib.F_COO_CURRENT, _lib.F_STRESS, _lib.F_EPS, _lib.F_VEL):
        np.testing.assert_array_equal(a.download(f), b.download(f))
    with pytest.raises(_lib.MegaError):  # FP64 records were not built
        b.step(1, 3e-8, mode="fp64")
    a.close()
    b.close()


def test_snapshot_equals_single_downloads(tmp_path):
    """One device-to-host copy of several fields equals their single
    downloads, and the output step writes them as VTK."""
    from taylor_b200 import vtk
    c = cases.taylor_bar(h=1.0e-3)
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    m.search_and_shapes()
    m.step(20, 3e-8)
    fields = (_lib.F_COO_CURRENT, _lib.F_STRESS, _lib.F_EPS, _lib.F_NEWTON_IT, _lib.F_VEL, _lib.F_DSP_TOT_PHY)
    snap = m.snapshot(fields)
    for f in fields:
        np.testing.assert_array_equal(snap[int(f)], m.download(f))
    p = tmp_path / "MEGAOUT_0001.vtk"
    vtk.write_output_step(m, p)
    lines = p.read_text().splitlines()
    assert lines[4].split() == ["POINTS", str(c["n"]), "double"]
    assert sum(1 for l in lines if l.startswith("SCALARS")) == 3 + 3 + 6 + 1
    m.close()


def test_release_cached_memory():
    """Finalised contexts leave their blocks cached in the library and the
    device pool; mega_release_cached_memory returns them to the driver (a
    host program with its own allocator sees the memory free again) and the
    library keeps working afterwards."""
    import torch
    c = cases.taylor_bar(h=0.4e-3)
    free0 = torch.cuda.mem_get_info()[0]
    m = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    m.search_and_shapes()
    held = m.device_bytes()
    m.close()
    assert held > 0
    free_cached = torch.cuda.mem_get_info()[0]
    assert _lib.lib().mega_release_cached_memory() == 0
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 >= free_cached
    assert free1 >= free0 - (64 << 20)  # back to within the driver's own granularity
    again = mega.Mega(c, _lib.params(**cases.param_kwargs(c)))
    again.search_and_shapes()
    again.step(5, 3.9e-8)
    again.close()
