"""CPU restatement of MEGA's mesh pre-processing for hexahedral and
tetrahedral meshes.

TEST INFRASTRUCTURE ONLY: imported by tests/ and the golden-fixture script,
never by the product package.  It follows the reference loops in element
order, so nodal sums come out bit for bit as the Fortran forms them:
  raw nodal windows (ADIAL): the largest per-axis distance between two nodes
      of any hex holding the node            PRE_MODEL_ADIAL.F90:64-153
  nodal volumes: 1/8 of each holding hex's volume, the hex split into three
      wedges about its 1-7 diagonal           PRE_MODEL_VOLUMES.F90:70-117,
                                              PRE_MODEL_VOL2.F90:36-52
  tetrahedra (block type 1): the window from the first four nodes, 1/4 of
      the GET_VOL1 volume to each              PRE_MODEL_ADIAL.F90:112-150,
                                              PRE_MODEL_VOL1.f90:37-45
  smoothing cells, second moments, DIST_MAX   PRE_MODEL_SMOOTHING_LENGTHS.F90:49-99
"""
import numpy as np

THRD = 0.333333333333333  # PRE_MODEL_SMOOTHING_LENGTHS.F90:41


def _det_abs_cols(c0, c1, c2):
    """DETERMINANT.F90:18-35 for the matrices with columns c0, c1, c2 (each
    (E, 3)), in the Fortran's operation order."""
    t1 = c1[:, 1] * c2[:, 2] - c1[:, 2] * c2[:, 1]
    t2 = c0[:, 2] * c2[:, 1] - c0[:, 1] * c2[:, 2]
    t3 = c0[:, 1] * c1[:, 2] - c0[:, 2] * c1[:, 1]
    return np.abs(c0[:, 0] * t1 + c1[:, 0] * t2 + c2[:, 0] * t3)


def hex_windows_and_volumes(coo, elems):
    """ADIAL (n, 3) and VOLUME (n) from hexes elems (E, 8), 0-based."""
    coo = np.asarray(coo, np.float64)
    elems = np.asarray(elems, np.int64)
    n = len(coo)
    x = coo[elems]                                   # (E, 8, 3)
    ext = x.max(axis=1) - x.min(axis=1)              # max over node pairs of |x_K - x_J|
    d71 = x[:, 6] - x[:, 0]
    ad = _det_abs_cols(d71, x[:, 1] - x[:, 0], x[:, 2] - x[:, 5])
    bd = _det_abs_cols(d71, x[:, 4] - x[:, 0], x[:, 5] - x[:, 7])
    cd = _det_abs_cols(d71, x[:, 3] - x[:, 0], x[:, 7] - x[:, 2])
    dvol = (ad + bd + cd) / 6.0
    adial = np.zeros((n, 3))
    np.maximum.at(adial, elems.ravel(), np.repeat(ext, 8, axis=0))
    vol = np.zeros(n)
    np.add.at(vol, elems.ravel(), np.repeat(0.125 * dvol, 8))  # element order, then node order
    return adial, vol


def windows_and_volumes(coo, elems, eltype=None):
    """ADIAL and VOLUME for a mesh of hexahedra (eltype 2) and tetrahedra
    (eltype 1; elems (E, 8) 0-based, a tetrahedron's first four nodes used),
    the nodal sums in element order."""
    coo = np.asarray(coo, np.float64)
    elems = np.asarray(elems, np.int64)
    if eltype is None:
        return hex_windows_and_volumes(coo, elems)
    et = np.asarray(eltype)
    n = len(coo)
    adial = np.zeros((n, 3))
    vol = np.zeros(n)
    x = coo[elems]
    tet = et == 1
    share = np.empty(len(elems))
    ext = np.where(tet[:, None], x[:, :4].max(axis=1) - x[:, :4].min(axis=1), x.max(axis=1) - x.min(axis=1))
    if np.any(~tet):
        h = x[~tet]
        d71 = h[:, 6] - h[:, 0]
        dv = (_det_abs_cols(d71, h[:, 1] - h[:, 0], h[:, 2] - h[:, 5]) + _det_abs_cols(d71, h[:, 4] - h[:, 0],
              h[:, 5] - h[:, 7]) + _det_abs_cols(d71, h[:, 3] - h[:, 0], h[:, 7] - h[:, 2])) / 6.0
        share[~tet] = 0.125 * dv
    if np.any(tet):
        t = x[tet]
        r1, r2, r3 = t[:, 3] - t[:, 2], t[:, 0] - t[:, 2], t[:, 1] - t[:, 2]   # rows of A (GET_VOL1)
        cols = [np.stack([r1[:, a], r2[:, a], r3[:, a]], axis=1) for a in range(3)]
        share[tet] = 0.25 * (_det_abs_cols(*cols) / 6.0)
    nk = np.where(tet, 4, 8)
    eidx = np.repeat(np.arange(len(elems)), nk)                     # element order, then node order
    kidx = np.concatenate([np.arange(k) for k in nk])
    nodes = elems[eidx, kidx]
    np.maximum.at(adial, nodes, ext[eidx])
    np.add.at(vol, nodes, share[eidx])
    return adial, vol


def smoothing_lengths(vol, win_raw):
    """SM_LEN (n, 6), X/Y/Z_MOM (n, 3) and (XDIST_MAX, YDIST_MAX, ZDIST_MAX)."""
    dim = 2.0 * np.asarray(win_raw, np.float64)
    vol_win = dim[:, 0] * dim[:, 1] * dim[:, 2]
    ratio = np.asarray(vol, np.float64) ** THRD / vol_win ** THRD
    m = dim * ratio[:, None]
    mom = m * m / 12.0
    half = dim * ratio[:, None] / 2.0
    sm = np.repeat(half, 2, axis=1)
    dmax = np.array([max(0.0, sm[:, 0].max()), max(0.0, sm[:, 2].max()), max(0.0, sm[:, 5].max())])
    return sm, mom, dmax
