"""A second, independent restatement of MEGA's Lagrangian DNI hot path in
numpy -- TEST INFRASTRUCTURE ONLY (imported by tests/ to cross-check the C++
oracle, never by the product package).

It is written from the Fortran alone, vectorised over nodes and list
entries, and shares no code with oracle/mega_oracle.cpp, so a transcription
error in one restatement shows up as a disagreement with the other.  It
covers what the resident GPU step computes on the reference's live path:

  rk1             RK1 with the cubic B-spline box kernel, QL and the singular
                  kernel of EBC neighbours (RK.f90:16-453, KERNEL.F90:57-71,
                  FILL_H / DERIV_H RK.f90:462-575, M44INV INVERSE.F90:185-223)
  hughes_winget   HUGHES_WINGET with INV3 as written (HUGHES_WINGET.F90:16-81,
                  INVERSE.F90:119-152), ROTATE_TENSOR (ROTATE_TENSOR.F90:21-87)
  von_mises       VON_MISES (CONSTITUTE_VONMISES.F90:21-158)
  construct_fint  the Lagrangian finite-strain DNI force (FINT.F90:577-870,
                  995-1116) for materials 1 and 2
  Step            MAIN.F90's predictor, DO_INTERP, force and corrector
                  (MAIN.F90:348-356, 377-386, 432-488; HANDELER.F90:114-139)

Sums over neighbours run in list order (np.add.at applies its additions in
index order), MATMUL-style sums in index order, so the two restatements
agree to rounding.
"""
import numpy as np

S23 = np.sqrt(2.0 / 3.0)
F32_1E5 = float(np.float32(1.0e-5))    # the single-precision literal 1.0E-05 (CONSTITUTE_VONMISES.F90:112)
F32_1E15 = float(np.float32(1.0e-15))  # the single-precision literal 1.0E-015 (RK.f90:221)


def _kernel(r):
    """MLS_KERNEL0 cubic B-spline (KERNEL.F90:57-71): value and d/dr at r >= 0."""
    r2 = r * r          # XSA**2 and XSA**3 as repeated products (integer powers)
    r3 = r2 * r
    phi = np.where(r <= 0.5, 2.0 / 3.0 - 4.0 * r2 + 4.0 * r3,
                   np.where(r <= 1.0, 4.0 / 3.0 - 4.0 * r + 4.0 * r2 - 4.0 / 3.0 * r3, 0.0))
    dphi = np.where(r <= 0.5, -8.0 * r + 12.0 * r2, np.where(r <= 1.0, -4.0 + 8.0 * r - 4.0 * r2, 0.0))
    return phi, dphi


def _sign_over(r, w):
    """DRDX of RK.f90:182-205: 0 at r = 0, else +-1/w."""
    return np.where(r == 0.0, 0.0, np.where(r >= 0.0, 1.0 / w, -1.0 / w))


def _mm(a, b):
    """Batched MATMUL with the inner sum in index order."""
    out = a[..., :, 0:1] * b[..., 0:1, :]
    for k in range(1, a.shape[-1]):
        out = out + a[..., :, k:k + 1] * b[..., k:k + 1, :]
    return out


def m44inv(A):
    """M44INV (INVERSE.F90:185-223): transpose of the cofactors over the determinant."""
    a = lambda i, j: A[:, i - 1, j - 1]  # noqa: E731  1-based like the Fortran
    det = (a(1, 1) * (a(2, 2) * (a(3, 3) * a(4, 4) - a(3, 4) * a(4, 3)) + a(2, 3) * (a(3, 4) * a(4, 2) - a(3, 2) * a(4, 4))
                      + a(2, 4) * (a(3, 2) * a(4, 3) - a(3, 3) * a(4, 2)))
           - a(1, 2) * (a(2, 1) * (a(3, 3) * a(4, 4) - a(3, 4) * a(4, 3)) + a(2, 3) * (a(3, 4) * a(4, 1) - a(3, 1) * a(4, 4))
                        + a(2, 4) * (a(3, 1) * a(4, 3) - a(3, 3) * a(4, 1)))
           + a(1, 3) * (a(2, 1) * (a(3, 2) * a(4, 4) - a(3, 4) * a(4, 2)) + a(2, 2) * (a(3, 4) * a(4, 1) - a(3, 1) * a(4, 4))
                        + a(2, 4) * (a(3, 1) * a(4, 2) - a(3, 2) * a(4, 1)))
           - a(1, 4) * (a(2, 1) * (a(3, 2) * a(4, 3) - a(3, 3) * a(4, 2)) + a(2, 2) * (a(3, 3) * a(4, 1) - a(3, 1) * a(4, 3))
                        + a(2, 3) * (a(3, 1) * a(4, 2) - a(3, 2) * a(4, 1))))
    c = np.empty_like(A)
    c[:, 0, 0] = a(2, 2) * (a(3, 3) * a(4, 4) - a(3, 4) * a(4, 3)) + a(2, 3) * (a(3, 4) * a(4, 2) - a(3, 2) * a(4, 4)) + a(2, 4) * (a(3, 2) * a(4, 3) - a(3, 3) * a(4, 2))
    c[:, 0, 1] = a(2, 1) * (a(3, 4) * a(4, 3) - a(3, 3) * a(4, 4)) + a(2, 3) * (a(3, 1) * a(4, 4) - a(3, 4) * a(4, 1)) + a(2, 4) * (a(3, 3) * a(4, 1) - a(3, 1) * a(4, 3))
    c[:, 0, 2] = a(2, 1) * (a(3, 2) * a(4, 4) - a(3, 4) * a(4, 2)) + a(2, 2) * (a(3, 4) * a(4, 1) - a(3, 1) * a(4, 4)) + a(2, 4) * (a(3, 1) * a(4, 2) - a(3, 2) * a(4, 1))
    c[:, 0, 3] = a(2, 1) * (a(3, 3) * a(4, 2) - a(3, 2) * a(4, 3)) + a(2, 2) * (a(3, 1) * a(4, 3) - a(3, 3) * a(4, 1)) + a(2, 3) * (a(3, 2) * a(4, 1) - a(3, 1) * a(4, 2))
    c[:, 1, 0] = a(1, 2) * (a(3, 4) * a(4, 3) - a(3, 3) * a(4, 4)) + a(1, 3) * (a(3, 2) * a(4, 4) - a(3, 4) * a(4, 2)) + a(1, 4) * (a(3, 3) * a(4, 2) - a(3, 2) * a(4, 3))
    c[:, 1, 1] = a(1, 1) * (a(3, 3) * a(4, 4) - a(3, 4) * a(4, 3)) + a(1, 3) * (a(3, 4) * a(4, 1) - a(3, 1) * a(4, 4)) + a(1, 4) * (a(3, 1) * a(4, 3) - a(3, 3) * a(4, 1))
    c[:, 1, 2] = a(1, 1) * (a(3, 4) * a(4, 2) - a(3, 2) * a(4, 4)) + a(1, 2) * (a(3, 1) * a(4, 4) - a(3, 4) * a(4, 1)) + a(1, 4) * (a(3, 2) * a(4, 1) - a(3, 1) * a(4, 2))
    c[:, 1, 3] = a(1, 1) * (a(3, 2) * a(4, 3) - a(3, 3) * a(4, 2)) + a(1, 2) * (a(3, 3) * a(4, 1) - a(3, 1) * a(4, 3)) + a(1, 3) * (a(3, 1) * a(4, 2) - a(3, 2) * a(4, 1))
    c[:, 2, 0] = a(1, 2) * (a(2, 3) * a(4, 4) - a(2, 4) * a(4, 3)) + a(1, 3) * (a(2, 4) * a(4, 2) - a(2, 2) * a(4, 4)) + a(1, 4) * (a(2, 2) * a(4, 3) - a(2, 3) * a(4, 2))
    c[:, 2, 1] = a(1, 1) * (a(2, 4) * a(4, 3) - a(2, 3) * a(4, 4)) + a(1, 3) * (a(2, 1) * a(4, 4) - a(2, 4) * a(4, 1)) + a(1, 4) * (a(2, 3) * a(4, 1) - a(2, 1) * a(4, 3))
    c[:, 2, 2] = a(1, 1) * (a(2, 2) * a(4, 4) - a(2, 4) * a(4, 2)) + a(1, 2) * (a(2, 4) * a(4, 1) - a(2, 1) * a(4, 4)) + a(1, 4) * (a(2, 1) * a(4, 2) - a(2, 2) * a(4, 1))
    c[:, 2, 3] = a(1, 1) * (a(2, 3) * a(4, 2) - a(2, 2) * a(4, 3)) + a(1, 2) * (a(2, 1) * a(4, 3) - a(2, 3) * a(4, 1)) + a(1, 3) * (a(2, 2) * a(4, 1) - a(2, 1) * a(4, 2))
    c[:, 3, 0] = a(1, 2) * (a(2, 4) * a(3, 3) - a(2, 3) * a(3, 4)) + a(1, 3) * (a(2, 2) * a(3, 4) - a(2, 4) * a(3, 2)) + a(1, 4) * (a(2, 3) * a(3, 2) - a(2, 2) * a(3, 3))
    c[:, 3, 1] = a(1, 1) * (a(2, 3) * a(3, 4) - a(2, 4) * a(3, 3)) + a(1, 3) * (a(2, 4) * a(3, 1) - a(2, 1) * a(3, 4)) + a(1, 4) * (a(2, 1) * a(3, 3) - a(2, 3) * a(3, 1))
    c[:, 3, 2] = a(1, 1) * (a(2, 4) * a(3, 2) - a(2, 2) * a(3, 4)) + a(1, 2) * (a(2, 1) * a(3, 4) - a(2, 4) * a(3, 1)) + a(1, 4) * (a(2, 2) * a(3, 1) - a(2, 1) * a(3, 2))
    c[:, 3, 3] = a(1, 1) * (a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2)) + a(1, 2) * (a(2, 3) * a(3, 1) - a(2, 1) * a(3, 3)) + a(1, 3) * (a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1))
    return np.transpose(c, (0, 2, 1)) / det[:, None, None]


def rk1(coo, win, ebc_nodes, rows, cols, n, ql=True, ql_coef=0.001, ql_len=0.0):
    """Shape functions and gradients of every list entry (rows i, cols j,
    0-based, in list order) at X_i: RK1 for linear basis, box support."""
    d = coo[rows] - coo[cols]                       # X - X_J, unnormalised
    w = win[cols]
    r = d / w                                       # normalised
    px, dpx = _kernel(np.abs(r[:, 0]))
    py, dpy = _kernel(np.abs(r[:, 1]))
    pz, dpz = _kernel(np.abs(r[:, 2]))
    phi = px * py * pz
    w1 = w[:, 0]                                    # DRDY, DRDZ divide by GWIN(1,II) as written
    phx = dpx * py * pz * _sign_over(r[:, 0], w1)
    phy = px * dpy * pz * _sign_over(r[:, 1], w1)
    phz = px * py * dpz * _sign_over(r[:, 2], w1)
    sing = np.asarray(ebc_nodes, bool)[cols]
    if np.any(sing):                                # singular kernel of EBC neighbours (RK.f90:217-228)
        wm = 1.0 / (np.sqrt(r[:, 0] ** 2 + r[:, 1] ** 2 + r[:, 2] ** 2) + F32_1E15)
        wm3 = wm * wm * wm
        phx = np.where(sing, phx * wm - phi * wm3 * r[:, 0] / w[:, 0], phx)
        phy = np.where(sing, phy * wm - phi * wm3 * r[:, 1] / w[:, 1], phy)
        phz = np.where(sing, phz * wm - phi * wm3 * r[:, 2] / w[:, 2], phz)
        phi = np.where(sing, phi * wm, phi)
    H = np.concatenate([np.ones((len(rows), 1)), d], axis=1)
    dphi = (phx, phy, phz)
    M = np.zeros((n, 4, 4))
    Md = [np.zeros((n, 4, 4)) for _ in range(3)]
    psum = np.zeros(n)
    np.add.at(psum, rows, phi)
    for j in range(4):
        for k in range(4):
            np.add.at(M[:, j, k], rows, H[:, j] * H[:, k] * phi)
            for a in range(3):
                hj = 1.0 if j == a + 1 else 0.0
                hk = 1.0 if k == a + 1 else 0.0
                np.add.at(Md[a][:, j, k], rows, hj * H[:, k] * phi + H[:, j] * hk * phi + H[:, j] * H[:, k] * dphi[a])
    hq = np.zeros(4)
    if ql:                                          # RK.f90:251-303
        mstar = np.zeros((4, 4))
        for sgn_axis in ((0, 1.0), (0, -1.0), (1, 1.0), (1, -1.0), (2, 1.0), (2, -1.0)):
            h = np.zeros(4)
            h[0] = 1.0
            h[1 + sgn_axis[0]] = -sgn_axis[1] * ql_len   # X - (X +- QL_LEN e)
            mstar = mstar + np.outer(h, h)
            hq = hq + h
        M = M + mstar[None] * psum[:, None, None] * ql_coef
    minv = m44inv(M)
    b = minv[:, 0, :]
    bd = [_mm(-minv, Md[a])[:, :, :] for a in range(3)]
    bd = [_mm(x, minv)[:, 0, :] for x in bd]
    Hs = H + hq[None] * ql_coef if ql else H
    bi = b[rows]
    c = bi[:, 0] * Hs[:, 0] + bi[:, 1] * Hs[:, 1] + bi[:, 2] * Hs[:, 2] + bi[:, 3] * Hs[:, 3]
    shp = c * phi
    dshp = np.empty((len(rows), 3))
    for a in range(3):
        ba = bd[a][rows]
        ca = ba[:, 0] * Hs[:, 0] + ba[:, 1] * Hs[:, 1] + ba[:, 2] * Hs[:, 2] + ba[:, 3] * Hs[:, 3]
        ca = ca + bi[:, a + 1]                      # MATMUL(B, H_X) = B(a + 1)
        dshp[:, a] = ca * phi + c * dphi[a]
    return shp, dshp


def inv3(A):
    """INV3 as written (INVERSE.F90:119-152): the adjugate times det(A)."""
    a = lambda i, j: A[..., i - 1, j - 1]  # noqa: E731
    det = (a(1, 1) * a(2, 2) * a(3, 3) - a(1, 1) * a(2, 3) * a(3, 2) - a(1, 2) * a(2, 1) * a(3, 3)
           + a(1, 2) * a(2, 3) * a(3, 1) + a(1, 3) * a(2, 1) * a(3, 2) - a(1, 3) * a(2, 2) * a(3, 1))
    o = np.empty_like(A)
    o[..., 0, 0] = (a(2, 2) * a(3, 3) - a(2, 3) * a(3, 2)) * det
    o[..., 1, 0] = -(a(2, 1) * a(3, 3) - a(2, 3) * a(3, 1)) * det
    o[..., 2, 0] = (a(2, 1) * a(3, 2) - a(2, 2) * a(3, 1)) * det
    o[..., 0, 1] = -(a(1, 2) * a(3, 3) - a(1, 3) * a(3, 2)) * det
    o[..., 1, 1] = (a(1, 1) * a(3, 3) - a(1, 3) * a(3, 1)) * det
    o[..., 2, 1] = -(a(1, 1) * a(3, 2) - a(1, 2) * a(3, 1)) * det
    o[..., 0, 2] = (a(1, 2) * a(2, 3) - a(1, 3) * a(2, 2)) * det
    o[..., 1, 2] = -(a(1, 1) * a(2, 3) - a(1, 3) * a(2, 1)) * det
    o[..., 2, 2] = (a(1, 1) * a(2, 2) - a(1, 2) * a(2, 1)) * det
    return o


def _v2t(v):
    t = np.empty(v.shape[:-1] + (3, 3))
    t[..., 0, 0], t[..., 1, 1], t[..., 2, 2] = v[..., 0], v[..., 1], v[..., 2]
    t[..., 1, 2] = t[..., 2, 1] = v[..., 3]
    t[..., 0, 2] = t[..., 2, 0] = v[..., 4]
    t[..., 0, 1] = t[..., 1, 0] = v[..., 5]
    return t


def _t2v(t):
    return np.stack([t[..., 0, 0], t[..., 1, 1], t[..., 2, 2], t[..., 1, 2], t[..., 0, 2], t[..., 0, 1]], axis=-1)


def hughes_winget(L):
    """HUGHES_WINGET: rotation, Voigt strain with engineering shear, and D."""
    eye = np.broadcast_to(np.eye(3), L.shape)
    A = eye + 0.5 * L
    G = _mm(L, inv3(A))
    Gt = np.swapaxes(G, -1, -2)
    W = 0.5 * (G - Gt)
    R = eye + _mm(inv3(eye - 0.5 * W), W)
    D = _t2v(0.5 * (G + Gt))
    strain = D.copy()
    strain[..., 3:] = 2.0 * strain[..., 3:]
    return R, strain, D


def rotate_tensor(R, v):
    """ROTATE_TENSOR: R T R^T of a Voigt tensor (shear as tensor components)."""
    return _t2v(_mm(_mm(R, _v2t(v)), np.swapaxes(R, -1, -2)))


def _tnorm(v):
    return np.sqrt(v[..., 0] ** 2 + v[..., 1] ** 2 + v[..., 2] ** 2 + 2.0 * (v[..., 3] ** 2 + v[..., 4] ** 2 + v[..., 5] ** 2))


def von_mises(spred, eps, props):
    """VON_MISES for every node (Newton capped at 20); returns stress, eps."""
    nu, E, s0, B, C = props[:, 0], props[:, 1], props[:, 3], props[:, 4], props[:, 5]
    mu = E / (2.0 * (1.0 + nu))
    kk = spred[:, 0] + spred[:, 1] + spred[:, 2]
    dev = spred.copy()
    dev[:, :3] = spred[:, :3] - (kk / 3.0)[:, None]
    sph = np.zeros_like(spred)
    sph[:, :3] = -(kk / 3.0)[:, None]
    tn = _tnorm(dev)
    sig23 = np.sqrt(2.0 / 3.0) * s0
    eps = eps.copy()
    out = dev.copy()
    xk = sig23 * (1.0 + B * eps) ** C
    for i in np.flatnonzero(tn - xk > 0.0):
        dg, epst = 0.0, eps[i]
        for it in range(1, 21):
            xki = sig23[i] * (1.0 + B[i] * eps[i]) ** C[i]
            y = tn[i] - xki - (2.0 * mu[i] * dg)
            if abs(y) > sig23[i] * F32_1E5:
                xkp = B[i] * C[i] * s0[i] * (1.0 + B[i] * eps[i]) ** (C[i] - 1.0)
                dg = dg - y / (-2.0 * mu[i] * (1.0 + xkp / 3.0 / mu[i]))
            else:
                eps[i] = epst + np.sqrt(2.0 / 3.0) * dg
                break
            eps[i] = epst + np.sqrt(2.0 / 3.0) * dg
        out[i] = dev[i] - dg * 2.0 * mu[i] * dev[i] / tn[i]
    return -sph + out, eps


def _cmat_times(props, e):
    """MATMUL(FORM_CMAT(LPROP), STRAIN) with the sum in index order."""
    lam, mu, l2m = props[:, 27], props[:, 28], props[:, 29]
    z = np.zeros_like(lam)
    C = np.stack([np.stack([l2m, lam, lam, z, z, z], -1), np.stack([lam, l2m, lam, z, z, z], -1),
                  np.stack([lam, lam, l2m, z, z, z], -1), np.stack([z, z, z, mu, z, z], -1),
                  np.stack([z, z, z, z, mu, z], -1), np.stack([z, z, z, z, z, mu], -1)], 1)
    out = C[:, :, 0] * e[:, 0:1]
    for k in range(1, 6):
        out = out + C[:, :, k] * e[:, k:k + 1]
    return out


def construct_fint(case, rows, cols, shp, dshp, stress, strain, eps, dinc, dinc_tot):
    """The Lagrangian finite-strain DNI force of one call after LINIT
    (FINT.F90:577-870, 995-1116), materials 1 and 2, no body force.
    Returns fint (n,3) and the updated stress, strain, eps."""
    n = case["n"]
    props = np.asarray(case["props"], np.float64)
    vol = np.asarray(case["vol"], np.float64)
    ut = dinc_tot.reshape(-1, 3)
    du = dinc.reshape(-1, 3)
    F = np.broadcast_to(np.eye(3), (n, 3, 3)).copy()  # FMAT = I, then the terms in list order
    for k in range(3):
        for l in range(3):
            acc = F[:, k, l].copy()
            np.add.at(acc, rows, dshp[:, l] * ut[cols, k])
            F[:, k, l] = acc
    det = np.abs(F[:, 0, 0] * (F[:, 1, 1] * F[:, 2, 2] - F[:, 2, 1] * F[:, 1, 2])
                 + F[:, 0, 1] * (F[:, 2, 0] * F[:, 1, 2] - F[:, 1, 0] * F[:, 2, 2])
                 + F[:, 0, 2] * (F[:, 1, 0] * F[:, 2, 1] - F[:, 2, 0] * F[:, 1, 1]))
    IF = inv3(F)
    IFe = IF[rows]
    g = np.zeros_like(dshp)
    for l in range(3):                              # SHPD(l) = sum_k SHPDTMP(k) IFMAT(k, l)
        for k in range(3):
            g[:, l] = g[:, l] + dshp[:, k] * IFe[:, k, l]
    L = np.zeros((n, 3, 3))
    for k in range(3):
        for l in range(3):
            np.add.at(L[:, k, l], rows, g[:, l] * du[cols, k])
    R, de, _ = hughes_winget(L)
    s = rotate_tensor(R, stress)
    e = rotate_tensor(R, strain) + de
    spred = s + _cmat_times(props, de)
    mat = np.asarray(case["mat_type"])
    snew, enew_eps = spred.copy(), eps.copy()
    vm = mat == 2
    if np.any(vm):
        sv, ev = von_mises(spred[vm], eps[vm], props[vm])
        snew[vm], enew_eps[vm] = sv, ev
    # FINT3 = MATMUL(BMAT^T, LSTRESS) (zero terms add nothing), times VOL then DET
    sr = snew[rows]
    f1 = (g[:, 0] * sr[:, 0] + g[:, 2] * sr[:, 4]) + g[:, 1] * sr[:, 5]
    f2 = (g[:, 1] * sr[:, 1] + g[:, 2] * sr[:, 3]) + g[:, 0] * sr[:, 5]
    f3 = (g[:, 2] * sr[:, 2] + g[:, 1] * sr[:, 3]) + g[:, 0] * sr[:, 4]
    vd = vol[rows]
    dd = det[rows]
    fint = np.zeros((n, 3))
    for k, fk in enumerate((f1, f2, f3)):
        np.add.at(fint[:, k], cols, fk * vd * dd)
    return fint, snew, e, enew_eps


class Step:
    """MAIN.F90's explicit loop after LINIT on the numpy restatement: the
    predictor (MAIN.F90:353-355), DO_INTERP (HANDELER.F90:114-139), the
    current coordinates (MAIN.F90:377-386), the force and the corrector with
    fixity 0/1 (MAIN.F90:432-488)."""

    def __init__(self, case, nb, ql=True, ql_coef=0.001, ql_len=None):
        self.case = case
        n = self.n = case["n"]
        gn = np.asarray(nb["gn"], np.int64)
        gs = np.asarray(nb["gstart"], np.int64) - 1
        self.rows = np.repeat(np.arange(n), gn)
        pos = np.concatenate([np.arange(s, s + k) for s, k in zip(gs, gn)]) if n else np.zeros(0, np.int64)
        self.cols = np.asarray(nb["gstack"], np.int64)[pos] - 1
        ebcn = np.any(np.asarray(case["ebc"]) == 1, axis=1)
        self.shp, self.dshp = rk1(np.asarray(case["coo"], np.float64), np.asarray(case["win"], np.float64), ebcn,
                                  self.rows, self.cols, n, ql, ql_coef,
                                  case["ql_len"] if ql_len is None else ql_len)
        ebc = np.asarray(case["ebc"]).reshape(-1)
        self.ebc = ebc
        self.vel = np.where(ebc == 1, 0.0, np.asarray(case["vinit"], np.float64).reshape(-1))
        z = np.zeros(3 * n)
        self.acl, self.dsp, self.dsp_tot, self.phy = z.copy(), z.copy(), z.copy(), z.copy()
        self.fint, self.fext = z.copy(), z.copy()
        self.stress, self.strain, self.eps = np.zeros((n, 6)), np.zeros((n, 6)), np.zeros(n)
        self.mass = np.asarray(case["mass"], np.float64).reshape(-1)
        self.damp = np.repeat(np.asarray(case["props"], np.float64)[:, 20], 3)

    def step(self, dt):
        self.dsp = dt * self.vel + dt * dt * 0.5 * self.acl
        self.dsp_tot = self.dsp_tot + self.dsp
        self.vel = self.vel + dt * 0.5 * self.acl
        dphy = np.zeros((self.n, 3))
        du = self.dsp.reshape(-1, 3)
        for k in range(3):
            np.add.at(dphy[:, k], self.rows, self.shp * du[self.cols, k])
        self.phy = self.phy + dphy.reshape(-1)
        f, self.stress, self.strain, self.eps = construct_fint(self.case, self.rows, self.cols, self.shp, self.dshp,
                                                               self.stress, self.strain, self.eps, self.dsp,
                                                               self.dsp_tot)
        self.fint = f.reshape(-1)
        fixed = self.ebc == 1
        mpdc = self.damp * self.mass
        acl = (self.fext - self.fint - mpdc * self.vel) / (self.mass + 0.5 * dt * mpdc)
        self.acl = np.where(fixed, 0.0, acl)
        self.vel = np.where(fixed, 0.0, self.vel + 0.5 * dt * self.acl)
        self.fext = np.where(fixed, -self.fint, self.fext)

    @property
    def coo_cur(self):
        return np.asarray(self.case["coo"], np.float64).reshape(-1) + self.phy
