"""Synthetic inputs for the explicit meshfree step.

The reference builds its model from an LS-DYNA keyword mesh (PRE_MODEL.F90)
and a Control.dat deck (PRE_CONTROL.F90 / READ.F90).  The configurations
measured here are lattices, so this module produces the arrays that
pre-processing would hand to the hot path: coordinates (3,N), raw and
normalised windows, nodal volumes, masses, fixities, initial velocities,
material properties PROPS(30,N) and smoothing lengths SM_LEN(6,N).

Arrays are numpy C-order (N,3)/(N,6)/(N,30), which is the Fortran
column-major (3,N)/(6,N)/(30,N) layout the C ABI takes.
"""
import math

import numpy as np

THRD = 0.333333333333333  # PRE_MODEL_SMOOTHING_LENGTHS.F90:41


def props_vector(mat_type, E, nu, rho, p4=0.0, p5=0.0, p6=0.0, p7=0.0, p8=0.0, damping=0.0):
    """PROPS(30) of one material (READ.F90:394-507): 1 nu, 2 E, 3 rho,
    4..8 law parameters, 21 mass-proportional damping, 28..30 lambda, mu,
    lambda + 2 mu."""
    p = np.zeros(30)
    p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7] = nu, E, rho, p4, p5, p6, p7, p8
    p[20] = damping
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    p[27], p[28], p[29] = lam, mu, lam + 2.0 * mu
    return p


def with_damage(case, mat_type, k_i, k_c, dam_max, q_phi=0.0, k_phi=0.0, q_psi=0.0):
    """The case with a damaged model on every node: material 6 (J2 with the
    case's hardening, isotropic damage) or 3 (Drucker-Prager shear yield
    with damage).  PROPS(9..11) = K_I, K_C, DAM_MAX (thresholds on the
    total-strain norm), PROPS(25..27) = Q_PHI, K_PHI, Q_PSI."""
    c = dict(case)
    pr = np.array(case["props"], copy=True)
    pr[:, 8], pr[:, 9], pr[:, 10] = k_i, k_c, dam_max
    pr[:, 24], pr[:, 25], pr[:, 26] = q_phi, k_phi, q_psi
    c["props"] = pr
    c["mat_type"] = np.full(case["n"], mat_type, np.int32)
    c["name"] = f"{case.get('name', 'case')}_mat{mat_type}"
    return c


def hex_box(nx, ny, nz, h, jitter=0.0, seed=1):
    """A structured hexahedral mesh of nx*ny*nz nodes at spacing h, each
    coordinate jittered by a seeded uniform +-jitter*h; hexes in the
    LS-DYNA node order (bottom face counter-clockwise, then the top face),
    0-based node ids, (nx-1)(ny-1)(nz-1) elements."""
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    coo = np.stack([i.ravel() * h, j.ravel() * h, k.ravel() * h], axis=1).astype(np.float64)
    if jitter:
        rng = np.random.Generator(np.random.PCG64(seed))
        coo += rng.uniform(-jitter * h, jitter * h, size=coo.shape)
    nid = lambda a, b, c: a + nx * (b + ny * c)
    ek, ej, ei = np.meshgrid(np.arange(nz - 1), np.arange(ny - 1), np.arange(nx - 1), indexing="ij")
    ei, ej, ek = ei.ravel(), ej.ravel(), ek.ravel()
    elems = np.stack([nid(ei, ej, ek), nid(ei + 1, ej, ek), nid(ei + 1, ej + 1, ek), nid(ei, ej + 1, ek),
                      nid(ei, ej, ek + 1), nid(ei + 1, ej, ek + 1), nid(ei + 1, ej + 1, ek + 1),
                      nid(ei, ej + 1, ek + 1)], axis=1).astype(np.int32)
    return coo, elems


def smoothing_lengths(vol, win_raw):
    """GET_SMOOTHING_LENGTHS (PRE_MODEL_SMOOTHING_LENGTHS.F90:49-99) with the
    raw windows: SM_LEN(6,N) and (XDIST_MAX, YDIST_MAX, ZDIST_MAX)."""
    dim = 2.0 * win_raw
    vol_win = dim[:, 0] * dim[:, 1] * dim[:, 2]
    ratio = vol ** THRD / vol_win ** THRD
    sm = np.empty((len(vol), 6))
    sm[:, 0] = sm[:, 1] = dim[:, 0] * ratio / 2.0
    sm[:, 2] = sm[:, 3] = dim[:, 1] * ratio / 2.0
    sm[:, 4] = sm[:, 5] = dim[:, 2] * ratio / 2.0
    dist_max = np.array([max(0.0, sm[:, 0].max()), max(0.0, sm[:, 2].max()), max(0.0, sm[:, 5].max())])
    return sm, dist_max


def cylinder_lattice(h, R, L, jitter=0.05, seed=1, planar_wall=True):
    """Nodes (i h, j h, k h) with i^2 + j^2 <= (R/h)^2, 0 <= k h <= L; x runs
    fastest, then y, then z.  Each coordinate gets a seeded uniform jitter of
    +-jitter*h (PCG64); the k = 0 layer keeps z exact so the wall is planar."""
    r = int(round(R / h))
    nk = int(round(L / h)) + 1
    ii, jj = np.meshgrid(np.arange(-r, r + 1), np.arange(-r, r + 1), indexing="xy")
    ii, jj = ii.ravel(), jj.ravel()
    keep = ii * ii + jj * jj <= r * r
    ii, jj = ii[keep], jj[keep]
    m = len(ii)
    k = np.repeat(np.arange(nk), m)
    coo = np.empty((m * nk, 3))
    coo[:, 0] = np.tile(ii, nk) * h
    coo[:, 1] = np.tile(jj, nk) * h
    coo[:, 2] = k * h
    rng = np.random.Generator(np.random.PCG64(seed))
    jit = rng.uniform(-jitter * h, jitter * h, size=coo.shape)
    if planar_wall:
        jit[k == 0, 2] = 0.0
    return coo + jit, k


def taylor_bar(h=0.4e-3, R=3.2e-3, L=32.4e-3, jitter=0.05, seed=1, v0=227.0, E=117e9, nu=0.35,
               rho=8930.0, sy=400e6, H=100e6, norm_win=2.0, mat_type=2, rate_law=None,
               planar_wall=True, damping=0.0):
    """Copper Taylor bar (D = 2R, length L, axis z) on a jittered cubic lattice
    against a rigid frictionless wall at z = 0 (fixity 0 0 1 on the k = 0
    layer).  Linear hardening sigma_y + H eps_p maps onto the reference law
    sigma_y (1 + B eps_p)^C with B = H / sigma_y, C = 1.  rate_law =
    (A, B, n, C, epsdot0) selects the power-law rate-dependent law (type 7)."""
    coo, k = cylinder_lattice(h, R, L, jitter, seed, planar_wall)
    n = len(coo)
    vol = np.full(n, math.pi * R * R * L / n)
    win_raw = np.full((n, 3), h)
    sm_len, dist_max = smoothing_lengths(vol, win_raw)
    if rate_law is not None:
        A, B, nexp, C, ed0 = rate_law
        pv = props_vector(7, E, nu, rho, A, B, nexp, C, ed0, damping=damping)
        mat_type = 7
    else:
        pv = props_vector(mat_type, E, nu, rho, sy, H / sy, 1.0, damping=damping)
    wall = k == 0
    ebc = np.zeros((n, 3), np.int32)
    ebc[wall, 2] = 1
    vinit = np.zeros((n, 3))
    vinit[:, 2] = -v0
    return dict(
        name=f"taylor_bar_h{h*1e3:.3g}mm", n=n, coo=coo, win=win_raw * norm_win, win_raw=win_raw, vol=vol,
        mass=np.repeat((vol * rho)[:, None], 3, axis=1).copy(), ebc=ebc, vinit=vinit,
        props=np.tile(pv, (n, 1)), mat_type=np.full(n, mat_type, np.int32), body_id=np.ones(n, np.int32),
        bodyforce=None, sm_len=sm_len, dist_max=dist_max, ql_len=0.1 * win_raw.min(), wall=wall, h=h,
        layer=k, R=R, L=L, v0=v0)


def bar_metrics(case, coo_cur, eps):
    """End-state measures of a Taylor test: bar length (z extent), mushroom
    radius (largest radius of the wall layer), peak equivalent plastic
    strain (the largest nodal value) and two aggregate measures of the same
    field that one node's history cannot move: its 99.9th percentile over the
    nodes and the mean of its largest 0.1 % of nodal values."""
    x = np.asarray(coo_cur).reshape(-1, 3)
    w = case["wall"]
    e = np.asarray(eps)
    top = np.sort(e)[-max(1, len(e) // 1000):]
    return dict(length=float(x[:, 2].max() - x[:, 2].min()),
                radius=float(np.sqrt(x[w, 0] ** 2 + x[w, 1] ** 2).max()),
                peak_eps=float(np.max(e)),
                eps_p999=float(np.percentile(e, 99.9)),
                eps_top_mean=float(np.mean(top)))


def batch_bars(nbars=256, seed=5, h_range=(0.15e-3, 0.6e-3), v0_range=(100.0, 300.0), sy_range=(200e6, 600e6),
               H=100e6, rate_law=None, **bar):
    """Many Taylor bars of uneven size stepped as one batch: instance k has
    lattice spacing h_k, impact speed v0_k and yield stress sy_k drawn
    uniformly from the ranges (one seed), linear hardening H -- or, with
    rate_law = (B, n, C, epsdot0), the power-law rate-dependent law with
    A = sy_k.  The bars keep their own coordinates (they overlap in space;
    each is searched alone).  Returns the concatenated case with `counts`,
    per-instance `dist_max` (nbars, 3), stable steps `dt` (nbars), `params`
    (h, v0, sy) and the instances themselves."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hs = rng.uniform(*h_range, nbars)
    v0s = rng.uniform(*v0_range, nbars)
    sys_ = rng.uniform(*sy_range, nbars)
    bars = [taylor_bar(h=float(hs[k]), v0=float(v0s[k]), sy=float(sys_[k]), H=H, seed=seed * 1000 + k,
                       rate_law=None if rate_law is None else (float(sys_[k]),) + tuple(rate_law), **bar)
            for k in range(nbars)]
    keys = ("coo", "win", "win_raw", "vol", "mass", "ebc", "vinit", "props", "mat_type", "body_id", "sm_len", "wall",
            "layer")
    out = {k: np.concatenate([b[k] for b in bars]) for k in keys}
    out.update(name=f"batch_{nbars}_bars", n=int(sum(b["n"] for b in bars)), bodyforce=None,
               counts=np.array([b["n"] for b in bars], np.int32),
               dist_max=np.stack([b["dist_max"] for b in bars]),
               ql_len=float(min(b["ql_len"] for b in bars)), params=np.stack([hs, v0s, sys_], axis=1), bars=bars,
               h=float(hs.min()), dt=np.array([lattice_dt(b) for b in bars]))
    return out


def lattice_dt(bar, cfl=0.2):
    """A stable step of a jittered lattice bar without its neighbour lists:
    cfl x (0.9 h, the closest two nodes of a +-5 % jitter can be) over the
    dilatational wave speed.  cfl = 0.2 keeps the impact of every bar of
    batch_bars finite through 1,500 steps (with 0.5 the fast bars' nodes
    close in at the wall and their steps go non-finite after 400-1,200)."""
    p = bar["props"][0]
    E, nu, rho = p[1], p[0], p[2]
    K, G = E / (3.0 * (1.0 - 2.0 * nu)), E / (2.0 * (1.0 + nu))
    return float(cfl * 0.9 * bar["h"] / np.sqrt((K + 4.0 * G / 3.0) / rho))


def param_kwargs(case, **over):
    """mega_params values for a case (Control.dat defaults: RK 1/3/0, QL 1
    0.001, DNI, Lagrangian finite strain, box support)."""
    dmax = np.asarray(case["dist_max"], dtype=np.float64).reshape(-1, 3).max(axis=0)  # a batch: the largest
    kw = dict(rk_degree=1, rk_cont=3, rk_impl=0, itype_int=0, ql=1, lagrangian=1, finite_strain=1, shsup=0,
              peridynamics=0, inv3_exact=0, newton_max_iter=20, ql_coef=0.001, ql_len=float(case["ql_len"]),
              gravity=(0.0, 0.0, 0.0), dist_max=tuple(float(v) for v in dmax), newton_rtol=1e-10)
    kw.update(over)
    return kw


def stable_dt(case, gn, gstart, gstack, cfl=0.5, chunk=1 << 22):
    """Fixed step 0.5 * min_i(d_min,i / c_i) (the CFL rule of FINT.F90:
    1280-1311, commented out in the reference, evaluated once): d_min = the
    nearest neighbour distance, c = sqrt(max(K + 4G/3, G) / rho).  Evaluated
    over list chunks of `chunk` entries to bound host memory."""
    coo = case["coo"]
    n = case["n"]
    gn = np.asarray(gn, np.int64)
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(gn, out=ptr[1:])
    dmin = np.full(n, np.inf)
    r0 = 0
    while r0 < n:
        r1 = int(np.searchsorted(ptr, ptr[r0] + chunk, side="right")) - 1
        r1 = min(n, max(r1, r0 + 1))
        rows = np.repeat(np.arange(r0, r1), gn[r0:r1])
        cols = np.asarray(gstack[ptr[r0]:ptr[r1]], np.int64) - 1
        d = np.linalg.norm(coo[cols] - coo[rows], axis=1)
        d[cols == rows] = np.inf
        np.minimum.at(dmin, rows, d)
        r0 = r1
    p = case["props"]
    E, nu, rho = p[:, 1], p[:, 0], p[:, 2]
    K = E / (3.0 * (1.0 - 2.0 * nu))
    G = E / (2.0 * (1.0 + nu))
    c = np.sqrt(np.maximum(K + 4.0 * G / 3.0, G) / rho)
    return float(cfl * np.min(dmin / c))


def pd_plate(h=0.25e-3, nx=400, ny=400, nz=16, horizon=3.015, E=72e9, rho=2440.0, s_c=1e-3,
             notch=20e-3, v_edge=5.0, seed=1, jitter=0.0):
    """Brittle glass-like plate for bond-based PMB peridynamics: a nx*ny*nz
    lattice at spacing h, horizon delta = horizon*h (spherical support),
    micromodulus c = 18 K / (pi delta^4) with K = E / (3 (1 - 2 nu)), nu =
    1/4 (bond-based restriction).  A pre-notch of length `notch` at mid-edge
    (plane y = mid, x < notch) starts with the bonds that cross it broken;
    the two halves of the edge x = 0 (three particle columns, `fixed`) are
    driven apart at a sustained +-v_edge in y."""
    xs = (np.arange(nx) + 0.5) * h
    ys = (np.arange(ny) + 0.5) * h
    zs = (np.arange(nz) + 0.5) * h
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    coo = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if jitter:
        rng = np.random.Generator(np.random.PCG64(seed))
        coo += rng.uniform(-jitter * h, jitter * h, size=coo.shape)
    n = len(coo)
    delta = horizon * h
    K = E / (3.0 * (1.0 - 2.0 * 0.25))
    c = 18.0 * K / (math.pi * delta ** 4)
    vol = np.full(n, h ** 3)
    ymid = 0.5 * ny * h
    vel = np.zeros((n, 3))
    edge = coo[:, 0] < 3 * h
    vel[edge & (coo[:, 1] > ymid), 1] = v_edge
    vel[edge & (coo[:, 1] < ymid), 1] = -v_edge
    return dict(name=f"pmb_plate_{nx}x{ny}x{nz}", n=n, coo=coo, win=np.full((n, 3), delta), vol=vol, rho=rho,
                c=c, s_c=s_c, delta=delta, h=h, notch=notch, ymid=ymid, vinit=vel, sm_len=np.zeros((n, 6)),
                dist_max=np.zeros(3), fixed=edge.astype(np.int32))


def crack_tip(case, damage, threshold=0.35):
    """Crack tip of a plate from the local damage of its particles: the
    largest x among particles within two horizons of the notch plane whose
    damage exceeds `threshold` (None when none does)."""
    coo = case["coo"]
    near = np.abs(coo[:, 1] - case["ymid"]) < 2.0 * case["delta"]
    hit = near & (np.asarray(damage) > threshold)
    if not np.any(hit):
        return None
    return float(coo[hit, 0].max())


def notch_broken(case, gn, gstart, gstack):
    """Bonds crossing the pre-notch plane y = ymid for x < notch start broken."""
    coo = case["coo"]
    n = case["n"]
    rows = np.repeat(np.arange(n), gn)
    cols = gstack - 1
    yi, yj = coo[rows, 1], coo[cols, 1]
    cross = ((yi - case["ymid"]) * (yj - case["ymid"]) < 0.0)
    # the segment crosses the plane at x = x_i + t (x_j - x_i)
    t = (case["ymid"] - yi) / np.where(yj != yi, yj - yi, 1.0)
    xc = coo[rows, 0] + t * (coo[cols, 0] - coo[rows, 0])
    return (cross & (xc < case["notch"])).astype(np.uint8)


def notch_rect(case):
    """The pre-notch of notch_broken as a cut rectangle (corner, edge a, edge
    b) for the device cut: plane y = ymid, x up to the notch length, through
    the whole thickness."""
    zmax = float(np.max(case["coo"][:, 2]))
    corner = np.array([-1.0, case["ymid"], -1.0])
    return corner, np.array([case["notch"] + 1.0, 0.0, 0.0]), np.array([0.0, 0.0, zmax + 2.0])


def case_a(npz):
    """Golden case A: the reference's Taylor_bar.k + Control.dat deck, from
    the arrays tests/golden/make_case_a.py extracted (raw windows, volumes,
    node sets).  Deck values: window 2.75 on BAR, fixity 0 0 1 on WALL,
    v = (0, 0, -373) on BAR, material type 2 with PROPS 0.3 78.2e9 2700
    0.29e9 125 0.1, QL 1 0.001 with QL_LEN = 0.1 * min raw window
    (PRE_CONTROL.F90:803-828), dt = 0.78363e-7, TIME_END = 5.5e-5."""
    z = np.load(npz)
    coo = z["coo"]
    n = len(coo)
    win_raw = z["win_raw"]
    norm = np.full(n, 1.8)                      # default normalised window (PRE_CONTROL.F90:604-609)
    norm[z["bar"] - 1] = float(z["norm_win"])
    win = win_raw * norm[:, None]               # PRE_CONTROL.F90:870-872
    vol = z["vol"]
    sm_len, dist_max = smoothing_lengths(vol, win_raw)
    pr = z["props"]
    pv = props_vector(int(z["mat_type"]), pr[1], pr[0], pr[2], pr[3], pr[4], pr[5])
    ebc = np.zeros((n, 3), np.int32)
    ebc[z["wall"] - 1, 2] = 1
    vinit = np.zeros((n, 3))
    vinit[z["bar"] - 1, 2] = -float(z["v0"])
    rho = pr[2]
    wall = np.zeros(n, bool)
    wall[z["wall"] - 1] = True
    dt = float(z["dt"])
    nsteps = 0
    t = 0.0
    while True:                                 # MAIN.F90:644-656: TIME = TIME + DLT until TIME > TIME_END
        t = t + dt
        nsteps += 1
        if t > float(z["time_end"]):
            break
    return dict(name="case_a_Taylor_bar_k", n=n, coo=coo, win=win, win_raw=win_raw, vol=vol,
                mass=np.repeat((vol * rho)[:, None], 3, axis=1).copy(), ebc=ebc, vinit=vinit,
                props=np.tile(pv, (n, 1)), mat_type=np.full(n, int(z["mat_type"]), np.int32),
                body_id=np.ones(n, np.int32), bodyforce=None, sm_len=sm_len, dist_max=dist_max,
                ql_len=0.1 * win_raw.min(), wall=wall, dt=dt, nsteps=nsteps, v0=float(z["v0"]))
