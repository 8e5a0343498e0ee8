"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.  See
mega_oracle.cpp for what it restates and which reference lines it follows.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double

_SIG = {
    "orc_bin_search": (I32, [I32, P, P, P, P, I32, I32, P, P, P, I64, P, P, P, P, P]),
    "orc_rk_shapes": (I32, [P, I32, P, P, P, P, P, P, P, P, I32]),
    "orc_hughes_winget": (None, [I32, P, P, P, P, I32]),
    "orc_rotate_tensor": (None, [I32, P, P]),
    "orc_constitution": (I32, [I32, P, P, P, D, P, P, P, I32, D, I32]),
    "orc_vm_rate": (I32, [I32, P, P, D, D, I32, P, P, P, P, P, I32]),
    "orc_damaged": (I32, [I32, P, P, P, P, P, P, P, I32]),
    "orc_construct_fint": (I32, [P, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, I32, D, P, P, P, P,
                                 P, I32, P, P, P, P, P]),
    "orc_interp": (None, [I32, P, P, P, P, P, P, I32]),
    "orc_pd_shape": (I32, [I32, P, P, P, P, P, P, P, P, I32]),
    "orc_construct_fint_pd": (I32, [P, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, I32, D, P, P, I32]),
    "orc_fixity2_velocity": (None, [I32, P, P, D, P]),
    "orc_corrector": (None, [I32, P, P, P, P, P, P, P, P, P, P, D, P]),
    "orc_step": (I32, [P, I32] + [P] * 31 + [D, I32, I32, P, P, P, P, P]),
    "orc_pmb_force": (I64, [I32, P, P, P, P, P, P, D, D, P, P, I32]),
    "orc_mlp_nparams": (I64, [I32]),
    "orc_mlp_forward_backward": (D, [I32, P, I32, P, P, P, P]),
    "orc_adam": (None, [I64, P, P, P, P, D, D, D, D, I32]),
}

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "mega_oracle.cpp")
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
            build()
        L = C.CDLL(LIB)
        for k, (r, a) in _SIG.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def bin_search(coo, win, sm_len, dist_max, itype_int=0, shsup=False, geom_in=None):
    """BIN_SEARCH; geom_in (9 values, as returned in "geom") reuses the bins
    laid out at LINIT, as the semi-Lagrangian re-search does."""
    coo, win, sm_len, dist_max = f64(coo), f64(win), f64(sm_len), f64(dist_max)
    n = len(coo)
    gn = np.zeros(n, np.int32)
    gstart = np.zeros(n, np.int32)
    ijk = np.zeros((n, 3), np.int32)
    cap = n * 128
    nnz = C.c_int64(0)
    gmaxn = C.c_int32(0)
    geom = np.zeros(9)
    while True:
        gstack = np.zeros(cap, np.int32)
        st = lib().orc_bin_search(n, _p(coo), _p(win), _p(sm_len), _p(dist_max), int(itype_int), int(bool(shsup)),
                                  _p(gn), _p(gstart), _p(gstack), cap, C.byref(nnz), C.byref(gmaxn), _p(ijk),
                                  _p(geom), _p(None if geom_in is None else f64(geom_in)))
        if not (st & 0x40):
            break
        cap = int(nnz.value)
    return dict(gn=gn, gstart=gstart, gstack=gstack[: nnz.value].copy(), gmaxn=gmaxn.value, ijk=ijk,
                nnz=nnz.value, geom=geom, status=st)


class Params(C.Structure):
    """Same layout as mega_params in include/mega_gpu.h."""
    _fields_ = [
        ("rk_degree", C.c_int32), ("rk_cont", C.c_int32), ("rk_impl", C.c_int32),
        ("itype_int", C.c_int32), ("ql", C.c_int32), ("lagrangian", C.c_int32),
        ("finite_strain", C.c_int32), ("shsup", C.c_int32), ("peridynamics", C.c_int32),
        ("inv3_exact", C.c_int32), ("newton_max_iter", C.c_int32), ("rate_solver", C.c_int32),
        ("ql_coef", C.c_double), ("ql_len", C.c_double), ("gravity", C.c_double * 3),
        ("dist_max", C.c_double * 3), ("newton_rtol", C.c_double),
        ("auto_ts", C.c_int32), ("reserved", C.c_int32), ("dlt_fac", C.c_double),
    ]


def params(**kw):
    p = Params()
    p.rk_degree, p.rk_cont, p.itype_int, p.ql, p.lagrangian, p.finite_strain = 1, 3, 0, 1, 1, 1
    p.newton_max_iter, p.ql_coef, p.newton_rtol = 20, 0.001, 1e-10
    for k, v in kw.items():
        if k in ("gravity", "dist_max"):
            for i in range(3):
                getattr(p, k)[i] = float(v[i])
        else:
            setattr(p, k, v)
    return p


def rk_shapes(p, coo, win, ebc_nodes, gn, gstart, gstack, nthreads=8):
    coo, win = f64(coo), f64(win)
    nnz = len(gstack)
    shp = np.zeros(nnz)
    dshp = np.zeros((nnz, 3))
    en = None if ebc_nodes is None else i32(ebc_nodes)
    st = lib().orc_rk_shapes(C.byref(p), len(coo), _p(coo), _p(win), _p(en), _p(i32(gn)), _p(i32(gstart)),
                             _p(i32(gstack)), _p(shp), _p(dshp), nthreads)
    return shp, dshp, st


def hughes_winget(lmat, exact=False):
    lm = np.ascontiguousarray(np.transpose(f64(lmat), (0, 2, 1)))
    n = len(lm)
    rot = np.zeros((n, 3, 3))
    strain = np.zeros((n, 6))
    d = np.zeros((n, 6))
    lib().orc_hughes_winget(n, _p(lm), _p(rot), _p(strain), _p(d), int(exact))
    return np.transpose(rot, (0, 2, 1)).copy(), strain, d


def rotate_tensor(rot, v):
    r = np.ascontiguousarray(np.transpose(f64(rot), (0, 2, 1)))
    v = f64(v).copy()
    lib().orc_rotate_tensor(len(v), _p(r), _p(v))
    return v


def constitution(spred, mat, props, dlt, state, maxit=20, rtol=1e-10, solver=0):
    spred = f64(spred)
    n = len(spred)
    state = f64(state).copy()
    stress = np.zeros((n, 6))
    it = np.zeros(n, np.int32)
    st = lib().orc_constitution(n, _p(spred), _p(i32(mat)), _p(f64(props)), float(dlt), _p(state), _p(stress),
                                _p(it), maxit, rtol, int(solver))
    return stress, state, it, st


def damaged(stress_rot, tot, inc, mat, props, state, maxit=20):
    """DRUCK_PRAG (3) / VON_MISES_DAM (6) from the rotated old stress, the
    total strain and the strain increment: (stress, state, passes, status)."""
    stress = f64(stress_rot).copy()
    n = len(stress)
    state = f64(state).copy()
    it = np.zeros(n, np.int32)
    st = lib().orc_damaged(n, _p(i32(mat)), _p(f64(props)), _p(f64(tot)), _p(f64(inc)), _p(state), _p(stress),
                           _p(it), int(maxit))
    return stress, state, it, st


def vm_rate(spred, props, dt, state, dg0=None, rtol=1e-10, maxit=50, solver=0):
    spred = f64(spred)
    n = len(spred)
    state = f64(state).copy()
    stress = np.zeros((n, 6))
    it = np.zeros(n, np.int32)
    dg = np.zeros(n)
    st = lib().orc_vm_rate(n, _p(spred), _p(f64(props)), float(dt), float(rtol), int(maxit),
                           _p(None if dg0 is None else f64(dg0)), _p(state), _p(stress), _p(it), _p(dg),
                           int(solver))
    return stress, state, it, dg, st


def construct_fint(p, case, state, stress, strain, dinc, dinc_tot, nb, shp, dshp, linit, dlt, nthreads=1,
                   gint_work=0.0, ddshp=None, sgrad=None, coo_current=None):
    """CONSTRUCT_FINT; with p.itype_int == 2 (NSNI) ddshp (6 per list entry,
    built when linit) and sgrad (18 per node, the stress gradients) are
    updated in place too; p.lagrangian == 0 (semi-Lagrangian) builds the
    shapes on coo_current every call."""
    n = case["n"]
    fint = np.zeros(3 * n)
    fext = np.zeros(3 * n)
    wv = np.zeros(n)
    seq = np.zeros(n)
    it = np.zeros(n, np.int32)
    gw = C.c_double(gint_work)
    en = i32(np.any(case["ebc"] == 1, axis=1))
    bf = case.get("bodyforce")
    st = lib().orc_construct_fint(
        C.byref(p), n, _p(f64(case["coo"])), _p(f64(case["win"])), _p(f64(case["vol"])), _p(f64(case["props"])),
        _p(i32(case["mat_type"])), _p(en), _p(None if bf is None else f64(bf)), _p(state), _p(stress), _p(strain),
        _p(f64(dinc)), _p(f64(dinc_tot)), _p(i32(nb["gn"])), _p(i32(nb["gstart"])), _p(i32(nb["gstack"])), _p(shp),
        _p(dshp), int(bool(linit)), float(dlt), _p(fint), _p(fext), _p(wv), _p(seq), C.byref(gw), int(nthreads),
        _p(it), _p(f64(case["sm_len"]) if ddshp is not None else None), _p(ddshp), _p(sgrad),
        _p(None if coo_current is None else f64(coo_current)))
    return dict(fint=fint, fext=fext, gmax_wvel=wv, gstrain_eq=seq, gint_work=gw.value, iters=it, status=st)


class Run:
    """MAIN.F90:304-658 on the CPU oracle: LINIT (search, RK1, zero-force
    CONSTRUCT_FINT) then steps of predictor / interp / force / corrector."""

    def __init__(self, case, p, nthreads=1, serial_interp=True):
        self.case, self.p = case, p
        self.n = n = case["n"]
        self.nthreads = nthreads
        self.serial_interp = serial_interp
        self.semi = p.lagrangian == 0
        self.nb = bin_search(case["coo"], case["win"], case["sm_len"], case["dist_max"], p.itype_int, p.shsup)
        self.geom = self.nb["geom"].copy()  # the LINIT bins (kept by the semi-Lagrangian re-search)
        nnz = self.nb["nnz"]
        self.shp = np.zeros(nnz)
        self.dshp = np.zeros(3 * nnz)
        self.state = np.zeros((n, 20))
        self.stress = np.zeros((n, 6))
        self.strain = np.zeros((n, 6))
        self.dsp = np.zeros(3 * n)
        self.dsp_tot = np.zeros(3 * n)
        self.dsp_tot_phy = np.zeros(3 * n)
        ebc = case["ebc"].reshape(-1)
        self.vel = np.where(ebc == 1, 0.0, case["vinit"].reshape(-1)).astype(np.float64)
        self.acl = np.zeros(3 * n)
        self.fint = np.zeros(3 * n)
        self.fext = np.zeros(3 * n)
        self.prforce = np.zeros(3 * n)
        self.coo_cur = f64(case["coo"]).reshape(-1).copy()
        self.wvel = np.zeros(n)
        self.strain_eq = np.zeros(n)
        self.en = np.zeros(4)
        self.total_force = np.zeros(6)
        self.iters = np.zeros(n, np.int32)
        self.time = 0.0
        self.steps = 0
        # NSNI: smoothed second derivatives (6 per entry), stress gradients (18 per node)
        self.ddshp = np.zeros(6 * nnz) if p.itype_int == 2 else None
        self.sgrad = np.zeros((n, 18)) if p.itype_int == 2 else None
        # LINIT: shapes + a force call at zero displacement (MAIN.F90:320-334)
        r = construct_fint(p, case, self.state, self.stress, self.strain, self.dsp, self.dsp_tot, self.nb,
                           self.shp, self.dshp, True, 0.0, nthreads, ddshp=self.ddshp, sgrad=self.sgrad,
                           coo_current=self.coo_cur if self.semi else None)
        self.init_status = r["status"]
        self.en[3] = r["gint_work"]
        self.fixity2 = None  # (FIXITY2_TIME (steps,2), FIXITY2_NONZERO_EBC (steps,3)) of fixity code 2

    def set_fixity2(self, times, disp):
        """The prescribed-displacement windows of fixity code 2 (MODEL.F90:61-62)."""
        t = np.asfortranarray(np.asarray(times, np.float64).reshape(-1, 2))
        d = np.asfortranarray(np.asarray(disp, np.float64).reshape(-1, 3))
        self.fixity2 = (len(t), t.ravel(order="F").copy(), d.ravel(order="F").copy())

    def _vel2(self):
        """Prescribed velocities of this step's TIME (MAIN.F90:448-462)."""
        v = np.zeros(3)
        if self.fixity2 is not None:
            k, t, d = self.fixity2
            lib().orc_fixity2_velocity(k, _p(t), _p(d), float(self.time), _p(v))
        return v

    def _semi_step(self, dt):
        """MAIN.F90:348-488 with LLAGRANGIAN = .FALSE.: predictor, DO_INTERP
        with the last lists and shapes, the current coordinates, a re-search
        on them in the LINIT bins (HANDELER.F90:145, 252-273), CONSTRUCT_FINT
        with shapes on the current coordinates, corrector, energies."""
        c, n, p = self.case, self.n, self.p
        dsp = dt * self.vel + dt * dt * 0.5 * self.acl                 # MAIN.F90:353-355
        self.dsp[:] = dsp
        self.dsp_tot += dsp
        self.vel += dt * 0.5 * self.acl
        dphy = np.zeros(3 * n)
        nb = self.nb
        lib().orc_interp(n, _p(nb["gn"]), _p(nb["gstart"]), _p(nb["gstack"]), _p(self.shp), _p(self.dsp), _p(dphy), 1)
        self.dsp_tot_phy += dphy                                         # MAIN.F90:377-386
        self.coo_cur[:] = f64(c["coo"]).reshape(-1) + self.dsp_tot_phy
        self.nb = bin_search(self.coo_cur.reshape(-1, 3), c["win"], c["sm_len"], c["dist_max"], p.itype_int,
                             p.shsup, geom_in=self.geom)
        self.shp = np.zeros(self.nb["nnz"])
        self.dshp = np.zeros(3 * self.nb["nnz"])
        fext_nmo = self.fext.copy()
        r = construct_fint(p, c, self.state, self.stress, self.strain, self.dsp, self.dsp_tot, self.nb, self.shp,
                           self.dshp, False, dt, self.nthreads, gint_work=self.en[3], coo_current=self.coo_cur)
        self.en[3] = r["gint_work"]
        self.fint[:], self.fext[:] = r["fint"], r["fext"]
        self.wvel[:], self.strain_eq[:], self.iters[:] = r["gmax_wvel"], r["gstrain_eq"], r["iters"]
        p21 = np.ascontiguousarray(f64(c["props"])[:, 20])
        lib().orc_corrector(n, _p(i32(c["ebc"])), _p(p21), _p(f64(c["mass"])), _p(self.fint), _p(self.fext),
                            _p(self.vel), _p(self.acl), _p(self.prforce), _p(i32(c["body_id"])),
                            _p(self.total_force), float(dt), _p(self._vel2()))
        mass = f64(c["mass"]).reshape(-1)
        self.en[0] = self.en[3]
        self.en[1] = float(np.sum(0.5 * mass * self.vel * self.vel))
        self.en[2] = self.en[2] + float(np.sum(0.5 * (self.fext + fext_nmo) * self.dsp))
        return r["status"] | (self.nb["status"] & ~0x40)

    def step(self, nsteps, dt):
        c = self.case
        st = 0
        if self.semi:
            for _ in range(nsteps):
                st |= self._semi_step(dt)
                self.time += dt
                self.steps += 1
            return st
        en_ebc = i32(np.any(c["ebc"] == 1, axis=1))
        bf = c.get("bodyforce")
        for _ in range(nsteps):
            st |= lib().orc_step(
                C.byref(self.p), self.n, _p(f64(c["coo"])), _p(f64(c["win"])), _p(f64(c["vol"])),
                _p(f64(c["mass"])), _p(i32(c["ebc"])), _p(f64(c["props"])), _p(i32(c["mat_type"])), _p(en_ebc),
                _p(None if bf is None else f64(bf)), _p(i32(c["body_id"])), _p(self.nb["gn"]), _p(self.nb["gstart"]),
                _p(self.nb["gstack"]), _p(self.shp), _p(self.dshp), _p(self.state), _p(self.stress), _p(self.strain),
                _p(self.dsp), _p(self.dsp_tot), _p(self.dsp_tot_phy), _p(self.vel), _p(self.acl), _p(self.fint),
                _p(self.fext), _p(self.prforce), _p(self.coo_cur), _p(self.wvel), _p(self.strain_eq), _p(self.en),
                _p(self.total_force), float(dt), int(self.nthreads), int(bool(self.serial_interp)), _p(self.iters),
                _p(f64(c["sm_len"]) if self.ddshp is not None else None), _p(self.ddshp), _p(self.sgrad),
                _p(self._vel2()))
            self.time += dt
            self.steps += 1
        return st


def pd_shape(case, nb, nthreads=8):
    n = case["n"]
    shp = np.zeros(nb["nnz"])
    ginvk = np.zeros((n, 3, 3))
    st = lib().orc_pd_shape(n, _p(f64(case["coo"])), _p(f64(case["win"])), _p(f64(case["vol"])), _p(i32(nb["gn"])),
                            _p(i32(nb["gstart"])), _p(i32(nb["gstack"])), _p(shp), _p(ginvk), nthreads)
    return shp, ginvk, st


def construct_fint_pd(p, case, cur, state, stress, strain, dinc, nb, shp, ginvk, linit, dlt, nthreads=1):
    n = case["n"]
    fint = np.zeros(3 * n)
    wv = np.zeros(n)
    st = lib().orc_construct_fint_pd(
        C.byref(p), n, _p(f64(case["coo"])), _p(f64(cur)), _p(f64(case["vol"])), _p(f64(case["props"])),
        _p(i32(case["mat_type"])), _p(state), _p(stress), _p(strain), _p(f64(dinc)), _p(i32(nb["gn"])),
        _p(i32(nb["gstart"])), _p(i32(nb["gstack"])), _p(f64(shp)), _p(f64(ginvk)), int(bool(linit)), float(dlt),
        _p(fint), _p(wv), int(nthreads))
    return fint, wv, st


def pmb_force(case, nb, u, broken, nthreads=8):
    n = case["n"]
    f = np.zeros(3 * n)
    nbk = lib().orc_pmb_force(n, _p(f64(case["coo"])), _p(f64(u)), _p(f64(case["vol"])), _p(i32(nb["gn"])),
                              _p(i32(nb["gstart"])), _p(i32(nb["gstack"])), float(case["c"]), float(case["s_c"]),
                              _p(broken), _p(f), nthreads)
    return f, int(nbk)


def mlp_nparams(H):
    return int(lib().orc_mlp_nparams(H))


def mlp_forward_backward(H, theta, x, t=None, grad=True):
    theta, x = f64(theta), f64(x)
    nb = len(x)
    y = np.zeros(nb)
    g = np.zeros(mlp_nparams(H)) if (grad and t is not None) else None
    loss = lib().orc_mlp_forward_backward(H, _p(theta), nb, _p(x), _p(None if t is None else f64(t)), _p(y), _p(g))
    return loss, y, g


def adam(theta, g, m, v, lr, t, b1=0.9, b2=0.999, eps=1e-8):
    lib().orc_adam(len(theta), _p(theta), _p(f64(g)), _p(m), _p(v), lr, b1, b2, eps, int(t))
