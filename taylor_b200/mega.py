"""Host-side mirror of MEGA's hot-path interface over libmega_gpu.so.

Function names and argument meanings follow the reference's subroutines:
  bin_search        GET_BINS + SOFT_SEARCH      (BIN_SEARCH.F90:2-328)
  rk_shapes         RK1 over all nodes           (RK.f90:16-453, FINT.F90:404-408)
  hughes_winget     HUGHES_WINGET                (HUGHES_WINGET.F90:16-81)
  rotate_tensor     ROTATE_TENSOR                (ROTATE_TENSOR.F90:21-87)
  constitution      CONSTITUTION                 (CONSTITUTION.F90:18-89)
  construct_fint    CONSTRUCT_FINT               (FINT.F90:16-1336)
  construct_fint_pd CONSTRUCT_FINT_PD            (FINT_PD.F90:16-759)
  Mega              the MAIN.F90:304-658 time loop, device resident.
Errors are raised as MegaError with the reference's message, the way
EXIT_PROGRAM would stop the Fortran program.  Neighbour lists are 1-based.
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, ptr


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def bin_search(coo, win, sm_len, dist_max, itype_int=0, shsup=False, dim_nn_list=None):
    """Neighbour lists of every node (GN, GSTART, GSTACK 1-based, GMAXN, GIJKSPC)."""
    coo, win, sm_len = _f64(coo), _f64(win), _f64(sm_len)
    dist_max = _f64(dist_max)
    n = len(coo)
    gn = np.zeros(n, np.int32)
    gstart = np.zeros(n, np.int32)
    ijk = np.zeros((n, 3), np.int32)
    gmaxn = C.c_int32(0)
    nnz = C.c_int64(0)
    cap = int(dim_nn_list) if dim_nn_list else n * 128
    while True:
        gstack = np.zeros(cap, np.int32)
        st = _lib.lib().mega_bin_search(n, ptr(coo), ptr(win), ptr(sm_len), ptr(dist_max), int(itype_int),
                                        int(bool(shsup)), ptr(gn), ptr(gstart), ptr(gstack), cap,
                                        C.byref(gmaxn), ptr(ijk), C.byref(nnz))
        if st > 0 and (st & _lib.ST_STACK_OVERFLOW) and not dim_nn_list:
            cap = int(nnz.value)
            continue
        check(st, "bin_search")
        break
    return dict(gn=gn, gstart=gstart, gstack=gstack[: nnz.value].copy(), gmaxn=gmaxn.value, ijk=ijk,
                nnz=int(nnz.value))


def rk_shapes(params, coo, win, ebc_nodes, gn, gstart, gstack):
    """GSTACK_SHP (nnz) and GSTACK_DSHP (nnz,3) from RK1 at every node."""
    coo, win = _f64(coo), _f64(win)
    gn, gstart, gstack = _i32(gn), _i32(gstart), _i32(gstack)
    n = len(coo)
    nnz = len(gstack)
    shp = np.zeros(nnz)
    dshp = np.zeros((nnz, 3))
    en = None if ebc_nodes is None else _i32(ebc_nodes)
    st = _lib.lib().mega_rk_shapes(C.byref(params), n, ptr(coo), ptr(win), ptr(en), ptr(gn), ptr(gstart),
                                   ptr(gstack), nnz, ptr(shp), ptr(dshp))
    check(st, "rk_shapes")
    return shp, dshp


def hughes_winget(params, lmat):
    """lmat (n,3,3) -> rot (n,3,3), strain (n,6), d (n,6)."""
    lm = np.ascontiguousarray(np.transpose(_f64(lmat), (0, 2, 1)))  # column-major per node
    n = len(lm)
    rot = np.zeros((n, 3, 3))
    strain = np.zeros((n, 6))
    d = np.zeros((n, 6))
    check(_lib.lib().mega_hughes_winget(C.byref(params), n, ptr(lm), ptr(rot), ptr(strain), ptr(d)),
          "hughes_winget")
    return np.transpose(rot, (0, 2, 1)).copy(), strain, d


def rotate_tensor(rot, v):
    r = np.ascontiguousarray(np.transpose(_f64(rot), (0, 2, 1)))
    v = _f64(v).copy()
    check(_lib.lib().mega_rotate_tensor(len(v), ptr(r), ptr(v)), "rotate_tensor")
    return v


def constitution(params, stress_pred, mat_type, props, dlt, state, allow_status=False):
    """Returns (stress (n,6), state (n,20), iterations (n), status)."""
    sp = _f64(stress_pred)
    n = len(sp)
    state = _f64(state).copy()
    stress = np.zeros((n, 6))
    it = np.zeros(n, np.int32)
    st = _lib.lib().mega_constitution(C.byref(params), n, ptr(sp), ptr(_i32(mat_type)), ptr(_f64(props)),
                                      float(dlt), ptr(state), ptr(stress), ptr(it))
    check(st, "constitution", allow_status)
    return stress, state, it, st


def construct_fint(params, coo, win, vol, props, mat_type, ebc_nodes, state, stress, strain, dinc, dinc_tot,
                   gn, gstart, gstack, shp, dshp, linit, dlt, bodyforce=None, gint_work=0.0, allow_status=False):
    """CONSTRUCT_FINT: returns a dict with fint, fext (3N), stress, strain,
    state, gmax_wvel, gstrain_eq, gint_work and (linit) the shape stacks."""
    n = len(coo)
    state, stress, strain = _f64(state).copy(), _f64(stress).copy(), _f64(strain).copy()
    shp, dshp = _f64(shp).copy(), _f64(dshp).copy()
    fint = np.zeros(3 * n)
    fext = np.zeros(3 * n)
    wv = np.zeros(n)
    seq = np.zeros(n)
    gw = C.c_double(gint_work)
    en = None if ebc_nodes is None else _i32(ebc_nodes)
    st = _lib.lib().mega_construct_fint(
        C.byref(params), n, ptr(_f64(coo)), ptr(_f64(win)), ptr(_f64(vol)), ptr(_f64(props)), ptr(_i32(mat_type)),
        ptr(en), ptr(None if bodyforce is None else _f64(bodyforce)), ptr(state), ptr(stress), ptr(strain),
        ptr(_f64(dinc)), ptr(_f64(dinc_tot)), ptr(_i32(gn)), ptr(_i32(gstart)), ptr(_i32(gstack)), len(gstack),
        ptr(shp), ptr(dshp), int(bool(linit)), float(dlt), ptr(fint), ptr(fext), ptr(wv), ptr(seq), C.byref(gw))
    check(st, "construct_fint", allow_status)
    return dict(fint=fint, fext=fext, stress=stress, strain=strain, state=state, gmax_wvel=wv, gstrain_eq=seq,
                gint_work=gw.value, shp=shp, dshp=dshp, status=st)


def _ref(v, ct):
    """A by-reference scalar, as gfortran passes every argument."""
    return C.byref(ct(v))


def construct_fint_full(params, coo, win, vol, props, mat_type, ebc_nodes, state, stress, strain, dinc, dinc_tot,
                        gn, gstart, gstack, shp, dshp, linit, dlt, coo_current=None, sm_len=None, ddshp=None,
                        sgrad=None, bodyforce=None, body_id=None, gint_work=0.0, allow_status=False):
    """CONSTRUCT_FINT through construct_fint_gpu: the reference's own 46
    arguments (FINT.F90:16-25) in order, all by reference.  ddshp (nnz, 6)
    and sgrad (n, 18: the x, y and z stress gradients) for NSNI; returns the
    outputs as construct_fint does, plus ddshp and sgrad."""
    n = len(coo)
    check(_lib.lib().mega_fint_control(C.byref(params)), "mega_fint_control")
    state, stress, strain = _f64(state).copy(), _f64(stress).copy(), _f64(strain).copy()
    shp, dshp = _f64(shp).copy(), _f64(dshp).copy()
    nnz = len(gstack)
    dd = np.zeros((nnz, 6)) if ddshp is None else _f64(ddshp).copy()
    sg = np.zeros((n, 18)) if sgrad is None else _f64(sgrad).copy()
    dx, dy, dz = (np.ascontiguousarray(sg[:, 6 * k:6 * k + 6]) for k in range(3))
    cur = _f64(coo if coo_current is None else coo_current)
    sml = _f64(np.zeros((n, 6)) if sm_len is None else sm_len)
    fint, fext = np.zeros(3 * n), np.zeros(3 * n)
    wv, seq, cdist = np.zeros(n), np.zeros(n), np.zeros(n)
    h_s, s_s = np.zeros((n, 6)), np.zeros((n, 6))
    z3n, zn = np.zeros((n, 3)), np.zeros(n)
    ginvk = np.zeros((n, 3, 3))
    gw = C.c_double(gint_work)
    dlt_fint = C.c_double(-1.0)
    en = _i32(np.zeros(n) if ebc_nodes is None else ebc_nodes)
    bid = _i32(np.ones(n) if body_id is None else body_id)
    bf = _f64(np.zeros((n, 3)) if bodyforce is None else bodyforce)
    st = _lib.lib().construct_fint_gpu(
        ptr(_f64(win)), ptr(_f64(vol)), _ref(n, C.c_int32), ptr(_f64(coo)), ptr(cur),
        ptr(sml), ptr(z3n), ptr(zn), ptr(z3n),
        ptr(_i32(np.zeros(n))), ptr(_f64(props)), ptr(state), ptr(stress),
        ptr(strain), ptr(h_s), ptr(s_s), ptr(_f64(dinc)), ptr(_f64(dinc_tot)), ptr(_i32(mat_type)),
        ptr(en),
        ptr(_i32(gn)), ptr(_i32(gstart)), _ref(nnz, C.c_int32),
        ptr(_i32(gstack)), ptr(shp), ptr(dshp), ptr(dd), _ref(int(np.max(gn)), C.c_int32), ptr(ginvk),
        _ref(int(bool(linit)), C.c_int32),
        ptr(fint), ptr(fext), C.byref(dlt_fint), ptr(cdist), ptr(wv),
        ptr(dx), ptr(dy), ptr(dz),
        ptr(zn), ptr(zn), ptr(zn), ptr(bf), C.byref(gw), ptr(bid), ptr(seq), _ref(float(dlt), C.c_double))
    check(st, "construct_fint_gpu", allow_status)
    return dict(fint=fint, fext=fext, stress=stress, strain=strain, state=state, gmax_wvel=wv, gstrain_eq=seq,
                gint_work=gw.value, shp=shp, dshp=dshp, ddshp=dd, sgrad=np.concatenate([dx, dy, dz], axis=1),
                dlt_fint=dlt_fint.value, status=st)


def construct_fint_pd_full(params, coo, coo_current, win, vol, props, mat_type, state, stress, strain, dinc, gn,
                           gstart, gstack, shp, ginvk, linit, dlt, allow_status=False):
    """CONSTRUCT_FINT_PD through construct_fint_pd_gpu (FINT_PD.F90:16-25, 43
    arguments by reference); ginvk (n,3,3) row-major here.  Returns fint,
    stress, strain, state, gmax_wvel, shp, ginvk, gchar_dist and dlt_fint."""
    n = len(coo)
    check(_lib.lib().mega_fint_control(C.byref(params)), "mega_fint_control")
    state, stress, strain = _f64(state).copy(), _f64(stress).copy(), _f64(strain).copy()
    shp = _f64(shp).copy()
    ik = np.ascontiguousarray(np.transpose(_f64(ginvk), (0, 2, 1)))
    nnz = len(gstack)
    fint, wv, cdist = np.zeros(3 * n), np.zeros(n), np.zeros(n)
    z6, z3n, zn = np.zeros((n, 6)), np.zeros((n, 3)), np.zeros(n)
    gw = C.c_double(0.0)
    dlt_fint = C.c_double(-1.0)
    st = _lib.lib().construct_fint_pd_gpu(
        ptr(_f64(win)), ptr(_f64(vol)), _ref(n, C.c_int32), ptr(_f64(coo)), ptr(_f64(coo_current)),
        ptr(z6), ptr(z3n), ptr(zn), ptr(z3n), ptr(_i32(np.zeros(n))), ptr(_f64(props)), ptr(state), ptr(stress),
        ptr(strain), ptr(z6.copy()), ptr(z6.copy()), ptr(_f64(dinc)), ptr(_f64(np.zeros(3 * n))), ptr(_i32(mat_type)),
        ptr(_i32(np.zeros(n))), ptr(_i32(gn)), ptr(_i32(gstart)), _ref(nnz, C.c_int32), ptr(_i32(gstack)), ptr(shp),
        ptr(np.zeros((nnz, 3))), ptr(np.zeros((nnz, 6))), _ref(int(np.max(gn)), C.c_int32), ptr(ik),
        _ref(int(bool(linit)), C.c_int32), ptr(fint), C.byref(dlt_fint), ptr(cdist), ptr(wv), ptr(z6.copy()),
        ptr(z6.copy()), ptr(z6.copy()), ptr(zn), ptr(zn), ptr(zn), ptr(z3n), C.byref(gw), _ref(float(dlt), C.c_double))
    check(st, "construct_fint_pd_gpu", allow_status)
    return dict(fint=fint, stress=stress, strain=strain, state=state, gmax_wvel=wv, shp=shp,
                ginvk=np.transpose(ik, (0, 2, 1)).copy(), gchar_dist=cdist, dlt_fint=dlt_fint.value, status=st)


def pre_model_hex(coo, elems, norm_win=None, allow_status=False):
    """Mesh pre-processing on the device (PRE_MODEL.F90:248-268, PRE_CONTROL.F90:
    803-871) for a hexahedral mesh: elems (E, 8) 0-based node ids.  Returns
    win_raw, win (scaled by norm_win, per node or scalar), vol, sm_len, mom
    (X/Y/Z_MOM), dist_max and the smallest raw window."""
    return pre_model(coo, elems, None, norm_win, allow_status)


def pre_model(coo, elems, eltype=None, norm_win=None, allow_status=False):
    """As pre_model_hex for hexahedral (eltype 2) and tetrahedral (eltype 1)
    elements, elems (E, 8) 0-based -- the arrays kfile.read_k returns."""
    coo = _f64(coo)
    n = len(coo)
    conn = np.ascontiguousarray(np.asarray(elems, np.int64) + 1, dtype=np.int32)
    nw = None
    if norm_win is not None:
        nw = _f64(np.broadcast_to(np.asarray(norm_win, np.float64), (n,)))
    win_raw, win, mom = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
    vol, sm_len, dmax = np.zeros(n), np.zeros((n, 6)), np.zeros(3)
    wmin = C.c_double(0.0)
    et = None if eltype is None else _i32(eltype)
    st = _lib.lib().mega_pre_model(n, ptr(coo), len(conn), ptr(conn), ptr(et), ptr(nw), ptr(win_raw), ptr(win),
                                   ptr(vol), ptr(sm_len), ptr(mom), ptr(dmax), C.byref(wmin))
    check(st, "pre_model", allow_status)
    return dict(win_raw=win_raw, win=win, vol=vol, sm_len=sm_len, mom=mom, dist_max=dmax, min_raw_window=wmin.value,
                status=st)


MLP_HIDDEN = 64


def mlp_nparams(hidden=MLP_HIDDEN):
    return int(check(_lib.lib().mega_mlp_nparams(int(hidden)), "mlp_nparams", allow_status=True))


def mlp_init(seed=0, hidden=MLP_HIDDEN):
    """Glorot-uniform weights, zero biases, in the packed parameter order."""
    rng = np.random.default_rng(seed)
    H = hidden
    parts = []
    for (o, i) in ((H, 4), (H, 0), (H, H), (H, 0), (1, H), (1, 0)):
        if i == 0:
            parts.append(np.zeros(o))
        else:
            a = np.sqrt(6.0 / (o + i))
            parts.append(rng.uniform(-a, a, o * i))
    return np.concatenate(parts).astype(np.float32)


def mlp_grad(theta, x, t):
    th = np.ascontiguousarray(theta, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    tt = np.ascontiguousarray(t, np.float32)
    g = np.zeros_like(th)
    loss = np.zeros(1, np.float32)
    check(_lib.lib().mega_mlp_grad(MLP_HIDDEN, ptr(th), len(tt), ptr(xx), ptr(tt), ptr(g), ptr(loss)), "mlp_grad")
    return float(loss[0]), g


def mlp_eval(theta, x, tensor_cores=False):
    th = np.ascontiguousarray(theta, np.float32)
    xx = np.ascontiguousarray(x, np.float32)
    y = np.zeros(len(xx), np.float32)
    check(_lib.lib().mega_mlp_eval(MLP_HIDDEN, ptr(th), len(xx), ptr(xx), ptr(y), int(bool(tensor_cores))),
          "mlp_eval")
    return y


def mlp_train(theta, x, t, epochs, batch=4096, lr=1e-3, seed=0):
    th = np.array(theta, np.float32, copy=True)
    xx = np.ascontiguousarray(x, np.float32)
    tt = np.ascontiguousarray(t, np.float32)
    loss = np.zeros(int(epochs), np.float32)
    check(_lib.lib().mega_mlp_train(MLP_HIDDEN, ptr(th), len(tt), ptr(xx), ptr(tt), int(epochs), int(batch),
                                    float(lr), int(seed), ptr(loss)), "mlp_train")
    return th, loss


class Mega:
    """Device-resident model: the MAIN.F90 time loop on the GPU.

    Construct from a case dict (taylor_b200.cases), call search_and_shapes()
    once (LINIT), then step(nsteps, dt, mode)."""

    def __init__(self, case, params):
        self.case = case
        self.n = int(case["n"])
        self.params = params
        h = C.c_int64(0)
        bf = case.get("bodyforce")
        check(_lib.lib().mega_gpu_init(
            C.byref(params), self.n, ptr(_f64(case["coo"])), ptr(_f64(case["win"])), ptr(_f64(case["vol"])),
            ptr(_f64(case["mass"])), ptr(_i32(case["ebc"])), ptr(_f64(case["vinit"])), ptr(_f64(case["props"])),
            ptr(_i32(case["mat_type"])), ptr(_i32(case["body_id"])), ptr(None if bf is None else _f64(bf)),
            ptr(_f64(case["sm_len"])), C.byref(h)), "mega_gpu_init")
        self.h = h.value
        self.nnz = 0

    def set_instances(self, counts, dist_max=None):
        """The nodes are len(counts) independent instances (searched apart,
        instance k with bin-grid DIST_MAX dist_max[k] when given)."""
        cnt = np.ascontiguousarray(counts, dtype=np.int32)
        dm = None if dist_max is None else _f64(dist_max, (len(cnt), 3))
        check(_lib.lib().mega_set_instances(self.h, len(cnt), ptr(cnt), ptr(dm)), "set_instances")

    def autotune(self, dt, mode="mixed", reps=5):
        """Pick the fastest launch variant of each gather; returns the chosen
        (defgrad, force) variants and the per-variant mean times (ms)."""
        ch = np.zeros(2, np.int32)
        t = np.zeros(2 * _lib.TUNE_VARIANTS, np.float32)
        check(_lib.lib().mega_autotune(self.h, float(dt), self.mode_bits(mode), int(reps), ptr(ch), ptr(t)),
              "autotune")
        return (int(ch[0]), int(ch[1])), t.reshape(2, _lib.TUNE_VARIANTS)

    def set_fixity2(self, times, disp):
        """Windows of fixity code 2 (FIXITY2_TIME (steps,2), FIXITY2_NONZERO_EBC
        (steps,3)): a code-2 DOF moves at disp[k, j] / (t2 - t1) inside window k."""
        t = np.asarray(times, np.float64).reshape(-1, 2)
        d = np.asarray(disp, np.float64).reshape(-1, 3)
        tf = np.ascontiguousarray(t.ravel(order="F"))
        df = np.ascontiguousarray(d.ravel(order="F"))
        check(_lib.lib().mega_set_fixity2(self.h, len(t), ptr(tf), ptr(df)), "set_fixity2")

    def set_instance_dt(self, dt_inst):
        """Each instance steps by its own dt (None: one dt for all)."""
        d = None if dt_inst is None else _f64(dt_inst)
        check(_lib.lib().mega_set_instance_dt(self.h, ptr(d)), "set_instance_dt")

    def set_variants(self, defgrad, force, mode="mixed"):
        """Pin the gathers' launch variants for one precision."""
        check(_lib.lib().mega_set_variants(self.h, self.mode_bits(mode), int(defgrad), int(force)), "set_variants")

    def set_precisions(self, fp64=True, mixed=True):
        check(_lib.lib().mega_set_precisions(self.h, (1 if fp64 else 0) | (2 if mixed else 0)), "set_precisions")

    def search_and_shapes(self, download=False, allow_status=False):
        nnz = C.c_int64(0)
        gmaxn = C.c_int32(0)
        L = _lib.lib()
        if not download:
            st = L.mega_search_and_shapes(self.h, None, None, None, 0, None, None, C.byref(nnz), C.byref(gmaxn))
            check(st, "search_and_shapes", allow_status)
            self.nnz, self.gmaxn = nnz.value, gmaxn.value
            return dict(nnz=self.nnz, gmaxn=self.gmaxn, status=st)
        # first pass learns nnz, second downloads (the device search is cheap)
        st = L.mega_search_and_shapes(self.h, None, None, None, 0, None, None, C.byref(nnz), C.byref(gmaxn))
        check(st, "search_and_shapes", allow_status)
        m = nnz.value
        gn = np.zeros(self.n, np.int32)
        gstart = np.zeros(self.n, np.int32)
        gstack = np.zeros(m, np.int32)
        shp = np.zeros(m)
        dshp = np.zeros((m, 3))
        st = L.mega_search_and_shapes(self.h, ptr(gn), ptr(gstart), ptr(gstack), m, ptr(shp), ptr(dshp),
                                      C.byref(nnz), C.byref(gmaxn))
        check(st, "search_and_shapes", allow_status)
        self.nnz, self.gmaxn = nnz.value, gmaxn.value
        return dict(gn=gn, gstart=gstart, gstack=gstack, shp=shp, dshp=dshp, nnz=m, gmaxn=gmaxn.value, status=st)

    @staticmethod
    def mode_bits(mode="fp64", interp_each_step=False, learned=False):
        b = {"fp64": _lib.MODE_FP64, "mixed": _lib.MODE_MIXED}[mode]
        if interp_each_step:
            b |= _lib.FLAG_INTERP_EACH_STEP
        if learned:
            b |= _lib.FLAG_LEARNED_GUESS
        return b

    def step(self, nsteps, dt, mode="fp64", interp_each_step=False, allow_status=False, learned=False):
        st = _lib.lib().mega_step_resident(self.h, int(nsteps), float(dt),
                                           self.mode_bits(mode, interp_each_step, learned))
        return check(st, "step", allow_status)

    def step_timed(self, nsteps, dt, mode="fp64", interp_each_step=False, learned=False, allow_status=False):
        """Device milliseconds of nsteps steps; the status bits of the call are
        kept in self.last_status (raised unless allow_status)."""
        ms = C.c_float(0.0)
        st = _lib.lib().mega_step_timed(self.h, int(nsteps), float(dt),
                                        self.mode_bits(mode, interp_each_step, learned), C.byref(ms))
        self.last_status = check(st, "step_timed", allow_status)
        return ms.value

    def kernel_times(self, reps, dt, mode="fp64", learned=False):
        out = np.zeros(3, np.float32)
        check(_lib.lib().mega_kernel_times(self.h, int(reps), float(dt), self.mode_bits(mode, learned=learned),
                                           ptr(out)), "kernel_times")
        return out

    # -- surrogate start of the rate-dependent return mapping
    def set_surrogate(self, theta):
        th = None if theta is None else np.ascontiguousarray(theta, np.float32)
        check(_lib.lib().mega_set_surrogate(self.h, MLP_HIDDEN, None if th is None else ptr(th)), "set_surrogate")

    def log_rate_samples(self, cap, stride=1, seed=0):
        check(_lib.lib().mega_log_rate_samples(self.h, int(cap), int(stride), int(seed)), "log_rate_samples")

    def rate_samples(self, cap=None):
        """Logged (x0..x3, y) rows, shape (m, 5)."""
        held = C.c_int64(0)
        check(_lib.lib().mega_rate_samples(self.h, None, 0, C.byref(held)), "rate_samples")
        m = held.value if cap is None else min(held.value, int(cap))
        out = np.zeros((max(m, 1), 5), np.float32)
        got = C.c_int64(0)
        if m:
            check(_lib.lib().mega_rate_samples(self.h, ptr(out), m, C.byref(got)), "rate_samples")
        return out[:got.value]

    def train_surrogate(self, theta, epochs, batch=4096, lr=1e-3, seed=0):
        """Adam on the logged samples without leaving the device; installs and
        returns the trained parameters and the per-epoch mean loss."""
        th = np.array(theta, np.float32, copy=True)
        loss = np.zeros(int(epochs), np.float32)
        check(_lib.lib().mega_train_surrogate(self.h, ptr(th), int(epochs), int(batch), float(lr), int(seed),
                                              ptr(loss)), "train_surrogate")
        return th, loss

    _SIZES = {0: 3, 1: 3, 2: 3, 3: 3, 4: 3, 5: 3, 6: 3, 7: 6, 8: 6, 9: 1, 10: 1, 11: 1, 12: 3, 13: 3, 14: 1, 15: 4, 16: 18}

    def download(self, field):
        k = self._SIZES[field]
        out = np.zeros(self.n * k)
        check(_lib.lib().mega_download(self.h, int(field), ptr(out)), "download")
        return out.reshape(self.n, k) if k > 1 else out

    def snapshot(self, fields):
        """Several fields in one device-to-host copy: {field code: array}."""
        codes = np.ascontiguousarray([int(f) for f in fields], dtype=np.int32)
        sizes = [self._SIZES[int(f)] for f in codes]
        out = np.zeros(self.n * sum(sizes))
        check(_lib.lib().mega_snapshot(self.h, len(codes), ptr(codes), ptr(out)), "snapshot")
        res, off = {}, 0
        for f, k in zip(codes, sizes):
            a = out[off:off + self.n * k]
            res[int(f)] = a.reshape(self.n, k).copy() if k > 1 else a.copy()
            off += self.n * k
        return res

    def upload(self, field, arr):
        check(_lib.lib().mega_upload(self.h, int(field), ptr(_f64(arr).ravel())), "upload")

    def scalars(self):
        s = _lib.MegaScalars()
        check(_lib.lib().mega_get_scalars(self.h, C.byref(s)), "scalars")
        return dict(time=s.time, int_energy=s.int_energy, kin_energy=s.kin_energy, ext_energy=s.ext_energy,
                    total_force=list(s.total_force), steps=s.steps, newton_iters=s.newton_iters,
                    plastic_nodes=s.plastic_nodes, newton_iters_total=s.newton_iters_total,
                    plastic_nodes_total=s.plastic_nodes_total)

    def device_bytes(self):
        return int(_lib.lib().mega_device_bytes(self.h))

    def kernel_launches(self):
        return int(_lib.lib().mega_kernel_launches(self.h))

    def close(self):
        if self.h:
            _lib.lib().mega_gpu_finalize(self.h)
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def construct_fint_pd(params, coo, coo_current, win, vol, props, mat_type, state, stress, strain, dinc, gn, gstart,
                      gstack, shp, ginvk, linit, dlt, allow_status=False):
    """CONSTRUCT_FINT_PD (correspondence peridynamics).  ginvk is (n,3,3)
    row-major here; returns fint (3N), stress, strain, state, gmax_wvel and
    (linit) the influence functions and K^-1."""
    n = len(coo)
    state, stress, strain = _f64(state).copy(), _f64(stress).copy(), _f64(strain).copy()
    shp = _f64(shp).copy()
    ik = np.ascontiguousarray(np.transpose(_f64(ginvk), (0, 2, 1)))  # column-major (3,3,n)
    fint = np.zeros(3 * n)
    wv = np.zeros(n)
    gw = C.c_double(0.0)
    st = _lib.lib().mega_construct_fint_pd(
        C.byref(params), n, ptr(_f64(coo)), ptr(_f64(coo_current)), ptr(_f64(win)), ptr(_f64(vol)),
        ptr(_f64(props)), ptr(_i32(mat_type)), ptr(state), ptr(stress), ptr(strain), ptr(_f64(dinc)), ptr(_i32(gn)),
        ptr(_i32(gstart)), ptr(_i32(gstack)), len(gstack), ptr(shp), ptr(ik), int(bool(linit)), float(dlt), ptr(fint),
        ptr(wv), C.byref(gw))
    check(st, "construct_fint_pd", allow_status)
    return dict(fint=fint, stress=stress, strain=strain, state=state, gmax_wvel=wv, shp=shp,
                ginvk=np.transpose(ik, (0, 2, 1)).copy(), status=st)


class Pmb:
    """Bond-based PMB peridynamics, device resident (no reference
    counterpart).  case from taylor_b200.cases.pd_plate."""

    def __init__(self, case, broken0=None, fixed=None, mode="mixed"):
        self.case = case
        self.n = int(case["n"])
        h = C.c_int64(0)
        nb = C.c_int64(0)
        b0 = None if broken0 is None else np.ascontiguousarray(broken0, dtype=np.uint8)
        fx = None if fixed is None else _i32(fixed)
        check(_lib.lib().mega_pmb_init(self.n, ptr(_f64(case["coo"])), ptr(_f64(case["vol"])),
                                       ptr(_f64(case["vinit"])), ptr(fx), float(case["delta"]), float(case["c"]),
                                       float(case["s_c"]), float(case["rho"]), ptr(b0),
                                       {"fp64": _lib.MODE_FP64, "mixed": _lib.MODE_MIXED}[mode], C.byref(h),
                                       C.byref(nb)),
              "pmb_init")
        self.h, self.nnz = h.value, nb.value

    def step(self, nsteps, dt, timed=False):
        ms = C.c_float(0.0)
        check(_lib.lib().mega_pmb_step(self.h, int(nsteps), float(dt), C.byref(ms) if timed else None), "pmb_step")
        return ms.value

    def cut(self, corner, edge_a, edge_b):
        """Break the bonds crossing the rectangle corner + s a + t b (0..1)."""
        k = C.c_int64(0)
        check(_lib.lib().mega_pmb_cut(self.h, ptr(_f64(corner)), ptr(_f64(edge_a)), ptr(_f64(edge_b)),
                                      C.byref(k)), "pmb_cut")
        return k.value

    def download(self, what):
        m = self.nnz if what == 3 else (self.n if what == 4 else 3 * self.n)
        out = np.zeros(m)
        nbk = C.c_int64(0)
        check(_lib.lib().mega_pmb_download(self.h, int(what), ptr(out), C.byref(nbk)), "pmb_download")
        return out, nbk.value

    def close(self):
        if self.h:
            _lib.lib().mega_pmb_finalize(self.h)
            self.h = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
