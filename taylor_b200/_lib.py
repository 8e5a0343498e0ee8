"""ctypes binding of libmega_gpu.so (the C ABI declared in include/mega_gpu.h).

The product path always goes through this library; there is no CPU
fallback.  Importing works without a GPU (the library loads, no CUDA call is
made); the first entry point that touches the device fails loudly when no
GPU is present.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmega_gpu.so")

# status bits and error codes (mega_gpu.h)
ST_NEWTON_CAP = 0x0001
ST_SINGULAR_MOMENT = 0x0002
ST_BIN_OVERFLOW = 0x0004
ST_CAND_OVERFLOW = 0x0008
ST_NONFINITE = 0x0010
ST_BAD_MATERIAL = 0x0020
ST_STACK_OVERFLOW = 0x0040
ST_SINGULAR_SHAPE = 0x0080
ST_BAD_MESH = 0x0100
ST_WAIT_TIMEOUT = 0x0200
ERR_CUDA, ERR_ARG, ERR_HANDLE, ERR_STATE, ERR_NOMEM, ERR_UNSUPPORTED = -1, -2, -3, -4, -5, -6

MODE_FP64 = 0
MODE_MIXED = 1
FLAG_INTERP_EACH_STEP = 0x100
FLAG_LEARNED_GUESS = 0x200
TUNE_VARIANTS = 8  # MEGA_TUNE_VARIANTS: launch variants of each per-step gather

MAT_ELASTIC, MAT_VONMISES, MAT_DRUCKER_PRAGER, MAT_VM_DAMAGE, MAT_VM_RATE = 1, 2, 3, 6, 7

F_COO_CURRENT, F_DSP, F_DSP_TOT, F_VEL, F_ACL, F_FINT, F_FEXT, F_STRESS, F_STRAIN, F_EPS = range(10)
F_STRAIN_EQ, F_WAVE_VEL, F_DSP_TOT_PHY, F_PRFORCE, F_NEWTON_IT, F_STATE_AUX, F_NSNI_SGRAD = range(10, 17)


class MegaParams(C.Structure):
    _fields_ = [
        ("rk_degree", C.c_int32), ("rk_cont", C.c_int32), ("rk_impl", C.c_int32),
        ("itype_int", C.c_int32), ("ql", C.c_int32), ("lagrangian", C.c_int32),
        ("finite_strain", C.c_int32), ("shsup", C.c_int32), ("peridynamics", C.c_int32),
        ("inv3_exact", C.c_int32), ("newton_max_iter", C.c_int32), ("rate_solver", C.c_int32),
        ("ql_coef", C.c_double), ("ql_len", C.c_double), ("gravity", C.c_double * 3),
        ("dist_max", C.c_double * 3), ("newton_rtol", C.c_double),
        ("auto_ts", C.c_int32), ("reserved", C.c_int32), ("dlt_fac", C.c_double),
    ]


class MegaScalars(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("int_energy", C.c_double), ("kin_energy", C.c_double),
        ("ext_energy", C.c_double), ("total_force", C.c_double * 6), ("steps", C.c_int64),
        ("newton_iters", C.c_int64), ("plastic_nodes", C.c_int64),
        ("newton_iters_total", C.c_int64), ("plastic_nodes_total", C.c_int64),
    ]


P = C.c_void_p
I32, I64, D, F32 = C.c_int32, C.c_int64, C.c_double, C.c_float
PP = C.POINTER(MegaParams)

# name -> (restype, argtypes)
SIGNATURES = {
    "mega_params_default": (None, [PP]),
    "mega_bin_search": (I32, [I32, P, P, P, P, I32, I32, P, P, P, I64, P, P, P]),
    "mega_bin_search_noalloc": (I32, [I32, P, P, P, P, I32, I32, P, P, P, I64, P, C.POINTER(I32),
                                      C.POINTER(I64), P]),
    "mega_rk_shapes": (I32, [PP, I32, P, P, P, P, P, P, I64, P, P]),
    "mega_hughes_winget": (I32, [PP, I32, P, P, P, P]),
    "mega_rotate_tensor": (I32, [I32, P, P]),
    "mega_constitution": (I32, [PP, I32, P, P, P, D, P, P, P]),
    "mega_construct_fint": (I32, [PP, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, I64, P, P,
                                  I32, D, P, P, P, P, P]),
    "mega_construct_fint_pd": (I32, [PP, I32, P, P, P, P, P, P, P, P, P, P, P, P, P, I64, P, P,
                                     I32, D, P, P, P]),
    "mega_gpu_init": (I32, [PP, I32, P, P, P, P, P, P, P, P, P, P, P, C.POINTER(I64)]),
    "mega_search_and_shapes": (I32, [I64, P, P, P, I64, P, P, P, P]),
    "mega_set_instances": (I32, [I64, I32, P, P]),
    "mega_set_precisions": (I32, [I64, I32]),
    "mega_set_fixity2": (I32, [I64, I32, P, P]),
    "mega_release_cached_memory": (I32, []),
    "mega_set_variants": (I32, [I64, I32, I32, I32]),
    "mega_set_instance_dt": (I32, [I64, P]),
    "mega_fint_control": (I32, [PP]),
    "construct_fint_gpu": (I32, [P] * 46),
    "construct_fint_pd_gpu": (I32, [P] * 43),
    "mega_autotune": (I32, [I64, D, I32, I32, P, P]),
    "mega_step_resident": (I32, [I64, I32, D, I32]),
    "mega_step_timed": (I32, [I64, I32, D, I32, C.POINTER(F32)]),
    "mega_kernel_times": (I32, [I64, I32, D, I32, P]),
    "mega_download": (I32, [I64, I32, P]),
    "mega_upload": (I32, [I64, I32, P]),
    "mega_snapshot": (I32, [I64, I32, P, P]),
    "mega_get_scalars": (I32, [I64, C.POINTER(MegaScalars)]),
    "mega_device_bytes": (I64, [I64]),
    "mega_kernel_launches": (I64, [I64]),
    "mega_pmb_init": (I32, [I32, P, P, P, P, D, D, D, D, P, I32, C.POINTER(I64), C.POINTER(I64)]),
    "mega_pmb_step": (I32, [I64, I32, D, C.POINTER(F32)]),
    "mega_pmb_download": (I32, [I64, I32, P, C.POINTER(I64)]),
    "mega_pmb_cut": (I32, [I64, P, P, P, C.POINTER(I64)]),
    "mega_pmb_finalize": (I32, [I64]),
    "mega_mlp_nparams": (I32, [I32]),
    "mega_mlp_grad": (I32, [I32, P, I64, P, P, P, P]),
    "mega_mlp_eval": (I32, [I32, P, I64, P, P, I32]),
    "mega_mlp_train": (I32, [I32, P, I64, P, P, I32, I32, F32, C.c_uint64, P]),
    "mega_set_surrogate": (I32, [I64, I32, P]),
    "mega_log_rate_samples": (I32, [I64, I64, I32, C.c_uint32]),
    "mega_rate_samples": (I32, [I64, P, I64, C.POINTER(I64)]),
    "mega_train_surrogate": (I32, [I64, P, I32, I32, F32, C.c_uint64, P]),
    "mega_pre_model_hex": (I32, [I32, P, I32, P, P, P, P, P, P, P, P, P]),
    "mega_pre_model": (I32, [I32, P, I32, P, P, P, P, P, P, P, P, P, P]),
    "mega_status_string": (C.c_char_p, [I32]),
    "mega_gpu_finalize": (I32, [I64]),
}

_lib = None


def lib():
    """Load libmega_gpu.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libmega_gpu.so is missing; build it with `python -m taylor_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class MegaError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        super().__init__(f"{what}: {status_string(code)} (code {code})")


def status_string(code):
    return lib().mega_status_string(int(code)).decode()


def check(code, what, allow_status=False):
    """Negative codes always raise; positive status bits raise unless allowed."""
    if code < 0 or (code > 0 and not allow_status):
        raise MegaError(code, what)
    return code


def ptr(a):
    if a is None:
        return None
    assert isinstance(a, np.ndarray) and a.flags["C_CONTIGUOUS"], "arrays must be contiguous numpy arrays"
    return a.ctypes.data_as(C.c_void_p)


def params(**kw):
    p = MegaParams()
    lib().mega_params_default(C.byref(p))
    for k, v in kw.items():
        if k in ("gravity", "dist_max"):
            arr = getattr(p, k)
            for i in range(3):
                arr[i] = float(v[i])
        else:
            setattr(p, k, v)
    return p
