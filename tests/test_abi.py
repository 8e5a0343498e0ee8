"""The C ABI library loads without a GPU, exports every entry point the
header declares, lays out mega_params exactly as C does, and rejects bad
arguments with negative codes before touching the device."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from taylor_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mega_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w \*]*?\b(mega_\w+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("mega_bin_search", "mega_rk_shapes", "mega_construct_fint", "mega_construct_fint_pd",
                 "mega_hughes_winget", "mega_constitution", "mega_gpu_init", "mega_step_resident",
                 "mega_download", "mega_gpu_finalize", "mega_status_string"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_params_layout_matches_c():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "mega_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(mega_params), offsetof(mega_params, ql_coef),
         offsetof(mega_params, gravity), offsetof(mega_params, dist_max), offsetof(mega_params, newton_rtol),
         sizeof(mega_scalars_t));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.check_output([exe]).split()]
    P = _lib.MegaParams
    assert got == [C.sizeof(P), P.ql_coef.offset, P.gravity.offset, P.dist_max.offset, P.newton_rtol.offset,
                   C.sizeof(_lib.MegaScalars)]


def test_bad_arguments_rejected_without_device():
    L = _lib.lib()
    assert L.mega_bin_search(0, None, None, None, None, 0, 0, None, None, None, 0, None, None, None) == _lib.ERR_ARG
    h = C.c_int64(0)
    assert L.mega_gpu_init(None, 10, *([None] * 11), C.byref(h)) == _lib.ERR_ARG
    assert L.mega_step_resident(12345, 1, 1e-8, 0) == _lib.ERR_HANDLE
    assert L.mega_gpu_finalize(12345) == _lib.ERR_HANDLE
    assert "invalid handle" in _lib.status_string(_lib.ERR_HANDLE)
    assert "DID NOT CONVERGE" in _lib.status_string(_lib.ST_NEWTON_CAP)
    assert "MAX_NEIGH" in _lib.status_string(_lib.ST_BIN_OVERFLOW | _lib.ST_NEWTON_CAP)


def test_params_defaults_follow_the_deck():
    p = _lib.params()
    assert (p.rk_degree, p.rk_cont, p.itype_int, p.ql, p.lagrangian, p.finite_strain) == (1, 3, 0, 1, 1, 1)
    assert p.ql_coef == 0.001 and p.newton_max_iter == 20 and p.inv3_exact == 0


def test_mirror_raises_on_error_codes():
    with pytest.raises(_lib.MegaError):
        _lib.check(_lib.ERR_ARG, "x")
    with pytest.raises(_lib.MegaError):
        _lib.check(_lib.ST_NEWTON_CAP, "x")
    assert _lib.check(_lib.ST_NEWTON_CAP, "x", allow_status=True) == _lib.ST_NEWTON_CAP


def _build_fortran_abi_check(tmp_path):
    """gcc-compiles tests/fortran_abi_check.c (the force subroutines called
    with Fortran's by-reference conventions) against include/mega_gpu.h and
    links it with the library."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib_dir = os.path.join(root, "taylor_b200")
    exe = str(tmp_path / "fortran_abi_check")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-O1", "-o", exe,
                    os.path.join(root, "tests", "fortran_abi_check.c"), "-L" + lib_dir, "-lmega_gpu",
                    "-Wl,-rpath," + lib_dir, "-lm"], check=True)
    return exe


def test_fortran_abi_check_compiles(tmp_path):
    assert os.path.exists(_build_fortran_abi_check(tmp_path))
