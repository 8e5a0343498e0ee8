"""The allocation-free neighbour search (mega_bin_search_noalloc).

It serves callers that cannot allocate GPU memory when they search -- their
device memory comes from another allocator or arena, or their loop may not
allocate.  The test hands it device buffers it owns beforehand, calls it
through the C ABI twice in a row on different inputs (and once more on the
first), and checks each result against the allocating entry point
mega_bin_search: the lists must be identical, element for element, since
neighbour lists are integer results.  Free device memory must not change
across the calls.  The file sorts last so that a failure here comes after
every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from taylor_b200 import _lib, cases, mega

pytestmark = pytest.mark.gpu


def _dev(a, torch, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _buffers(case, torch, cap):
    n = case["n"]
    return dict(
        coo=_dev(case["coo"], torch, torch.float64), win=_dev(case["win"], torch, torch.float64),
        sm=_dev(case["sm_len"], torch, torch.float64), gn=torch.zeros(n, dtype=torch.int32, device="cuda"),
        gstart=torch.zeros(n, dtype=torch.int32, device="cuda"),
        gstack=torch.zeros(cap, dtype=torch.int32, device="cuda"),
        ijk=torch.zeros((n, 3), dtype=torch.int32, device="cuda"), n=n, cap=cap,
        dist=np.ascontiguousarray(case["dist_max"], dtype=np.float64))


def _call(b):
    gmaxn, nnz = C.c_int32(0), C.c_int64(0)
    st = _lib.lib().mega_bin_search_noalloc(
        b["n"], C.c_void_p(b["coo"].data_ptr()), C.c_void_p(b["win"].data_ptr()), C.c_void_p(b["sm"].data_ptr()),
        b["dist"].ctypes.data_as(C.c_void_p), 0, 0, C.c_void_p(b["gn"].data_ptr()),
        C.c_void_p(b["gstart"].data_ptr()), C.c_void_p(b["gstack"].data_ptr()), b["cap"],
        C.c_void_p(b["ijk"].data_ptr()), C.byref(gmaxn), C.byref(nnz), None)
    return st, gmaxn.value, nnz.value


def _check(b, ref, st, gmaxn, nnz):
    assert st == 0, _lib.status_string(st)
    assert nnz == ref["nnz"] and gmaxn == ref["gmaxn"]
    np.testing.assert_array_equal(b["gn"].cpu().numpy(), ref["gn"])
    np.testing.assert_array_equal(b["gstart"].cpu().numpy(), ref["gstart"])
    np.testing.assert_array_equal(b["gstack"].cpu().numpy()[:nnz], ref["gstack"])
    np.testing.assert_array_equal(b["ijk"].cpu().numpy(), ref["ijk"])


def test_noalloc_search_matches_allocating_entry(golden_dir):
    import os

    import torch
    ca = cases.taylor_bar(h=0.4e-3)
    cb = cases.case_a(os.path.join(golden_dir, "case_a.npz"))
    ra = mega.bin_search(ca["coo"], ca["win"], ca["sm_len"], ca["dist_max"])
    rb = mega.bin_search(cb["coo"], cb["win"], cb["sm_len"], cb["dist_max"])
    ba = _buffers(ca, torch, ra["nnz"] + 1024)
    bb = _buffers(cb, torch, rb["nnz"])
    torch.cuda.synchronize()
    _check(ba, ra, *_call(ba))          # first call on this device does the set-up
    free0 = torch.cuda.mem_get_info()[0]
    _check(bb, rb, *_call(bb))          # second call, other input, same scratch array
    ba["gstack"].fill_(-7)
    ba["gn"].fill_(-7)
    _check(ba, ra, *_call(ba))          # the previous call's contents do not leak in
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_search_rejects_too_large_and_small_stack():
    import torch
    c = cases.taylor_bar(h=0.8e-3, L=8e-3)
    ref = mega.bin_search(c["coo"], c["win"], c["sm_len"], c["dist_max"])
    b = _buffers(c, torch, ref["nnz"] - 1)
    st, _, nnz = _call(b)
    assert st > 0 and st & _lib.ST_STACK_OVERFLOW and nnz == ref["nnz"]
    np.testing.assert_array_equal(b["gn"].cpu().numpy(), ref["gn"])
    big = dict(b)
    big["n"] = 4_000_000  # rejected before any input is read
    st, _, _ = _call(big)
    assert st == _lib.ERR_UNSUPPORTED
    assert "fixed" in _lib.status_string(st)
