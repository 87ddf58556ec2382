"""hsc_spmv_noalloc, the allocation-free matrix product, against H x.

hsc_spmv_noalloc serves callers that cannot allocate device memory when they
need H x (an engine whose device memory is all reserved up front in its own
pool, or a multi-stream loop that must not take the device-wide synchronisation
of cudaFree).  It keeps its sums in a static device array shared by every call,
so this test makes two calls in a row with different vectors (the second must
not see the first one's sums), checks both against the assembled H @ x on the
CPU and against the context entry point hsc_spmv, then a call whose output
aliases its input, and a matrix with one out-of-range triplet, which the kernel
skips and the call reports.  It runs last (file name) so that a stop at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_noalloc_spmv_matches_H_x_twice(cube_system):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import _lib
    from hsc_reimpl_b200.solver import HSCContext, DeviceSystem
    lib = _lib.load()
    s = cube_system
    ds = DeviceSystem.from_system(s)
    ctx = HSCContext()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(11)
    for call in range(2):
        xh = rng.standard_normal(s.N) * (10.0 ** call)
        x = torch.from_numpy(xh).cuda()
        y_ctx = ctx.spmv(ds, x)                                   # the existing entry point
        y = torch.full_like(x, float("nan"))
        rc = lib.hsc_spmv_noalloc(C.byref(ds.bcoo()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                  C.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize()
        assert rc == _lib.HSC_OK
        a = y.cpu().numpy()
        assert _rel(a, s.H @ xh) <= 1e-13, call
        assert _rel(a, y_ctx.cpu().numpy()) <= 1e-13, call
    # y aliasing x: the product of a copy of x, written over it
    xh = rng.standard_normal(s.N)
    xy = torch.from_numpy(xh.copy()).cuda()
    rc = lib.hsc_spmv_noalloc(C.byref(ds.bcoo()), C.c_void_p(xy.data_ptr()), C.c_void_p(xy.data_ptr()),
                              C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    assert rc == _lib.HSC_OK
    assert _rel(xy.cpu().numpy(), s.H @ xh) <= 1e-13
    assert _rel(xy.cpu().numpy(), ctx.spmv(ds, torch.from_numpy(xh).cuda()).cpu().numpy()) <= 1e-13


def test_noalloc_spmv_skips_and_reports_out_of_range_triplets(cube_system):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import _lib
    lib = _lib.load()
    s = cube_system
    nb = s.nblock
    # one extra triplet whose row lies past the last block row
    rows = np.concatenate([s.rows, [nb + 5]]).astype(np.int32)
    cols = np.concatenate([s.cols, [0]]).astype(np.int32)
    vals = np.concatenate([s.values_colmajor(), np.ones((1, 9))])
    dr, dc = torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda()
    dv = torch.from_numpy(np.ascontiguousarray(vals)).cuda()
    A = _lib.BCOO3(dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), int(rows.size), int(nb))
    xh = np.random.default_rng(3).standard_normal(s.N)
    x = torch.from_numpy(xh).cuda()
    y = torch.full_like(x, float("nan"))
    rc = lib.hsc_spmv_noalloc(C.byref(A), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == _lib.HSC_ERR_INVALID
    assert _rel(y.cpu().numpy(), s.H @ xh) <= 1e-13   # the valid triplets' product
    # the next valid call is clean again (the flag is per call)
    rc = lib.hsc_spmv_noalloc(C.byref(A.__class__(dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), int(s.rows.size),
                                                   int(nb))),
                              C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == _lib.HSC_OK


def test_noalloc_spmv_rejects_systems_beyond_its_array():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import _lib
    lib = _lib.load()
    too_big = _lib.BCOO3(0, 0, 0, 0, (1 << 20) // 3 + 1)
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.hsc_spmv_noalloc(C.byref(too_big), C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), None)
    assert rc == _lib.HSC_ERR_INVALID
