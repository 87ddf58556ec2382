"""hsc_spmv_noalloc, the allocation-free matrix product, against hsc_spmv.

hsc_spmv_noalloc serves callers that cannot allocate device memory when they
need H x (an engine whose device memory is all reserved up front in its own
pool, or a multi-stream loop that must not take the device-wide synchronisation
of cudaFree).  It keeps its sums in a static device array shared by every call,
so this test makes two calls in a row with different vectors: the second must
not see the first one's sums.  It runs last (file name) so that a stop at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_spmv_matches_hsc_spmv_twice(cube_system):
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
        x = torch.from_numpy(rng.standard_normal(s.N) * (10.0 ** call)).cuda()
        y_ref = ctx.spmv(ds, x)                                   # the existing entry point
        y = torch.full_like(x, float("nan"))
        rc = lib.hsc_spmv_noalloc(C.byref(ds.bcoo()), C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()),
                                  C.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize()
        assert rc == _lib.HSC_OK
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.linalg.norm(a - b) <= 1e-13 * np.linalg.norm(b), call


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
