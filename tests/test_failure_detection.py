"""Failure detection of the persistent PCG's grid barrier, tested without a GPU
fault: a CTA that never arrives makes one waiter give up after its poll limit;
it raises the abort flag and the counter's top bit, every other waiter leaves
at once with a failure, the host reads the flag, and the context stays usable."""
import ctypes as C
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from hsc_reimpl_b200 import _lib
    return _lib.load()


def selftest(lib, ctas, absent, first_limit, limit):
    st = (C.c_int32 * ctas)()
    ab, wh = C.c_int32(-1), C.c_int32(-1)
    rc = lib.hsc_debug_barrier_selftest(ctas, absent, first_limit, limit, st, C.byref(ab), C.byref(wh))
    return rc, list(st), ab.value, wh.value


def test_barrier_passes_when_every_cta_arrives(lib):
    rc, st, ab, _ = selftest(lib, 8, -1, 200_000, 5_000_000)
    assert rc == 0 and st == [1] * 8 and ab == 0


def test_absent_cta_times_out_and_the_abort_reaches_every_waiter(lib):
    t = time.time()
    rc, st, ab, wh = selftest(lib, 8, 3, 2000, 5_000_000)
    elapsed = time.time() - t
    assert rc == 0
    assert st[3] == 2 and all(s == 0 for i, s in enumerate(st) if i != 3), st
    assert ab == 1 and wh == 0
    # the waiters with the large limit left on the abort bit, not after their own limit
    assert elapsed < 3.0, elapsed


def test_context_usable_after_the_failed_barrier(lib, cube_system):
    from hsc_reimpl_b200.solver import DeviceSystem, HSCContext, HSCOptions
    rc, _, ab, _ = selftest(lib, 4, 0, 1000, 1_000_000)
    assert rc == 0 and ab == 1
    ctx = HSCContext(HSCOptions(omega=2 / 3))
    x, st = ctx.solve(DeviceSystem.from_system(cube_system))
    assert st["status"] == 0 and st["full_relative_residual"] <= 1e-6


def test_selftest_rejects_bad_arguments(lib):
    from hsc_reimpl_b200 import _lib
    assert selftest(lib, 1, -1, 10, 10)[0] == _lib.HSC_ERR_INVALID          # one CTA cannot wait on another
    assert selftest(lib, 8, -1, 100, 10)[0] == _lib.HSC_ERR_INVALID         # limit below the first limit
    assert selftest(lib, 100000, -1, 10, 10)[0] == _lib.HSC_ERR_INVALID     # more CTAs than SMs
