"""kpzb_roughness_noalloc: roughness of a caller's device lattice with no device allocation.

This entry point serves callers that cannot allocate device memory when they measure: an
application whose allocator owns the whole GPU, or a timing loop where cudaMalloc/cudaFree
would synchronize the device.  Its scratch is a fixed file-scope device array (ly <= 16).
The test calls it through the C ABI on a lattice owned by a scheduler handle and checks the
result against kpzb_roughness (same tolerance as the other roughness tests, rtol 1e-12) on
two calls in a row -- the second on a different lattice size, so stale scratch from the
first call would show -- and checks the size limit.  It runs last in the suite and also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def noalloc(lib, ptr, lx, ly):
    out = (C.c_double * 8)()
    st = lib.kpzb_roughness_noalloc(C.c_void_p(ptr), lx, ly, out, None)
    return st, np.array(out[:])


@pytest.mark.parametrize("first,second", [((10, 9), (12, 7)), ((14, 14), (9, 9))])
def test_noalloc_matches_roughness_twice(kpzb, first, second):
    from cudakpz_b200._lib import lib
    for lx, ly in (first, second):
        s = kpzb.Scheduler(lx, ly)
        s.setPQ(0.6, 0.3)
        s.supplySeed(17)
        s.mcsPQSyncRng(9)
        ref = s.roughness()
        st, got = noalloc(lib, s.devicePtr(), lx, ly)
        assert st == 0, lib.kpzb_last_error()
        np.testing.assert_allclose(got, [ref.w2] + ref.h, rtol=RTOL, atol=1e-12)
        # a repeated call on the same lattice gives the same numbers
        st, again = noalloc(lib, s.devicePtr(), lx, ly)
        assert st == 0 and np.array_equal(got, again)
        s.close()


def test_noalloc_rejects_rows_beyond_scratch(kpzb):
    from cudakpz_b200._lib import lib
    s = kpzb.Scheduler(8, 17)
    st, _ = noalloc(lib, s.devicePtr(), 8, 17)
    assert st == 1 and b"ly > 16" in lib.kpzb_last_error()
    s.close()
