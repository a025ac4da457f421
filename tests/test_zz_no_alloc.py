"""kpzb_roughness_noalloc: roughness of a caller's device lattice with no device allocation.

This entry point serves callers that cannot allocate device memory when they measure: an
application whose allocator owns the whole GPU, or a timing loop where cudaMalloc/cudaFree
would synchronize the device.  Its scratch is a fixed file-scope device array (ly <= 16).
The test calls it through the C ABI on a lattice owned by a scheduler handle and checks the
result against kpzb_roughness (same tolerance as the other roughness tests, rtol 1e-12) on
two calls in a row -- the second on a different lattice size, so stale scratch from the
first call would show -- checks that calls after the first leave the device's free memory and
the default memory pool's reserved and used bytes unchanged, and checks the size limit.  It
runs last in the suite and also passes on its own in a fresh process.
"""
import ctypes as C
import glob
import os

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


def _cudart():
    """The CUDA runtime shipped with torch (a second runtime instance in this process; device
    memory and memory pools belong to the device's primary context, which both share)."""
    import nvidia
    libs = []
    for root in nvidia.__path__:
        libs += glob.glob(os.path.join(root, "cuda_runtime", "lib", "libcudart.so*"))
    return C.CDLL(sorted(libs)[0]) if libs else None


def _device_memory_state(rt, dev):
    free, total = C.c_size_t(), C.c_size_t()
    assert rt.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
    pool = C.c_void_p()
    assert rt.cudaDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    vals = []
    for attr in (5, 7):  # cudaMemPoolAttrReservedMemCurrent, cudaMemPoolAttrUsedMemCurrent
        v = C.c_uint64()
        assert rt.cudaMemPoolGetAttribute(pool, attr, C.byref(v)) == 0
        vals.append(v.value)
    return free.value, vals[0], vals[1]


def test_noalloc_calls_allocate_nothing(kpzb):
    """After one call (which may load the module and look up the scratch address), further
    calls change neither the device's free memory nor the default pool's reserved/used bytes."""
    from cudakpz_b200._lib import lib
    rt = _cudart()
    if rt is None:
        pytest.skip("no CUDA runtime library beside torch to read memory counters with")
    lx, ly = 12, 12
    s = kpzb.Scheduler(lx, ly)
    s.setPQ(0.5, 0.5)
    s.supplySeed(3)
    s.mcsPQSyncRng(4)
    ref = s.roughness()
    st, _ = noalloc(lib, s.devicePtr(), lx, ly)
    assert st == 0, lib.kpzb_last_error()
    before = _device_memory_state(rt, 0)
    for _ in range(2):
        st, got = noalloc(lib, s.devicePtr(), lx, ly)
        assert st == 0, lib.kpzb_last_error()
        np.testing.assert_allclose(got, [ref.w2] + ref.h, rtol=RTOL, atol=1e-12)
        assert _device_memory_state(rt, 0) == before
    s.close()


def test_noalloc_rejects_rows_beyond_scratch(kpzb):
    from cudakpz_b200._lib import lib
    s = kpzb.Scheduler(8, 17)
    st, _ = noalloc(lib, s.devicePtr(), 8, 17)
    assert st == 1 and b"ly > 16" in lib.kpzb_last_error()
    s.close()
