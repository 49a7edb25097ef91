"""The bounded device waits (failure detection without a GPU fault).

Every spin-wait in the library's kernels -- the grid barrier of the
persistent solvers, the mbarrier wait for tensor-core completion -- ends
after a limit with an error that the host reads.  These tests make each wait
run out on purpose through the library's self-test entry points (a block that
leaves without arriving at the barrier, a barrier that nothing signals),
check the error code and message, and then run a normal solve to show that
the CUDA context is still usable.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve_still_works():
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    g = GpuModel(mg.beam_brick(6, 2, 2, 3.0, 1.0, 1.0))
    rv, it = g.fem_solve()
    assert rv == 0 and it > 0 and np.isfinite(g.u()).all()


def test_grid_barrier_times_out_and_reports():
    from ufem_b200 import _lib
    L = _lib.load()
    L.ufem_selftest_barrier_timeout.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    sm, ma, mi, mem = C.c_int(), C.c_int(), C.c_int(), C.c_long()
    L.ufem_device_info(C.byref(sm), C.byref(ma), C.byref(mi), C.byref(mem))
    nblocks = sm.value
    nto, ms = C.c_int(), C.c_double()
    rv = L.ufem_selftest_barrier_timeout(nblocks, 200, C.byref(nto), C.byref(ms))
    assert rv == -1                                   # AF_ERR
    assert b"grid barrier timed out" in L.ufem_last_error()
    assert nto.value == nblocks - 1                   # every waiting block left the barrier
    assert 150.0 <= ms.value < 5000.0                 # it waited about its limit, then returned
    _solve_still_works()


def test_tensor_core_wait_times_out_and_reports():
    from ufem_b200 import _lib
    L = _lib.load()
    L.ufem_selftest_mma_wait_timeout.argtypes = [C.c_long, C.POINTER(C.c_int)]
    to = C.c_int()
    rv = L.ufem_selftest_mma_wait_timeout(4096, C.byref(to))
    assert rv == -1 and to.value == 1
    assert b"wait timed out" in L.ufem_last_error()
    _solve_still_works()


def test_selftests_refuse_bad_arguments():
    from ufem_b200 import _lib
    L = _lib.load()
    L.ufem_selftest_barrier_timeout.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.ufem_selftest_mma_wait_timeout.argtypes = [C.c_long, C.POINTER(C.c_int)]
    assert L.ufem_selftest_barrier_timeout(1, 200, None, None) == -3   # AF_ERR_VAL
    assert L.ufem_selftest_barrier_timeout(4, 0, None, None) == -3
    assert L.ufem_selftest_mma_wait_timeout(0, None) == -3
