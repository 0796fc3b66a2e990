"""GPU: the device-side failure path without a GPU fault.  A kernel waits on
a barrier nothing arrives at; the bounded wait gives up after its limit, the
host reads SAPB_ETIMEOUT, and the same process keeps computing correct
forces afterwards."""
import time

import pytest

import sapporo2_b200 as sp
from tests import cases as T

pytestmark = pytest.mark.gpu

SAPB_EINVAL, SAPB_ETIMEOUT = -2, -4


def test_bounded_wait_gives_up_and_the_device_stays_usable(gpu):
    with sp.Sapporo(order=sp.SIXTH) as s:
        assert s.lib.sapb_wait_selftest(s.dev, 0) == SAPB_EINVAL
        assert s.lib.sapb_wait_selftest(s.dev, 5000) == SAPB_EINVAL
        for limit_ms in (20, 80):
            t0 = time.perf_counter()
            rc = s.lib.sapb_wait_selftest(s.dev, limit_ms)
            dt = time.perf_counter() - t0
            assert rc == SAPB_ETIMEOUT, s.lib.sapb_last_error(s.dev)
            assert b"gave up" in s.lib.sapb_last_error(s.dev)
            assert 0.9 * limit_ms * 1e-3 <= dt < 5.0
    # the context is usable: a force call afterwards gives the oracle's answer
    case = T.build_case(2, 800, seed=31)
    want = T.oracle_force(case)
    got = T.run_library(case, sp.DOUBLESINGLE)
    T.check_forces(got, want, 2)


SAPB_ENOMEM = -3


def test_bad_arguments_and_allocation_failure_leave_the_device_usable(gpu):
    """Error codes instead of the reference's asserts and exits: bad order,
    precision, device, launch shape and sizes return SAPB_EINVAL; a j store
    too large for the GPU returns SAPB_ENOMEM (a failed cudaMalloc, not a
    fault); the handle keeps working afterwards."""
    import ctypes as C
    import numpy as np

    lib = sp.load_library()
    h = C.c_void_p()
    assert lib.sapb_open(C.byref(h), 0, 7, sp.DOUBLESINGLE, 0, 0) == SAPB_EINVAL
    assert lib.sapb_open(C.byref(h), 0, sp.SIXTH, 5, 0, 0) == SAPB_EINVAL
    assert lib.sapb_open(C.byref(h), 99, sp.SIXTH, sp.DOUBLESINGLE, 0, 0) == SAPB_EINVAL
    with sp.Sapporo(order=sp.SIXTH) as s:
        assert s.lib.sapb_set_launch(s.dev, 3, 2, 0) == SAPB_EINVAL
        assert s.lib.sapb_set_launch(s.dev, 1, 4, -1) == SAPB_EINVAL
        assert s.lib.sapb_predict(s.dev, 10 ** 9, 0.0) == SAPB_EINVAL
        assert s.lib.sapb_force(s.dev, 100, 10 ** 8, 0.0, 0.0, 0) == SAPB_EINVAL
        # 2e9 j need ~350 GB of device memory: the allocation fails cleanly
        assert s.lib.sapb_reserve_j(s.dev, 2_000_000_000) == SAPB_ENOMEM
        assert b"cannot allocate" in s.lib.sapb_last_error(s.dev)
    case = T.build_case(2, 700, seed=32)
    want = T.oracle_force(case)
    got = T.run_library(case, sp.DOUBLESINGLE)
    T.check_forces(got, want, 2)
