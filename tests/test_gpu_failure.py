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
