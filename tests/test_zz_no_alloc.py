"""GPU: the force call that allocates nothing (sapb_force_device_noalloc).

Some integrators cannot let a library allocate device memory while they run:
they give the whole GPU to their own pool allocator, or they cannot afford
the device-wide synchronisation that cudaFree implies in the middle of a time
step.  For them the library offers a force call whose partial sums live in a
fixed 32 MiB device array instead of a buffer grown with cudaMalloc.  These
tests call it through the C ABI and check it against the ordinary
device-resident force call on the same inputs, twice in a row (the array is
shared by all calls and keeps the previous call's contents), plus the size
limit.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import sapporo2_b200 as sp
from tests import cases as T

pytestmark = pytest.mark.gpu

# Same kernel on the same inputs; only the number of j slices (and so the
# FP64 summation order of the partial sums) may differ.
FORCE_TOL = (1e-12, 1e-10)


def _records(case, sel, id_offset=0):
    ids = case["id"][sel] + id_offset
    return sp.pack_i_records(2, case["px"][sel], case["pv"][sel], case["h2"][sel], ids,
                             case["pa"][sel])


def _call(lib, dev, fn, nj, rec, torch, lists=True, mem=None):
    """One force call through the C ABI on device buffers made beforehand;
    `mem` (a list) receives the device's free bytes just before and after
    the library call."""
    ni = len(rec)
    i_dev = torch.from_numpy(rec).cuda()
    res = torch.full((ni, sp.RES_STRIDE), np.nan, dtype=torch.float64, device="cuda")
    cnt = torch.full((ni,), -7, dtype=torch.int32, device="cuda")
    lst = torch.full((ni * sp.NGB_PB,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    if mem is not None:
        mem.append(torch.cuda.mem_get_info()[0])
    rc = getattr(lib, fn)(dev, nj, ni, ctypes.c_void_p(i_dev.data_ptr()), 1e-6,
                          sp.F_NGB_LIST if lists else 0, ctypes.c_void_p(res.data_ptr()),
                          ctypes.c_void_p(cnt.data_ptr()), ctypes.c_void_p(lst.data_ptr()))
    assert rc == 0, lib.sapb_last_error(dev).decode()
    torch.cuda.synchronize()
    if mem is not None:
        mem.append(torch.cuda.mem_get_info()[0])
    return res.cpu().numpy(), cnt.cpu().numpy(), lst.cpu().numpy().reshape(ni, sp.NGB_PB)


def _compare(a, b):
    ra, ca, la = a
    rb, cb, lb = b
    got = {"acc": ra[:, 0:3], "pot": ra[:, 3], "jrk": ra[:, 4:7], "snp": ra[:, 7:10]}
    want = {"acc": rb[:, 0:3], "pot": rb[:, 3], "jrk": rb[:, 4:7], "snp": rb[:, 7:10]}
    T.check_forces(got, want, 2, *FORCE_TOL)
    assert np.array_equal(ra[:, 10:12], rb[:, 10:12])  # nearest neighbour ds2 and id
    assert np.array_equal(ca, cb)
    # below the capacity the lists hold every neighbour (order is arrival
    # order, so compare sorted); at or above it the call reports overflow and,
    # as in the reference, which ids were stored is not defined
    for i in np.nonzero(ca < sp.NGB_PB)[0]:
        k = int(ca[i])
        assert np.array_equal(np.sort(la[i, :k]), np.sort(lb[i, :k]))


def test_noalloc_matches_device_call_twice(gpu):
    torch = pytest.importorskip("torch")
    case = T.build_case(2, 16384, seed=61, binaries=0.1)
    n = case["n"]
    limit = sp.NOALLOC_SCRATCH_BYTES // (8 * sp.RES_STRIDE)
    with sp.Sapporo(order=sp.SIXTH, precision=sp.DOUBLESINGLE) as s:
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        s.force_prediction(n)
        lib, dev = s.lib, s.dev
        s.set_spatial(0)  # both calls in address order: the same arithmetic per pair
        # 16 j slices (64 tiles of 256 j): the first call fits them in the
        # fixed scratch (16384 i x 16 slices), the second (100000 i) does not
        # and is capped to limit // 100000 = 3 slices
        s.set_launch(1, 4, 16)
        assert s.plan(n, n) == (1, 4, 16) and s.plan(100_000, n) == (1, 4, 16)
        assert 16 * n <= limit and 16 > limit // 100_000
        # a small call first loads the kernels (module loading may take device
        # memory); no sapb_force_device call has run yet, so the handle holds
        # no growable partial-sum buffer: had the next call used one, it
        # would have had to allocate it and the free memory would show it
        _call(lib, dev, "sapb_force_device_noalloc", n, _records(case, np.arange(512)), torch)
        # first compared call: every particle
        rec1 = _records(case, np.arange(n))
        mem = []
        first = _call(lib, dev, "sapb_force_device_noalloc", n, rec1, torch, mem=mem)
        assert mem[0] == mem[1], f"free device memory changed by {mem[0] - mem[1]} bytes"
        _compare(first, _call(lib, dev, "sapb_force_device", n, rec1, torch))
        # second call in a row on other inputs, over the stale 16-slice
        # records of the first (ids offset: no self pairs)
        sel = np.random.default_rng(3).integers(0, n, 100_000)
        rec2 = _records(case, sel, id_offset=1_000_000 + np.arange(len(sel)) - case["id"][sel])
        _compare(_call(lib, dev, "sapb_force_device_noalloc", n, rec2, torch),
                 _call(lib, dev, "sapb_force_device", n, rec2, torch))
        # an empty call does nothing, as sapb_force_device
        buf = torch.zeros(16, dtype=torch.float64, device="cuda")
        for fn in ("sapb_force_device_noalloc", "sapb_force_device"):
            assert getattr(lib, fn)(dev, 0, 0, ctypes.c_void_p(buf.data_ptr()), 0.0, 0,
                                    ctypes.c_void_p(buf.data_ptr()), None, None) == 0


def test_noalloc_rejects_oversize(gpu):
    torch = pytest.importorskip("torch")
    limit = sp.NOALLOC_SCRATCH_BYTES // (8 * sp.RES_STRIDE)
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLESINGLE) as s:
        buf = torch.zeros(16, dtype=torch.float64, device="cuda")
        rc = s.lib.sapb_force_device_noalloc(s.dev, 1, limit + 1,
                                             ctypes.c_void_p(buf.data_ptr()), 0.0, 0,
                                             ctypes.c_void_p(buf.data_ptr()), None, None)
        assert rc == -2  # SAPB_EINVAL, nothing launched
        assert "exceeds the fixed scratch" in s.lib.sapb_last_error(s.dev).decode()
