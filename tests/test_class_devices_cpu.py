"""CPU: the host logic of the `sapporo` class over several devices, with the
device side (include/sapporo_b200.h) replaced by an FP64 stand-in on the
oracle (tests/host_fake/sapb_cpu_fake.cpp).  The class sources and its C and
GRAPE-6 bindings are compiled unchanged against it.

What the reference fixes and these tests check (lib/src/sapporohostclass.cpp):
the device list of open (:90-163), j address a on device a % G at a / G
(:473-474), j memory grown by 10 % rounded to a multiple of G (:560-583), the
first nj addresses split as nj / G (+1 on the first nj % G devices,
:687-691), forces summed and the nearest neighbour taken over the devices
(:749-799), neighbour-list overflow per device in read_ngb_list (:804-835)
and the running-total rule of get_ngb_list (:837-880).  The nearest
neighbour at equal distance on two devices is the lower id (the library's
rule inside one device)."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

import sapporo2_b200 as sp
from sapporo2_b200 import ic
from oracle import oracle as O
from tests import cases as T

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "sapporo2_b200" / "csrc"
ORACLE_DIR = ROOT / "oracle"


@pytest.fixture(scope="module")
def fake(tmp_path_factory):
    O.lib()  # builds oracle/liboracle.so when missing
    out = tmp_path_factory.mktemp("fake") / "libsapporo_fake.so"
    cmd = ["g++", "-O2", "-shared", "-fPIC", "-std=c++17", "-Wall", f"-I{ROOT / 'include'}",
           f"-I{CSRC}", str(ROOT / "tests" / "host_fake" / "sapb_cpu_fake.cpp"),
           str(CSRC / "sapporohostclass.cpp"), str(CSRC / "sapporo_cbind.cpp"),
           str(CSRC / "sapporoG6lib.cpp"), "-o", str(out), f"-L{ORACLE_DIR}", "-loracle",
           f"-Wl,-rpath,{ORACLE_DIR}"]
    subprocess.run(cmd, check=True)
    lib = C.CDLL(str(out))
    for name, res, args in sp._SIGS:
        if hasattr(lib, name):
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
    lib.fake_sapb_pushes.restype = C.c_int
    lib.fake_sapb_open_devices.restype = C.c_int
    lib.fake_sapb_open_devices.argtypes = [C.POINTER(C.c_int), C.c_int]
    return lib


def open_class(lib, order, devices, precision=sp.DOUBLESINGLE):
    """A sapporo2_b200.Sapporo bound to the stand-in library."""
    s = sp.Sapporo.__new__(sp.Sapporo)
    s.lib, s.order, s.precision = lib, order, precision
    s.h = lib.sapporo_c_new()
    ids = np.ascontiguousarray(devices, dtype=np.int32)
    rc = lib.sapporo_c_open_devices(s.h, len(ids), ids if len(ids) else None, order, precision)
    assert rc == 0, rc
    s.dev = lib.sapporo_c_device(s.h)
    s.devs = [lib.sapporo_c_device_at(s.h, k) for k in range(lib.sapporo_c_n_devices(s.h))]
    return s


def run(lib, case, devices, sel, maxlength=sp.NGB_PB, h2=None):
    o, n = case["order"], case["n"]
    s = open_class(lib, o, devices)
    try:
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        h2 = case["h2"][sel] if h2 is None else h2
        s.start(n, case["id"][sel], case["px"][sel], case["pv"][sel],
                case["pa"][sel] if case["pa"] is not None else None, case["eps2"], h2)
        r = s.results(n)
        r["overflow"] = s.read_ngb_list()
        r["lists"] = [s.get_ngb_list(q, maxlength) for q in range(len(sel))]
    finally:
        s.close()
    return r


def want_for(case, sel, h2=None):
    o = case["order"]
    return O.force(o, case["px"][sel], case["pv"][sel],
                   case["pa"][sel] if case["pa"] is not None else None,
                   case["h2"][sel] if h2 is None else h2, case["id"][sel], case["px"],
                   case["pv"], case["pa"], case["m"], case["id"], case["eps2"])


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("devices", [[0], [0, 1], [0, 1, 2], [3, 1, 2, 0]])
def test_split_matches_oracle(fake, order, devices):
    case = T.build_case(order, 3000, seed=40 + order, binaries=0.1)
    sel = np.sort(np.random.default_rng(3).choice(case["n"], 400, replace=False))
    got = run(fake, case, devices, sel)
    want = want_for(case, sel)
    tol = 0.0 if len(devices) == 1 else 1e-12  # other summation order over the devices
    for f in ("acc", "jrk", "pot") + (("snp",) if order >= 2 else ()):
        assert T.rel_err(got[f], want[f]).max() <= tol, f
    T.check_nn(case, got["nnb"], want, sel)
    ok = want["nnb"] >= 0
    np.testing.assert_array_equal(got["ds2min"][ok],
                                  want["ds2min"][ok].astype(np.float32).astype(np.float64))
    counts = np.array([q[1] for q in got["lists"]])
    small = want["ngb_count"] < sp.NGB_PB
    np.testing.assert_array_equal(counts[small], want["ngb_count"][small])
    for q in np.nonzero(small)[0]:
        ovf, nb, ids = got["lists"][q]
        assert ovf == 0
        np.testing.assert_array_equal(ids, np.sort(want["ngb_list"][q, :nb]))


def test_nearest_neighbour_tie_takes_lower_id(fake):
    # two j at the same distance from the i, on devices 0 and 1: the lower id
    # wins whichever device holds it
    for ids_j in ([7, 3], [3, 7]):
        n = 4
        x = np.array([[1.0, 0, 0], [0, 1.0, 0], [5.0, 5.0, 5.0], [0, 0, 0]])
        ids = np.array(ids_j + [11, 20], dtype=np.int32)
        z = np.zeros((n, 3))
        s = open_class(fake, 1, [0, 1])
        try:
            s.set_j_particles(np.arange(n), ids, np.zeros(n), np.full(n, 1e-3), x, z, z, z)
            s.set_time(0.0)
            s.start(n, ids[3:], x[3:], z[3:], None, 1e-4, np.zeros(1))
            r = s.results(n)
        finally:
            s.close()
        assert r["nnb"][0] == 3 and r["ds2min"][0] == 1.0


def test_growth_restaging_and_few_j(fake):
    # 20000 j on three devices (past the initial 16384 addresses), two
    # addresses staged twice before the push (the second values count), then
    # a call on fewer j than devices
    case = T.build_case(1, 20000, seed=44)
    n = case["n"]
    sel = np.arange(0, n, 97)
    s = open_class(fake, 1, [0, 1, 2])
    pushes0 = fake.fake_sapb_pushes()
    try:
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"])
        m2 = case["m"].copy()
        m2[[5, 19999]] *= 3.0
        s.set_j_particles(np.array([5, 19999]), case["id"][[5, 19999]], case["t0"][[5, 19999]],
                          m2[[5, 19999]], case["x"][[5, 19999]], case["v"][[5, 19999]],
                          case["a"][[5, 19999]], case["j"][[5, 19999]])
        s.set_time(case["ti"])
        s.start(n, case["id"][sel], case["px"][sel], case["pv"][sel], None, case["eps2"],
                case["h2"][sel])
        got = s.results(n)
        assert fake.fake_sapb_pushes() - pushes0 == 3  # the staged j travel once per device
        # each device holds its share: 6667, 6667 and 6666 j below capacity
        caps = []
        for d in s.devs:
            c = C.c_int()
            assert fake.sapb_info(d, None, None, None, C.byref(c), None) == 0
            caps.append(c.value)
        assert min(caps) >= 6667
        # two j on three devices: the third takes no force call
        s.set_time(case["ti"])
        s.start(2, case["id"][:2], case["px"][:2], case["pv"][:2], None, case["eps2"],
                np.full(2, 1e3))
        few = s.results(2)
        few_lists = [s.get_ngb_list(q) for q in range(2)]
        assert fake.fake_sapb_pushes() - pushes0 == 3  # nothing new staged
    finally:
        s.close()
    want = O.force(1, case["px"][sel], case["pv"][sel], None, case["h2"][sel], case["id"][sel],
                   case["px"], case["pv"], None, m2, case["id"], case["eps2"])
    for f in ("acc", "jrk", "pot"):
        assert T.rel_err(got[f], want[f]).max() <= 1e-12, f
    np.testing.assert_array_equal(few["nnb"], case["id"][[1, 0]])
    for q, (ovf, nb, ids) in enumerate(few_lists):
        assert (ovf, nb, list(ids)) == (0, 1, [int(case["id"][1 - q])])


def test_list_overflow_rules(fake):
    # counts per device below NGB_PB but their total above: read_ngb_list
    # reports no overflow (it checks each device), get_ngb_list does once the
    # running total reaches maxlength; with a short maxlength the count stops
    # at the device whose list crossed it
    case = T.build_case(1, 2000, seed=45)
    n, G = case["n"], 3
    sel = np.arange(0, 40)
    d2 = ((case["px"][None, :, :] - case["px"][sel][:, None, :]) ** 2).sum(-1)
    # h2 between the k-th and (k+1)-th neighbour: 400 (about 133 per device)
    # for the first 20 i, 30 for the others
    srt = np.sort(d2, axis=1)  # column 0 is the i itself
    k = np.where(sel < 20, 400, 30)
    h2 = 0.5 * (srt[np.arange(len(sel)), k] + srt[np.arange(len(sel)), k + 1])
    got = run(fake, case, list(range(G)), sel, h2=h2)
    want = want_for(case, sel, h2=h2)
    inside = (h2[:, None] > d2) & (case["id"][None, :] != case["id"][sel][:, None])
    per_dev = np.stack([inside[:, g::G].sum(1) for g in range(G)], 1)
    np.testing.assert_array_equal(per_dev.sum(1), want["ngb_count"])
    assert got["overflow"] == int(np.any(per_dev >= sp.NGB_PB))
    for q, (ovf, nb, ids) in enumerate(got["lists"]):
        total = 0
        for g in range(G):
            total += per_dev[q, g]
            if total >= sp.NGB_PB:
                break
        assert nb == total
        assert ovf == int(total >= sp.NGB_PB or np.any(per_dev[q] >= sp.NGB_PB))
        assert set(ids.tolist()) <= set(case["id"][inside[q]].tolist())
    assert np.any(want["ngb_count"] >= sp.NGB_PB) and np.all(per_dev < sp.NGB_PB)
    short = run(fake, case, list(range(G)), sel, maxlength=10, h2=h2)
    for q, (ovf, nb, ids) in enumerate(short["lists"]):
        total = 0
        for g in range(G):
            total += per_dev[q, g]
            if total >= 10:
                break
        assert nb == total and len(ids) == min(total, 10)
        assert ovf == int(total >= 10)
    # maxlength above NGB_PB: the devices' lists together (400 ids for the
    # first 20 i) come back whole and sorted
    long = run(fake, case, list(range(G)), sel, maxlength=1024, h2=h2)
    for q, (ovf, nb, ids) in enumerate(long["lists"]):
        assert ovf == 0 and nb == per_dev[q].sum() and len(ids) == nb
        np.testing.assert_array_equal(ids, np.sort(case["id"][inside[q]]))
    assert max(len(ids) for _, _, ids in long["lists"]) > sp.NGB_PB


def test_g6_interface_over_devices(fake):
    # g6_open_special with a device list, j set one by one through
    # g6_set_j_particle_ (a2 = a/2, j6 = jerk/6)
    case = T.build_case(1, 1500, seed=46, binaries=0.1)
    n = case["n"]
    g6 = sp.G6.__new__(sp.G6)
    g6.lib = fake
    assert g6.open_special((0, 2, 1)) == 0
    try:
        z3 = np.zeros(3)
        for k in range(n):
            g6.set_j_particle(k, int(case["id"][k]), float(case["t0"][k]), 0.0,
                              float(case["m"][k]), z3, case["j"][k] / 6.0, case["a"][k] / 2.0,
                              case["v"][k], case["x"][k])
        g6.set_ti(case["ti"])
        zi = np.zeros((n, 3))
        g6.calc_firsthalf(n, case["id"], case["px"], case["pv"], zi, zi, np.zeros(n),
                          case["eps2"], case["h2"])
        rc, acc, jrk, pot, inn = g6.calc_lasthalf2(n, case["id"], case["px"], case["pv"],
                                                   case["eps2"], case["h2"])
        assert rc == 0
        lists = [g6.get_neighbour_list(i, sp.NGB_PB) for i in range(n)]
    finally:
        g6.close()
    want = T.oracle_force(case)
    for f, g in (("acc", acc), ("jrk", jrk), ("pot", pot)):
        assert T.rel_err(g, want[f]).max() <= 1e-12, f
    T.check_nn(case, inn, want)
    small = want["ngb_count"] < sp.NGB_PB
    np.testing.assert_array_equal(np.array([q[1] for q in lists])[small],
                                  want["ngb_count"][small])


def test_g6_open_reads_the_device_list(fake, tmp_path, monkeypatch):
    # ./sapporo2.config: the device count, then one id per line
    # (lib/interfaces/sapporoG6lib.cpp:46-77); g6_open_ opens those devices
    (tmp_path / "sapporo2.config").write_text("2\n0\n3\n")
    monkeypatch.chdir(tmp_path)
    g6 = sp.G6.__new__(sp.G6)
    g6.lib = fake
    assert g6.open() == 0
    try:
        ids = np.zeros(8, dtype=np.int32)
        n = fake.fake_sapb_open_devices(ids.ctypes.data_as(C.POINTER(C.c_int)), 8)
        assert list(ids[:n]) == [0, 3]
    finally:
        g6.close()
    assert fake.fake_sapb_open_devices(ids.ctypes.data_as(C.POINTER(C.c_int)), 8) == 0


def test_device_lists_and_readback(fake):
    case = T.build_case(2, 700, seed=47)
    n = case["n"]
    # nprocs = 0: every visible device (the stand-in has four); nprocs < 0: the first -nprocs
    for nprocs, expect in ((0, 4), (-2, 2)):
        h = fake.sapporo_c_new()
        assert fake.sapporo_c_open_devices(h, nprocs, None, 2, sp.DOUBLESINGLE) == 0
        assert fake.sapporo_c_n_devices(h) == expect
        fake.sapporo_c_close(h)
        fake.sapporo_c_delete(h)
    # a device id that does not exist: an error, no device left open
    h = fake.sapporo_c_new()
    bad = np.array([0, 9], dtype=np.int32)
    assert fake.sapporo_c_open_devices(h, 2, bad, 2, sp.DOUBLESINGLE) == -5  # SAPB_ENODEV
    assert fake.sapporo_c_n_devices(h) == 0
    fake.sapporo_c_delete(h)
    # predicted and raw state of each address, found on its device
    s = open_class(fake, 2, [0, 1, 2])
    try:
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        s.force_prediction(n)
        for k in (0, 1, 2, 3, 350, 698, 699):
            p = s.retrieve_predicted(k)
            st = s.retrieve_state(k)
            assert p["id"] == case["id"][k] and p["mass"] == case["m"][k]
            np.testing.assert_array_equal(p["pos"], case["px"][k])
            np.testing.assert_array_equal(p["vel"], case["pv"][k])
            np.testing.assert_array_equal(p["acc"], case["pa"][k])
            np.testing.assert_array_equal(st["pos"], case["x"][k])
            np.testing.assert_array_equal(st["jrk"], case["j"][k])
    finally:
        s.close()


@pytest.mark.parametrize("devices", [[0], [0, 1]])
def test_bulk_upload_repeated_address_keeps_call_order(fake, devices):
    # one set_j_particles call that names an address twice keeps the later
    # entry, as set_j_particle one by one would.  70001 entries are packed in
    # chunks of 35001 when two threads are free; the repeated address is the
    # last entry of the first chunk and the first of the second, where a
    # threaded fill would write one record from two threads
    n = 70000
    x, v, m = ic.plummer(n, 12)
    ids = (np.arange(n) + 100).astype(np.int32)
    k2 = 35001
    addr = np.concatenate([np.arange(k2), [k2 - 1], np.arange(k2, n)]).astype(np.int32)
    rows = np.concatenate([np.arange(k2), [n], np.arange(k2, n)])
    xr = np.vstack([x, x[k2 - 1] + [0.25, -0.5, 0.125]])[rows]
    vr = np.vstack([v, -v[k2 - 1]])[rows]
    mr = np.append(m, 3.0 * m[k2 - 1])[rows]
    zero = np.zeros_like(xr)
    s = open_class(fake, 1, devices)
    try:
        s.set_j_particles(addr, np.append(ids, ids[k2 - 1])[rows], np.ones(n + 1), mr, xr, vr,
                          zero, zero)
        s.set_time(1.0)
        s.force_prediction(n)
        for k in (0, k2 - 2, k2 - 1, k2, n - 1):
            st = s.retrieve_state(k)
            src = n if k == k2 - 1 else k
            want_x = x[k2 - 1] + [0.25, -0.5, 0.125] if src == n else x[k]
            want_m = 3.0 * m[k2 - 1] if src == n else m[k]
            assert st["mass"] == want_m, k
            np.testing.assert_array_equal(st["pos"], want_x)
            np.testing.assert_array_equal(st["vel"], -v[k2 - 1] if src == n else v[k])
    finally:
        s.close()


def test_wrapper_refuses_arrays_of_the_wrong_length(fake):
    # per-particle arrays shorter or longer than the address list are refused
    # in Python, before the C side could read past their end
    case = T.build_case(1, 64, seed=13)
    n = case["n"]
    s = open_class(fake, 1, [0])
    args = [np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"], case["a"],
            case["j"]]
    try:
        for k, what in ((1, "id"), (2, "t"), (3, "mass")):
            bad = list(args)
            bad[k] = args[k][:-1]
            with pytest.raises(ValueError, match=what):
                s.set_j_particles(*bad)
        with pytest.raises(ValueError, match="eps"):
            s.set_j_particles(*args, eps=np.zeros(n + 1))
        with pytest.raises(ValueError):
            s.set_j_particles(*args[:4], case["x"][:-1], *args[5:])
        s.set_j_particles(*args)
        s.set_time(case["ti"])
        with pytest.raises(ValueError, match="h2"):
            s.start(n, case["id"], case["px"], case["pv"], None, case["eps2"], case["h2"][:-1])
        s.start(n, case["id"], case["px"], case["pv"], None, case["eps2"], case["h2"])
        s.results(n)
    finally:
        s.close()
    # the GRAPE-6 wrapper: 3-vectors of a j particle and per-i h2 / phiold
    g6 = sp.G6.__new__(sp.G6)
    g6.lib = fake
    assert g6.open_special((0,)) == 0
    try:
        z3, zi = np.zeros(3), np.zeros((n, 3))
        with pytest.raises(ValueError):
            g6.set_j_particle(0, 5, 0.0, 0.0, 1.0, z3, z3, z3, z3, np.zeros(2))
        with pytest.raises(ValueError, match="h2"):
            g6.calc_firsthalf(n, case["id"], case["px"], case["pv"], zi, zi, np.zeros(n),
                              case["eps2"], case["h2"][:-1])
        with pytest.raises(ValueError, match="phiold"):
            g6.calc_firsthalf(n, case["id"], case["px"], case["pv"], zi, zi, np.zeros(n - 1),
                              case["eps2"], case["h2"])
        with pytest.raises(ValueError, match="h2"):
            g6.calc_lasthalf2(n, case["id"], case["px"], case["pv"], case["eps2"],
                              case["h2"][:-1])
    finally:
        g6.close()
