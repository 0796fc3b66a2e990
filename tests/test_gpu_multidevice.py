"""GPU: the sapporo class over several devices (sapporo::open with a device
list, lib/src/sapporohostclass.cpp:90-163).  The j are spread round-robin by
address (:473-474), each device computes the partial forces of its j on the
same i, and getGravResults sums them, takes the closest nearest neighbour and
concatenates the neighbour lists (:687-691, :749-799, :837-880).

A test box has one GPU, so the device lists repeat device 0: every entry
still gets its own handle, stream, j memory and force launches, which is
what the split and the combine exercise.  Checked against the FP64 oracle
and against the one-device class on the same inputs (nearest neighbours,
distances, neighbour sets and the predicted j state identical; forces within
the parity tolerances)."""
import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from tests import cases as T

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,precision,devices", [
    (1, sp.DOUBLESINGLE, [0, 0, 0]),
    (2, sp.DOUBLESINGLE, [0, 0]),
    (2, sp.DOUBLE, [0, 0, 0]),
])
def test_split_matches_oracle_and_one_device(gpu, order, precision, devices):
    # 20000 j: past the initial 16384 addresses (j memory grows by 10 %,
    # rounded to a multiple of the device count) and not a multiple of 3
    case = T.build_case(order, 20000, seed=61 + order, binaries=0.1)
    sel = np.sort(np.random.default_rng(5).choice(case["n"], 900, replace=False))
    one = T.run_library(case, precision, sel=sel)
    many = T.run_library(case, precision, sel=sel, devices=devices)
    want = T.oracle_force(case, sel)
    T.check_forces(many, want, order)
    T.check_nn(case, many["nnb"], want, sel)
    T.check_neighbours(case, many["ngb_sets"], many["ngb_count"], want, sel)
    # per pair the devices compute what one device does: the same nearest
    # neighbour (lower id at equal ds2), distance and neighbour sets
    np.testing.assert_array_equal(many["nnb"], one["nnb"])
    np.testing.assert_array_equal(many["ds2min"], one["ds2min"])
    # (an overflowing i's count stops at the device whose list crossed
    # maxlength, so counts and lists are compared below NGB_PB)
    small = one["ngb_count"] < sp.NGB_PB
    np.testing.assert_array_equal(many["ngb_count"][small], one["ngb_count"][small])
    assert np.all(many["ngb_count"][~small] >= sp.NGB_PB)
    for a, b, ok in zip(many["ngb_sets"], one["ngb_sets"], small):
        if ok:
            np.testing.assert_array_equal(a, b)
    assert many["overflow"] == one["overflow"]
    # forces: other partial sums, so equal only to rounding (each run is
    # within the parity tolerances of the oracle, checked above)
    for f in ("acc", "jrk", "pot") + (("snp",) if order >= 2 else ()):
        e = T.rel_err(many[f], one[f])
        assert np.median(e) <= 1e-6 and e.max() <= 2e-4, (f, np.median(e), e.max())
    if precision == sp.DOUBLE:
        for f in ("acc", "jrk", "pot", "snp"):
            assert T.rel_err(many[f], one[f]).max() <= 1e-10, f


def test_fewer_j_than_devices(gpu):
    # nj = 2 on three devices: the third holds no j and adds nothing
    case = T.build_case(2, 64, seed=71)
    n = 2
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE, devices=[0, 0, 0]) as s:
        assert len(s.devs) == 3
        s.set_j_particles(np.arange(n), case["id"][:n], case["t0"][:n], case["m"][:n],
                          case["x"][:n], case["v"][:n], case["a"][:n], case["j"][:n],
                          case["s"][:n], case["c"][:n])
        s.set_time(case["ti"])
        h2 = np.full(n, 1e3)
        s.start(n, case["id"][:n], case["px"][:n], case["pv"][:n], case["pa"][:n],
                case["eps2"], h2)
        got = s.results(n)
        lists = [s.get_ngb_list(i, sp.NGB_PB) for i in range(n)]
    want = O.force(2, case["px"][:n], case["pv"][:n], case["pa"][:n], h2, case["id"][:n],
                   case["px"][:n], case["pv"][:n], case["pa"][:n], case["m"][:n],
                   case["id"][:n], case["eps2"])
    T.check_forces(got, want, 2)
    # each body's only neighbour is the other one
    np.testing.assert_array_equal(got["nnb"], case["id"][[1, 0]])
    for i, (ovf, nb, ids) in enumerate(lists):
        assert ovf == 0 and nb == 1 and list(ids) == [int(case["id"][1 - i])]


def test_list_concatenation_and_overflow(gpu):
    # get_ngb_list over devices: the lists in device order until the total
    # reaches maxlength (overflow), then sorted; every id returned is a true
    # neighbour
    case = T.build_case(1, 3000, seed=81, nngb=48.0)
    sel = np.arange(0, 3000, 7)
    with sp.Sapporo(order=1, precision=sp.DOUBLESINGLE, devices=[0, 0]) as s:
        s.set_j_particles(np.arange(case["n"]), case["id"], case["t0"], case["m"], case["x"],
                          case["v"], case["a"], case["j"])
        s.set_time(case["ti"])
        s.start(case["n"], case["id"][sel], case["px"][sel], case["pv"][sel], None,
                case["eps2"], case["h2"][sel])
        s.results(case["n"])
        full = [s.get_ngb_list(q, sp.NGB_PB) for q in range(len(sel))]
        short = [s.get_ngb_list(q, 8) for q in range(len(sel))]
    want = T.oracle_force(case, sel)
    counts = np.array([f[1] for f in full])
    T.check_neighbours(case, [f[2] for f in full], counts, want, sel)
    tested = 0
    for q, ((ovf, nb, ids), (fo, fn, fids)) in enumerate(zip(short, full)):
        if fn >= 8:
            assert ovf == 1 and nb >= 8 and len(ids) == 8
            tested += 1
        else:
            assert ovf == 0 and nb == fn
            np.testing.assert_array_equal(ids, fids)
        assert np.all(np.diff(ids) > 0)
        assert set(ids.tolist()) <= set(fids.tolist())
    assert tested > 100


def test_predicted_state_readback(gpu):
    # retrieve_predicted_j_particle / retrieve_j_particle_state find each
    # address on its device (a % G at a / G)
    case = T.build_case(2, 5000, seed=91)
    n = case["n"]
    out = []
    for devices in (None, [0, 0, 0]):
        with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE, devices=devices) as s:
            s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"],
                              case["v"], case["a"], case["j"], case["s"], case["c"])
            s.set_time(case["ti"])
            s.force_prediction(n)
            picks = [0, 1, 2, 3, 1234, 4998, 4999]
            out.append([(s.retrieve_predicted(k), s.retrieve_state(k)) for k in picks])
    for (p1, s1), (p3, s3) in zip(*out):
        for key in p1:
            np.testing.assert_array_equal(p3[key], p1[key])
        for key in s1:
            np.testing.assert_array_equal(s3[key], s1[key])
    for k, (p, _) in zip([0, 1, 2, 3, 1234, 4998, 4999], out[1]):
        assert p["id"] == case["id"][k]
        np.testing.assert_allclose(p["pos"], case["px"][k], rtol=0, atol=1e-12)
