"""GPU: spatial mode of the mixed-precision force calls.

In spatial mode the predicted j records and the call's i positions are taken
in Morton order, and (warp, j tile) pairs whose boxes are far apart use the
single-float difference of the high position parts instead of the
double-single difference of the reference (kernels.cu:169-177).  Tiles that
could hold a nearest neighbour or a list member always take the
double-single path.  So, against the same call in address order (mode 0):
nearest neighbours, their ds2 and the neighbour lists are identical, and the
forces agree with the FP64 oracle within the mixed-precision tolerance.
"""
import numpy as np
import pytest

import sapporo2_b200 as sp
from sapporo2_b200 import ic
from tests import cases as T

pytestmark = pytest.mark.gpu

EVERY_CALL = 2  # spatial mode for every call, whatever its size


def _same_neighbours(a, b):
    """Nearest neighbours (id and ds2 bits) and neighbour lists identical."""
    assert np.array_equal(a["raw"][:, 10:12], b["raw"][:, 10:12])
    assert np.array_equal(a["nnb"], b["nnb"])
    assert a["overflow"] == b["overflow"]
    assert np.array_equal(a["ngb_count"], b["ngb_count"])
    for q in np.nonzero(np.asarray(a["ngb_count"]) < sp.NGB_PB)[0]:
        assert np.array_equal(a["ngb_sets"][q], b["ngb_sets"][q]), q


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("delta", [0.0, 1e-5])
def test_spatial_matches_oracle_and_address_order(gpu, order, delta):
    """Shape (1, 4): at this size the planner would pick one i per thread,
    which takes the Morton order but not the far tiles."""
    case = T.build_case(order, 6000, seed=21, binaries=0.1)
    want = T.oracle_force(case)
    got = T.run_library(case, sp.DOUBLESINGLE, launch=(1, 4, 0), spatial=(EVERY_CALL, delta))
    ref = T.run_library(case, sp.DOUBLESINGLE, launch=(1, 4, 0), spatial=(0, 0.0))
    st = T.check_forces(got, want, order)
    assert T.check_nn(case, got["nnb"], want) == T.check_nn(case, ref["nnb"], want)
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want)
    _same_neighbours(got, ref)
    far, tiles = got["far_tiles"]
    assert tiles > 0 and far > 0, (far, tiles)  # the far path ran
    print(st, far / tiles)


@pytest.mark.parametrize("launch", [(1, 4, 0), (2, 4, 3), (1, 2, 0), (2, 2, 3), (4, 2, 0),
                                    (8, 2, 5), (16, 1, 2), (32, 1, 0)])
def test_spatial_launch_shapes(gpu, launch):
    """Every shape: the packed ones (two i per instruction) take far tiles,
    the one-i-per-thread ones only the Morton order of i and j."""
    case = T.build_case(2, 6000, seed=22, binaries=0.1)
    sel = np.random.default_rng(5).choice(6000, 5000, replace=False)
    want = T.oracle_force(case, sel=sel)
    got = T.run_library(case, sp.DOUBLESINGLE, sel=sel, launch=launch,
                        spatial=(EVERY_CALL, 1e-5))
    ref = T.run_library(case, sp.DOUBLESINGLE, sel=sel, launch=launch, spatial=(0, 0.0))
    far, tiles = got["far_tiles"]
    assert (far > 0) == (launch[1] > 1), (far, tiles)  # packed shapes only
    T.check_forces(got, want, 2)
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], want, sel=sel)
    _same_neighbours(got, ref)


def test_spatial_foreign_i_outside_the_j_box(gpu):
    """i that are not among the j (other ids) and partly far outside the j
    box, where their Morton keys clamp to its faces."""
    case = T.build_case(2, 4000, seed=23, binaries=0.1)
    rng = np.random.default_rng(8)
    ni = 3000
    xi = case["px"][rng.choice(4000, ni)] + rng.normal(scale=1e-3, size=(ni, 3))
    xi[: ni // 3] += np.array([40.0, -25.0, 10.0])
    vi = rng.normal(scale=0.3, size=(ni, 3))
    ai = rng.normal(scale=0.1, size=(ni, 3))
    ids = np.arange(ni, dtype=np.int32) + 10_000_000
    h2 = np.full(ni, 0.01)
    from oracle import oracle as O
    want = O.force(2, xi, vi, ai, h2, ids, case["px"], case["pv"], case["pa"], case["m"],
                   case["id"], case["eps2"], lists=True)
    out = {}
    for mode in (EVERY_CALL, 0):
        with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
            s.set_spatial(mode, 1e-5)
            n = case["n"]
            s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"],
                              case["v"], case["a"], case["j"], case["s"], case["c"])
            s.set_time(case["ti"])
            s.start(n, ids, xi, vi, ai, case["eps2"], h2)
            r = s.results(n, ngb=True)
            r["raw"] = s.raw_results(ni).copy()
            out[mode] = r
    got = out[EVERY_CALL]
    T.check_forces(got, want, 2)
    assert np.array_equal(got["raw"][:, 10:12], out[0]["raw"][:, 10:12])
    jpos = {int(k): p for k, p in zip(case["id"], case["px"])}
    for q in np.nonzero(got["nnb"] != want["nnb"])[0]:  # near-ties only
        d = [float(((jpos[int(k)] - xi[q]) ** 2).sum()) for k in (got["nnb"][q], want["nnb"][q])]
        assert abs(d[0] - d[1]) <= 1e-6 * d[1], (q, d)


def test_spatial_self_pair_on_a_far_tile(gpu):
    """i given far from their own j (same id, positions displaced by 40):
    the self pair then lies on a far tile, whose loop reads the id from the
    record's velocity row, and is skipped by id as the reference skips it
    (kernels.cu:565).  Its force would shift acc and pot by ~2.5e-4."""
    from oracle import oracle as O
    case = T.build_case(2, 4000, seed=29, binaries=0.1)
    n = case["n"]
    sel = np.arange(0, n, 4)
    xi = case["px"][sel] + np.array([40.0, -25.0, 10.0])
    vi, ai = case["pv"][sel], case["pa"][sel]
    h2 = np.full(len(sel), 0.01)
    want = O.force(2, xi, vi, ai, h2, case["id"][sel], case["px"], case["pv"], case["pa"],
                   case["m"], case["id"], case["eps2"], lists=True)
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
        s.set_launch(1, 4, 0)
        s.set_spatial(EVERY_CALL, 1e-5)
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"],
                          case["v"], case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        s.start(n, case["id"][sel], xi, vi, ai, case["eps2"], h2)
        got = s.results(n, ngb=True)
        far, tiles = s.spatial_stats()
    assert tiles > 0 and far > 0, (far, tiles)
    T.check_forces(got, want, 2)


def test_spatial_reorders_after_j_change(gpu):
    """The ordering follows the predicted records: a second call after new j
    data and a new prediction time uses them, not the first call's order."""
    a = T.build_case(2, 5000, seed=24, binaries=0.1)
    b = T.build_case(2, 5000, seed=25, binaries=0.1)
    n = a["n"]
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
        s.set_spatial(EVERY_CALL, 1e-5)
        for case in (a, b):
            s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"],
                              case["v"], case["a"], case["j"], case["s"], case["c"])
            s.set_time(case["ti"])
            s.start(n, case["id"], case["px"], case["pv"], case["pa"], case["eps2"], case["h2"])
            got = s.results(n, ngb=True)
            want = T.oracle_force(case, lists=False)
            T.check_forces(got, want, 2)
            T.check_nn(case, got["nnb"], want)


def test_spatial_forces_do_not_depend_on_h2(gpu):
    """The far test ignores h2 (list members on far tiles are found by an exact
    rescan), so two radii give bit-identical forces and nearest neighbours;
    a radius reaching well into far tiles still gives the address-order
    lists."""
    case = T.build_case(2, 6000, seed=27, binaries=0.1)
    wide = dict(case)
    wide["h2"] = np.full(case["n"], 0.15 ** 2)
    a = T.run_library(case, sp.DOUBLESINGLE, launch=(1, 4, 0), spatial=(EVERY_CALL, 1e-5))
    b = T.run_library(wide, sp.DOUBLESINGLE, launch=(1, 4, 0), spatial=(EVERY_CALL, 1e-5))
    ref = T.run_library(wide, sp.DOUBLESINGLE, launch=(1, 4, 0), spatial=(0, 0.0))
    assert b["far_tiles"][0] > 0
    assert np.array_equal(a["raw"], b["raw"])
    _same_neighbours(b, ref)
    assert np.mean(b["ngb_count"]) > 10  # lists reach far beyond the near tiles


def test_spatial_grape5_order(gpu):
    """GRAPE-5 order (acceleration and potential only, the self pair kept,
    no neighbours) in spatial mode against the oracle; far tiles are taken."""
    from oracle import oracle as O
    case = T.build_case(1, 6000, seed=28, binaries=0.1)
    n, eps2 = case["n"], 1e-6
    x, m = case["x"], case["m"]
    z = np.zeros((n, 3))
    with sp.Sapporo(order=sp.GRAPE5, precision=sp.DOUBLESINGLE) as s:
        s.set_launch(1, 4, 0)
        s.set_spatial(EVERY_CALL, 1e-5)
        s.set_j_particles(np.arange(n), case["id"], np.zeros(n), m, x, z, z, z)
        s.start(n, case["id"], x, z, None, eps2, np.full(n, 1.0))
        got = s.results(n)
        far, tiles = s.spatial_stats()
    want = O.force(1, x, z, None, np.zeros(n), np.full(n, -7, dtype=np.int32), x, z, None, m,
                   case["id"], eps2, lists=False)
    T.check_forces({"acc": got["acc"], "pot": got["pot"]}, want, 1, fields=["acc", "pot"])
    assert tiles > 0 and far > tiles // 4, (far, tiles)


def test_spatial_default_mode_threshold(gpu):
    """Mode 1 (the default) orders only calls of >= 2^28 pairs and >= 65536 j: a small call
    gives bit-identical results to mode 0."""
    case = T.build_case(2, 2000, seed=26, binaries=0.1)
    got = T.run_library(case, sp.DOUBLESINGLE, spatial=(1, 0.0))
    ref = T.run_library(case, sp.DOUBLESINGLE, spatial=(0, 0.0))
    assert np.array_equal(got["raw"], ref["raw"])


def test_spatial_default_mode_turns_on_at_threshold(gpu):
    """Mode 1 orders a call from 2^28 pairs and 1024 i on: 1023 i x 2^18 j
    runs in address order, 1024 i x 2^18 j (2^28 pairs) in spatial mode."""
    n = 1 << 18
    x, v, m = ic.plummer(n, 27)
    z = np.zeros((n, 3))
    ids = np.arange(n, dtype=np.int32)
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
        s.set_spatial(1, 0.0)
        s.set_j_particles(np.arange(n), ids, np.zeros(n), m, x, v, z, z, z, z)
        s.set_time(0.0)
        for ni, on in ((1023, False), (1024, True)):
            sel = (np.arange(ni) * 257) % n
            s.start(n, ids[sel], x[sel], v[sel], z[sel], 1e-6, np.zeros(ni))
            r = s.results(n)
            assert np.all(np.isfinite(r["acc"]))
            far, tiles = s.spatial_stats(reset=True)
            assert (tiles > 0) == on, (ni, far, tiles)


def test_spatial_rejects_bad_arguments(gpu):
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
        for mode, delta in [(3, 0.0), (-1, 0.0), (1, -1e-6), (1, 2e-4), (1, float("nan"))]:
            with pytest.raises(sp.SapporoError):
                s.set_spatial(mode, delta)
        s.set_spatial(0, 0.0)
