"""GPU: the documented workloads at their full sizes against the FP64 oracle
(on seeded samples of i where all of them would take the oracle minutes).

C1  4th order, N = 16384 Plummer, all i, lists off (mixed and FP64 kernels)
C2  6th order, N = 131072, block steps dt = 2^-k, k in 3..12, active sets
    from the block-bin occupancy, lists on (h2 for ~32 neighbours), NN on
C3  N = 2^20 precision form (Salpeter masses, 10 % binaries), mixed kernel
    on every i against the FP64 kernel (itself checked against the oracle on
    a seeded sample), spatial mode on and off
C4  512 Plummer clusters in one persistent launch (batch API)
"""
import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from sapporo2_b200 import ic
from sapporo2_b200.direct import fp64_direct
from tests import cases as T

pytestmark = pytest.mark.gpu


def test_c1_fourth_order_16384_all_active(gpu):
    cfg = ic.make_config("C1")
    n = cfg["n"]
    fn = O.derivative_fn()
    cfg["a"], cfg["j"], _ = fn(1, cfg["x"], cfg["v"], None, cfg["m"], cfg["id"], cfg["eps2"])
    px, pv, _ = O.predict(1, cfg["ti"], cfg["t0"], cfg["x"], cfg["v"], cfg["a"], cfg["j"])
    case = dict(order=1, n=n, x=cfg["x"], v=cfg["v"], m=cfg["m"], a=cfg["a"], j=cfg["j"],
                s=None, c=None, id=cfg["id"], t0=cfg["t0"], ti=cfg["ti"], px=px, pv=pv, pa=None,
                h2=np.zeros(n), eps2=cfg["eps2"])
    want = T.oracle_force(case, lists=False)
    for prec, tol in ((sp.DOUBLESINGLE, (T.MEDIAN_TOL, T.MAX_TOL)), (sp.DOUBLE, (1e-13, 1e-9))):
        got = T.run_library(case, prec, lists=False)
        st = T.check_forces(got, want, 1, *tol)
        T.check_nn(case, got["nnb"], want)
        print(prec, st)


def test_c2_sixth_order_131072_block_steps(gpu):
    cfg = ic.make_config("C2")
    n, k = cfg["n"], cfg["k"]
    x, v, m, ids, eps2 = cfg["x"], cfg["v"], cfg["m"], cfg["id"], cfg["eps2"]
    a, j, _ = fp64_direct(1, x, v, None, m, ids, eps2)
    _, _, s = fp64_direct(2, x, v, a, m, ids, eps2)
    c = ic.crackle_from(x, a, j)
    rng = np.random.default_rng(2)
    with sp.Sapporo(order=sp.SIXTH, precision=sp.DOUBLESINGLE, n_pipes=n) as lib:
        for step in (1, 6, 64, 512):
            T_, t0, act = ic.block_state(k, step)
            px, pv, pa = O.predict(2, T_, t0, x, v, a, j, s, c)
            lib.set_j_particles(np.arange(n), ids, t0, m, x, v, a, j, s, c)
            lib.set_time(T_)
            lib.start(n, ids[act], px[act], pv[act], pa[act], eps2, cfg["h2"][act])
            got = lib.results(n)
            cnt, lst = lib.neighbour_lists()
            q = np.sort(rng.choice(len(act), min(len(act), 768), replace=False))
            sel = act[q]
            want = O.force(2, px[sel], pv[sel], pa[sel], cfg["h2"][sel], ids[sel], px, pv, pa, m,
                           ids, eps2)
            sub = {f: got[f][q] for f in ("acc", "jrk", "snp", "pot")}
            st = T.check_forces(sub, want, 2)
            case = dict(n=n, px=px, id=ids, h2=cfg["h2"])
            T.check_nn(case, got["nnb"][q], want, sel=sel)
            np.testing.assert_array_equal(cnt[q], want["ngb_count"])
            sets = [lst[i, :min(cnt[i], sp.NGB_PB)] for i in q]
            T.check_neighbours(case, sets, cnt[q], want, sel=sel)
            assert np.median(want["ngb_count"]) > 10  # lists are really exercised
            print(step, len(act), st)


@pytest.fixture(scope="module")
def c3():
    """The N = 2^20 precision form (seed 3, as the benchmark) and the all-FP64
    kernel's results on every i (the FP64 kernel is pinned to the oracle in
    test_c3_fp64_kernel_matches_oracle)."""
    import bench
    cfg = bench.build_inputs(1 << 20, seed=3)
    cfg["f64"] = _c3_run(cfg, sp.DOUBLE)
    return cfg


def _c3_run(cfg, precision, spatial=None, near=None):
    n = cfg["n"]
    with sp.Sapporo(order=sp.SIXTH, precision=precision, n_pipes=n) as lib:
        if spatial is not None:
            lib.set_spatial(spatial, 0.0)
        if near is not None:
            lib.set_near(near)
        lib.set_j_particles(np.arange(n), cfg["id"], cfg["t0"], cfg["m"], cfg["x"], cfg["v"],
                            cfg["a"], cfg["j"], cfg["s"], cfg["c"])
        lib.set_time(cfg["ti"])
        lib.start(n, cfg["id"], cfg["px"], cfg["pv"], cfg["pa"], cfg["eps2"], np.zeros(n))
        got = lib.results(n)
        got["far_tiles"] = lib.spatial_stats()
    return got


def test_c3_fp64_kernel_matches_oracle(gpu, c3):
    n = c3["n"]
    sel = np.sort(np.random.default_rng(33).choice(n, 512, replace=False)).astype(np.int32)
    px, pv, pa = O.predict(2, c3["ti"], c3["t0"], c3["x"], c3["v"], c3["a"], c3["j"], c3["s"],
                           c3["c"])
    want = O.force_subset(2, sel, c3["px"], c3["pv"], c3["pa"], np.zeros(n), c3["id"], px, pv,
                          pa, c3["m"], c3["id"], c3["eps2"])
    sub = {f: c3["f64"][f][sel] for f in ("acc", "jrk", "snp", "pot")}
    print(T.check_forces(sub, want, 2, 1e-12, 1e-10))


@pytest.mark.parametrize("spatial", [1, 0])
def test_c3_precision_form_2_20_every_i(gpu, c3, spatial):
    """Mixed precision on all 2^20 i against the FP64 kernel: median <= 1e-6
    and max <= 1e-4 relative for acc, jerk, snap and pot, in spatial mode (the
    default for this call size) and in address order."""
    got = _c3_run(c3, sp.DOUBLESINGLE, spatial=spatial)
    far, tiles = got["far_tiles"]
    assert (far > 0.9 * tiles) if spatial else (tiles == 0)
    st = T.check_forces(got, c3["f64"], 2)
    assert st["acc"][0] <= 1e-6  # the required median relative acc error vs FP64
    print(spatial, st)


def test_c3_near_pairs_are_summed_in_fp64(gpu, c3):
    """The FP64 near-pair sums change the results where a j sits within 4
    softening lengths of an i and nowhere else."""
    on = _c3_run(c3, sp.DOUBLESINGLE, spatial=0)
    off = _c3_run(c3, sp.DOUBLESINGLE, spatial=0, near=0.0)
    changed = np.any(on["snp"] != off["snp"], axis=1)
    near = (on["ds2min"] < 16 * c3["eps2"]) & (on["ds2min"] > 0)
    assert changed.sum() > 1000 and np.all(near[changed])
    e_on = T.rel_err(on["snp"], c3["f64"]["snp"])[changed]
    e_off = T.rel_err(off["snp"], c3["f64"]["snp"])[changed]
    print(f"{changed.sum()} i with near pairs: snap max {e_off.max():.2e} -> {e_on.max():.2e}, "
          f"median {np.median(e_off):.2e} -> {np.median(e_on):.2e}")
    assert np.median(e_on) < 0.5 * np.median(e_off)


def test_c4_ensemble_of_512_clusters(gpu):
    import bench
    cl, first, ns = bench.ensemble_inputs(512, seed=4)
    total = int(ns.sum())
    act = np.array([len(c["active"]) for c in cl])
    with sp.Sapporo(order=sp.FOURTH, precision=sp.DOUBLESINGLE) as s:
        s.set_j_particles(np.arange(total), np.concatenate([c["id"] for c in cl]),
                          np.concatenate([c["t0"] for c in cl]), np.concatenate([c["m"] for c in cl]),
                          np.concatenate([c["x"] for c in cl]), np.concatenate([c["v"] for c in cl]),
                          np.concatenate([c["a"] for c in cl]), np.concatenate([c["j"] for c in cl]))
        s.force_prediction(total)
        with sp.Batch(s, len(cl), int(act.sum())) as b:
            b.plan(first, ns, act, [c["ti"] for c in cl], [c["eps2"] for c in cl])
            row = 0
            for c in cl:
                a_ = c["active"]
                b.i_stage[row:row + len(a_)] = sp.pack_i_records(1, c["px"][a_], c["pv"][a_],
                                                                 None, c["id"][a_])
                row += len(a_)
            b.run(sp.F_PREDICT)
            res = b.results()
    rows = np.concatenate([[0], np.cumsum(act)])
    for ci in np.random.default_rng(44).choice(len(cl), 8, replace=False):
        c = cl[ci]
        px, pv, _ = O.predict(1, c["ti"], c["t0"], c["x"], c["v"], c["a"], c["j"])
        a_ = c["active"]
        want = O.force(1, c["px"][a_], c["pv"][a_], None, np.zeros(len(a_)), c["id"][a_], px, pv,
                       None, c["m"], c["id"], c["eps2"], lists=False)
        r = res[rows[ci]:rows[ci + 1]]
        got = {"acc": r[:, 0:3], "pot": r[:, 3], "jrk": r[:, 4:7]}
        T.check_forces(got, want, 1)
