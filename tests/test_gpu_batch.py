"""GPU: batched force evaluation (one persistent launch in a captured CUDA
graph) against the FP64 oracle -- ensembles of independent clusters of mixed
N with their own prediction times and active fractions, and block-timestep
steps of one system."""
import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from sapporo2_b200 import ic
from tests import cases as T

pytestmark = pytest.mark.gpu


def make_ensemble(order, k, seed, nmin=64, nmax=1500):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), k)).astype(int)
    clusters = []
    for c, n in enumerate(ns):
        case = T.build_case(order, int(n), seed=seed * 100 + c, binaries=0.1, id_offset=0)
        # each cluster has its own prediction time
        case["ti"] = 1.0 + 0.01 * c
        case["t0"] = case["ti"] - rng.integers(0, 8, n) * 2.0 ** -10
        case["px"], case["pv"], case["pa"] = O.predict(order, case["ti"], case["t0"], case["x"],
                                                       case["v"], case["a"], case["j"],
                                                       case["s"], case["c"])
        case["h2"] = ic.plummer_h2(case["px"], case["m"], 24.0)
        frac = np.exp(rng.uniform(np.log(1.0 / n), 0.0))
        na = max(1, int(round(frac * n)))
        case["active"] = np.sort(rng.choice(n, na, replace=False))
        clusters.append(case)
    return clusters


def run_ensemble(order, precision, clusters, lists=True, tuning=0, reps=1, near=None):
    total = sum(c["n"] for c in clusters)
    with sp.Sapporo(order=order, precision=precision) as s:
        if near is not None:
            s.set_near(near)
        addr = 0
        j_first, j_count, i_count, t_pred, eps2 = [], [], [], [], []
        for c in clusters:
            n = c["n"]
            s.set_j_particles(np.arange(addr, addr + n), c["id"], c["t0"], c["m"], c["x"],
                              c["v"], c["a"], c["j"], c["s"], c["c"])
            j_first.append(addr)
            j_count.append(n)
            i_count.append(len(c["active"]))
            t_pred.append(c["ti"])
            eps2.append(c["eps2"])
            addr += n
        s.force_prediction(total)  # upload (the batch graph predicts per cluster)
        max_i = sum(i_count) + 16
        with sp.Batch(s, len(clusters), max_i) as b:
            b.set_tuning(tuning)
            b.plan(j_first, j_count, i_count, t_pred, eps2)
            row = 0
            for c in clusters:
                a = c["active"]
                rec = sp.pack_i_records(order, c["px"][a], c["pv"][a], c["h2"][a], c["id"][a],
                                        c["pa"][a] if order >= 2 else None)
                b.i_stage[row:row + len(a)] = rec
                row += len(a)
            flags = sp.F_PREDICT | (sp.F_NGB_LIST if lists else 0)
            for _ in range(reps):
                b.run(flags)
                res = b.results()
            info = b.info()
            cnt, lst = b.neighbours() if lists else (None, None)
    return res, cnt, lst, info


def check_cluster(order, precision, c, res, cnt, lst):
    a = c["active"]
    want = T.oracle_force(c, sel=a)
    got = {"acc": res[:, 0:3], "pot": res[:, 3], "jrk": res[:, 4:7], "snp": res[:, 7:10],
           "nnb": res[:, 11].astype(np.int32)}
    tol = (1e-13, 1e-9) if precision == sp.DOUBLE else (T.MEDIAN_TOL, T.MAX_TOL)
    T.check_forces(got, want, order, *tol)
    T.check_nn(c, got["nnb"], want, sel=a)
    if cnt is not None:
        sets = [np.sort(lst[q, :min(cnt[q], sp.NGB_PB)]) for q in range(len(a))]
        T.check_neighbours(c, sets, cnt, want, sel=a)


@pytest.mark.parametrize("order,precision", [(1, sp.DOUBLESINGLE), (2, sp.DOUBLESINGLE),
                                             (2, sp.DOUBLE)])
def test_ensemble_matches_oracle(gpu, order, precision):
    clusters = make_ensemble(order, 24, seed=7 + order)
    res, cnt, lst, info = run_ensemble(order, precision, clusters, reps=2)
    assert info["runs"] == 2 and info["items"] >= len(clusters)
    row = 0
    for c in clusters:
        k = len(c["active"])
        check_cluster(order, precision, c, res[row:row + k], cnt[row:row + k], lst[row:row + k])
        row += k


@pytest.mark.parametrize("order", [1, 2])
def test_ensemble_near_pairs_in_fp64(gpu, order):
    """The batch kernel sums the rows of tiles holding a near pair (ds2 < 16
    eps2) in FP64: results change exactly for the i with such a pair, and
    the changed ones move closer to the oracle."""
    clusters = make_ensemble(order, 12, seed=31 + order)
    for c in clusters:  # a softening of 1e-2: pairs within 4e-2 are near ones
        c["eps2"] = 1e-4
    on = run_ensemble(order, sp.DOUBLESINGLE, clusters, lists=False)[0]
    off = run_ensemble(order, sp.DOUBLESINGLE, clusters, lists=False, near=0.0)[0]
    row, e_on, e_off, n_changed = 0, [], [], 0
    for c in clusters:
        a = c["active"]
        k = len(a)
        ro, rf = on[row:row + k], off[row:row + k]
        changed = np.any(ro[:, 0:10] != rf[:, 0:10], axis=1)
        near = (ro[:, 10] < 16 * c["eps2"]) & (ro[:, 11] >= 0)
        assert np.array_equal(changed, near), c["n"]
        want = T.oracle_force(c, sel=a, lists=False)
        f, sl = ("snp", slice(7, 10)) if order >= 2 else ("jrk", slice(4, 7))
        for r, e in ((ro, e_on), (rf, e_off)):
            e.append(T.rel_err(r[:, sl], want[f])[changed])
        n_changed += int(changed.sum())
        row += k
    e_on, e_off = np.concatenate(e_on), np.concatenate(e_off)
    assert n_changed > 30, n_changed
    assert np.median(e_on) < np.median(e_off), (np.median(e_on), np.median(e_off))


@pytest.mark.parametrize("tuning", [-2, 1, 3])
def test_ensemble_tuning_shapes_agree(gpu, tuning):
    clusters = make_ensemble(1, 10, seed=21)
    res, cnt, lst, _ = run_ensemble(1, sp.DOUBLESINGLE, clusters, tuning=tuning)
    row = 0
    for c in clusters:
        k = len(c["active"])
        check_cluster(1, sp.DOUBLESINGLE, c, res[row:row + k], cnt[row:row + k],
                      lst[row:row + k])
        row += k


def test_block_steps_one_system(gpu):
    """Block time steps dt = 2^-k: at each block time the active set is the
    particles whose step divides it, every j is predicted from its own last
    time; consecutive steps replay the same graph with different sizes."""
    n = 3000
    case = T.build_case(2, n, seed=91, binaries=0.1, t_spread=False)
    k, dt = ic.block_timesteps(n, seed=5, kmin=3, kmax=8)
    with sp.Sapporo(order=2, precision=sp.DOUBLESINGLE) as s:
        with sp.Batch(s, 1, n) as b:
            for step in (37, 64, 96, 128):
                T_, t0, active = ic.block_state(k, 256 + step, kmax=8)
                s.set_j_particles(np.arange(n), case["id"], t0, case["m"], case["x"],
                                  case["v"], case["a"], case["j"], case["s"], case["c"])
                s.force_prediction(n)
                px, pv, pa = O.predict(2, T_, t0, case["x"], case["v"], case["a"], case["j"],
                                       case["s"], case["c"])
                c = dict(case, ti=T_, t0=t0, px=px, pv=pv, pa=pa, active=active)
                b.plan([0], [n], [len(active)], [T_], [case["eps2"]])
                b.i_stage[:len(active)] = sp.pack_i_records(2, px[active], pv[active],
                                                            c["h2"][active], c["id"][active],
                                                            pa[active])
                b.run(sp.F_PREDICT | sp.F_NGB_LIST)
                res = b.results()
                cnt, lst = b.neighbours()
                check_cluster(2, sp.DOUBLESINGLE, c, res, cnt, lst)
            assert b.info()["runs"] == 4
