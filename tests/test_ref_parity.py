"""GPU parity against the reference's own CUDA kernels (oracle/_ref: the
reference's kernels.cu compiled unchanged for sm_100a, launched with the
reference geometry) on fresh seeded inputs."""
import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from tests import cases as T

pytestmark = pytest.mark.gpu


def _ref_ready():
    if not O.ref_available():
        pytest.skip("oracle/_ref not built (reference tree absent when the repo was built)")


def _run(order, precision, n, seed, sel=None):
    case = T.build_case(order, n, seed, binaries=0.1)
    rpx, rpv, rpa = O.ref_predict(order, case["ti"], case["t0"], case["x"], case["m"], case["v"],
                                  case["a"], case["j"], case["s"], case["c"])
    # i = reference-predicted state, so both sides see identical i and j
    case = dict(case, px=rpx, pv=rpv, pa=rpa if order == 2 else None)
    idx = np.arange(n) if sel is None else sel
    ref = O.ref_gravity(order, precision, rpx[idx], rpv[idx],
                        rpa[idx] if order == 2 else None, case["h2"][idx], case["id"][idx],
                        rpx, rpv, rpa if order == 2 else None, case["m"], case["id"],
                        case["eps2"])
    ref["ngb_list"] = np.sort(np.where(np.arange(256)[None, :] < ref["ngb_count"][:, None],
                                       ref["ngb_list"], np.iinfo(np.int32).max), axis=1)
    got = T.run_library(case, precision, sel=sel)
    return case, ref, got


# The reference's 6th-order snap is not a defined value: devForce2's default
# constructor (lib/CUDAKernels/kernels.cu:519-524) zeroes acc, pot and jerk but
# leaves snpx/snpy/snpz uninitialised before `+=` (:661-663).  Acc, jerk, pot,
# nearest neighbour and lists are compared with the reference kernels; snap is
# compared with the FP64 oracle, which sums the same expression from zero.
REF_FIELDS = ["acc", "pot", "jrk"]


def _snap_vs_oracle(case, got, sel=None):
    if case["order"] < 2:
        return
    want = T.oracle_force(case, sel=sel, lists=False)
    T.check_forces(got, want, 2, fields=["snp"])


@pytest.mark.parametrize("order,precision", [(1, sp.DOUBLESINGLE), (1, sp.DOUBLE),
                                             (2, sp.DOUBLESINGLE), (2, sp.DOUBLE)])
def test_matches_reference_kernels(gpu, order, precision):
    _ref_ready()
    case, ref, got = _run(order, precision, 4096, seed=31 + order)
    stats = T.check_forces(got, ref, order, fields=REF_FIELDS)
    _snap_vs_oracle(case, got)
    nn_ties = T.check_nn(case, got["nnb"], ref)
    exempt = T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], ref)
    assert nn_ties <= 2
    print(f"order {order} prec {precision}: {stats} nn-ties {nn_ties} boundary pairs {exempt}")


@pytest.mark.parametrize("order", [1, 2])
def test_predictor_matches_reference(gpu, order):
    _ref_ready()
    case = T.build_case(order, 3000, seed=41)
    rpx, rpv, rpa = O.ref_predict(order, case["ti"], case["t0"], case["x"], case["m"], case["v"],
                                  case["a"], case["j"], case["s"], case["c"])
    n = case["n"]
    with sp.Sapporo(order=order, precision=sp.DOUBLE) as s:
        s.set_j_particles(np.arange(n), case["id"], case["t0"], case["m"], case["x"], case["v"],
                          case["a"], case["j"], case["s"], case["c"])
        s.set_time(case["ti"])
        s.force_prediction(n)
        out = np.zeros((n, 24))
        assert s.lib.sapb_read_j(s.dev, 0, n, case["ti"], 1, out) == 0
    px, pv = out[:, 14:17], out[:, 17:20]
    assert np.max(np.abs(px - rpx) / np.maximum(np.abs(rpx), 1e-300)) <= 2e-16
    assert np.max(np.abs(pv - rpv) / np.maximum(np.abs(rpv), 1e-300)) <= 2e-16
    if order == 2:
        pa = out[:, 20:23]
        assert np.max(np.abs(pa - rpa) / np.maximum(np.abs(rpa), 1e-300)) <= 2e-16


@pytest.mark.parametrize("ni", [1, 7, 96, 100, 256])
def test_small_steps_match_reference(gpu, ni):
    """Block-step sized active sets (6th order never rounds i in the
    reference launch, so every size is a valid reference run)."""
    _ref_ready()
    sel = np.sort(np.random.default_rng(ni).choice(2500, ni, replace=False))
    case, ref, got = _run(2, sp.DOUBLESINGLE, 2500, seed=51, sel=sel)
    T.check_forces(got, ref, 2, fields=REF_FIELDS)
    _snap_vs_oracle(case, got, sel=sel)
    T.check_nn(case, got["nnb"], ref, sel=sel)
    T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], ref, sel=sel)


# ---- the workloads at their own sizes (reference geometry: 256-i launches) ----
def _c1_case():
    from sapporo2_b200 import ic
    cfg = ic.make_config("C1")
    n = cfg["n"]
    a, j, _ = O.derivative_fn()(1, cfg["x"], cfg["v"], None, cfg["m"], cfg["id"], cfg["eps2"])
    rpx, rpv, _ = O.ref_predict(1, cfg["ti"], cfg["t0"], cfg["x"], cfg["m"], cfg["v"], a, j)
    return dict(order=1, n=n, x=cfg["x"], v=cfg["v"], m=cfg["m"], a=a, j=j, s=None, c=None,
                id=cfg["id"], t0=cfg["t0"], ti=cfg["ti"], px=rpx, pv=rpv, pa=None,
                h2=np.zeros(n), eps2=cfg["eps2"])


@pytest.mark.parametrize("precision", [sp.DOUBLESINGLE, sp.DOUBLE])
def test_c1_16384_all_i_matches_reference(gpu, precision):
    """C1 (4th order, N = 16384 Plummer, all i, lists off) against the
    reference's fourth_DS / fourth_double (kernels.cu:1100-1102)."""
    _ref_ready()
    case = _c1_case()
    n = case["n"]
    assert O.ref_size_ok(1, n)  # no padded i-threads in the reference launch
    ref = O.ref_gravity(1, precision, case["px"], case["pv"], None, case["h2"], case["id"],
                        case["px"], case["pv"], None, case["m"], case["id"], case["eps2"])
    got = T.run_library(case, precision, lists=False)
    stats = T.check_forces(got, ref, 1, fields=REF_FIELDS)
    ties = T.check_nn(case, got["nnb"], ref)
    assert ties <= 2 and n == 16384
    print(f"C1 prec {precision}: {stats} nn-ties {ties}")


_C2 = {}


def _c2_case(step):
    """C2 (6th order, N = 131072 Plummer, block steps dt = 2^-k, k in 3..12,
    h2 for ~32 neighbours) at block time step * 2^-12: j predicted by the
    reference's own predictor, the active set from the block-bin occupancy."""
    from sapporo2_b200 import ic
    from sapporo2_b200.direct import fp64_direct
    if "base" not in _C2:
        cfg = ic.make_config("C2")
        x, v, m, ids, eps2 = cfg["x"], cfg["v"], cfg["m"], cfg["id"], cfg["eps2"]
        a, j, _ = fp64_direct(1, x, v, None, m, ids, eps2)
        _, _, s = fp64_direct(2, x, v, a, m, ids, eps2)
        _C2["base"] = (cfg, a, j, s, ic.crackle_from(x, a, j))
    cfg, a, j, s, c = _C2["base"]
    T_, t0, act = ic.block_state(cfg["k"], step)
    rpx, rpv, rpa = O.ref_predict(2, T_, t0, cfg["x"], cfg["m"], cfg["v"], a, j, s, c)
    case = dict(order=2, n=cfg["n"], x=cfg["x"], v=cfg["v"], m=cfg["m"], a=a, j=j, s=s, c=c,
                id=cfg["id"], t0=t0, ti=T_, px=rpx, pv=rpv, pa=rpa, h2=cfg["h2"],
                eps2=cfg["eps2"])
    return case, act


def _c2_ref(case, sel, precision):
    ref = O.ref_gravity(2, precision, case["px"][sel], case["pv"][sel], case["pa"][sel],
                        case["h2"][sel], case["id"][sel], case["px"], case["pv"], case["pa"],
                        case["m"], case["id"], case["eps2"])
    ref["ngb_list"] = np.sort(np.where(np.arange(256)[None, :] < ref["ngb_count"][:, None],
                                       ref["ngb_list"], np.iinfo(np.int32).max), axis=1)
    return ref


@pytest.mark.parametrize("precision", [sp.DOUBLESINGLE, sp.DOUBLE])
def test_c2_block_step_matches_reference(gpu, precision):
    """C2's first block step (the 12983 particles with dt = 2^-12) on all
    131072 j, lists and nearest neighbours on, against the reference's
    sixth_DS / sixth_double (kernels.cu:1104-1106); snap against the oracle."""
    _ref_ready()
    case, act = _c2_case(1)
    assert len(act) >= 12983
    ref = _c2_ref(case, act, precision)
    got = T.run_library(case, precision, sel=act)
    stats = T.check_forces(got, ref, 2, fields=REF_FIELDS)
    _snap_vs_oracle(case, got, sel=act)
    ties = T.check_nn(case, got["nnb"], ref, sel=act)
    exempt = T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], ref, sel=act)
    assert ties <= 2 and np.median(ref["ngb_count"]) > 10
    print(f"C2 step 1 prec {precision}: {len(act)} i {stats} nn-ties {ties} boundary {exempt}")


def test_spatial_call_matches_reference(gpu):
    """One call above the spatial-mode threshold (4096 i x 131072 j = 2^29
    pairs: Morton order, single-float difference on far tiles) against the
    reference's sixth_DS, lists and nearest neighbours on."""
    _ref_ready()
    case, _ = _c2_case(1)
    sel = np.sort(np.random.default_rng(71).choice(case["n"], 4096, replace=False))
    ref = _c2_ref(case, sel, sp.DOUBLESINGLE)
    got = T.run_library(case, sp.DOUBLESINGLE, sel=sel, spatial=(1, 0.0))
    far, tiles = got["far_tiles"]
    assert far > 0.5 * tiles > 0  # the call really ran in spatial mode
    stats = T.check_forces(got, ref, 2, fields=REF_FIELDS)
    _snap_vs_oracle(case, got, sel=sel)
    ties = T.check_nn(case, got["nnb"], ref, sel=sel)
    exempt = T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], ref, sel=sel)
    assert ties <= 2
    print(f"spatial call: far {far}/{tiles} {stats} nn-ties {ties} boundary {exempt}")


def test_c3_headline_config_matches_reference(gpu):
    """C3, the workload of the headline figure (N = 2^20 Plummer, Salpeter
    masses, 10 % binaries 1e-6..1e-4 apart, 6th order): 2048 seeded i against
    all 2^20 j (2^31 pairs, spatial mode by the default rule), lists and
    nearest neighbours on, against the reference's sixth_DS; snap against the
    oracle."""
    _ref_ready()
    from sapporo2_b200 import ic
    from sapporo2_b200.direct import fp64_direct
    cfg = ic.make_config("C3")
    x, v, m, ids, eps2 = cfg["x"], cfg["v"], cfg["m"], cfg["id"], cfg["eps2"]
    a, j, _ = fp64_direct(1, x, v, None, m, ids, eps2)
    _, _, sn = fp64_direct(2, x, v, a, m, ids, eps2)
    c = ic.crackle_from(x, a, j)
    rpx, rpv, rpa = O.ref_predict(2, cfg["ti"], cfg["t0"], x, m, v, a, j, sn, c)
    case = dict(order=2, n=cfg["n"], x=x, v=v, m=m, a=a, j=j, s=sn, c=c, id=ids, t0=cfg["t0"],
                ti=cfg["ti"], px=rpx, pv=rpv, pa=rpa, h2=cfg["h2"], eps2=eps2)
    sel = np.sort(np.random.default_rng(73).choice(case["n"], 2048, replace=False))
    ref = _c2_ref(case, sel, sp.DOUBLESINGLE)
    got = T.run_library(case, sp.DOUBLESINGLE, sel=sel, spatial=(1, 0.0))
    far, tiles = got["far_tiles"]
    assert far > 0.5 * tiles > 0  # the default rule ordered the call
    stats = T.check_forces(got, ref, 2, fields=REF_FIELDS)
    _snap_vs_oracle(case, got, sel=sel)
    ties = T.check_nn(case, got["nnb"], ref, sel=sel)
    exempt = T.check_neighbours(case, got["ngb_sets"], got["ngb_count"], ref, sel=sel)
    assert ties <= 2 and np.median(ref["ngb_count"]) > 10
    print(f"C3: far {far}/{tiles} {stats} nn-ties {ties} boundary {exempt}")
