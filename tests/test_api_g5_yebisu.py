"""GPU: the GRAPE-5 interface (in libsapporo_b200.so, the reference's
lib/interfaces/sapporoG5lib.cpp API) and the Yebisu 6th-order interface
(libsapporoyeb_b200.so, lib/interfaces/sapporoYeblib.cpp) against the FP64
oracle."""
import ctypes as C

import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from tests import cases as T

gpu = pytest.mark.gpu


@gpu
def test_g5_forces_include_the_self_potential(gpu):
    """GRAPE-5 computes every pair, the self pair included: zero force and
    -m/eps in the potential (kernels.cu:565 skips nothing for GRAPE5)."""
    case = T.build_case(1, 3000, seed=91, binaries=0.0)
    n, eps = case["n"], 1e-3
    x, m = case["x"], case["m"]
    g5 = sp.G5()
    try:
        g5.set_eps(eps)
        g5.set_j(x, m)
        assert g5.lib.g5_get_number_of_pipelines() > 0
        a, phi = g5.force(x)
        a2, phi2 = g5.force_chunk(x[:700])
    finally:
        g5.close()
    z = np.zeros((n, 3))
    want = O.force(1, x, z, None, np.zeros(n), np.full(n, -7, dtype=np.int32), x, z, None, m,
                   np.arange(n, dtype=np.int32), eps * eps, lists=False)
    T.check_forces({"acc": a, "pot": phi, "jrk": want["jrk"]}, want, 1, fields=["acc", "pot"])
    # g5_set_xi / g5_get_force on a chunk (another launch shape: same physics)
    part = {k: (v[:700] if v is not None else None) for k, v in want.items()}
    T.check_forces({"acc": a2, "pot": phi2}, part, 1, fields=["acc", "pot"])
    # the self term is in: it alone is -m/eps, far beyond the tolerance
    assert np.all(m / eps > 1e-3 * np.abs(want["pot"]))


class Pred(C.Structure):
    _fields_ = [("pos", C.c_double * 3), ("vel", C.c_double * 3), ("acc", C.c_double * 3),
                ("mass", C.c_double), ("id", C.c_double), ("eps2", C.c_double)]


class Force(C.Structure):
    _fields_ = [("acc", C.c_double * 3), ("jrk", C.c_double * 3), ("snp", C.c_double * 3),
                ("phi", C.c_double), ("nnb_id", C.c_int), ("nnb_r2", C.c_float)]


def test_yebisu_records_have_the_reference_layout():
    assert C.sizeof(Pred) == 96 and C.sizeof(Force) == 88


@gpu
def test_yebisu_api_forces_and_predictor(gpu):
    L = C.CDLL(str(sp.LIB_PATH.parent / "libsapporoyeb_b200.so"))
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    L.initialize_special.argtypes = [C.c_int, C.POINTER(C.c_int)]
    L.set_jp_2.argtypes = [C.c_int, dp, dp, dp, dp, dp, dp, C.c_double, C.c_double, C.c_int,
                           C.c_double]
    L.predict_all.argtypes = [C.c_double, C.c_int]
    L.pick_up_predictor_2.argtypes = [C.c_int, C.POINTER(Pred)]
    L.calc_force_on_predictors.argtypes = [C.c_int, C.POINTER(Pred), C.POINTER(Force), C.c_int]
    L.initialize_special(1, (C.c_int * 1)(0))
    case = T.build_case(2, 2500, seed=92, binaries=0.1)
    n = case["n"]
    for k in range(n):
        L.set_jp_2(k, case["x"][k].copy(), case["v"][k].copy(), case["a"][k].copy(),
                   case["j"][k].copy(), case["s"][k].copy(), case["c"][k].copy(),
                   float(case["m"][k]), float(case["t0"][k]), int(case["id"][k]), case["eps2"])
    L.predict_all(case["ti"], n)
    for addr in (0, 33, n - 1):
        p = Pred()
        L.pick_up_predictor_2(addr, C.byref(p))
        assert int(p.id) == case["id"][addr] and p.mass == case["m"][addr]
        scale = np.maximum(np.abs(case["px"][addr]), np.abs(case["x"][addr]))
        assert np.all(np.abs(np.array(p.pos) - case["px"][addr]) <= 2e-14 * scale)
    preds = (Pred * n)()
    for i in range(n):
        preds[i].pos[:] = case["px"][i]
        preds[i].vel[:] = case["pv"][i]
        preds[i].acc[:] = case["pa"][i]
        preds[i].mass, preds[i].id, preds[i].eps2 = case["m"][i], case["id"][i], case["eps2"]
    forces = (Force * n)()
    L.calc_force_on_predictors(n, preds, forces, n)
    f = np.frombuffer(forces, dtype=np.dtype([("acc", "3f8"), ("jrk", "3f8"), ("snp", "3f8"),
                                              ("phi", "f8"), ("nnb", "i4"), ("r2", "f4")]))
    want = T.oracle_force(case, lists=False)
    got = {"acc": f["acc"], "jrk": f["jrk"], "snp": f["snp"], "pot": -f["phi"]}
    T.check_forces(got, want, 2, median_tol=1e-13, max_tol=1e-9)
    T.check_nn(case, f["nnb"], want)
    ok = want["nnb"] == f["nnb"]
    np.testing.assert_allclose(f["r2"][ok], want["ds2min"][ok].astype(np.float32), rtol=1e-6)


@gpu
def test_grape5_order_keeps_the_self_pair_whatever_the_ids(gpu):
    """Order GRAPE5 through the class: ids are passed and equal the j ids,
    yet, as on GRAPE-5, the self pair is not skipped and no neighbour is
    searched."""
    case = T.build_case(1, 1500, seed=93)
    n, eps2 = case["n"], 1e-6
    x, m = case["x"], case["m"]
    z = np.zeros((n, 3))
    with sp.Sapporo(order=sp.GRAPE5, precision=sp.DOUBLESINGLE) as s:
        s.set_j_particles(np.arange(n), case["id"], np.zeros(n), m, x, z, z, z)
        s.start(n, case["id"], x, z, None, eps2, np.full(n, 1.0))
        got = s.results(n)
        counts = s.neighbour_counts()
    want = O.force(1, x, z, None, np.zeros(n), np.full(n, -7, dtype=np.int32), x, z, None, m,
                   case["id"], eps2, lists=False)
    T.check_forces({"acc": got["acc"], "pot": got["pot"]}, want, 1, fields=["acc", "pot"])
    assert np.all(got["nnb"] == 0) and np.all(counts == 0)
