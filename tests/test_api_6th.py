"""GPU: the 6th-order C interface (libsapporo6th_b200.so, the reference's
lib/interfaces/sapporo6thlib.cpp API) against the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

import sapporo2_b200 as sp
from oracle import oracle as O
from tests import cases as T

pytestmark = pytest.mark.gpu

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


@pytest.fixture(scope="module")
def lib6(gpu):
    L = C.CDLL(str(sp.LIB_PATH.parent / "libsapporo6th_b200.so"))
    L.initialize_special.argtypes = [C.c_int, C.POINTER(C.c_int)]
    L.set_j_particle.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                 C.c_int, C.c_double]
    L.predict_all.argtypes = [C.c_double, C.c_int]
    L.no_predict_all.argtypes = [C.c_double, C.c_int]
    L.pick_up_predictor_2.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), _dp, _dp, _dp]
    L.calc_force_on_predictors.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, _dp, _dp, _dp, _dp,
                                           _dp, _dp, _dp, _dp, _ip, _dp]
    dev = (C.c_int * 1)(0)
    L.initialize_special(1, dev)
    return L


def test_6th_api_forces_and_predictor(lib6):
    case = T.build_case(2, 3000, seed=81, binaries=0.1)
    n = case["n"]
    for k in range(n):
        lib6.set_j_particle(k, case["x"][k].copy(), case["v"][k].copy(), case["a"][k].copy(),
                            case["j"][k].copy(), case["s"][k].copy(), case["c"][k].copy(),
                            float(case["m"][k]), float(case["t0"][k]), int(case["id"][k]), 0.0)
    lib6.predict_all(case["ti"], n)
    # predicted state read back = the FP64 prediction
    for addr in (0, 17, n - 1):
        pid, m, e2 = C.c_int(), C.c_double(), C.c_double()
        pos, vel, acc = np.zeros(3), np.zeros(3), np.zeros(3)
        lib6.pick_up_predictor_2(addr, C.byref(pid), C.byref(m), C.byref(e2), pos, vel, acc)
        assert pid.value == case["id"][addr] and m.value == case["m"][addr]
        scale = np.maximum(np.abs(case["px"][addr]), np.abs(case["x"][addr]))
        assert np.all(np.abs(pos - case["px"][addr]) <= 2e-14 * scale)
    # force on every particle (all-FP64 kernels by default)
    ids = case["id"].astype(np.int32)
    eps2 = np.full(n, case["eps2"])
    out = {k: np.zeros((n, 3)) for k in ("acc", "jrk", "snp", "crk")}
    phi, nnb, r2 = np.zeros(n), np.zeros(n, dtype=np.int32), np.zeros(n)
    lib6.calc_force_on_predictors(n, n, ids, case["px"], case["pv"], case["pa"], case["m"], eps2,
                                  out["acc"], out["jrk"], out["snp"], out["crk"], phi, nnb, r2)
    want = T.oracle_force(case, lists=False)
    got = {"acc": out["acc"], "jrk": out["jrk"], "snp": out["snp"], "pot": phi}
    T.check_forces(got, want, 2, median_tol=1e-13, max_tol=1e-9)
    assert np.all(out["crk"] == 0)
    assert T.check_nn(case, nnb, want) == 0
