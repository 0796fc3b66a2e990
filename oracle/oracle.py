"""ctypes wrapper of the FP64 CPU oracle (liboracle.so, sapporo_oracle.c)
and of the reference-kernel launcher (_ref/libsapref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
CPU-baseline leg of bench.py, always as the checker or the timed CPU
baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_DIR = HERE / "_ref"
REF_SO = REF_DIR / "libsapref.so"
REF_CUBIN = REF_DIR / "ref_kernels.cubin"

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def _opt(t):
    class _P(t):  # type: ignore[misc, valid-type]
        @classmethod
        def from_param(cls, obj):
            return None if obj is None else t.from_param(obj)
    return _P


_dpo, _ipo = _opt(_dp), _opt(_ip)
_lib = None
_ref = None


def build() -> None:
    """Builds liboracle.so (and _ref/ when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            build()
        L = C.CDLL(str(ORACLE_SO))
        L.orc_predict.argtypes = [C.c_int, C.c_double, C.c_int, _dp, _dp, _dp, _dp, _dp, _dpo,
                                  _dpo, _dp, _dp, _dpo, C.c_int]
        L.orc_predict.restype = None
        L.orc_force.argtypes = [C.c_int, C.c_int, _dp, _dp, _dpo, _dpo, _ip, C.c_int, _dp, _dp,
                                _dpo, _dp, _ip, C.c_double, _dp, _dpo, _dpo, _dpo, _ipo, _dpo,
                                _ipo, _ipo, C.c_int, C.c_int]
        L.orc_force.restype = None
        L.orc_force_subset.argtypes = [C.c_int, C.c_int, _ip, _dp, _dp, _dpo, _dpo, _ip, C.c_int,
                                       _dp, _dp, _dpo, _dp, _ip, C.c_double, _dp, _dpo, _dpo,
                                       _dpo, _ipo, _dpo, _ipo, C.c_int]
        L.orc_force_subset.restype = None
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def max_threads() -> int:
    return lib().orc_max_threads()


def _f(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.reshape(shape) if shape is not None else a


def predict(order, ti, t, x, v, a, j, s=None, c=None, nthreads=0):
    """FP64 Taylor prediction of every j to ti (kernels.cu:331-383)."""
    n = len(t)
    px, pv = np.empty((n, 3)), np.empty((n, 3))
    pa = np.empty((n, 3)) if order >= 2 else None
    lib().orc_predict(n, float(ti), int(order), _f(t), _f(x, (n, 3)), _f(v, (n, 3)),
                      _f(a, (n, 3)), _f(j, (n, 3)), _f(s, (n, 3)), _f(c, (n, 3)), px, pv, pa,
                      int(nthreads))
    return px, pv, pa


def force(order, xi, vi, ai, h2, idi, xj, vj, aj, mj, idj, eps2, ngb_cap=256, nthreads=0,
          lists=True):
    """FP64 direct summation on every i (kernels.cu:552-669 semantics)."""
    ni, nj = len(idi), len(idj)
    acc, jrk, pot = np.empty((ni, 3)), np.empty((ni, 3)), np.empty(ni)
    snp = np.zeros((ni, 3))
    nnb, cnt = np.empty(ni, dtype=np.int32), np.empty(ni, dtype=np.int32)
    ds2 = np.empty(ni)
    lst = np.full((ni, ngb_cap), -1, dtype=np.int32) if lists else None
    lib().orc_force(int(order), ni, _f(xi, (ni, 3)), _f(vi, (ni, 3)),
                    _f(ai, (ni, 3)) if order >= 2 else None, _f(h2),
                    np.ascontiguousarray(idi, dtype=np.int32), nj, _f(xj, (nj, 3)),
                    _f(vj, (nj, 3)), _f(aj, (nj, 3)) if order >= 2 else None, _f(mj),
                    np.ascontiguousarray(idj, dtype=np.int32), float(eps2), acc, jrk, snp, pot,
                    nnb, ds2, cnt, lst, int(ngb_cap), int(nthreads))
    return {"acc": acc, "jrk": jrk, "snp": snp, "pot": pot, "nnb": nnb, "ds2min": ds2,
            "ngb_count": cnt, "ngb_list": lst}


def force_subset(order, sel, xi, vi, ai, h2, idi, xj, vj, aj, mj, idj, eps2, nthreads=0):
    """FP64 direct summation for the i listed in `sel` (sampled checks)."""
    sel = np.ascontiguousarray(sel, dtype=np.int32)
    ns, ni, nj = len(sel), len(idi), len(idj)
    acc, jrk, snp, pot = np.empty((ns, 3)), np.empty((ns, 3)), np.zeros((ns, 3)), np.empty(ns)
    nnb, cnt, ds2 = np.empty(ns, dtype=np.int32), np.empty(ns, dtype=np.int32), np.empty(ns)
    lib().orc_force_subset(int(order), ns, sel, _f(xi, (ni, 3)), _f(vi, (ni, 3)),
                           _f(ai, (ni, 3)) if order >= 2 else None, _f(h2),
                           np.ascontiguousarray(idi, dtype=np.int32), nj, _f(xj, (nj, 3)),
                           _f(vj, (nj, 3)), _f(aj, (nj, 3)) if order >= 2 else None, _f(mj),
                           np.ascontiguousarray(idj, dtype=np.int32), float(eps2), acc, jrk,
                           snp, pot, nnb, ds2, cnt, int(nthreads))
    return {"acc": acc, "jrk": jrk, "snp": snp, "pot": pot, "nnb": nnb, "ds2min": ds2,
            "ngb_count": cnt}


def derivative_fn(nthreads=0):
    """force_fn for sapporo2_b200.ic.fill_derivatives (all particles act on
    all particles, FP64)."""
    def fn(order, x, v, a, m, ids, eps2):
        r = force(order, x, v, a, None, ids, x, v, a, m, ids, eps2, ngb_cap=1,
                  nthreads=nthreads, lists=False)
        return r["acc"], r["jrk"], r["snp"]
    return fn


# ---------------------------------------------------------------------------
# Reference kernels (oracle/_ref, built from the reference sources)
# ---------------------------------------------------------------------------
def ref_available() -> bool:
    return REF_SO.exists() and REF_CUBIN.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        R = C.CDLL(str(REF_SO))
        R.sapref_open.argtypes = [C.c_char_p, C.c_int]
        R.sapref_last_error.restype = C.c_char_p
        R.sapref_size_ok.argtypes = [C.c_int, C.c_int]
        R.sapref_predict.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp,
                                     _dpo, _dpo, _dp, _dp, _dpo]
        R.sapref_gravity.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp, _dpo, _ip, C.c_int,
                                     _dp, _dp, _dpo, _ip, C.c_double, _dp, _fp, _ip, _ipo,
                                     C.c_int, C.POINTER(C.c_float)]
        rc = R.sapref_open(str(REF_CUBIN).encode(), 0)
        if rc != 0:
            raise RuntimeError(f"sapref_open: {R.sapref_last_error().decode()}")
        _ref = R
    return _ref


def ref_size_ok(order, ni) -> bool:
    return bool(ref().sapref_size_ok(int(order), int(ni)))


def _pack4(a3, w):
    n = len(a3)
    o = np.zeros((n, 4))
    o[:, :3] = a3
    o[:, 3] = w
    return o


def ref_predict(order, ti, t, x, m, v, a, j, s=None, c=None):
    n = len(t)
    t2 = np.zeros((n, 2))
    t2[:, 0] = t
    pos, vel, acc, jrk = _pack4(x, m), _pack4(v, 0.0), _pack4(a, 0.0), _pack4(j, 0.0)
    snp = _pack4(s, 0.0) if order >= 2 else None
    crk = _pack4(c, 0.0) if order >= 2 else None
    pp, pv, pa = np.zeros((n, 4)), np.zeros((n, 4)), np.zeros((n, 4))
    rc = ref().sapref_predict(int(order), n, float(ti), t2, pos, vel, acc, jrk, snp, crk, pp, pv,
                              pa)
    if rc != 0:
        raise RuntimeError(f"sapref_predict {rc}: {ref().sapref_last_error().decode()}")
    return pp[:, :3].copy(), pv[:, :3].copy(), pa[:, :3].copy()


def ref_gravity(order, precision, xi, vi, ai, h2, idi, xj, vj, aj, mj, idj, eps2, reps=1,
                lists=True):
    """The reference's dev_evaluate_gravity_* with its own launch geometry.
    Returns the same dict as `force` plus `ms` (mean time per sweep)."""
    ni, nj = len(idi), len(idj)
    jpos, jvel = _pack4(xj, mj), _pack4(vj, 0.0)
    jacc = _pack4(aj, 0.0) if order >= 2 else None
    ipos, ivel = _pack4(xi, h2), _pack4(vi, eps2)
    iacc = _pack4(ai, 0.0) if order >= 2 else None
    res = np.zeros((3 * ni, 4))
    ds = np.zeros((ni, 2), dtype=np.float32)
    cnt = np.zeros(ni, dtype=np.int32)
    lst = np.zeros((ni, 256), dtype=np.int32) if lists else None
    ms = C.c_float(0)
    rc = ref().sapref_gravity(int(order), int(precision), nj, jpos, jvel, jacc,
                              np.ascontiguousarray(idj, dtype=np.int32), ni, ipos, ivel, iacc,
                              np.ascontiguousarray(idi, dtype=np.int32), float(eps2), res, ds,
                              cnt, lst, int(reps), C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"sapref_gravity {rc}: {ref().sapref_last_error().decode()}")
    acc = res[:ni, :3].copy()
    pot = res[:ni, 3].copy()
    jrk = res[ni:2 * ni, :3].copy()
    snp = res[2 * ni:3 * ni, :3].copy()
    nnb = ds[:, 0].view(np.int32).copy()
    return {"acc": acc, "jrk": jrk, "snp": snp, "pot": pot, "nnb": nnb,
            "ds2min": ds[:, 1].astype(np.float64), "ngb_count": cnt, "ngb_list": lst,
            "ms": ms.value}


if __name__ == "__main__":
    build()
    print("oracle threads:", max_threads(), "reference kernels:", ref_available(),
          os.environ.get("OMP_NUM_THREADS"))
