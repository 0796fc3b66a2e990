"""Python mirror of the Sapporo2 B200 library interfaces.

The product is the native library ``sapporo2_b200/lib/libsapporo_b200.so``
(CUDA kernels for sm_100a + the C++ ``sapporo`` class + the GRAPE-6 ``g6_*``
exports).  This module binds it with ctypes so that tests, the benchmark and
Python integrators can drive it:

* :class:`Sapporo` -- the ``sapporo`` C++ class (reference
  lib/include/sapporohostclass.h:125-175) through ``include/sapporo_c.h``;
* :class:`G6` -- the GRAPE-6 functions (reference
  lib/interfaces/sapporoG6lib.cpp), called exactly as a C/Fortran caller
  would;
* :class:`G5` -- the GRAPE-5 functions (reference lib/interfaces/sapporoG5lib.cpp);
* :class:`Batch` -- batched force calls over many clusters (``sapb_batch_*``);
* the lower sapb_* C ABI (``include/sapporo_b200.h``) through ``_SIGS``
  (``load_library()`` returns the bound library; :class:`Sapporo` exposes the
  handles of its devices as ``dev`` / ``devs``), including the device-resident
  force calls ``sapb_force_device`` and ``sapb_force_device_noalloc``.

There is no CPU fallback: if the library is missing or no sm_100 GPU is
present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

GRAPE5, FOURTH, SIXTH = 0, 1, 2
FLOAT, DOUBLESINGLE, DOUBLE = 0, 1, 2
NGB_PB = 256
NPIPES = 16384
NOALLOC_SCRATCH_BYTES = 32 << 20  # fixed scratch of sapb_force_device_noalloc
RES_STRIDE = 12
F_PREDICT = 1
F_NGB_LIST = 2

_PKG = Path(__file__).resolve().parent
# SAPPORO_B200_LIB selects another build of the library (e.g. a variant
# compiled with different kernel options); default: the in-tree build
LIB_PATH = Path(os.environ.get("SAPPORO_B200_LIB", _PKG / "lib" / "libsapporo_b200.so"))

_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class SapporoError(RuntimeError):
    pass


def _opt(ptr_type):
    """ndpointer that also accepts None."""

    class _P(ptr_type):  # type: ignore[misc, valid-type]
        @classmethod
        def from_param(cls, obj):
            if obj is None:
                return None
            return ptr_type.from_param(obj)

    return _P


_dpo = _opt(_dp)
_ipo = _opt(_ip)

# (name, restype, argtypes)
_SIGS = [
    ("sapb_version", C.c_char_p, []),
    ("sapb_error_string", C.c_char_p, [C.c_int]),
    ("sapb_last_error", C.c_char_p, [C.c_void_p]),
    ("sapb_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("sapb_open", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    ("sapb_close", C.c_int, [C.c_void_p]),
    ("sapb_info", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int)] * 5),
    ("sapb_set_stream", C.c_int, [C.c_void_p, C.c_void_p]),
    ("sapb_reserve_j", C.c_int, [C.c_void_p, C.c_int]),
    ("sapb_j_stage", C.c_void_p, [C.c_void_p, C.c_int]),
    ("sapb_j_stage_stride", C.c_int, [C.c_void_p]),
    ("sapb_push_j", C.c_int, [C.c_void_p, C.c_int]),
    ("sapb_predict", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("sapb_i_stage", C.c_void_p, [C.c_void_p, C.c_int]),
    ("sapb_i_stage_stride", C.c_int, [C.c_void_p]),
    ("sapb_force", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]),
    ("sapb_results", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int)]),
    ("sapb_ngb_fetch", C.c_int, [C.c_void_p, _ipo, _ipo, C.c_int]),
    ("sapb_wait_selftest", C.c_int, [C.c_void_p, C.c_int]),
    ("sapb_force_device", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_double,
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("sapb_force_device_noalloc", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                            C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                                            C.c_void_p]),
    ("sapb_read_j", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, _dp]),
    ("sapb_set_launch", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    ("sapb_set_spatial", C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    ("sapb_spatial_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong),
                                     C.POINTER(C.c_ulonglong), C.c_int]),
    ("sapb_set_near", C.c_int, [C.c_void_p, C.c_double]),
    ("sapb_get_plan", C.c_int, [C.c_void_p, C.c_int, C.c_int] + [C.POINTER(C.c_int)] * 3),
    ("sapb_batch_create", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    ("sapb_batch_destroy", C.c_int, [C.c_void_p]),
    ("sapb_batch_i_stage", C.c_void_p, [C.c_void_p]),
    ("sapb_batch_plan", C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _ip, _dpo, _dpo]),
    ("sapb_batch_run", C.c_int, [C.c_void_p, C.c_int]),
    ("sapb_batch_results", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int)]),
    ("sapb_batch_ngb_fetch", C.c_int, [C.c_void_p, _ipo, _ipo]),
    ("sapb_batch_info", C.c_int, [C.c_void_p] + [C.POINTER(C.c_int)] * 3),
    ("sapb_batch_set_tuning", C.c_int, [C.c_void_p, C.c_int]),
    ("sapb_batch_autotune", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int),
                                      C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    ("sapb_mlp_num_params", C.c_int, []),
    ("sapb_mlp_create", C.c_int, [C.c_void_p, C.c_ulonglong, C.POINTER(C.c_void_p)]),
    ("sapb_mlp_destroy", C.c_int, [C.c_void_p]),
    ("sapb_mlp_set_params", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("sapb_mlp_get_params", C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    ("sapb_mlp_forward", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float)]),
    ("sapb_mlp_gradient", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float),
                                    C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float)]),
    ("sapb_mlp_propose", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                   C.c_float, C.c_float, C.c_float, C.POINTER(C.c_float)]),
    ("sapb_mlp_train", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                 C.c_int, C.c_float, C.POINTER(C.c_float)]),
    # class binding
    ("sapporo_c_new", C.c_void_p, []),
    ("sapporo_c_delete", None, [C.c_void_p]),
    ("sapporo_c_open", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    ("sapporo_c_open_devices", C.c_int, [C.c_void_p, C.c_int, _ipo, C.c_int, C.c_int]),
    ("sapporo_c_close", C.c_int, [C.c_void_p]),
    ("sapporo_c_get_n_pipes", C.c_int, [C.c_void_p]),
    ("sapporo_c_set_time", C.c_int, [C.c_void_p, C.c_double]),
    ("sapporo_c_set_no_time", C.c_int, [C.c_void_p]),
    ("sapporo_c_set_j_particles", C.c_int, [C.c_void_p, C.c_int, _ip, _ip, _dpo, _dp, _dp, _dp,
                                            _dp, _dp, _dpo, _dpo, _dpo]),
    ("sapporo_c_start", C.c_int, [C.c_void_p, C.c_int, C.c_int, _ip, _dp, _dp, _dpo, C.c_double,
                                  _dpo]),
    ("sapporo_c_results", C.c_int, [C.c_void_p, C.c_int, C.c_int, _dp, _dpo, _dpo, _dp, _ipo,
                                    _dpo, C.c_int]),
    ("sapporo_c_force_prediction", C.c_int, [C.c_void_p, C.c_int]),
    ("sapporo_c_read_ngb_list", C.c_int, [C.c_void_p]),
    ("sapporo_c_get_ngb_list", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), _ip]),
    ("sapporo_c_ngb_list_copied", C.c_int, [C.c_void_p]),
    ("sapporo_c_retrieve_predicted", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("sapporo_c_retrieve_state", C.c_int, [C.c_void_p, C.c_int, _dp]),
    ("sapporo_c_last_status", C.c_int, [C.c_void_p]),
    ("sapporo_c_device", C.c_void_p, [C.c_void_p]),
    ("sapporo_c_device_at", C.c_void_p, [C.c_void_p, C.c_int]),
    ("sapporo_c_n_devices", C.c_int, [C.c_void_p]),
    # GRAPE-6
    # GRAPE-5 interface
    ("g5_open_special", C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    ("g5_open", None, []),
    ("g5_close", None, []),
    ("g5_get_number_of_pipelines", C.c_int, []),
    ("g5_set_n", None, [C.c_int]),
    ("g5_set_eps2_to_all", None, [C.c_double]),
    ("g5_set_eps_to_all", None, [C.c_double]),
    ("g5_set_xmj", None, [C.c_int, C.c_int, _dp, _dp]),
    ("g5_set_jp", None, [C.c_int, C.c_int, _dp, _dp]),
    ("g5_set_xi", None, [C.c_int, _dp]),
    ("g5_run", None, []),
    ("g5_get_force", None, [C.c_int, _dp, _dp]),
    ("g5_calculate_force_on_x", None, [_dp, _dp, _dp, C.c_int]),
    ("g5_set_range", None, [C.c_double, C.c_double, C.c_double]),
    ("g5_get_jmemsize", C.c_int, []),
    ("g5_get_number_of_real_pipelines", C.c_int, []),
    ("g5_get_pcibus_freq", C.c_int, []),
    ("g6_open_", C.c_int, [C.POINTER(C.c_int)]),
    ("g6_open_special", C.c_int, [C.c_int, C.POINTER(C.c_int)]),
    ("g6_close_", C.c_int, [C.POINTER(C.c_int)]),
    ("g6_npipes_", C.c_int, []),
    ("g6_set_tunit_", C.c_int, [C.POINTER(C.c_double)]),
    ("g6_set_xunit_", C.c_int, [C.POINTER(C.c_double)]),
    ("g6_set_ti_", C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    ("g6_set_j_particle_", C.c_int, [C.POINTER(C.c_int)] * 3 + [C.POINTER(C.c_double)] * 3
     + [_dp] * 5),
    ("g6calc_firsthalf_", None, [C.POINTER(C.c_int)] * 3 + [_ip, _dp, _dp, _dp, _dp, _dp,
                                                             C.POINTER(C.c_double), _dp]),
    ("g6calc_lasthalf_", C.c_int, [C.POINTER(C.c_int)] * 3 + [_ip, _dp, _dp,
                                                              C.POINTER(C.c_double), _dp, _dp,
                                                              _dp, _dp]),
    ("g6calc_lasthalf2_", C.c_int, [C.POINTER(C.c_int)] * 3 + [_ip, _dp, _dp,
                                                               C.POINTER(C.c_double), _dp, _dp,
                                                               _dp, _dp, _ip]),
    ("g6_initialize_jp_buffer_", C.c_int, [C.POINTER(C.c_int)] * 2),
    ("g6_flush_jp_buffer_", C.c_int, [C.POINTER(C.c_int)]),
    ("g6_reset_", C.c_int, [C.POINTER(C.c_int)]),
    ("g6_reset_fofpga_", C.c_int, [C.POINTER(C.c_int)]),
    ("g6_read_neighbour_list_", C.c_int, [C.POINTER(C.c_int)]),
    ("g6_get_neighbour_list_", C.c_int, [C.POINTER(C.c_int)] * 4 + [_ip]),
]


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libsapporo_b200.so (built by ``python -m sapporo2_b200.build``)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise SapporoError(f"{p} is missing; build it with `python -m sapporo2_b200.build`")
    lib = C.CDLL(str(p))
    for name, res, args in _SIGS:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return [s[0] for s in _SIGS]


def _check(rc: int, what: str, handle=None) -> int:
    if rc < 0:
        lib = load_library()
        detail = lib.sapb_last_error(handle).decode() if handle is not None else \
            lib.sapb_last_error(None).decode()
        raise SapporoError(f"{what}: {lib.sapb_error_string(rc).decode()} ({detail})")
    return rc


def device_count() -> int:
    lib = load_library()
    n = C.c_int(0)
    lib.sapb_device_count(C.byref(n))
    return n.value


def _f64(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


def _i32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.int32)


def _per_particle(a, n, what):
    """`a` (already converted) as n scalars, one per particle (or per
    cluster): the C side reads n values, so a shorter or longer array is
    refused here."""
    if a is not None and a.shape != (n,):
        raise ValueError(f"{what}: {n} values expected, got shape {a.shape}")
    return a


class Sapporo:
    """The ``sapporo`` class (C++).  Method names follow the reference; array
    arguments are numpy arrays ([n, 3] for vectors).  ``devices`` (a list of
    device ids, ids may repeat) spreads the j round-robin over one handle per
    entry, as ``sapporo::open(…, devices, len(devices), …)``; the default is
    the one device ``device``."""

    def __init__(self, device: int = 0, order: int = FOURTH, precision: int = DOUBLESINGLE,
                 n_pipes: int | None = None, devices=None):
        self.lib = load_library()
        self.h = self.lib.sapporo_c_new()
        if not self.h:
            raise SapporoError("allocation failed")
        self.order = order
        self.precision = precision
        # n_pipes (max i per start) is read from SAPPORO_NPIPES at open, as in the C++ class
        old = os.environ.get("SAPPORO_NPIPES")
        if n_pipes:
            os.environ["SAPPORO_NPIPES"] = str(int(n_pipes))
        try:
            if devices is None:
                _check(self.lib.sapporo_c_open(self.h, device, order, precision), "open")
            else:
                ids = _i32(list(devices))
                _check(self.lib.sapporo_c_open_devices(self.h, len(ids), ids if len(ids) else None,
                                                       order, precision), "open")
        finally:
            if n_pipes:
                if old is None:
                    del os.environ["SAPPORO_NPIPES"]
                else:
                    os.environ["SAPPORO_NPIPES"] = old
        self.dev = self.lib.sapporo_c_device(self.h)
        self.devs = [self.lib.sapporo_c_device_at(self.h, k)
                     for k in range(self.lib.sapporo_c_n_devices(self.h))]

    def _one_device(self, what):
        if len(self.devs) != 1:
            raise SapporoError(f"{what} reads one device; this object drives {len(self.devs)}")

    def close(self):
        if self.h:
            self.lib.sapporo_c_close(self.h)
            self.lib.sapporo_c_delete(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_n_pipes(self) -> int:
        return self.lib.sapporo_c_get_n_pipes(self.h)

    def set_time(self, t: float):
        _check(self.lib.sapporo_c_set_time(self.h, float(t)), "set_time")

    def set_no_time(self):
        _check(self.lib.sapporo_c_set_no_time(self.h), "set_no_time")

    def set_j_particles(self, address, id, t, mass, x, v, a, jrk, snp=None, crk=None, eps=None):
        address = _i32(address).reshape(-1)
        n = len(address)
        if mass is None or x is None:
            raise ValueError("set_j_particles: mass and x are required")
        _check(self.lib.sapporo_c_set_j_particles(
            self.h, n, address, _per_particle(_i32(id), n, "id"), _per_particle(_f64(t), n, "t"),
            _per_particle(_f64(mass), n, "mass"), _f64(x, (n, 3)), _f64(v, (n, 3)),
            _f64(a, (n, 3)), _f64(jrk, (n, 3)), _f64(snp, (n, 3)) if snp is not None else None,
            _f64(crk, (n, 3)) if crk is not None else None, _per_particle(_f64(eps), n, "eps")),
            "set_j_particle", self.dev)

    def start(self, nj, id, xi, vi, ai=None, eps2=0.0, h2=None):
        id = _i32(id).reshape(-1)
        ni = len(id)
        _check(self.lib.sapporo_c_start(self.h, int(nj), ni, id, _f64(xi, (ni, 3)),
                                        _f64(vi, (ni, 3)),
                                        _f64(ai, (ni, 3)) if ai is not None else None,
                                        float(eps2), _per_particle(_f64(h2), ni, "h2")),
               "startGravCalc", self.dev)
        self._ni = ni

    def results(self, nj, ni=None, ngb=True) -> dict:
        ni = self._ni if ni is None else ni
        acc = np.zeros((ni, 3))
        jrk = np.zeros((ni, 3))
        snp = np.zeros((ni, 3))
        pot = np.zeros(ni)
        nnb = np.zeros(ni, dtype=np.int32)
        dsmin = np.full(ni, np.nan)
        _check(self.lib.sapporo_c_results(self.h, int(nj), ni, acc, jrk, snp, pot, nnb, dsmin,
                                          1 if ngb else 0), "getGravResults", self.dev)
        return {"acc": acc, "jrk": jrk, "snp": snp, "pot": pot, "nnb": nnb, "ds2min": dsmin}

    def force_prediction(self, nj):
        _check(self.lib.sapporo_c_force_prediction(self.h, int(nj)), "forcePrediction", self.dev)

    def read_ngb_list(self) -> int:
        return self.lib.sapporo_c_read_ngb_list(self.h)

    def neighbour_counts(self, ni=None) -> np.ndarray:
        """Exact neighbour counts of the last force call (the lists hold at most
        NGB_PB ids; a count >= NGB_PB is an overflow)."""
        self._one_device("neighbour_counts")
        ni = self._ni if ni is None else ni
        cnt = np.zeros(max(ni, 1), dtype=np.int32)
        self.results_ready()
        _check(self.lib.sapb_ngb_fetch(self.dev, cnt, None, ni), "ngb_fetch", self.dev)
        return cnt[:ni]

    def raw_results(self, ni=None) -> np.ndarray:
        """Result records of the last force call as the device wrote them:
        [ni, RES_STRIDE] doubles = acc[3], pot, jerk[3], snap[3], ds2 of the
        nearest neighbour (float value; 1e11 when none), its id (-1 when
        none).  The input of the multi-GPU combine (sum, min-loc)."""
        self._one_device("raw_results")
        ni = self._ni if ni is None else ni
        p, n = C.c_void_p(), C.c_int()
        _check(self.lib.sapb_results(self.dev, C.byref(p), C.byref(n)), "results", self.dev)
        if n.value < ni:
            raise SapporoError(f"results hold {n.value} records, {ni} requested")
        buf = (C.c_double * (ni * RES_STRIDE)).from_address(p.value)
        return np.frombuffer(buf, dtype=np.float64).reshape(ni, RES_STRIDE).copy()

    def neighbour_lists(self, ni=None):
        """Counts [ni] and lists [ni, NGB_PB] of the last force call (entries
        past min(count, NGB_PB) are undefined)."""
        self._one_device("neighbour_lists")
        ni = self._ni if ni is None else ni
        cnt = np.zeros(max(ni, 1), dtype=np.int32)
        lst = np.zeros(max(ni, 1) * NGB_PB, dtype=np.int32)
        self.results_ready()
        _check(self.lib.sapb_ngb_fetch(self.dev, cnt, lst, ni), "ngb_fetch", self.dev)
        return cnt[:ni], lst.reshape(-1, NGB_PB)[:ni]

    def results_ready(self):
        self._one_device("results_ready")
        p, n = C.c_void_p(), C.c_int()
        _check(self.lib.sapb_results(self.dev, C.byref(p), C.byref(n)), "results", self.dev)

    def get_ngb_list(self, ipipe: int, maxlength: int = NGB_PB):
        buf = np.zeros(max(maxlength, 1), dtype=np.int32)
        n = C.c_int(0)
        ovf = self.lib.sapporo_c_get_ngb_list(self.h, int(ipipe), int(maxlength), C.byref(n), buf)
        # the ids written: several devices' lists together may hold more than NGB_PB
        return ovf, n.value, buf[:self.lib.sapporo_c_ngb_list_copied(self.h)].copy()

    def retrieve_predicted(self, addr: int) -> dict:
        o = np.zeros(12)
        _check(self.lib.sapporo_c_retrieve_predicted(self.h, int(addr), o), "retrieve", self.dev)
        return {"mass": o[0], "id": o[1], "eps2": o[2], "pos": o[3:6].copy(),
                "vel": o[6:9].copy(), "acc": o[9:12].copy()}

    def retrieve_state(self, addr: int) -> dict:
        o = np.zeros(24)
        _check(self.lib.sapporo_c_retrieve_state(self.h, int(addr), o), "retrieve", self.dev)
        keys = ["pos", "vel", "acc", "jrk", "ppos", "pvel", "pacc"]
        d = {"mass": o[0], "id": o[1], "eps2": o[2]}
        for k, name in enumerate(keys):
            d[name] = o[3 + 3 * k: 6 + 3 * k].copy()
        return d

    # lower level (settings go to every device of the object)
    def set_launch(self, tpi=0, ip=0, nslices=0):
        for d in self.devs:
            _check(self.lib.sapb_set_launch(d, tpi, ip, nslices), "set_launch", d)

    def set_spatial(self, mode=1, delta=0.0):
        """Spatial mode of the mixed-precision force calls: 0 off (address
        order, double-single difference for every pair), 1 on for calls of
        >= 2^28 pairs, >= 1024 i and >= 65536 j (default), 2 on for every call; far tiles use the
        single-float difference, accurate to `delta` (0: 1e-6)."""
        for d in self.devs:
            _check(self.lib.sapb_set_spatial(d, int(mode), float(delta)), "set_spatial", d)

    def set_near(self, factor=16.0):
        """Mixed precision: an i's share of a j tile holding a pair with
        ds2 < factor * eps2 is summed in FP64 (0: every pair in FP32)."""
        for d in self.devs:
            _check(self.lib.sapb_set_near(d, float(factor)), "set_near", d)

    def spatial_stats(self, reset=False):
        """(far, all) (warp, j tile) pairs of the spatial-mode calls since the
        last reset."""
        far = total = 0
        for d in self.devs:
            f, a = C.c_ulonglong(), C.c_ulonglong()
            _check(self.lib.sapb_spatial_stats(d, C.byref(f), C.byref(a), int(reset)),
                   "spatial_stats", d)
            far, total = far + f.value, total + a.value
        return far, total

    def plan(self, ni, nj):
        t, i, s = C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.sapb_get_plan(self.dev, ni, nj, C.byref(t), C.byref(i), C.byref(s)),
               "plan", self.dev)
        return t.value, i.value, s.value

    def set_stream(self, stream_ptr: int | None):
        self._one_device("set_stream")
        _check(self.lib.sapb_set_stream(self.dev, C.c_void_p(stream_ptr or 0)), "set_stream",
               self.dev)


class G5:
    """The GRAPE-5 interface (positions and masses in, acceleration and
    potential out), through its C ABI; one process-wide instance."""

    def __init__(self, devices=(0,)):
        self.lib = load_library()
        arr = (C.c_int * len(devices))(*devices)
        _check(self.lib.g5_open_special(len(devices), arr), "g5_open_special")

    def close(self):
        self.lib.g5_close()

    def set_eps(self, eps):
        self.lib.g5_set_eps_to_all(float(eps))

    def set_j(self, x, m):
        m = _f64(m).reshape(-1)
        x = _f64(x, (len(m), 3))
        self.lib.g5_set_n(len(m))
        self.lib.g5_set_xmj(0, len(m), x, m)

    def force(self, xi):
        xi = _f64(xi).reshape(-1, 3)
        a, phi = np.zeros((len(xi), 3)), np.zeros(len(xi))
        self.lib.g5_calculate_force_on_x(xi, a, phi, len(xi))
        return a, phi

    def force_chunk(self, xi):
        """g5_set_xi + g5_get_force (ni <= n_pipes)."""
        xi = _f64(xi).reshape(-1, 3)
        a, phi = np.zeros((len(xi), 3)), np.zeros(len(xi))
        self.lib.g5_set_xi(len(xi), xi)
        self.lib.g5_run()
        self.lib.g5_get_force(len(xi), a, phi)
        return a, phi


class G6:
    """The GRAPE-6 interface, called through its C ABI (one process-wide
    instance, as in the reference)."""

    def __init__(self):
        self.lib = load_library()

    @staticmethod
    def _i(v):
        return C.byref(C.c_int(int(v)))

    @staticmethod
    def _d(v):
        return C.byref(C.c_double(float(v)))

    def open(self, cluster=0):
        return self.lib.g6_open_(self._i(cluster))

    def open_special(self, devices=(0,)):
        arr = (C.c_int * len(devices))(*devices)
        return self.lib.g6_open_special(len(devices), arr)

    def close(self, cluster=0):
        return self.lib.g6_close_(self._i(cluster))

    def npipes(self):
        return self.lib.g6_npipes_()

    def set_ti(self, ti, cluster=0):
        return self.lib.g6_set_ti_(self._i(cluster), self._d(ti))

    def set_j_particle(self, address, index, tj, dtj, mass, k18, j6, a2, v, x, cluster=0):
        return self.lib.g6_set_j_particle_(self._i(cluster), self._i(address), self._i(index),
                                           self._d(tj), self._d(dtj), self._d(mass),
                                           _f64(k18, (3,)), _f64(j6, (3,)), _f64(a2, (3,)),
                                           _f64(v, (3,)), _f64(x, (3,)))

    def calc_firsthalf(self, nj, index, xi, vi, aold, j6old, phiold, eps2, h2, cluster=0):
        index = _i32(index).reshape(-1)
        ni = len(index)
        self.lib.g6calc_firsthalf_(self._i(cluster), self._i(nj), self._i(ni), index,
                                   _f64(xi, (ni, 3)), _f64(vi, (ni, 3)), _f64(aold, (ni, 3)),
                                   _f64(j6old, (ni, 3)), _per_particle(_f64(phiold), ni, "phiold"),
                                   self._d(eps2), _per_particle(_f64(h2), ni, "h2"))

    def calc_lasthalf(self, nj, index, xi, vi, eps2, h2, cluster=0):
        index = _i32(index).reshape(-1)
        ni = len(index)
        acc, jrk, pot = np.zeros((ni, 3)), np.zeros((ni, 3)), np.zeros(ni)
        rc = self.lib.g6calc_lasthalf_(self._i(cluster), self._i(nj), self._i(ni), index,
                                       _f64(xi, (ni, 3)), _f64(vi, (ni, 3)), self._d(eps2),
                                       _per_particle(_f64(h2), ni, "h2"), acc, jrk, pot)
        return rc, acc, jrk, pot

    def calc_lasthalf2(self, nj, index, xi, vi, eps2, h2, cluster=0):
        index = _i32(index).reshape(-1)
        ni = len(index)
        acc, jrk, pot = np.zeros((ni, 3)), np.zeros((ni, 3)), np.zeros(ni)
        inn = np.zeros(ni, dtype=np.int32)
        rc = self.lib.g6calc_lasthalf2_(self._i(cluster), self._i(nj), self._i(ni), index,
                                        _f64(xi, (ni, 3)), _f64(vi, (ni, 3)), self._d(eps2),
                                        _per_particle(_f64(h2), ni, "h2"), acc, jrk, pot, inn)
        return rc, acc, jrk, pot, inn

    def read_neighbour_list(self, cluster=0):
        return self.lib.g6_read_neighbour_list_(self._i(cluster))

    def get_neighbour_list(self, ipipe, maxlength=NGB_PB, cluster=0):
        buf = np.zeros(max(maxlength, 1), dtype=np.int32)
        n = C.c_int(0)
        ovf = self.lib.g6_get_neighbour_list_(self._i(cluster), self._i(ipipe),
                                              self._i(maxlength), C.byref(n), buf)
        # without overflow every id counted was written (several devices'
        # lists together may exceed NGB_PB); with it, at least the first
        # min(count, maxlength, NGB_PB)
        k = n.value if ovf == 0 else min(n.value, maxlength, NGB_PB)
        return ovf, n.value, buf[:k].copy()


class Batch:
    """Batched force evaluation (sapb_batch_*): many clusters -- independent
    systems or the active set of a block step -- in one persistent launch
    replayed from a captured CUDA graph.  Clusters are contiguous,
    address-ordered j ranges of the device's j store (set through the
    owning :class:`Sapporo`)."""

    def __init__(self, owner: "Sapporo", max_clusters: int, max_i: int):
        self.lib, self.owner = owner.lib, owner
        self.order = owner.order
        self.stride = 12 if self.order >= SIXTH else 8
        self.max_i = max_i
        h = C.c_void_p()
        _check(self.lib.sapb_batch_create(owner.dev, max_clusters, max_i, C.byref(h)),
               "batch_create", owner.dev)
        self.h = h
        ptr = self.lib.sapb_batch_i_stage(self.h)
        buf = (C.c_double * (max_i * self.stride)).from_address(ptr)
        self.i_stage = np.ctypeslib.as_array(buf).reshape(max_i, self.stride)

    def close(self):
        if self.h:
            self.lib.sapb_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def plan(self, j_first, j_count, i_count, t_pred=None, eps2=None):
        j_first = _i32(j_first).reshape(-1)
        n = len(j_first)
        _check(self.lib.sapb_batch_plan(self.h, n, j_first,
                                        _per_particle(_i32(j_count), n, "j_count"),
                                        _per_particle(_i32(i_count), n, "i_count"),
                                        _per_particle(_f64(t_pred), n, "t_pred"),
                                        _per_particle(_f64(eps2), n, "eps2")),
               "batch_plan", self.owner.dev)
        self.total_i = int(np.sum(i_count))

    def run(self, flags=F_PREDICT):
        _check(self.lib.sapb_batch_run(self.h, int(flags)), "batch_run", self.owner.dev)

    def results(self) -> np.ndarray:
        p, n = C.c_void_p(), C.c_int()
        _check(self.lib.sapb_batch_results(self.h, C.byref(p), C.byref(n)), "batch_results",
               self.owner.dev)
        if n.value == 0:
            return np.zeros((0, RES_STRIDE))
        buf = (C.c_double * (n.value * RES_STRIDE)).from_address(p.value)
        return np.ctypeslib.as_array(buf).reshape(n.value, RES_STRIDE).copy()

    def neighbours(self):
        n = self.total_i
        cnt = np.zeros(max(n, 1), dtype=np.int32)
        lst = np.zeros(max(n, 1) * NGB_PB, dtype=np.int32)
        _check(self.lib.sapb_batch_ngb_fetch(self.h, cnt, lst), "batch_ngb", self.owner.dev)
        return cnt[:n], lst[:n * NGB_PB].reshape(n, NGB_PB)

    def info(self):
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(self.lib.sapb_batch_info(self.h, C.byref(a), C.byref(b), C.byref(c)), "info",
               self.owner.dev)
        return {"items": a.value, "force_blocks": b.value, "runs": c.value}

    def set_tuning(self, tpi_scale: int):
        _check(self.lib.sapb_batch_set_tuning(self.h, int(tpi_scale)), "tuning", self.owner.dev)

    def autotune(self, flags=F_PREDICT, reps=2) -> dict:
        sc, sf, ms = C.c_int(), C.c_int(), C.c_float()
        _check(self.lib.sapb_batch_autotune(self.h, int(flags), int(reps), C.byref(sc),
                                            C.byref(sf), C.byref(ms)), "autotune", self.owner.dev)
        return {"tpi_scale": sc.value, "split_factor": sf.value, "ms": ms.value}


def pack_i_records(order, x, v, h2, ids, a=None) -> np.ndarray:
    """i records in the layout of sapb_i_stage (for device-resident calls)."""
    n = len(ids)
    stride = 12 if order >= SIXTH else 8
    rec = np.zeros((n, stride))
    rec[:, 0:3] = x
    rec[:, 3] = 0.0 if h2 is None else h2
    rec[:, 4:7] = v
    idw = np.zeros(n, dtype=np.int64)
    idw[:] = np.asarray(ids, dtype=np.int64) & 0xFFFFFFFF
    rec[:, 7] = idw.view(np.float64)
    if order >= SIXTH and a is not None:
        rec[:, 8:11] = a
    return rec
