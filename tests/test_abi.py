"""CPU: the shared library loads without a GPU and exports every entry point
that include/*.h declares (C names via dlsym, class methods via the
demangled dynamic symbol table)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

import sapporo2_b200 as sp

INCLUDE = Path(__file__).resolve().parents[1] / "include"
C_HEADERS = ["sapporo_b200.h", "sapporo_c.h", "sapporo_g6.h", "sapporo_g5.h"]
# interfaces with generic names live in libraries of their own
OWN_LIBS = {"sapporo6th.h": "libsapporo6th_b200.so", "sapporo_yebisu.h": "libsapporoyeb_b200.so"}
DECL = re.compile(r"^\s*(?:const\s+)?(?:struct\s+)?[A-Za-z_][\w]*\s*\**\s*\**\s*([a-z_][\w]*)\s*\(",
                  re.M)


def declared_c_functions(headers=C_HEADERS):
    names = []
    for h in headers:
        text = (INCLUDE / h).read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"#.*", "", text)
        names += [n for n in DECL.findall(text) if n not in ("if", "while", "return")]
    return sorted(set(names))


def test_library_loads_without_gpu():
    lib = sp.load_library()
    assert lib.sapb_version().startswith(b"sapporo-b200")


def test_declared_c_symbols_exported():
    names = declared_c_functions()
    assert len(names) >= 40, names
    lib = ctypes.CDLL(str(sp.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("header", sorted(OWN_LIBS))
def test_interface_libraries_export_their_headers(header):
    names = declared_c_functions([header])
    assert len(names) >= 6, names
    lib = ctypes.CDLL(str(sp.LIB_PATH.parent / OWN_LIBS[header]))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_bindings_cover_c_api():
    bound = set(sp.exported_symbols())
    decl = set(declared_c_functions())
    # every declared C function except the C++-only helper has a binding
    assert decl - bound <= {"get_j_part_data"}, decl - bound


CLASS_METHODS = ["open", "close", "get_n_pipes", "set_time", "set_no_time", "set_j_particle",
                 "startGravCalc", "getGravResults", "forcePrediction",
                 "retrieve_predicted_j_particle", "retrieve_j_particle_state",
                 "fetch_ngb_list_from_device", "read_ngb_list", "get_ngb_list",
                 "send_j_particles_to_device", "send_i_particles_to_device"]


def test_class_methods_exported():
    out = subprocess.run(["nm", "-DC", "--defined-only", str(sp.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    missing = [m for m in CLASS_METHODS if f"sapporo::{m}(" not in out]
    assert not missing, missing
    assert "sapporo::sapporo()" in out and "sapporo::~sapporo()" in out


def test_open_without_gpu_fails_cleanly():
    if sp.device_count() > 0:
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    lib = sp.load_library()
    rc = lib.sapb_open(ctypes.byref(h), 0, sp.SIXTH, sp.DOUBLESINGLE, 0, 0)
    assert rc == -5  # SAPB_ENODEV
    assert not h.value
    with pytest.raises(sp.SapporoError):
        sp.Sapporo(order=sp.SIXTH)
