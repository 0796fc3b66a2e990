"""Builds libsapporo_b200.so in-tree (sapporo2_b200/lib/) for sm_100a.

    python -m sapporo2_b200.build [--force] [--jobs N]

CUDA sources are compiled with nvcc for sm_100a only (the library refuses
other devices at open time); C++ host sources with the system g++.  The CUDA
runtime is linked statically, so the .so needs only the driver at run time.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIBNAME = "libsapporo_b200.so"
LIB6TH = "libsapporo6th_b200.so"  # 6th-order C interface (generic names, own library)
LIBYEB = "libsapporoyeb_b200.so"  # the Yebisu 6th-order interface (same generic names)

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
HOST_CXX = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-ccbin", HOST_CXX,
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "-Xcompiler", "-Wall",
    f"-I{INCLUDE}", f"-I{CSRC}",
]
CXX_FLAGS = ["-O3", "-fPIC", "-std=c++17", "-Wall", "-Wextra", f"-I{INCLUDE}", f"-I{CSRC}",
             f"-I{CUDA_HOME / 'include'}"]

CU_SOURCES = ["sapb_kernels.cu", "sapb_capi.cu", "sapb_batch_kernels.cu", "sapb_batch.cu",
              "sapb_mlp.cu", "sapb_spatial.cu"]
CXX_SOURCES = ["sapporohostclass.cpp", "sapporoG6lib.cpp", "sapporoG5lib.cpp", "sapporo_cbind.cpp"]


def _headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} {cmd[-1]}")


def library_path() -> Path:
    return LIBDIR / LIBNAME


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    deps = _headers()
    steps = []
    objs = []
    for s in CU_SOURCES:
        src, obj = CSRC / s, BUILD / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            steps.append([NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    for s in CXX_SOURCES:
        src, obj = CSRC / s, BUILD / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src, deps):
            steps.append([HOST_CXX, *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        list(ex.map(_run, steps))
    lib = library_path()
    relinked = False
    if force or steps or not lib.exists():
        tmp = lib.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-ccbin", HOST_CXX,
              "-o", str(tmp), *map(str, objs)])
        shutil.move(str(tmp), str(lib))
        relinked = True
    src6, obj6, lib6 = CSRC / "sapporo6thlib.cpp", BUILD / "sapporo6thlib.cpp.o", LIBDIR / LIB6TH
    if force or _stale(obj6, src6, deps):
        _run([HOST_CXX, *CXX_FLAGS, "-c", str(src6), "-o", str(obj6)])
        relinked = True
    if relinked or not lib6.exists():
        _run([HOST_CXX, "-shared", "-o", str(lib6), str(obj6), f"-L{LIBDIR}", "-lsapporo_b200",
              "-Wl,-rpath,$ORIGIN", "-Wl,-Bsymbolic"])
    srcy, objy, liby = CSRC / "sapporoYeblib.cpp", BUILD / "sapporoYeblib.cpp.o", LIBDIR / LIBYEB
    rely = relinked
    if force or _stale(objy, srcy, deps):
        _run([HOST_CXX, *CXX_FLAGS, "-c", str(srcy), "-o", str(objy)])
        rely = True
    if rely or not liby.exists():
        _run([HOST_CXX, "-shared", "-o", str(liby), str(objy), f"-L{LIBDIR}", "-lsapporo_b200",
              "-Wl,-rpath,$ORIGIN", "-Wl,-Bsymbolic"])
    if verbose:
        print(f"built {lib}")
    return lib


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    build(force=a.force, jobs=a.jobs, verbose=True)


if __name__ == "__main__":
    main()
