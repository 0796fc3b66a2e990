"""The reference's own test programs against this library.

CPU: testCodes/src/test_integrator.cpp (a GRAPE-6 Hermite integrator),
test_gravity_block.cpp and test_gravity_block_6th.cpp (sapporo class
drivers) compile and link *unchanged* against include/ and
libsapporo_b200.so -- checked wherever the reference tree is present.

GPU: the binaries built that way by oracle/Makefile (oracle/_ref/) run on
the GPU and their own printed checks are asserted: energy conservation of
the integrator and the relative force errors against their CPU FP64 loop.
"""
import os
import re
import subprocess
from pathlib import Path

import pytest

import sapporo2_b200 as sp

ROOT = Path(__file__).resolve().parents[1]
REF_BIN = ROOT / "oracle" / "_ref"


def _reference_tree() -> Path | None:
    """The reference tree: SAPPORO_REFERENCE, else the one oracle/Makefile
    built oracle/_ref/ from (recorded in oracle/_ref/reference_path)."""
    env = os.environ.get("SAPPORO_REFERENCE")
    if env:
        return Path(env)
    rec = REF_BIN / "reference_path"
    return Path(rec.read_text().strip()) if rec.exists() else None

PROGRAMS = ["test_integrator", "test_gravity_block", "test_gravity_block_6th"]


@pytest.mark.parametrize("prog", PROGRAMS)
def test_reference_program_links_unchanged(prog, tmp_path):
    ref = _reference_tree()
    src = ref / "testCodes" / "src" / f"{prog}.cpp" if ref else None
    if src is None or not src.exists():
        pytest.skip("reference tree not present")
    lib = sp.LIB_PATH
    cmd = ["/usr/bin/g++", "-O1", "-w", "-fopenmp", f"-I{ROOT / 'include'}",
           f"-I{ref / 'testCodes' / 'src'}", str(src), "-o", str(tmp_path / prog),
           f"-L{lib.parent}", "-lsapporo_b200", f"-Wl,-rpath,{lib.parent}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]


def _binary(prog):
    b = REF_BIN / prog
    if not b.exists():
        pytest.skip(f"{b} not built (make -C oracle where the reference tree exists)")
    return str(b)


@pytest.mark.gpu
def test_integrator_conserves_energy(gpu, tmp_path):
    r = subprocess.run([_binary("test_integrator"), "512"], capture_output=True, text=True,
                       cwd=tmp_path, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    de = [float(m) for m in re.findall(r"dE = (\S+) d\(dE\)", r.stderr)]
    assert len(de) > 50, r.stderr[-2000:]
    worst = max(abs(x) for x in de)
    print(f"\ntest_integrator N=512: {len(de)} steps to t=1, max |dE/E| = {worst:.3e}")
    assert worst < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("prog,args,tol", [
    ("test_gravity_block", ["1024", "linked", "1", "1"], (1e-5, 1e-3, 1e-6)),     # 4th, mixed
    ("test_gravity_block", ["1024", "linked", "1", "2"], (1e-12, 1e-10, 1e-12)),  # 4th, FP64
    ("test_gravity_block_6th", ["1024", "linked", "2", "2"], (1e-12, 1e-10, 1e-12)),
    ("test_gravity_block_6th", ["1024", "linked", "2", "1"], (1e-5, 1e-3, 1e-6)),
])
def test_gravity_block_programs(gpu, prog, args, tol, tmp_path):
    r = subprocess.run([_binary(prog), *args], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    last = [ln for ln in r.stdout.strip().splitlines() if ln.strip()][-1].split()
    acc_err, jrk_err, pot_err = (abs(float(x)) for x in last[:3])
    print(f"\n{prog} {' '.join(args)}: rel err acc {acc_err:.2e} jerk {jrk_err:.2e} "
          f"pot {pot_err:.2e}")
    assert acc_err < tol[0] and jrk_err < tol[1] and pot_err < tol[2]
