"""The maintainer-side adapter shown for the reference (an mxmOp over the
reference's own spMtx calling the C ABI) compiles against the reference's
unmodified include/matrix.h (through the oracle's Kokkos-API shim) and links
against libgk_b200.so.  Compile and link only: no GPU here."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_adapter_compiles_and_links(gk, orc, tmp_path):
    if not orc.reference_present():
        pytest.skip("reference headers not present on this host")
    REF_INCLUDE = os.path.join(orc.REFERENCE_DIR, "include")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    lib = os.path.dirname(gk.LIB_PATH)
    exe = tmp_path / "adapter"
    cmd = [cxx, "-std=c++2a", "-O1", "-fopenmp", "-w", "-I", os.path.join(ROOT, "oracle", "kokkos_shim"),
           "-I", REF_INCLUDE, "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "ref_adapter.cpp"), "-L", lib, "-lgk_b200", f"-Wl,-rpath,{lib}",
           "-o", str(exe)]
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr[-4000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and "compiled" in run.stdout
