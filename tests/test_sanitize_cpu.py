"""The host-side C++ (graph builder, matrix-file IO, the oracle's CPU
restatement) built with -fsanitize=address,undefined and run on seeded
graphs: no sanitizer report and every consistency check passes.  CPU only."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_host_code_under_asan_and_ubsan(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "sanitize"
    src = [os.path.join(ROOT, "tests", "cpp", "sanitize_main.cpp"), os.path.join(ROOT, "oracle", "gk_oracle.cpp"),
           os.path.join(ROOT, "graphkokkos_b200", "csrc", "graph_io.cpp"),
           os.path.join(ROOT, "graphkokkos_b200", "csrc", "graph_host.cpp")]
    cmd = [cxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=undefined", "-fopenmp", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "graphkokkos_b200", "csrc"), *src, "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0", UBSAN_OPTIONS="halt_on_error=1",
               OMP_NUM_THREADS="2")
    out = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, env=env, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "OK" in out.stdout
    assert "runtime error" not in out.stderr and "AddressSanitizer" not in out.stderr
