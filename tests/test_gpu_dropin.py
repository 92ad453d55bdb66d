"""The header-only C++ drop-in (include/gk/graphkokkos.hpp), compiled here
against libgk_b200.so and run as the reference's driver would call its
operators; results checked against the oracle."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def dropin_exe(tmp_path_factory, gk):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    out = tmp_path_factory.mktemp("dropin") / "dropin"
    lib = os.path.dirname(gk.LIB_PATH)
    cmd = [cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp"), "-L", lib, "-lgk_b200", f"-Wl,-rpath,{lib}",
           "-o", str(out)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return str(out)


@pytest.mark.parametrize("scale,seed", [(10, 3), (12, 5)])
def test_dropin_matches_oracle(dropin_exe, gk, orc, cuda, scale, seed):
    res = json.loads(subprocess.run([dropin_exe, str(scale), str(seed)], check=True, capture_output=True,
                                    text=True).stdout)
    A = gk.gen_rmat(scale, 16, seed=seed)
    tri = orc.tc_lower(gk.lower_host(A))
    assert res["tc_msa"] == res["tc_mca"] == res["tc_user"] == tri
    assert res["mxm_sum"] == int(orc.mxmm(A, A, A).astype(np.int64).sum())
    rp, col, iters, _ = orc.ktruss(A, 5)
    assert res["ktruss_nnz"] == len(col) and res["ktruss_iters"] == iters
    bc = orc.bc_f64(A, np.arange(32))
    assert res["bc_f64_sum"] == pytest.approx(bc.sum(), rel=1e-12)
    assert res["bc_float_sum"] == pytest.approx(bc.sum(), rel=1e-5)
    assert res["symm_roundtrip"] and res["transpose_nnz"]
    assert res["tc_lu"] == tri
    crp, ccol, cval = orc.mxmm_cmask(A, A, A)
    assert res["cmask_nnz"] == len(ccol) and res["cmask_sum"] == int(cval.astype(np.int64).sum())
    assert res["vertex_sum"] == int(orc.ref_tc_vertex(A).astype(np.int64).sum())
    assert res["add_nointersect_ok"] and res["spd_ok"]
    deg = np.diff(np.asarray(A.rowptr)).astype(np.float64)
    assert res["ewise_sum"] == float(2.0 * np.sum(deg ** 3))  # deg(i)^2 on deg(i) entries, twice


def test_dropin_learned_schedule_from_environment(dropin_exe, gk, cuda):
    """GK_SCHED=learned with the shipped model files: every drop-in call runs
    the learned schedule, with the plain schedule's results."""
    from graphkokkos_b200 import sched
    env = dict(os.environ, GK_SCHED="learned", GK_SCHED_MODEL=sched.bin_path(sched.MODEL_PATH),
               GK_BC_SCHED_MODEL=sched.bin_path(sched.BC_MODEL_PATH))
    plain = json.loads(subprocess.run([dropin_exe, "12", "5"], check=True, capture_output=True, text=True).stdout)
    learned = json.loads(subprocess.run([dropin_exe, "12", "5"], check=True, capture_output=True, text=True,
                                        env=env).stdout)
    for key in ("tc_msa", "tc_mca", "tc_user", "mxm_sum", "ktruss_nnz", "ktruss_iters", "tc_lu", "vertex_sum"):
        assert learned[key] == plain[key], key
    assert learned["bc_f64_sum"] == pytest.approx(plain["bc_f64_sum"], rel=1e-12)
    bad = dict(env, GK_SCHED_MODEL=os.path.join(ROOT, "README.md"))
    run = subprocess.run([dropin_exe, "10", "3"], capture_output=True, text=True, env=bad)
    assert run.returncode != 0 and "GKMLP001" in run.stderr


def test_reference_adapter_learned(gk, cuda):
    """The integration guide's reference-side adapter (built against the
    reference's own include/matrix.h) loads the learned models from their
    files and runs gk_mxmm_masked / gk_tc_count / gk_bc_batch with
    GK_SCHED_LEARNED."""
    from graphkokkos_b200 import sched
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_adapter")
    if not os.path.exists(exe):
        pytest.skip("the adapter is built only where the reference headers are present")
    run = subprocess.run([exe, sched.bin_path(sched.MODEL_PATH), sched.bin_path(sched.BC_MODEL_PATH)],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout + run.stderr
    res = json.loads(run.stdout)
    assert res["K64"]["tc_on_A"] == 64 * 63 * 62 and res["K4"]["mxm_sum"] == 24
