"""CPU-side checks of the product: the C-ABI library loads and exports every
symbol include/gk_b200.h declares; the host graph builder is deterministic and
canonical and matches an independent numpy restatement of the generator.
No compute entry point is called (no GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", fn)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(gk_\w+)\s*\(", txt, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(gk):
    lib = ctypes.CDLL(gk.LIB_PATH)
    decl = declared_symbols()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing
    from graphkokkos_b200._lib import SIGNATURES
    assert decl == set(SIGNATURES), decl ^ set(SIGNATURES)


def test_scheduler_shape(gk):
    lib = gk.load()
    assert lib.gk_sched_num_variants() == 24
    assert lib.gk_sched_num_features() == 8
    assert lib.gk_sched_model_size() > 0
    assert lib.gk_version() >= 100


def test_bad_model_rejected(gk):
    lib = gk.load()
    w = np.zeros(3, dtype=np.float32)
    assert lib.gk_sched_set_model(w.ctypes.data, 3) == 1  # GK_ERR_ARG
    assert b"gk_sched_model_size" in lib.gk_last_error_string()


def test_model_files_load_from_c(gk, tmp_path):
    """The shipped model files load through the C entry points a C/C++ host
    calls (host code only), equal the training output (.npz), and malformed
    files are refused with a reason."""
    from graphkokkos_b200 import sched
    lib = gk.load()
    for npz, loader in ((sched.MODEL_PATH, lib.gk_sched_load_model_file),
                        (sched.BC_MODEL_PATH, lib.gk_bc_load_model_file)):
        path = sched.bin_path(npz)
        assert loader(path.encode()) == 0, lib.gk_last_error_string()
        np.testing.assert_array_equal(sched.read_model_bin(path), np.load(npz)["w"].astype(np.float32))
        raw = open(path, "rb").read()
        for name, data, why in (("short", raw[:-4], b"wrong length"), ("long", raw + b"\0\0\0\0", b"wrong length"),
                                ("magic", b"XXXXXXXX" + raw[8:], b"GKMLP001"),
                                ("count", raw[:8] + b"\x05\0\0\0" + raw[12:], b"holds 5 weights")):
            bad = tmp_path / name
            bad.write_bytes(data)
            assert loader(str(bad).encode()) == 1, name
            assert why in lib.gk_last_error_string(), (name, lib.gk_last_error_string())
        assert loader(str(tmp_path / "absent.bin").encode()) == 1
        assert b"cannot open" in lib.gk_last_error_string()
    assert lib.gk_sched_has_model() == 1 and lib.gk_bc_has_model() == 1


def test_missing_library_fails_loudly(monkeypatch):
    import graphkokkos_b200._lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", "/nonexistent/libgk_b200.so")
    with pytest.raises(RuntimeError, match="not found"):
        L.load()


# ---------------------------------------------------------------------------
# host graph builder
# ---------------------------------------------------------------------------
MASK64 = (1 << 64) - 1


def mix64_np(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15))
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def rmat_numpy(scale, ef, seed, a=0.57, b=0.19, c=0.19):
    """Independent numpy restatement of the generator in gk_gen.h."""
    with np.errstate(over="ignore"):
        key = mix64_np(np.uint64(seed) ^ np.uint64(0x6A09E667F3BCC909))
        s = 4294967296.0
        ta, tab, tabc = np.uint32(int(a * s)), np.uint32(int((a + b) * s)), np.uint32(int((a + b + c) * s))
        e = np.arange(ef << scale, dtype=np.uint64)
        u = np.zeros_like(e)
        v = np.zeros_like(e)
        for lvl in range(scale):
            r = (mix64_np(key ^ ((e << np.uint64(6)) | np.uint64(lvl))) >> np.uint64(32)).astype(np.uint32)
            bu = (r >= tab).astype(np.uint64)
            bv = (((r >= ta) & (r < tab)) | (r >= tabc)).astype(np.uint64)
            u = (u << np.uint64(1)) | bu
            v = (v << np.uint64(1)) | bv
    keep = u != v
    u, v = u[keep].astype(np.int64), v[keep].astype(np.int64)
    n = 1 << scale
    keys = np.unique(np.concatenate([u * n + v, v * n + u]))
    rows, cols = keys // n, keys % n
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    return rp, cols.astype(np.int32)


@pytest.mark.parametrize("scale,seed", [(6, 1), (10, 7), (12, 3)])
def test_host_rmat_matches_numpy(gk, scale, seed):
    A = gk.gen_rmat(scale, 16, seed=seed)
    rp, col = rmat_numpy(scale, 16, seed)
    np.testing.assert_array_equal(A.rowptr, rp)
    np.testing.assert_array_equal(A.col, col)


def test_host_graph_canonical(gk):
    A = gk.gen_rmat(13, 16, seed=5)
    rp, col = A.rowptr, A.col
    rows = np.repeat(np.arange(A.m), np.diff(rp))
    assert np.all(col != rows), "self-loop"
    # sorted, strictly increasing within rows
    same = rows[1:] == rows[:-1]
    assert np.all(col[1:][same] > col[:-1][same])
    # symmetric
    fwd = rows.astype(np.int64) * A.m + col
    bwd = col.astype(np.int64) * A.m + rows
    np.testing.assert_array_equal(np.sort(fwd), np.sort(bwd))
    # deterministic
    B = gk.gen_rmat(13, 16, seed=5)
    np.testing.assert_array_equal(A.col, B.col)
    C = gk.gen_rmat(13, 16, seed=6)
    assert C.nnz != A.nnz or not np.array_equal(C.col, A.col)


def test_host_er(gk):
    A = gk.gen_er(5000, 40000, seed=9)
    assert A.m == 5000
    rp, col = A.rowptr, A.col
    rows = np.repeat(np.arange(A.m), np.diff(rp))
    assert np.all(col != rows)
    assert col.max() < 5000
    # ~ 2 * 40000 directed entries minus duplicates/self-loops
    assert 79000 < A.nnz <= 80000


def test_lower_host(gk, orc):
    A = gk.gen_rmat(9, 8, seed=2)
    L = gk.lower_host(A)
    orp, ocol = orc.extract_lower(A)
    np.testing.assert_array_equal(L.rowptr, orp)
    np.testing.assert_array_equal(L.col, ocol)


def test_dense_operator_arguments_are_checked_before_any_call(gk):
    """The Python operators refuse mismatched dense shapes and a non-float64
    in-place output before reaching the library (no GPU needed)."""
    from tests import graphs as G
    M = G.random_csr(4, 5, 0.5, seed=1)
    with pytest.raises(ValueError):
        gk.dense_ewise_mult_masked(np.zeros((4, 5)), np.zeros((4, 6)), M)
    with pytest.raises(ValueError):
        gk.dense_fuse_ewise_mult_add(np.zeros(6), np.zeros(6), np.zeros(6, dtype=np.float32))
    with pytest.raises(ValueError):
        gk.dense_fuse_ewise_mult_add(np.zeros(6), np.zeros(5), np.zeros(6))
    S = G.random_csr(4, 3, 0.5, seed=2)
    with pytest.raises(ValueError):
        gk.mxmm_spd(S, np.zeros((4, 5)), M)  # B must have S.n = 3 rows


def test_c_abi_refuses_bad_arguments_without_a_gpu(gk):
    """Shape and null-pointer errors come back as GK_ERR_ARG from the host
    side of the C ABI, before any device work."""
    lib = gk.load()
    A = gk.Csr(3, 3, np.array([0, 1, 2, 3]), np.array([1, 2, 0], dtype=np.int32), None, 3).as_gk()
    B = gk.Csr(4, 4, np.zeros(5, dtype=np.int64), np.zeros(0, dtype=np.int32), None, 0).as_gk()
    rp = np.zeros(4, dtype=np.int64)
    assert lib.gk_add_nointersect(ctypes.byref(A), ctypes.byref(B), rp.ctypes.data, None, None, None) == 1
    assert lib.gk_mxmm_spd(ctypes.byref(A), None, None, 2, ctypes.byref(B), None, None) == 1
    assert lib.gk_dense_ewise_mult_masked(-1, 2, None, None, ctypes.byref(A), None, None) == 1
    assert b"shape" in lib.gk_last_error_string() or b"negative" in lib.gk_last_error_string()
