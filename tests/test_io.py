"""Matrix files in the reference's formats (include/matrix.h:44-60, 210-533):
the library's readers give the reference readers' CSR entry for entry (rows
in file order), its writers round-trip, and bad files are refused with a
message.  Host code only: no GPU needed."""
import numpy as np
import pytest

from tests import graphs as G


def need_ref(orc):
    if not orc.ref_available():
        pytest.skip("reference oracle not built")


def same(a, b, values=True):
    assert (a.m, a.nnz) == (b.m, b.nnz)
    np.testing.assert_array_equal(np.asarray(a.rowptr), np.asarray(b.rowptr))
    np.testing.assert_array_equal(np.asarray(a.col), np.asarray(b.col))
    if values:
        np.testing.assert_array_equal(np.asarray(a.val), np.asarray(b.val))


def write_mtx(path, m, entries, field="pattern", symmetry="general"):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {symmetry}\n% a comment\n")
        f.write(f"{m} {m} {len(entries)}\n")
        for e in entries:
            f.write(" ".join(str(x) for x in e) + "\n")


def random_entries(m, n, seed, values):
    rng = np.random.default_rng(seed)
    r = rng.integers(1, m + 1, n)
    c = rng.integers(1, m + 1, n)
    if values:
        return [(int(i), int(j), int(v)) for i, j, v in zip(r, c, rng.integers(-9, 10, n))]
    return [(int(i), int(j)) for i, j in zip(r, c)]


@pytest.mark.parametrize("field,symmetry", [("pattern", "general"), ("pattern", "symmetric"),
                                            ("integer", "general"), ("integer", "symmetric")])
def test_mtx_matches_reference_reader(gk, orc, tmp_path, field, symmetry):
    need_ref(orc)
    path = tmp_path / "a.mtx"
    write_mtx(path, 300, random_entries(300, 2000, 7, field == "integer"), field, symmetry)
    mine = gk.read_matrix(path)
    ref = orc.ref_read_matrix(path, "mtx")
    same(mine, ref, values=field == "integer")
    if field == "pattern":
        assert mine.val is None
    # diagonal entries are dropped, as the reference does
    rows = np.repeat(np.arange(mine.m), np.diff(mine.rowptr))
    assert not np.any(rows == mine.col)


def test_rmat_format(gk, tmp_path):
    # each pair adds (x, y) and (y, x) in file order (matrix.h:488-533).  The
    # reference's reader cannot be run here: it sizes its buffers to 2·nz and
    # then reads 2·nz pairs from a file of nz (resizeVals doubles nz before the
    # loop, :494-505), overrunning them.
    p = tmp_path / "g.rmat"
    p.write_text("4 4 3\n0 1\n2 1\n3 0\n")
    A = gk.read_matrix(p)
    assert A.m == 4 and A.nnz == 6 and A.val is None
    np.testing.assert_array_equal(A.rowptr, [0, 2, 4, 5, 6])
    np.testing.assert_array_equal(A.col, [1, 3, 0, 2, 1, 0])


def test_crs_matches_reference_reader(gk, orc, tmp_path):
    need_ref(orc)
    A = G.random_csr(150, 150, 0.05, seed=4, values=True)
    p = tmp_path / "a.crs"
    # a three-letter code: the reference reads the code into a char[4]
    # (matrix.h:403), which with C++20 stream semantics stops after three
    # characters and would leave a fourth in the stream
    p.write_text(f"{A.m} {A.nnz} MCI\n" + " ".join(map(str, A.col)) + "\n" + " ".join(map(str, A.val)) + "\n"
                 + " ".join(map(str, A.rowptr)) + "\n")
    mine = gk.read_matrix(p)
    same(mine, orc.ref_read_matrix(p, "crs"))
    same(mine, A)


def test_bin_written_here_reads_in_the_reference(gk, orc, tmp_path):
    need_ref(orc)
    A = G.random_csr(250, 250, 0.04, seed=9, values=True)
    p = tmp_path / "a.bin"
    gk.write_matrix(p, A)
    same(gk.read_matrix(p), A)
    same(orc.ref_read_matrix(p, "bin"), A)


def test_round_trips(gk, tmp_path):
    A = gk.gen_rmat(10, 8, seed=2)
    for ext in ("mtx", "bin"):
        p = tmp_path / f"a.{ext}"
        gk.write_matrix(p, A)
        B = gk.read_matrix(p)
        same(B, A, values=False)
    V = G.random_csr(120, 120, 0.1, seed=1, values=True)
    gk.write_matrix(tmp_path / "v.bin", V)  # bin keeps everything
    same(gk.read_matrix(tmp_path / "v.bin"), V)
    gk.write_matrix(tmp_path / "v.mtx", V)  # mtx reading drops the diagonal, as the reference does
    rows = np.repeat(np.arange(V.m), np.diff(V.rowptr))
    keep = rows != V.col
    W = gk.read_matrix(tmp_path / "v.mtx", fmt="mtx")
    np.testing.assert_array_equal(W.col, V.col[keep])
    np.testing.assert_array_equal(W.val, V.val[keep])
    np.testing.assert_array_equal(np.diff(W.rowptr), np.bincount(rows[keep], minlength=V.m))


def test_graph_format_rows_start_after_the_header(gk, tmp_path):
    p = tmp_path / "a.graph"
    p.write_text("4 6\n1 2\n0 3\n0\n1\n")
    A = gk.read_matrix(p)
    assert A.m == 4 and A.nnz == 6 and A.val is None
    np.testing.assert_array_equal(A.rowptr, [0, 2, 4, 5, 6])
    np.testing.assert_array_equal(A.col, [1, 2, 0, 3, 0, 1])


def test_sort_rows(gk, tmp_path):
    p = tmp_path / "s.mtx"
    write_mtx(p, 5, [(1, 5, 3), (1, 2, 4), (2, 4, 1), (2, 1, 2)], "integer")
    A = gk.read_matrix(p)
    np.testing.assert_array_equal(A.col, [4, 1, 3, 0])
    S = gk.read_matrix(p, sort=True)
    np.testing.assert_array_equal(S.col, [1, 4, 0, 3])
    np.testing.assert_array_equal(S.val, [4, 3, 2, 1])


def test_bad_files_are_refused(gk, tmp_path):
    with pytest.raises(gk.GkError, match="cannot open"):
        gk.read_matrix(tmp_path / "missing.mtx")
    p = tmp_path / "bad.mtx"
    p.write_text("hello\n")
    with pytest.raises(gk.GkError, match="MatrixMarket"):
        gk.read_matrix(p)
    p = tmp_path / "rect.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n3 4 1\n1 2\n")
    with pytest.raises(gk.GkError, match="square"):
        gk.read_matrix(p)
    p = tmp_path / "short.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern general\n3 3 5\n1 2\n")
    with pytest.raises(gk.GkError, match="ends before"):
        gk.read_matrix(p)
    with pytest.raises(gk.GkError, match="format"):
        gk.read_matrix(tmp_path / "x.unknown")
