"""Matrix file loaders (krans_csr_read_host; host only, no GPU): IJA triplet
files and Matrix Market coordinate files parsed with the reference's rules
(src/IO/MatrixLoader.cpp:12-56): IJA header "rows cols nnz" then 0-based
triplets, duplicates summed, a count mismatch only warns; Matrix Market
1-based, symmetric / skew-symmetric mirrored, pattern entries = 1."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_golden_matrix


def _write_ija(path, A, extra=(), shuffle_seed=0, header_nnz=None):
    C = A.tocoo()
    rows, cols, vals = list(C.row), list(C.col), list(C.data)
    for (i, j, v) in extra:
        rows.append(i); cols.append(j); vals.append(v)
    order = np.random.default_rng(shuffle_seed).permutation(len(vals))
    with open(path, "w") as f:
        f.write(f"{A.shape[0]} {A.shape[1]} {header_nnz if header_nnz is not None else len(vals)}\n")
        for k in order:
            f.write(f"{int(rows[k])} {int(cols[k])} {float(vals[k])!r}\n")


@pytest.mark.parametrize("k", [1, 3, 6])
def test_ija_golden_round_trip(tmp_path, k):
    import krans_b200 as kb
    A, _ = load_golden_matrix(k)
    p = tmp_path / f"mat{k}.ija"
    _write_ija(p, A, shuffle_seed=k)
    B = kb.read_matrix(str(p))
    assert B.shape == A.shape
    assert (B != A).nnz == 0
    assert np.all(np.diff(B.indptr) >= 0)
    for r in range(min(B.shape[0], 50)):
        c = B.indices[B.indptr[r]:B.indptr[r + 1]]
        assert np.all(np.diff(c) > 0)


def test_ija_duplicates_summed_and_count_warning(tmp_path, capfd):
    import krans_b200 as kb
    A = sp.csr_matrix(np.array([[1.0, 0, 2.0], [0, 3.0, 0]]))
    p = tmp_path / "dup.ija"
    _write_ija(p, A, extra=[(0, 0, 0.5), (1, 2, -1.25)], header_nnz=7)
    B = kb.read_matrix(str(p))
    want = A.toarray()
    want[0, 0] += 0.5
    want[1, 2] += -1.25
    np.testing.assert_array_equal(B.toarray(), want)
    assert "Expected 7 entries but read 5" in capfd.readouterr().err


def test_ija_errors(tmp_path):
    import krans_b200 as kb
    with pytest.raises(kb.KransError, match="Cannot open file"):
        kb.read_matrix(str(tmp_path / "missing.ija"))
    bad = tmp_path / "bad.ija"
    bad.write_text("x y z\n")
    with pytest.raises(kb.KransError, match="Invalid IJA file header"):
        kb.read_matrix(str(bad))
    out = tmp_path / "out.ija"
    out.write_text("2 2 1\n2 0 1.0\n")
    with pytest.raises(kb.KransInvalidArgument):
        kb.read_matrix(str(out))
    with pytest.raises(kb.KransInvalidArgument, match="Unsupported input format"):
        kb.read_matrix(str(tmp_path / "m.txt"))


def test_matrix_market_general_symmetric_pattern(tmp_path):
    import krans_b200 as kb
    g = tmp_path / "g.mtx"
    g.write_text("%%MatrixMarket matrix coordinate real general\n% comment\n\n3 4 4\n1 1 2.5\n3 4 -1\n1 1 0.5\n2 3 7e-3\n")
    B = kb.read_matrix(str(g)).toarray()
    want = np.zeros((3, 4))
    want[0, 0] = 3.0
    want[2, 3] = -1
    want[1, 2] = 7e-3
    np.testing.assert_array_equal(B, want)
    s = tmp_path / "s.mtx"
    s.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 3\n1 1 1\n3 1 2\n3 2 4\n")
    np.testing.assert_array_equal(kb.read_matrix(str(s)).toarray(),
                                  np.array([[1.0, 0, 2], [0, 0, 4], [2, 4, 0]]))
    k = tmp_path / "k.mtx"
    k.write_text("%%MatrixMarket matrix coordinate real skew-symmetric\n2 2 1\n2 1 3\n")
    np.testing.assert_array_equal(kb.read_matrix(str(k)).toarray(), np.array([[0.0, -3], [3, 0]]))
    pt = tmp_path / "p.mtx"
    pt.write_text("%%MatrixMarket matrix coordinate pattern general\n2 3 2\n1 3\n2 1\n")
    np.testing.assert_array_equal(kb.read_matrix(str(pt)).toarray(), np.array([[0.0, 0, 1], [1, 0, 0]]))
    arr = tmp_path / "a.mtx"
    arr.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(kb.KransError, match="coordinate"):
        kb.read_matrix(str(arr))
