"""MatrixMarket input (zolo_read_mm, host only; prepare_matrix.f90:154-321, 638-759)
against SciPy's reader of the same files: a symmetric coordinate file becomes the full
symmetric matrix, a general file is used as stored, array files in both symmetry classes,
duplicates keep the last value (the reference's assignment loop), and malformed files
are reported with their error codes."""
import os

import numpy as np
import pytest
import scipy.io
import scipy.sparse

import zolo_svd_b200 as zb


def write(tmp_path, name, text):
    p = os.path.join(str(tmp_path), name)
    with open(p, "w") as f:
        f.write(text)
    return p


@pytest.mark.parametrize("symmetry", ["general", "symmetric"])
def test_coordinate_matches_scipy(tmp_path, symmetry):
    rng = np.random.default_rng(7)
    n = 37
    a = scipy.sparse.random(n, n, density=0.15, random_state=3, format="coo")
    a.data = rng.standard_normal(a.nnz)
    if symmetry == "symmetric":
        a = scipy.sparse.tril(a + a.T).tocoo()
        a = (a + scipy.sparse.triu(a.T, 1)).tocoo()  # full symmetric; mmwrite stores one triangle
    p = os.path.join(str(tmp_path), f"m_{symmetry}.mtx")
    scipy.io.mmwrite(p, a, symmetry=symmetry)
    got, kind = zb.read_mm(p)
    assert kind == symmetry
    assert np.array_equal(got, scipy.io.mmread(p).toarray())
    if symmetry == "symmetric":
        assert np.array_equal(got, got.T)


def test_array_formats(tmp_path):
    rng = np.random.default_rng(8)
    g = rng.standard_normal((5, 3))
    p = os.path.join(str(tmp_path), "g.mtx")
    scipy.io.mmwrite(p, g)
    got, kind = zb.read_mm(p)
    assert kind == "general" and np.array_equal(got, g)
    s = rng.standard_normal((6, 6))
    s = s + s.T
    p = os.path.join(str(tmp_path), "s.mtx")
    scipy.io.mmwrite(p, s, symmetry="symmetric")
    got, kind = zb.read_mm(p)
    assert kind == "symmetric" and np.allclose(got, s, rtol=0, atol=1e-14 * np.abs(s).max())


def test_duplicates_comments_and_other_classes(tmp_path):
    p = write(tmp_path, "d.mtx", "%%MatrixMarket matrix coordinate real general\n% a comment\n\n"
                                 "3 2 4\n1 1 1.5\n3 2 -2\n1 1 4.0\n2 2 7\n")
    got, kind = zb.read_mm(p)
    assert kind == "general"
    assert np.array_equal(got, np.array([[4.0, 0.0], [0.0, 7.0], [0.0, -2.0]]))
    p = write(tmp_path, "k.mtx", "%%MatrixMarket matrix coordinate integer skew-symmetric\n2 2 1\n2 1 3\n")
    got, kind = zb.read_mm(p)
    assert kind == "other" and np.array_equal(got, np.array([[0.0, 0.0], [3.0, 0.0]]))


@pytest.mark.parametrize("text,code", [
    ("not a matrix market file\n1 1 1\n", -11),
    ("%%MatrixMarket matrix coordinate complex general\n1 1 1\n1 1 1 0\n", -13),
    ("%%MatrixMarket matrix coordinate pattern general\n1 1 1\n1 1\n", -13),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 2\n", -15),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", -16),
    ("%%MatrixMarket matrix coordinate real symmetric\n2 3 1\n1 1 1\n", -17),
])
def test_malformed_files(tmp_path, text, code):
    p = write(tmp_path, "bad.mtx", text)
    with pytest.raises(zb.ZoloError) as e:
        zb.read_mm(p)
    assert str(code) in str(e.value)
    with pytest.raises(zb.ZoloError):
        zb.read_mm(os.path.join(str(tmp_path), "missing.mtx"))
